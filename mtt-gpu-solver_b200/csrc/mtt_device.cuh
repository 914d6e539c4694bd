// mtt_device.cuh — device primitives shared by the sm_100a kernels.
//
// Hand evaluation reproduces the reference scoring function fast_7card_score
// (src/tools/mtt_ev_dumper.cu:53-83; copies at honest_multistreet_solver.cu:24-54
// and preflop_grid_generator.cu:47-77) bit for bit, including its
// non-standard parts: no kickers for quads/trips/pairs, a full house takes
// the second trips before the best pair, and high-card hands compare by the
// whole 7-rank mask.  Instead of the reference's per-thread count arrays and
// rank loops it keeps four rank bit-planes (rank seen >=1, >=2, >=3, 4 times)
// and four 13-bit suit masks packed in one 64-bit word, so every case is a
// handful of bit operations, __popc and __clz with no local memory.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mtt {

struct Planes {
    uint32_t one, two, three, four;
    uint64_t suits;   // 4 x 16-bit lanes, lane s holds the 13-bit rank mask of suit s
};

__host__ __device__ __forceinline__ void planes_clear(Planes& p) {
    p.one = p.two = p.three = p.four = 0u;
    p.suits = 0ull;
}

__host__ __device__ __forceinline__ void planes_add(Planes& p, int card) {
    const uint32_t b = 1u << (card >> 2);
    p.four |= p.three & b;
    p.three |= p.two & b;
    p.two |= p.one & b;
    p.one |= b;
    p.suits |= (uint64_t)b << ((card & 3) * 16);
}

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ int hi_bit(uint32_t m) { return 31 - __clz(m); }
__device__ __forceinline__ int bit_count(uint32_t m) { return __popc(m); }
#else
inline int hi_bit(uint32_t m) { return 31 - __builtin_clz(m); }
inline int bit_count(uint32_t m) { return __builtin_popcount(m); }
#endif

// Highest card of a 5-rank run in m, 3 for the wheel A-2-3-4-5, else -1
// (f_str, mtt_ev_dumper.cu:57-61).
__host__ __device__ __forceinline__ int straight_high(uint32_t m) {
    const uint32_t s = m & (m >> 1) & (m >> 2) & (m >> 3) & (m >> 4);
    if (s) return hi_bit(s) + 4;
    return ((m & 0x100Fu) == 0x100Fu) ? 3 : -1;
}

// Mask of the suit holding >= 5 cards (at most one can with 7 cards), else 0.
__host__ __device__ __forceinline__ uint32_t flush_mask(uint64_t suits) {
    const uint32_t m0 = (uint32_t)(suits) & 0x1FFFu, m1 = (uint32_t)(suits >> 16) & 0x1FFFu;
    const uint32_t m2 = (uint32_t)(suits >> 32) & 0x1FFFu, m3 = (uint32_t)(suits >> 48) & 0x1FFFu;
    uint32_t fm = 0u;
    fm = bit_count(m0) >= 5 ? m0 : fm;
    fm = bit_count(m1) >= 5 ? m1 : fm;
    fm = bit_count(m2) >= 5 ? m2 : fm;
    fm = bit_count(m3) >= 5 ? m3 : fm;
    return fm;
}

// Exact reference score (uint32) of the 7 cards in p.
__host__ __device__ __forceinline__ uint32_t score_planes(const Planes& p) {
    const uint32_t fm = flush_mask(p.suits);
    if (fm) {
        const int sf = straight_high(fm);
        if (sf >= 0) return (8u << 24) | (uint32_t)sf;
        uint32_t m = fm, score = 5u << 24;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int r = hi_bit(m);
            score |= (uint32_t)r << (4 * (4 - k));
            m ^= 1u << r;
        }
        return score;
    }
    if (p.four) return (7u << 24) | ((uint32_t)hi_bit(p.four) << 4);
    const uint32_t trips = p.three & ~p.four, pairs = p.two & ~p.three;
    const int t1 = trips ? hi_bit(trips) : -1;
    const uint32_t trips2 = trips & ~(t1 >= 0 ? (1u << t1) : 0u);
    const int t2 = trips2 ? hi_bit(trips2) : -1;
    const int p1 = pairs ? hi_bit(pairs) : -1;
    const uint32_t pairs2 = pairs & ~(p1 >= 0 ? (1u << p1) : 0u);
    const int p2 = pairs2 ? hi_bit(pairs2) : -1;
    if (t1 >= 0 && (t2 >= 0 || p1 >= 0))
        return (6u << 24) | ((uint32_t)t1 << 4) | (uint32_t)(t2 >= 0 ? t2 : p1);
    const int st = straight_high(p.one);
    if (st >= 0) return (4u << 24) | (uint32_t)st;
    if (t1 >= 0) return (3u << 24) | ((uint32_t)t1 << 8);
    if (p1 >= 0 && p2 >= 0) return (2u << 24) | ((uint32_t)p1 << 8) | ((uint32_t)p2 << 4);
    if (p1 >= 0) return (1u << 24) | ((uint32_t)p1 << 12);
    return p.one;
}

// Monotone 16-bit key of the same score: key(a) < key(b) <=> score(a) <
// score(b) and equal keys <=> equal scores.  Each category's payload is
// re-based into one contiguous range (high card and flush use their 13-bit
// rank masks, which order like the reference's nibble lists); 16,973 keys
// in all, never 0 and never 0xFFFF, which the scans use as sentinels.
constexpr uint32_t KEY_PAIR = 8192, KEY_TWO_PAIR = 8208, KEY_TRIPS = 8464,
                   KEY_STRAIGHT = 8480, KEY_FLUSH = 8496, KEY_FULL = 16688,
                   KEY_QUADS = 16944, KEY_SFLUSH = 16960;

__host__ __device__ __forceinline__ uint32_t key_planes(const Planes& p) {
    const uint32_t fm = flush_mask(p.suits);
    if (fm) {
        const int sf = straight_high(fm);
        if (sf >= 0) return KEY_SFLUSH + (uint32_t)sf;
        uint32_t m = fm;
        while (bit_count(m) > 5) m &= m - 1u;   // drop the lowest ranks
        return KEY_FLUSH + m;
    }
    if (p.four) return KEY_QUADS + (uint32_t)hi_bit(p.four);
    const uint32_t trips = p.three & ~p.four, pairs = p.two & ~p.three;
    const int t1 = trips ? hi_bit(trips) : -1;
    const uint32_t trips2 = trips & ~(t1 >= 0 ? (1u << t1) : 0u);
    const int t2 = trips2 ? hi_bit(trips2) : -1;
    const int p1 = pairs ? hi_bit(pairs) : -1;
    const uint32_t pairs2 = pairs & ~(p1 >= 0 ? (1u << p1) : 0u);
    const int p2 = pairs2 ? hi_bit(pairs2) : -1;
    if (t1 >= 0 && (t2 >= 0 || p1 >= 0))
        return KEY_FULL + (((uint32_t)t1 << 4) | (uint32_t)(t2 >= 0 ? t2 : p1));
    const int st = straight_high(p.one);
    if (st >= 0) return KEY_STRAIGHT + (uint32_t)st;
    if (t1 >= 0) return KEY_TRIPS + (uint32_t)t1;
    if (p1 >= 0 && p2 >= 0) return KEY_TWO_PAIR + (((uint32_t)p1 << 4) | (uint32_t)p2);
    if (p1 >= 0) return KEY_PAIR + (uint32_t)p1;
    return p.one;
}

__host__ __device__ __forceinline__ uint32_t score7(const uint8_t* c) {
    Planes p; planes_clear(p);
#pragma unroll
    for (int i = 0; i < 7; ++i) planes_add(p, c[i]);
    return score_planes(p);
}

// combo id (0..1325) <-> cards, lexicographic over c1 < c2.
__host__ __device__ __forceinline__ int combo_id(int c1, int c2) {
    // pairs before (c1, c1+1): sum_{k<c1} (51-k) = c1*51 - c1*(c1-1)/2
    return c1 * 51 - (c1 * (c1 - 1)) / 2 + (c2 - c1 - 1);
}

}  // namespace mtt
