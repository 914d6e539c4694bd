// eval.cu — hand evaluation, board showdown counts and the flop-EV dumper chain.
//
//  * mtt_eval7: 7 bytes per hand in, uint32 reference score out.  Tiles of
//    1,024 hands (7,168 B) are staged into shared memory with 1-D TMA bulk
//    copies, double-buffered on two mbarriers, by a persistent grid.
//  * mtt_eval7_enumerate: all C(52,7) hands, category histogram + checksum.
//  * mtt_board_showdown_counts: exact win/tie/loss counts per (hero,
//    villain) pair over every completion of a 3/4/5-card board
//    (kernel_gen_49_turn_matrices, honest_multistreet_solver.cu:56-86, as
//    integer counts).  Each (completion, hand) is evaluated ONCE into a
//    16-bit key; pairs are then counted two completions per 32-bit word with
//    SIMD half-word compares (__vcmpgtu2 / __vcmpeq2) on shared-memory tiles.
//  * mtt_flop_ev / mtt_ev_dump: the reference dumper (mtt_ev_dumper.cu:85-168)
//    with the same subsampled runouts, villain stride, ½ tie weight, FMA
//    accumulation order and host aggregation, reproduced bit-exactly.
#include <cuda.h>   // CUcontext / CUresult types only: the driver entry points are resolved at run time
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "mtt_bulk.cuh"
#include "mtt_common.h"
#include "mtt_device.cuh"

namespace mtt {

// ============================================================ mtt_eval7
constexpr int EV_TILE = 1024;                // hands per tile
constexpr int EV_TILE_BYTES = EV_TILE * 7;   // 7,168 B, a multiple of 16
constexpr int EV_THREADS = 256;

__global__ void __launch_bounds__(EV_THREADS)
k_eval7_bulk(const uint8_t* __restrict__ cards, uint32_t* __restrict__ out, long long n_tiles,
             int* __restrict__ err) {
    __shared__ alignas(128) uint8_t buf[2][EV_TILE_BYTES];
    __shared__ alignas(8) uint64_t bar[2];
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    long long tile = blockIdx.x;
    const long long stride = gridDim.x;
    if (tid == 0 && tile < n_tiles) {
        mbar_arrive_expect_tx(&bar[0], EV_TILE_BYTES);
        bulk_g2s(buf[0], cards + tile * EV_TILE_BYTES, EV_TILE_BYTES, &bar[0]);
    }
    uint32_t parity = 0u;   // bit b = phase of bar[b]
    int s = 0;
    bool ok = true;
    for (; tile < n_tiles; tile += stride, s ^= 1) {
        const long long next = tile + stride;
        if (tid == 0 && next < n_tiles) {   // buffer s^1 was released by the trailing barrier
            mbar_arrive_expect_tx(&bar[s ^ 1], EV_TILE_BYTES);
            bulk_g2s(buf[s ^ 1], cards + next * EV_TILE_BYTES, EV_TILE_BYTES, &bar[s ^ 1]);
        }
        if (!mbar_wait_bounded(&bar[s], (parity >> s) & 1u)) { ok = false; }
        parity ^= 1u << s;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(err, 1);
            // drain the copy that may still be in flight into the other buffer
            if (next < n_tiles) (void)mbar_wait_bounded(&bar[s ^ 1], (parity >> (s ^ 1)) & 1u);
            return;
        }
        const uint8_t* b = buf[s];
        uint32_t* o = out + tile * EV_TILE;
#pragma unroll 4
        for (int h = tid; h < EV_TILE; h += EV_THREADS) {
            Planes p; planes_clear(p);
#pragma unroll
            for (int k = 0; k < 7; ++k) planes_add(p, b[7 * h + k]);
            o[h] = score_planes(p);
        }
        __syncthreads();
    }
}

__global__ void k_eval7_plain(const uint8_t* __restrict__ cards, uint32_t* __restrict__ out,
                              long long begin, long long n) {
    const long long i = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* c = cards + 7 * i;
    Planes p; planes_clear(p);
#pragma unroll
    for (int k = 0; k < 7; ++k) planes_add(p, c[k]);
    out[i] = score_planes(p);
}

static int sm_count(int* out) {
    int dev = 0;
    MTT_TRY_CUDA(cudaGetDevice(&dev));
    MTT_TRY_CUDA(cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev));
    return MTT_OK;
}

// ============================================================ enumeration
constexpr int ENUM_CHUNK = 64;
constexpr long long N_HANDS7 = 133784560LL;

__device__ __forceinline__ unsigned long long binom_dev(int n, int k) {
    if (k < 0 || n < k) return 0ull;
    unsigned long long b = 1ull;
    for (int i = 0; i < k; ++i) b = b * (unsigned long long)(n - i) / (unsigned long long)(i + 1);
    return b;
}

// colex unranking: idx -> c0 < c1 < ... < c6
__device__ __forceinline__ void unrank7(unsigned long long idx, int c[7]) {
    int top = 52;
    for (int i = 7; i >= 1; --i) {
        int cc = top - 1;
        unsigned long long b = binom_dev(cc, i);
        while (b > idx) { b = b * (unsigned long long)(cc - i) / (unsigned long long)cc; --cc; }
        c[i - 1] = cc;
        idx -= b;
        top = cc;
    }
}

__global__ void __launch_bounds__(256)
k_enumerate7(unsigned long long* __restrict__ hist, unsigned long long* __restrict__ checksum,
             uint32_t* __restrict__ key_table, int* __restrict__ err) {
    __shared__ unsigned long long s_hist[9];
    if (threadIdx.x < 9) s_hist[threadIdx.x] = 0ull;
    __syncthreads();
    const long long n_chunks = (N_HANDS7 + ENUM_CHUNK - 1) / ENUM_CHUNK;
    unsigned int cnt[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) cnt[k] = 0u;
    unsigned long long cs = 0ull;
    for (long long ch = (long long)blockIdx.x * blockDim.x + threadIdx.x; ch < n_chunks;
         ch += (long long)gridDim.x * blockDim.x) {
        unsigned long long idx = (unsigned long long)ch * ENUM_CHUNK;
        int c[7];
        unrank7(idx, c);
        int c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3], c4 = c[4], c5 = c[5], c6 = c[6];
        const unsigned long long end = min((unsigned long long)N_HANDS7, idx + ENUM_CHUNK);
        for (; idx < end; ++idx) {
            Planes p; planes_clear(p);
            planes_add(p, c0); planes_add(p, c1); planes_add(p, c2); planes_add(p, c3);
            planes_add(p, c4); planes_add(p, c5); planes_add(p, c6);
            const uint32_t s = score_planes(p);
            const uint32_t cat = s >> 24;
#pragma unroll
            for (int k = 0; k < 9; ++k) cnt[k] += (cat == (uint32_t)k) ? 1u : 0u;
            cs += (unsigned long long)s * (idx + 1ull);
            if (key_table) {
                const uint32_t key = key_planes(p);
                if (key_table[key] != s) {
                    const uint32_t old = atomicCAS(&key_table[key], 0xFFFFFFFFu, s);
                    if (old != 0xFFFFFFFFu && old != s) atomicOr(err, 2);
                }
            }
            // colex successor
            if (c0 + 1 < c1) { ++c0; }
            else if (c1 + 1 < c2) { ++c1; c0 = 0; }
            else if (c2 + 1 < c3) { ++c2; c0 = 0; c1 = 1; }
            else if (c3 + 1 < c4) { ++c3; c0 = 0; c1 = 1; c2 = 2; }
            else if (c4 + 1 < c5) { ++c4; c0 = 0; c1 = 1; c2 = 2; c3 = 3; }
            else if (c5 + 1 < c6) { ++c5; c0 = 0; c1 = 1; c2 = 2; c3 = 3; c4 = 4; }
            else { ++c6; c0 = 0; c1 = 1; c2 = 2; c3 = 3; c4 = 4; c5 = 5; }
        }
    }
    // warp reduce then shared then global
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        unsigned int v = cnt[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_hist[k], (unsigned long long)v);
    }
    for (int o = 16; o > 0; o >>= 1) cs += __shfl_down_sync(0xFFFFFFFFu, cs, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(checksum, cs);
    __syncthreads();
    if (threadIdx.x < 9 && s_hist[threadIdx.x]) atomicAdd(&hist[threadIdx.x], s_hist[threadIdx.x]);
}

// ============================================================ board counts
// keys[w][h] packs the 16-bit keys of completions 2w (low) and 2w+1 (high)
// for hand h; 0 marks a completion that uses one of h's cards (or padding).
__device__ __forceinline__ void pair_unrank(int k, int n, int& a, int& b) {
    // lexicographic (a<b) over n items
    a = 0;
    int row = n - 1;
    while (k >= row) { k -= row; ++a; --row; }
    b = a + 1 + k;
}

__global__ void k_completion_keys(const uint8_t* __restrict__ board, int nboard,
                                  const uint8_t* __restrict__ hands, int H, int Hp, int ncomp,
                                  uint32_t* __restrict__ keys) {
    __shared__ uint8_t rest[52];
    __shared__ int nrest;
    if (threadIdx.x == 0) {
        uint64_t bm = 0;
        for (int k = 0; k < nboard; ++k) bm |= 1ull << board[k];
        int n = 0;
        for (int c = 0; c < 52; ++c) if (!((bm >> c) & 1ull)) rest[n++] = (uint8_t)c;
        nrest = n;
    }
    __syncthreads();
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = blockIdx.y;
    if (h >= Hp) return;
    uint32_t word = 0u;
    if (h < H) {
        const int hc1 = hands[2 * h], hc2 = hands[2 * h + 1];
        uint64_t bm = 0;
        for (int k = 0; k < nboard; ++k) bm |= 1ull << board[k];
        const uint64_t hm = (1ull << hc1) | (1ull << hc2);
        if (!(hm & bm) && hc1 != hc2) {
            Planes base; planes_clear(base);
            for (int k = 0; k < nboard; ++k) planes_add(base, board[k]);
            planes_add(base, hc1); planes_add(base, hc2);
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int k = 2 * w + half;
                if (k >= ncomp) continue;
                Planes p = base;
                uint64_t cm = 0;
                if (nboard == 4) {
                    const int c = rest[k];
                    cm = 1ull << c;
                    planes_add(p, c);
                } else if (nboard == 3) {
                    int a, b;
                    pair_unrank(k, nrest, a, b);
                    cm = (1ull << rest[a]) | (1ull << rest[b]);
                    planes_add(p, rest[a]); planes_add(p, rest[b]);
                }
                if (cm & hm) continue;
                word |= key_planes(p) << (16 * half);
            }
        }
    }
    keys[(size_t)w * Hp + h] = word;
}

constexpr int BC_TILE = 64, BC_WCHUNK = 32;

__global__ void __launch_bounds__(256)
k_board_counts(const uint32_t* __restrict__ keys, int ncw, int H, int Hp,
               const uint8_t* __restrict__ hands, const uint8_t* __restrict__ board, int nboard,
               int n_const, int32_t* __restrict__ W, int32_t* __restrict__ T, int32_t* __restrict__ L) {
    __shared__ alignas(16) uint32_t hk[BC_WCHUNK][BC_TILE];
    __shared__ alignas(16) uint32_t vk[BC_WCHUNK][BC_TILE];
    const int tid = threadIdx.x, ti = tid & 15, tj = tid >> 4;
    const int i0 = blockIdx.x * BC_TILE, j0 = blockIdx.y * BC_TILE;
    uint32_t wc[4][4], tc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) { wc[a][b] = 0u; tc[a][b] = 0u; }
    for (int w0 = 0; w0 < ncw; w0 += BC_WCHUNK) {
        for (int e = tid; e < BC_WCHUNK * BC_TILE; e += 256) {
            const int w = e / BC_TILE, x = e % BC_TILE;
            uint32_t hv = 0u, vv = 0xFFFFFFFFu;
            if (w0 + w < ncw) {
                if (i0 + x < Hp) hv = keys[(size_t)(w0 + w) * Hp + i0 + x];
                if (j0 + x < Hp) { vv = keys[(size_t)(w0 + w) * Hp + j0 + x]; vv |= __vcmpeq2(vv, 0u); }
            }
            hk[w][x] = hv;
            vk[w][x] = vv;
        }
        __syncthreads();
#pragma unroll 4
        for (int w = 0; w < BC_WCHUNK; ++w) {
            const uint4 h4 = *reinterpret_cast<const uint4*>(&hk[w][ti * 4]);
            const uint4 v4 = *reinterpret_cast<const uint4*>(&vk[w][tj * 4]);
            const uint32_t hv[4] = {h4.x, h4.y, h4.z, h4.w};
            const uint32_t vv[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    wc[a][b] += __vcmpgtu2(hv[a], vv[b]) & 0x00010001u;
                    tc[a][b] += __vcmpeq2(hv[a], vv[b]) & 0x00010001u;
                }
        }
        __syncthreads();
    }
    uint64_t bm = 0;
    for (int k = 0; k < nboard; ++k) bm |= 1ull << board[k];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + ti * 4 + a;
        if (i >= H) continue;
        const uint64_t mi = (1ull << hands[2 * i]) | (1ull << hands[2 * i + 1]);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int j = j0 + tj * 4 + b;
            if (j >= H) continue;
            const uint64_t mj = (1ull << hands[2 * j]) | (1ull << hands[2 * j + 1]);
            int32_t wv = 0, tv = 0, lv = 0;
            if (!(mi & mj) && !(mi & bm) && !(mj & bm)) {
                wv = (int32_t)((wc[a][b] & 0xFFFFu) + (wc[a][b] >> 16));
                tv = (int32_t)((tc[a][b] & 0xFFFFu) + (tc[a][b] >> 16));
                lv = n_const - wv - tv;
            }
            const size_t o = (size_t)i * H + j;
            W[o] = wv; T[o] = tv; L[o] = lv;
        }
    }
}

// ============================================================ flop EV chain
// Runout subsample of the reference loop (mtt_ev_dumper.cu:98-103): turn
// index r1 = 0,2,..,46 into the 49-card deck, river index r2 = r1+1, r1+4,
// .. < 47.  192 (r1, r2) pairs, packed two per key word.
constexpr int FE_RUNOUTS = 192, FE_WORDS = 96, FE_ALIVE = 1176, FE_VILL = 294, FE_VMASK = 6;
__constant__ uint8_t c_runout_r1[FE_RUNOUTS];
__constant__ uint8_t c_runout_r2[FE_RUNOUTS];

static void host_runouts(uint8_t* r1s, uint8_t* r2s) {
    int k = 0;
    for (int r1 = 0; r1 < 47; r1 += 2)
        for (int r2 = r1 + 1; r2 < 47; r2 += 3) { r1s[k] = (uint8_t)r1; r2s[k] = (uint8_t)r2; ++k; }
}

__device__ __forceinline__ void flop_deck(const uint8_t* f, uint8_t* deck) {
    const uint64_t fm = (1ull << f[0]) | (1ull << f[1]) | (1ull << f[2]);
    int n = 0;
    for (int c = 0; c < 52; ++c) if (!((fm >> c) & 1ull)) deck[n++] = (uint8_t)c;
}

// keys[f][w][i] (hand-minor) and validity bits vmask[f][i][6] (bit k = runout k usable by hand i)
__global__ void __launch_bounds__(128)
k_flop_keys(const uint8_t* __restrict__ flops, uint32_t* __restrict__ keys, uint32_t* __restrict__ vmask) {
    __shared__ uint8_t deck[52];
    const int f = blockIdx.y;
    const uint8_t* fl = flops + 3 * f;
    if (threadIdx.x == 0) flop_deck(fl, deck);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= FE_ALIVE) return;
    int a, b;
    pair_unrank(i, 49, a, b);
    const int hc1 = deck[a], hc2 = deck[b];
    Planes base; planes_clear(base);
    planes_add(base, fl[0]); planes_add(base, fl[1]); planes_add(base, fl[2]);
    planes_add(base, hc1); planes_add(base, hc2);
    uint32_t* kout = keys + (size_t)f * FE_WORDS * FE_ALIVE + i;
    uint32_t vm[FE_VMASK] = {0u, 0u, 0u, 0u, 0u, 0u};
    for (int w = 0; w < FE_WORDS; ++w) {
        uint32_t word = 0u;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int k = 2 * w + half;
            const int t = deck[c_runout_r1[k]], r = deck[c_runout_r2[k]];
            if (t == hc1 || t == hc2 || r == hc1 || r == hc2) continue;
            Planes p = base;
            planes_add(p, t); planes_add(p, r);
            word |= key_planes(p) << (16 * half);
            vm[k >> 5] |= 1u << (k & 31);
        }
        kout[(size_t)w * FE_ALIVE] = word;
    }
    uint32_t* vo = vmask + ((size_t)f * FE_ALIVE + i) * FE_VMASK;
#pragma unroll
    for (int q = 0; q < FE_VMASK; ++q) vo[q] = vm[q];
}

// eqT[f][m][i]: equity of hero i vs villain j = 4m over the usable runouts
// ((2W+T)/(2N) as in mtt_ev_dumper.cu:105-110), -1 when the pair is skipped.
constexpr int FE_TH = 64, FE_TV = 64, FE_WCH = 32;
__global__ void __launch_bounds__(256)
k_flop_pair_eq(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vmask,
               const uint8_t* __restrict__ flops, float* __restrict__ eqT) {
    __shared__ alignas(16) uint32_t hk[FE_WCH][FE_TH];
    __shared__ alignas(16) uint32_t vk[FE_WCH][FE_TV];
    __shared__ uint8_t deck[52];
    const int f = blockIdx.z;
    const int tid = threadIdx.x, ti = tid & 15, tj = tid >> 4;
    const int i0 = blockIdx.x * FE_TH, m0 = blockIdx.y * FE_TV;
    if (tid == 0) flop_deck(flops + 3 * f, deck);
    const uint32_t* kf = keys + (size_t)f * FE_WORDS * FE_ALIVE;
    uint32_t wc[4][4], tc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) { wc[a][b] = 0u; tc[a][b] = 0u; }
    for (int w0 = 0; w0 < FE_WORDS; w0 += FE_WCH) {
        for (int e = tid; e < FE_WCH * FE_TH; e += 256) {
            const int w = e / FE_TH, x = e % FE_TH;
            const int i = i0 + x, m = m0 + x;
            hk[w][x] = (i < FE_ALIVE) ? kf[(size_t)(w0 + w) * FE_ALIVE + i] : 0u;
            uint32_t vv = 0xFFFFFFFFu;
            if (m < FE_VILL) { vv = kf[(size_t)(w0 + w) * FE_ALIVE + 4 * m]; vv |= __vcmpeq2(vv, 0u); }
            vk[w][x] = vv;
        }
        __syncthreads();
#pragma unroll 4
        for (int w = 0; w < FE_WCH; ++w) {
            const uint4 h4 = *reinterpret_cast<const uint4*>(&hk[w][ti * 4]);
            const uint4 v4 = *reinterpret_cast<const uint4*>(&vk[w][tj * 4]);
            const uint32_t hv[4] = {h4.x, h4.y, h4.z, h4.w};
            const uint32_t vv[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    wc[a][b] += __vcmpgtu2(hv[a], vv[b]) & 0x00010001u;
                    tc[a][b] += __vcmpeq2(hv[a], vv[b]) & 0x00010001u;
                }
        }
        __syncthreads();
    }
    const uint32_t* vmf = vmask + (size_t)f * FE_ALIVE * FE_VMASK;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + ti * 4 + a;
        if (i >= FE_ALIVE) continue;
        int ia, ib;
        pair_unrank(i, 49, ia, ib);
        const uint64_t mi = (1ull << deck[ia]) | (1ull << deck[ib]);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int m = m0 + tj * 4 + b;
            if (m >= FE_VILL) continue;
            const int j = 4 * m;
            int ja, jb;
            pair_unrank(j, 49, ja, jb);
            const uint64_t mj = (1ull << deck[ja]) | (1ull << deck[jb]);
            float eq = -1.0f;
            if (!(mi & mj)) {
                int n = 0;
#pragma unroll
                for (int q = 0; q < FE_VMASK; ++q)
                    n += __popc(vmf[(size_t)i * FE_VMASK + q] & vmf[(size_t)j * FE_VMASK + q]);
                if (n > 0) {
                    const int wins = 2 * (int)((wc[a][b] & 0xFFFFu) + (wc[a][b] >> 16));
                    const int ties = (int)((tc[a][b] & 0xFFFFu) + (tc[a][b] >> 16));
                    eq = __fdiv_rn((float)(wins + ties), (float)(2 * n));
                }
            }
            eqT[((size_t)f * FE_VILL + m) * FE_ALIVE + i] = eq;
        }
    }
}

// Per hero, villains in increasing order, the reference's contracted FMAs.
__global__ void k_flop_accumulate(const float* __restrict__ eqT, const float* __restrict__ reach0,
                                  const float* __restrict__ reach1, int nflops,
                                  float* __restrict__ ev0, float* __restrict__ ev1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (i >= FE_ALIVE || f >= nflops) return;
    const float uni = __fdiv_rn(1.0f, 1176.0f);
    const float* e = eqT + (size_t)f * FE_VILL * FE_ALIVE + i;
    float t0 = 0.0f, t1 = 0.0f;
    for (int m = 0; m < FE_VILL; ++m) {
        const float eq = e[(size_t)m * FE_ALIVE];
        if (eq < 0.0f) continue;
        const float r1 = reach1 ? reach1[4 * m] : uni;
        const float r0 = reach0 ? reach0[4 * m] : uni;
        t0 = __fmaf_rn(r1, __fmaf_rn(eq, 2.0f, -1.0f), t0);
        t1 = __fmaf_rn(r0, __fmaf_rn(__fsub_rn(1.0f, eq), 2.0f, -1.0f), t1);
    }
    ev0[(size_t)f * FE_ALIVE + i] = t0;
    ev1[(size_t)f * FE_ALIVE + i] = t1;
}

// dump[f][scen][player][class]: the host loop of mtt_ev_dumper.cu:160-168,
// one thread per output, its class's combos in increasing combo order.
__global__ void k_dump_aggregate(const uint8_t* __restrict__ flops, const float* __restrict__ ev0,
                                 const float* __restrict__ ev1, int nflops, float* __restrict__ out) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nflops * 4 * 2 * 169) return;
    const int cls = idx % 169, pl = (idx / 169) % 2, scen = (idx / 338) % 4, f = idx / 1352;
    const uint8_t* fl = flops + 3 * f;
    const uint64_t fm = (1ull << fl[0]) | (1ull << fl[1]) | (1ull << fl[2]);
    // class -> ranks (mtt_ev_dumper.cu:26-32 inverted)
    int hi, lo, kind;   // kind 0 pair, 1 suited, 2 offsuit
    if (cls < 13) { hi = lo = 12 - cls; kind = 0; }
    else {
        kind = cls < 91 ? 1 : 2;
        int off = cls - (kind == 1 ? 13 : 91);
        hi = 12;
        while (off >= hi) { off -= hi; --hi; }
        lo = hi - 1 - off;
    }
    const float* ev = (pl == 0 ? ev0 : ev1) + (size_t)f * FE_ALIVE;
    const float mult = __fadd_rn(1.0f, __fmul_rn(0.1f, (float)scen));
    float acc = 0.0f;
    for (int s1 = 0; s1 < 4; ++s1) {
        for (int s2 = 0; s2 < 4; ++s2) {
            int c1, c2;
            if (kind == 0) { if (s2 <= s1) continue; c1 = 4 * lo + s1; c2 = 4 * hi + s2; }
            else if (kind == 1) { if (s2 != s1) continue; c1 = 4 * lo + s1; c2 = 4 * hi + s2; }
            else { if (s2 == s1) continue; c1 = 4 * lo + s1; c2 = 4 * hi + s2; }
            if (((fm >> c1) & 1ull) || ((fm >> c2) & 1ull)) continue;
            // alive index = lexicographic pair index over the 49-card deck
            const int a = c1 - __popcll(fm & ((1ull << c1) - 1ull));
            const int b = c2 - __popcll(fm & ((1ull << c2) - 1ull));
            const int i = a * 49 - (a * (a + 1)) / 2 + (b - a - 1);
            acc = __fadd_rn(acc, __fmul_rn(ev[i], mult));
        }
    }
    out[idx] = acc;
}

static int upload_runouts(cudaStream_t st) {
    uint8_t r1[FE_RUNOUTS], r2[FE_RUNOUTS];
    host_runouts(r1, r2);
    MTT_TRY_CUDA(cudaMemcpyToSymbolAsync(c_runout_r1, r1, sizeof(r1), 0, cudaMemcpyHostToDevice, st));
    MTT_TRY_CUDA(cudaMemcpyToSymbolAsync(c_runout_r2, r2, sizeof(r2), 0, cudaMemcpyHostToDevice, st));
    return MTT_OK;
}

constexpr int FE_BATCH = 256;   // flops per scratch batch (~470 MB of scratch)

static int flop_ev_batched(const uint8_t* d_flops, int nflops, const float* d_reach0,
                           const float* d_reach1, float* d_ev0, float* d_ev1, cudaStream_t st) {
    MTT_TRY(upload_runouts(st));
    const int nb = nflops < FE_BATCH ? nflops : FE_BATCH;
    uint32_t *keys = nullptr, *vm = nullptr;
    float* eqT = nullptr;
    MTT_TRY_CUDA(cudaMallocAsync(&keys, (size_t)nb * FE_WORDS * FE_ALIVE * 4, st));
    int s = cuda_status(cudaMallocAsync(&vm, (size_t)nb * FE_ALIVE * FE_VMASK * 4, st));
    if (s == MTT_OK) s = cuda_status(cudaMallocAsync(&eqT, (size_t)nb * FE_VILL * FE_ALIVE * 4, st));
    for (int f0 = 0; s == MTT_OK && f0 < nflops; f0 += nb) {
        const int n = (nflops - f0) < nb ? (nflops - f0) : nb;
        const uint8_t* fl = d_flops + 3 * (size_t)f0;
        k_flop_keys<<<dim3(ceil_div(FE_ALIVE, 128), n), 128, 0, st>>>(fl, keys, vm);
        k_flop_pair_eq<<<dim3(ceil_div(FE_ALIVE, FE_TH), ceil_div(FE_VILL, FE_TV), n), 256, 0, st>>>(
            keys, vm, fl, eqT);
        k_flop_accumulate<<<dim3(ceil_div(FE_ALIVE, 128), n), 128, 0, st>>>(
            eqT, d_reach0, d_reach1, n, d_ev0 + (size_t)f0 * FE_ALIVE, d_ev1 + (size_t)f0 * FE_ALIVE);
        s = cuda_status(cudaGetLastError());
    }
    if (eqT) cudaFreeAsync(eqT, st);
    if (vm) cudaFreeAsync(vm, st);
    cudaFreeAsync(keys, st);
    return s;
}

}  // namespace mtt

using namespace mtt;

extern "C" int mtt_eval7(const uint8_t* d_cards7, uint32_t* d_out, int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!d_cards7 || !d_out))) return MTT_ERR_INVALID;
    if (n == 0) return MTT_OK;
    cudaStream_t st = as_stream(stream);
    long long n_tiles = 0;
    int* d_err = nullptr;
    if ((reinterpret_cast<uintptr_t>(d_cards7) & 15u) == 0u) n_tiles = n / EV_TILE;
    if (n_tiles > 0) {
        int sms = 0;
        MTT_TRY(sm_count(&sms));
        long long grid = (long long)sms * 4;
        if (grid > n_tiles) grid = n_tiles;
        MTT_TRY_CUDA(cudaMallocAsync(&d_err, sizeof(int), st));
        MTT_TRY_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
        k_eval7_bulk<<<(unsigned)grid, EV_THREADS, 0, st>>>(d_cards7, d_out, n_tiles, d_err);
        MTT_CHECK_LAUNCH();
    }
    const long long begin = n_tiles * EV_TILE;
    if (begin < n) {
        const long long rem = n - begin;
        k_eval7_plain<<<(unsigned)ceil_div_ll(rem, 256), 256, 0, st>>>(d_cards7, d_out, begin, n);
        MTT_CHECK_LAUNCH();
    }
    if (d_err) {
        int h_err = 0;
        MTT_TRY_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        MTT_TRY_CUDA(cudaFreeAsync(d_err, st));
        MTT_TRY_CUDA(cudaStreamSynchronize(st));
        if (h_err) return MTT_ERR_TIMEOUT;
    }
    return MTT_OK;
}

extern "C" int mtt_eval7_enumerate(uint64_t* d_hist9, uint64_t* d_checksum, uint32_t* d_key_table,
                                   int32_t* d_err, void* stream) {
    if (!d_hist9 || !d_checksum || !d_err) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    int sms = 0;
    MTT_TRY(sm_count(&sms));
    MTT_TRY_CUDA(cudaMemsetAsync(d_hist9, 0, 9 * sizeof(uint64_t), st));
    MTT_TRY_CUDA(cudaMemsetAsync(d_checksum, 0, sizeof(uint64_t), st));
    MTT_TRY_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int32_t), st));
    if (d_key_table) MTT_TRY_CUDA(cudaMemsetAsync(d_key_table, 0xFF, 65536 * sizeof(uint32_t), st));
    k_enumerate7<<<sms * 8, 256, 0, st>>>(reinterpret_cast<unsigned long long*>(d_hist9),
                                          reinterpret_cast<unsigned long long*>(d_checksum), d_key_table,
                                          reinterpret_cast<int*>(d_err));
    MTT_CHECK_LAUNCH();
    return MTT_OK;
}

extern "C" int mtt_board_showdown_counts(const uint8_t* d_board, int32_t nboard, const uint8_t* d_hands,
                                         int32_t H, int32_t* d_w, int32_t* d_t, int32_t* d_l,
                                         void* stream) {
    if (nboard < 3 || nboard > 5 || H < 0 || H > 1326) return MTT_ERR_INVALID;
    if (H == 0) return MTT_OK;
    if (!d_board || !d_hands || !d_w || !d_t || !d_l) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    const int nrest = 52 - nboard;
    const int ncomp = nboard == 5 ? 1 : nboard == 4 ? nrest : nrest * (nrest - 1) / 2;
    const int ncw = (ncomp + 1) / 2;
    const int Hp = (H + 63) / 64 * 64;
    // compatible pairs see every completion that avoids their 4 cards
    const int free_cards = nrest - 4;
    const int n_const = nboard == 5 ? 1 : nboard == 4 ? free_cards : free_cards * (free_cards - 1) / 2;
    uint32_t* keys = nullptr;
    MTT_TRY_CUDA(cudaMallocAsync(&keys, (size_t)ncw * Hp * sizeof(uint32_t), st));
    k_completion_keys<<<dim3(Hp / 64, ncw), 64, 0, st>>>(d_board, nboard, d_hands, H, Hp, ncomp, keys);
    int s = cuda_status(cudaGetLastError());
    if (s == MTT_OK) {
        k_board_counts<<<dim3(Hp / BC_TILE, Hp / BC_TILE), 256, 0, st>>>(keys, ncw, H, Hp, d_hands, d_board,
                                                                        nboard, n_const, d_w, d_t, d_l);
        s = cuda_status(cudaGetLastError());
    }
    cudaFreeAsync(keys, st);
    return s;
}

// ------------------------------------------------ counts without allocation
// Key scratch of mtt_board_showdown_counts_noalloc: one per device, in the
// module's static device memory, so a call needs no allocator.  1 MiB.
static __device__ __align__(256) uint32_t g_counts_scratch[MTT_COUNTS_NOALLOC_MAX_WORDS];

namespace mtt {
constexpr int kMaxDevices = 64;
static std::mutex g_counts_scratch_mu;
static uint32_t* g_counts_scratch_ptr[kMaxDevices] = {};
static unsigned long long g_counts_scratch_ctx[kMaxDevices] = {};

// Unique id of the calling thread's current context (0 if none or if the
// driver does not offer the query).  Ids are never reused within a process,
// so a context created after a cudaDeviceReset always has a new one.  The two
// driver functions are resolved at run time, so the library does not link the
// driver and still loads on machines without one.
static unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
    return 0;
}

// Address of this device's scratch in the current context.  It is looked up
// with the device current on the first call in each context (the first call
// on the device, and again after a cudaDeviceReset replaced its context).
static int counts_scratch(uint32_t** out) {
    int dev = 0;
    MTT_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return MTT_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_counts_scratch_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_counts_scratch_ptr[dev] || ctx == 0 || ctx != g_counts_scratch_ctx[dev]) {
        void* p = nullptr;
        MTT_TRY_CUDA(cudaGetSymbolAddress(&p, g_counts_scratch));   // makes the device's context current
        g_counts_scratch_ptr[dev] = static_cast<uint32_t*>(p);
        g_counts_scratch_ctx[dev] = current_context_id();
    }
    *out = g_counts_scratch_ptr[dev];
    return MTT_OK;
}
}  // namespace mtt

extern "C" int mtt_board_showdown_counts_noalloc(const uint8_t* d_board, int32_t nboard, const uint8_t* d_hands,
                                                 int32_t H, int32_t* d_w, int32_t* d_t, int32_t* d_l,
                                                 void* stream) {
    if (nboard < 3 || nboard > 5 || H < 0 || H > 1326) return MTT_ERR_INVALID;
    if (H == 0) return MTT_OK;
    if (!d_board || !d_hands || !d_w || !d_t || !d_l) return MTT_ERR_INVALID;
    const int nrest = 52 - nboard;
    const int ncomp = nboard == 5 ? 1 : nboard == 4 ? nrest : nrest * (nrest - 1) / 2;
    const int ncw = (ncomp + 1) / 2;
    const int Hp = (H + 63) / 64 * 64;
    if ((long long)ncw * Hp > MTT_COUNTS_NOALLOC_MAX_WORDS) return MTT_ERR_UNSUPPORTED;
    const int free_cards = nrest - 4;
    const int n_const = nboard == 5 ? 1 : nboard == 4 ? free_cards : free_cards * (free_cards - 1) / 2;
    uint32_t* keys = nullptr;
    MTT_TRY(counts_scratch(&keys));
    cudaStream_t st = as_stream(stream);
    // Nothing in the scratch has to start at zero: k_completion_keys writes
    // all ncw * Hp words before k_board_counts reads any of them.
    k_completion_keys<<<dim3(Hp / 64, ncw), 64, 0, st>>>(d_board, nboard, d_hands, H, Hp, ncomp, keys);
    MTT_TRY_CUDA(cudaGetLastError());
    k_board_counts<<<dim3(Hp / BC_TILE, Hp / BC_TILE), 256, 0, st>>>(keys, ncw, H, Hp, d_hands, d_board, nboard,
                                                                    n_const, d_w, d_t, d_l);
    MTT_TRY_CUDA(cudaGetLastError());
    return MTT_OK;
}

extern "C" int mtt_canonical_flops(uint8_t* h_out, int32_t capacity, int32_t* n_out) {
    if (!n_out) return MTT_ERR_INVALID;
    // mtt_ev_dumper.cu:34-51: trips, paired, then unpaired families, orbit weights 4/12/24
    std::vector<uint8_t> v;
    v.reserve(1755 * 4);
    auto mc = [](int r, int s) { return (uint8_t)(r * 4 + s); };
    auto push = [&](uint8_t a, uint8_t b, uint8_t c, uint8_t w) { v.push_back(a); v.push_back(b); v.push_back(c); v.push_back(w); };
    for (int r = 12; r >= 0; --r) push(mc(r, 0), mc(r, 1), mc(r, 2), 4);
    for (int rp = 12; rp >= 0; --rp)
        for (int rk = 12; rk >= 0; --rk) {
            if (rp == rk) continue;
            push(mc(rp, 0), mc(rp, 1), mc(rk, 0), 12);
            push(mc(rp, 0), mc(rp, 1), mc(rk, 2), 12);
        }
    for (int r1 = 12; r1 >= 2; --r1)
        for (int r2 = r1 - 1; r2 >= 1; --r2)
            for (int r3 = r2 - 1; r3 >= 0; --r3) {
                push(mc(r1, 0), mc(r2, 0), mc(r3, 0), 4);
                push(mc(r1, 0), mc(r2, 0), mc(r3, 1), 12);
                push(mc(r1, 0), mc(r2, 1), mc(r3, 0), 12);
                push(mc(r1, 1), mc(r2, 0), mc(r3, 0), 12);
                push(mc(r1, 0), mc(r2, 1), mc(r3, 2), 24);
            }
    *n_out = (int32_t)(v.size() / 4);
    if (h_out) {
        if (capacity < *n_out) return MTT_ERR_INVALID;
        std::memcpy(h_out, v.data(), v.size());
    }
    return MTT_OK;
}

extern "C" int mtt_flop_ev(const uint8_t* d_flops, int32_t nflops, const float* d_reach0,
                           const float* d_reach1, float* d_ev0, float* d_ev1, void* stream) {
    if (nflops < 0) return MTT_ERR_INVALID;
    if (nflops == 0) return MTT_OK;
    if (!d_flops || !d_ev0 || !d_ev1) return MTT_ERR_INVALID;
    return flop_ev_batched(d_flops, nflops, d_reach0, d_reach1, d_ev0, d_ev1, as_stream(stream));
}

extern "C" int mtt_ev_dump(const uint8_t* d_flops, int32_t nflops, float* d_out, void* stream) {
    if (nflops < 0) return MTT_ERR_INVALID;
    if (nflops == 0) return MTT_OK;
    if (!d_flops || !d_out) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    float *ev0 = nullptr, *ev1 = nullptr;
    MTT_TRY_CUDA(cudaMallocAsync(&ev0, (size_t)nflops * FE_ALIVE * 4, st));
    int s = cuda_status(cudaMallocAsync(&ev1, (size_t)nflops * FE_ALIVE * 4, st));
    if (s == MTT_OK) s = flop_ev_batched(d_flops, nflops, nullptr, nullptr, ev0, ev1, st);
    if (s == MTT_OK) {
        const int total = nflops * 1352;
        k_dump_aggregate<<<ceil_div(total, 256), 256, 0, st>>>(d_flops, ev0, ev1, nflops, d_out);
        s = cuda_status(cudaGetLastError());
    }
    if (ev1) cudaFreeAsync(ev1, st);
    cudaFreeAsync(ev0, st);
    return s;
}
