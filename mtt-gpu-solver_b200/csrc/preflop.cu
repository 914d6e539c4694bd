// preflop.cu — the preflop anchor chain (src/preflop/preflop_grid_generator.cu):
// the 169 x 169 all-in equity matrix, class-reduced flop equity matrices of
// a flop subset, and DCFR over the closed BTN-vs-BB preflop tree whose flop
// play is co-solved over those matrices.
//
// Two modes.  MTT_PF_REFERENCE reproduces the reference bit for bit where
// its arithmetic is integer (win/tie counts) or order-fixed float (the
// equities and their class averages): the all-in matrix's board samples are
// drawn with replacement from the reference's LCG and its class_to_cards
// mapping (:79-92) is used as written; the flop matrices cover only the
// first 1,176 combos in lexicographic order (:476-491), count a tie as a
// quarter win (wins += 2, ties += 1, total += 2 per runout, :169-171), and
// entries the reference never writes (hero combos touching the flop) are 0.
// MTT_PF_CORRECT draws boards without replacement from a valid card pair per
// class, uses every combo that avoids the flop and counts a tie as half.
//
// Flop matrices: per flop, every combo's 16-bit score key for every
// (turn, river) pair of the 49-card deck is evaluated once into a
// pair-major table; a CTA per hero combo then walks the hero's runout list
// (the reference's subsample: turn index r1 = 0, 2, .. and river r2 = r1+1,
// r1+4, .. into the hero's 47-card deck) comparing keys against every
// villain, with coalesced loads of the table.  The combo matrix is reduced
// to classes in the reference's summation order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mtt_common.h"
#include "mtt_device.cuh"

namespace mtt {
namespace pf {

constexpr int NC = 169, PAD = 192, ALIVE = 1176, NPAIR = 1176;   // NPAIR = C(49, 2) turn-river pairs
constexpr int LD_REF = 1216, LD_OK = 1344;   // row length of the combo matrices (reference: 1,216)
constexpr int SAMPLES = 3000;

// class_to_cards of the reference (:79-92), boundary behaviour included: the
// last class of each rank group maps into the next group (A2s becomes two
// copies of the king of clubs).  For classes 90 and 168 the reference's loop
// only ends in signed overflow (undefined); those take their own cards.
__host__ __device__ inline void class_cards_ref(int cls, int& h1, int& h2) {
    if (cls < 13) { const int r = 12 - cls; h1 = r * 4; h2 = r * 4 + 1; return; }
    int base = cls < 91 ? 13 : 91, r1 = 12;
    while (r1 > 0 && base + (r1 - 1) <= cls) base += r1--;
    if (r1 == 0) { h1 = 4; h2 = cls < 91 ? 0 : 1; return; }
    const int r2 = r1 - 1 - (cls - base);
    h1 = r1 * 4;
    h2 = r2 * 4 + (cls < 91 ? 0 : 1);
}

// A valid pair of cards of class cls: pairs c/d, suited c/c, offsuit c/d.
__host__ __device__ inline void class_cards_ok(int cls, int& h1, int& h2) {
    if (cls < 13) { const int r = 12 - cls; h1 = r * 4; h2 = r * 4 + 1; return; }
    const bool suited = cls < 91;
    int k = cls - (suited ? 13 : 91), hi = 12;
    while (k >= hi) { k -= hi; --hi; }
    const int lo = hi - 1 - k;
    h1 = hi * 4;
    h2 = lo * 4 + (suited ? 0 : 1);
}

// First combo of class cls (fixed suit order) that avoids the cards in dead.
__host__ __device__ inline void class_cards_avoid(int cls, uint64_t dead, int& c1, int& c2) {
    int hi, lo;
    bool pair = cls < 13, suited = false;
    if (pair) { hi = lo = 12 - cls; }
    else {
        suited = cls < 91;
        int k = cls - (suited ? 13 : 91);
        hi = 12;
        while (k >= hi) { k -= hi; --hi; }
        lo = hi - 1 - k;
    }
    for (int s1 = 0; s1 < 4; ++s1)
        for (int s2 = 0; s2 < 4; ++s2) {
            if (pair ? s2 <= s1 : (suited ? s2 != s1 : s2 == s1)) continue;
            const int a = hi * 4 + s1, b = lo * 4 + s2;
            if (((dead >> a) & 1ull) || ((dead >> b) & 1ull)) continue;
            c1 = a; c2 = b;
            return;
        }
    c1 = hi * 4; c2 = lo * 4 + 1;   // not reached: two dead cards leave a combo of every class
}

// combo -> class (host set-up, :475-483).
__host__ __device__ inline int combo_class(int c1, int c2) {
    const int r1 = c1 / 4, s1 = c1 % 4, r2 = c2 / 4, s2 = c2 % 4;
    const int hi = r1 > r2 ? r1 : r2, lo = r1 < r2 ? r1 : r2;
    if (r1 == r2) return 12 - hi;
    int base = s1 == s2 ? 13 : 91;
    for (int r = 12; r > hi; --r) base += r;
    return base + (hi - 1 - lo);
}

// Reference score of 7 cards that may repeat: rank counts are exact (a rank
// seen 5+ times is neither quads, trips nor a pair, as with the reference's
// rc[r] == 4 / 3 / 2 tests) and a suit flushes on its card count (sc[s] >= 5)
// with the ranks it holds (sm[s]), as the reference does.
__device__ inline uint32_t score_dup(const int* c) {
    uint32_t one = 0, two = 0, three = 0, four = 0, five = 0;
    uint32_t sm[4] = {0, 0, 0, 0};
    int sc[4] = {0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const uint32_t b = 1u << (c[i] >> 2);
        five |= four & b; four |= three & b; three |= two & b; two |= one & b; one |= b;
        sm[c[i] & 3] |= b;
        sc[c[i] & 3] += 1;
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        if (sc[s] >= 5) {
            const int sf = straight_high(sm[s]);
            if (sf >= 0) return (8u << 24) | (uint32_t)sf;
            uint32_t m = sm[s], score = 5u << 24;
            for (int p = 0; p < 5 && m; ++p) {
                const int r = hi_bit(m);
                score |= (uint32_t)r << (4 * (4 - p));
                m ^= 1u << r;
            }
            return score;
        }
    }
    const uint32_t quads = four & ~five, trips = three & ~four, pairs = two & ~three;
    if (quads) return (7u << 24) | ((uint32_t)hi_bit(quads) << 4);
    const int t1 = trips ? hi_bit(trips) : -1;
    const uint32_t trips2 = trips & ~(t1 >= 0 ? (1u << t1) : 0u);
    const int t2 = trips2 ? hi_bit(trips2) : -1;
    const int p1 = pairs ? hi_bit(pairs) : -1;
    const uint32_t pairs2 = pairs & ~(p1 >= 0 ? (1u << p1) : 0u);
    const int p2 = pairs2 ? hi_bit(pairs2) : -1;
    if (t1 >= 0 && (t2 >= 0 || p1 >= 0)) return (6u << 24) | ((uint32_t)t1 << 4) | (uint32_t)(t2 >= 0 ? t2 : p1);
    const int st = straight_high(one);
    if (st >= 0) return (4u << 24) | (uint32_t)st;
    if (t1 >= 0) return (3u << 24) | ((uint32_t)t1 << 8);
    if (p1 >= 0 && p2 >= 0) return (2u << 24) | ((uint32_t)p1 << 8) | ((uint32_t)p2 << 4);
    if (p1 >= 0) return (1u << 24) | ((uint32_t)p1 << 12);
    return one;
}

// kernel_gen_preflop_matrix (:95-127): thread per (hero, villain) class pair.
__global__ void __launch_bounds__(128) k_pf_allin(int mode, float* __restrict__ out, int* __restrict__ wins_out,
                                                  int* __restrict__ ties_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NC * NC) return;
    const int hc = i / NC, vc = i % NC;
    if (hc == vc) {
        out[i] = 0.5f;
        if (wins_out) { wins_out[i] = 0; ties_out[i] = 0; }
        return;
    }
    int h1, h2, v1, v2;
    if (mode == MTT_PF_REFERENCE) {
        class_cards_ref(hc, h1, h2);
        class_cards_ref(vc, v1, v2);
        if (h1 == v1 || h1 == v2 || h2 == v1 || h2 == v2) {   // the reference's suit switch (:104-107)
            if (h1 == v1 || h2 == v1) v1 = (v1 / 4) * 4 + 2;
            if (h1 == v2 || h2 == v2) v2 = (v2 / 4) * 4 + 3;
        }
    } else {
        class_cards_ok(hc, h1, h2);
        class_cards_avoid(vc, (1ull << h1) | (1ull << h2), v1, v2);
    }
    const uint64_t dead = (1ull << h1) | (1ull << h2) | (1ull << v1) | (1ull << v2);
    uint8_t deck[52];
    int dsz = 0;
    for (int c = 0; c < 52; ++c) if (!((dead >> c) & 1ull)) deck[dsz++] = (uint8_t)c;
    uint32_t rng = (uint32_t)(hc * 169 + vc) * 2654435761u + 0x9E3779B9u;
    int wins = 0, ties = 0;
    int a[7] = {h1, h2, 0, 0, 0, 0, 0}, b[7] = {v1, v2, 0, 0, 0, 0, 0};
    for (int s = 0; s < SAMPLES; ++s) {
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            rng = rng * 1664525u + 1013904223u;
            const int pick = k + (int)((rng >> 16) % (uint32_t)(dsz - k));
            int card = deck[pick];
            if (mode != MTT_PF_REFERENCE) {   // without replacement: partial Fisher-Yates
                deck[pick] = deck[k];
                deck[k] = (uint8_t)card;
            }
            a[2 + k] = card;
            b[2 + k] = card;
        }
        const uint32_t sh = score_dup(a), sv = score_dup(b);
        wins += sh > sv;
        ties += sh == sv;
    }
    out[i] = ((float)wins + 0.5f * (float)ties) / (float)SAMPLES;
    if (wins_out) { wins_out[i] = wins; ties_out[i] = ties; }
}

// Key table of one flop: KT[pair][combo] = 16-bit score key of combo with
// the flop and the (turn, river) pair (0xFFFF where cards collide).
__global__ void __launch_bounds__(256) k_pf_keys(const uint8_t* __restrict__ flops, const uint16_t* __restrict__ cc,
                                                 int ncombo, int ld, uint16_t* __restrict__ KT) {
    const int f = blockIdx.y;
    const int p = blockIdx.x;            // pair index over the 49-card deck
    const uint8_t f0 = flops[3 * f], f1 = flops[3 * f + 1], f2 = flops[3 * f + 2];
    const uint64_t fm = (1ull << f0) | (1ull << f1) | (1ull << f2);
    // unrank p -> (a < b) over the 49-card deck
    int a = 0, k = p, row = 48;
    while (k >= row) { k -= row; ++a; --row; }
    const int b = a + 1 + k;
    int n = 0, ta = -1, tb = -1;
    for (int c = 0; c < 52; ++c) {
        if ((fm >> c) & 1ull) continue;
        if (n == a) ta = c;
        if (n == b) tb = c;
        ++n;
    }
    uint16_t* out = KT + ((size_t)f * NPAIR + p) * ld;
    for (int j = threadIdx.x; j < ld; j += blockDim.x) {
        uint16_t key = 0xFFFFu;
        if (j < ncombo) {
            const int c1 = cc[2 * j], c2 = cc[2 * j + 1];
            const uint64_t m = (1ull << c1) | (1ull << c2);
            if (!(m & fm) && c1 != ta && c1 != tb && c2 != ta && c2 != tb) {
                Planes pl; planes_clear(pl);
                planes_add(pl, f0); planes_add(pl, f1); planes_add(pl, f2);
                planes_add(pl, c1); planes_add(pl, c2); planes_add(pl, ta); planes_add(pl, tb);
                key = (uint16_t)key_planes(pl);
            }
        }
        out[j] = key;
    }
}

// kernel_gen_100_flop_matrices (:130-183) from the key table: CTA per hero
// combo; E[f][j][h] = (wins + ties / 2) / total with the mode's tie weight.
__global__ void __launch_bounds__(256) k_pf_flop_eq(const uint8_t* __restrict__ flops, const uint16_t* __restrict__ cc,
                                                    const int* __restrict__ cidx, int ncombo, int ld, int mode,
                                                    const uint16_t* __restrict__ KT, float* __restrict__ E) {
    __shared__ uint16_t rp[256];     // pair index of each hero runout
    __shared__ uint16_t rk[256];     // hero key there
    __shared__ uint64_t rm[256];     // card mask of the runout
    __shared__ int nr;
    const int f = blockIdx.y, h = blockIdx.x;
    if (h >= ncombo) return;
    const uint8_t f0 = flops[3 * f], f1 = flops[3 * f + 1], f2 = flops[3 * f + 2];
    const uint64_t fm = (1ull << f0) | (1ull << f1) | (1ull << f2);
    const int hc1 = cc[2 * h], hc2 = cc[2 * h + 1];
    const uint64_t hm = (1ull << hc1) | (1ull << hc2);
    const int hcol = cidx[h];      // column of this hero in the padded matrix
    float* Ef = E + (size_t)f * ld * ld;
    if (hm & fm) {
        // the reference never writes these entries; here they are 0
        for (int j = threadIdx.x; j < ncombo; j += blockDim.x) Ef[(size_t)cidx[j] * ld + hcol] = 0.0f;
        return;
    }
    if (threadIdx.x == 0) {
        // the hero's 47-card deck and its runout subsample
        uint8_t deck[52];
        int dsz = 0;
        for (int c = 0; c < 52; ++c) if (!(((hm | fm) >> c) & 1ull)) deck[dsz++] = (uint8_t)c;
        // position of a card in the 49-card flop deck
        auto fpos = [&](int c) { int n = 0; for (int x = 0; x < c; ++x) n += !((fm >> x) & 1ull); return n; };
        int n = 0;
        for (int r1 = 0; r1 < dsz; r1 += 2)
            for (int r2 = r1 + 1; r2 < dsz; r2 += 3) {
                const int t = deck[r1], r = deck[r2];
                const int a = fpos(t), b = fpos(r);     // a < b since the deck is ascending
                const int p = a * 48 - (a * (a - 1)) / 2 + (b - a - 1);
                rp[n] = (uint16_t)p;
                rm[n] = (1ull << t) | (1ull << r);
                ++n;
            }
        nr = n;
    }
    __syncthreads();
    const int n = nr;
    const uint16_t* KTf = KT + (size_t)f * NPAIR * ld;
    for (int k = threadIdx.x; k < n; k += blockDim.x) rk[k] = KTf[(size_t)rp[k] * ld + h];
    __syncthreads();
    for (int j = threadIdx.x; j < ncombo; j += blockDim.x) {
        const int v1 = cc[2 * j], v2 = cc[2 * j + 1];
        const uint64_t vm = (1ull << v1) | (1ull << v2);
        float eq = 0.0f;
        if (!(vm & hm) && !(vm & fm)) {
            int wins = 0, ties = 0, total = 0;
            for (int k = 0; k < n; ++k) {
                if (rm[k] & vm) continue;
                const uint16_t hk = rk[k], vk = KTf[(size_t)rp[k] * ld + j];
                if (mode == MTT_PF_REFERENCE) {
                    wins += hk > vk ? 2 : 0;
                    ties += hk == vk ? 1 : 0;
                    total += 2;
                } else {
                    wins += hk > vk ? 2 : 0;
                    ties += hk == vk ? 2 : 0;
                    total += 2;
                }
            }
            eq = total > 0 ? ((float)wins + 0.5f * (float)ties) / (float)total : 0.0f;
        }
        Ef[(size_t)cidx[j] * ld + hcol] = eq;
    }
}

// kernel_reduce_combo_to_class_matrices (:189-223): out[f][v][h].
__global__ void k_pf_reduce(const float* __restrict__ E, int ld, const int* __restrict__ lists,
                            const int* __restrict__ counts, float* __restrict__ out) {
    const int f = blockIdx.y, hcl = blockIdx.x, vcl = threadIdx.x;
    if (hcl >= NC || vcl >= NC) return;
    const float* Ef = E + (size_t)f * ld * ld;
    float sum = 0.0f;
    int valid = 0;
    for (int i = 0; i < counts[hcl]; ++i) {
        const int ch = lists[hcl * 12 + i];
        for (int j = 0; j < counts[vcl]; ++j) {
            const float eq = Ef[(size_t)lists[vcl * 12 + j] * ld + ch];
            if (eq > 0.0f) { sum = __fadd_rn(sum, eq); valid++; }
        }
    }
    out[((size_t)f * NC + vcl) * NC + hcl] = valid > 0 ? __fdiv_rn(sum, (float)valid) : 0.5f;
}

// Host lists: combos of the matrix (reference: the first 1,176 in
// lexicographic order; correct: all 1,326, those touching a flop are zeroed
// per flop by the kernels) and up to `cap` combos per class.
struct Lists {
    std::vector<uint16_t> cc;     // 2 per combo
    std::vector<int> cidx;        // padded-matrix column of each combo
    std::vector<int> lists, counts;
    int ncombo = 0;
};

static Lists make_lists(int mode) {
    Lists L;
    const int limit = mode == MTT_PF_REFERENCE ? ALIVE : 1326;
    const int cap = 12;                  // the largest class (offsuit) has 12 combos
    L.lists.assign(NC * 12, 0);
    L.counts.assign(NC, 0);
    for (int c1 = 0; c1 < 52; ++c1)
        for (int c2 = c1 + 1; c2 < 52; ++c2) {
            if (L.ncombo >= limit) continue;
            const int cls = combo_class(c1, c2);
            L.cc.push_back((uint16_t)c1);
            L.cc.push_back((uint16_t)c2);
            L.cidx.push_back(L.ncombo);
            if (L.counts[cls] < cap) L.lists[cls * 12 + L.counts[cls]++] = L.ncombo;
            ++L.ncombo;
        }
    return L;
}

}  // namespace pf
}  // namespace mtt

using namespace mtt;
using namespace mtt::pf;

extern "C" int mtt_pf_allin_matrix(int32_t mode, float* d_out, int32_t* d_wins, int32_t* d_ties, void* stream) {
    if (!d_out || (mode != MTT_PF_REFERENCE && mode != MTT_PF_CORRECT) || (!d_wins != !d_ties)) return MTT_ERR_INVALID;
    k_pf_allin<<<(NC * NC + 127) / 128, 128, 0, as_stream(stream)>>>(mode, d_out, d_wins, d_ties);
    MTT_CHECK_LAUNCH();
    return MTT_OK;
}

extern "C" int mtt_pf_flop_class_matrices(int32_t mode, const uint8_t* d_flops, int32_t n, float* d_out, void* stream) {
    if (!d_flops || !d_out || n < 0 || (mode != MTT_PF_REFERENCE && mode != MTT_PF_CORRECT)) return MTT_ERR_INVALID;
    if (n == 0) return MTT_OK;
    cudaStream_t st = as_stream(stream);
    const Lists L = make_lists(mode);
    const int ld = mode == MTT_PF_REFERENCE ? LD_REF : LD_OK;
    constexpr int CHUNK = 8;   // flops per pass: 8 x (up to 3.2 MB of keys + 7.2 MB of matrix)
    uint16_t* d_cc = nullptr;
    int *d_cidx = nullptr, *d_lists = nullptr, *d_counts = nullptr;
    uint16_t* d_KT = nullptr;
    float* d_E = nullptr;
    int s = MTT_OK;
    if (!s) s = cuda_status(cudaMallocAsync(&d_cc, sizeof(uint16_t) * L.cc.size(), st));
    if (!s) s = cuda_status(cudaMallocAsync(&d_cidx, sizeof(int) * L.cidx.size(), st));
    if (!s) s = cuda_status(cudaMallocAsync(&d_lists, sizeof(int) * L.lists.size(), st));
    if (!s) s = cuda_status(cudaMallocAsync(&d_counts, sizeof(int) * L.counts.size(), st));
    if (!s) s = cuda_status(cudaMallocAsync(&d_KT, sizeof(uint16_t) * (size_t)CHUNK * NPAIR * ld, st));
    if (!s) s = cuda_status(cudaMallocAsync(&d_E, sizeof(float) * (size_t)CHUNK * ld * ld, st));
    if (!s) s = cuda_status(cudaMemcpyAsync(d_cc, L.cc.data(), sizeof(uint16_t) * L.cc.size(), cudaMemcpyHostToDevice, st));
    if (!s) s = cuda_status(cudaMemcpyAsync(d_cidx, L.cidx.data(), sizeof(int) * L.cidx.size(), cudaMemcpyHostToDevice, st));
    if (!s) s = cuda_status(cudaMemcpyAsync(d_lists, L.lists.data(), sizeof(int) * L.lists.size(), cudaMemcpyHostToDevice, st));
    if (!s) s = cuda_status(cudaMemcpyAsync(d_counts, L.counts.data(), sizeof(int) * L.counts.size(), cudaMemcpyHostToDevice, st));
    for (int f0 = 0; f0 < n && !s; f0 += CHUNK) {
        const int nf = std::min(CHUNK, n - f0);
        k_pf_keys<<<dim3(NPAIR, nf), 256, 0, st>>>(d_flops + 3 * f0, d_cc, L.ncombo, ld, d_KT);
        s = cuda_status(cudaGetLastError());
        if (!s) {
            k_pf_flop_eq<<<dim3(L.ncombo, nf), 256, 0, st>>>(d_flops + 3 * f0, d_cc, d_cidx, L.ncombo, ld, mode, d_KT,
                                                              d_E);
            s = cuda_status(cudaGetLastError());
        }
        if (!s) {
            k_pf_reduce<<<dim3(NC, nf), PAD, 0, st>>>(d_E, ld, d_lists, d_counts, d_out + (size_t)f0 * NC * NC);
            s = cuda_status(cudaGetLastError());
        }
    }
    cudaFreeAsync(d_cc, st); cudaFreeAsync(d_cidx, st); cudaFreeAsync(d_lists, st); cudaFreeAsync(d_counts, st);
    cudaFreeAsync(d_KT, st); cudaFreeAsync(d_E, st);
    return s;
}

extern "C" int mtt_pf_combo_class(int32_t c1, int32_t c2) {
    if (c1 < 0 || c2 <= c1 || c2 > 51) return -1;
    return combo_class(c1, c2);
}

// ============================================================ preflop DCFR
namespace mtt {
namespace pf {

// Closed preflop tree state; blocks of [A][PAD] floats in node order BTN root
// (3), BB vs min-raise (3), BTN vs 3-bet jam (2), BB vs open jam (2).
__host__ __device__ constexpr int node_off(int k) { return k == 0 ? 0 : k == 1 ? 3 * PAD : k == 2 ? 6 * PAD : 8 * PAD; }
__host__ __device__ constexpr int node_actions(int k) { return k < 2 ? 3 : 2; }
constexpr int STATE = 10 * PAD;

struct PfDev {
    const float* fw;        // flop weights [nf]
    const float* mats;      // class matrices [nf][v][h]
    const float* allin;     // [h][v]
    const float* tab;       // per iteration: w_pos, w_strat
    int* iter;              // 1-based iteration counter
    float *R, *G, *S, *C;   // regrets, current strategy, strategy sums, action values [STATE]
    float *root, *rbc, *rbb, *evb, *evbb;
    int nf;
    float stack, bf, dead;
};

__global__ void k_pf_init(PfDev d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *d.iter = 1;
    if (i < STATE) {
        d.R[i] = 0.0f;
        d.S[i] = 0.0f;
        d.C[i] = 0.0f;
        d.G[i] = i < 6 * PAD ? 1.0f / 3.0f : 0.5f;
    }
    if (i < PAD) d.root[i] = i < NC ? (i < 13 ? 6.0f : i < 91 ? 4.0f : 12.0f) / 1326.0f : 0.0f;
}

// kernel_update_dynamic_reaches (:412-421)
__global__ void k_pf_reach(PfDev d) {
    const int c = threadIdx.x;
    if (c >= NC) return;
    d.rbc[c] = __fmul_rn(d.root[c], d.G[node_off(0) + 1 * PAD + c]);
    d.rbb[c] = __fmul_rn(d.root[c], d.G[node_off(1) + 1 * PAD + c]);
}

// kernel_cosolve_100_board_matrices (:228-285): CTA per class; threads
// evaluate the flops' net EVs in parallel, thread 0 accumulates them in flop
// order, so the float sums follow the reference's loop exactly.
__global__ void __launch_bounds__(128) k_pf_cosolve(PfDev d) {
    __shared__ float nb_s[128], nbb_s[128];
    __shared__ float acc[3];
    const int cls = blockIdx.x, tid = threadIdx.x;
    const float pot_flop = __fadd_rn(d.dead, 3.1f);
    if (tid == 0) { acc[0] = 0.0f; acc[1] = 0.0f; acc[2] = 0.0f; }
    for (int f0 = 0; f0 < d.nf; f0 += 128) {
        const int f = f0 + tid;
        if (f < d.nf) {
            const float* eq = d.mats + (size_t)f * NC * NC;
            float s1 = 0.0f, e0 = 0.0f, s0 = 0.0f, e1 = 0.0f;
            for (int o = 0; o < NC; ++o) {
                const float r = d.rbb[o];
                s1 = __fadd_rn(s1, r);
                e0 = __fadd_rn(e0, __fmul_rn(r, eq[o * NC + cls]));
            }
            if (s1 > 1e-7f) e0 = __fdiv_rn(e0, s1);
            for (int o = 0; o < NC; ++o) {
                const float r = d.rbc[o];
                s0 = __fadd_rn(s0, r);
                e1 = __fadd_rn(e1, __fmul_rn(r, __fsub_rn(1.0f, eq[cls * NC + o])));
            }
            if (s0 > 1e-7f) e1 = __fdiv_rn(e1, s0);
            const float shb = __fmul_rn(__fmul_rn(e0, 1.06f), pot_flop);
            const float shbb = __fmul_rn(__fmul_rn(e1, 0.94f), pot_flop);
            nb_s[tid] = shb >= 2.1f ? __fsub_rn(shb, 2.1f) : -__fmul_rn(__fsub_rn(2.1f, shb), d.bf);
            nbb_s[tid] = shbb >= 2.1f ? __fsub_rn(shbb, 2.1f) : -__fmul_rn(__fsub_rn(2.1f, shbb), d.bf);
        }
        __syncthreads();
        if (tid == 0) {
            const int n = min(128, d.nf - f0);
            for (int k = 0; k < n; ++k) {
                const float w = d.fw[f0 + k];
                acc[2] = __fadd_rn(acc[2], w);
                acc[0] = __fadd_rn(acc[0], __fmul_rn(w, nb_s[k]));
                acc[1] = __fadd_rn(acc[1], __fmul_rn(w, nbb_s[k]));
            }
        }
        __syncthreads();
    }
    if (tid == 0 && acc[2] > 0.0f) {
        d.evb[cls] = __fdiv_rn(acc[0], acc[2]);
        d.evbb[cls] = __fdiv_rn(acc[1], acc[2]);
    }
}

// kernel_build_closed_preflop_cfvs (:290-385)
__global__ void k_pf_cfvs(PfDev d) {
    const int cls = threadIdx.x;
    if (cls >= NC) return;
    const float *sbr = d.G + node_off(0), *sbd = d.G + node_off(1), *s3b = d.G + node_off(2), *sbj = d.G + node_off(3);
    float *cbr = d.C + node_off(0), *cbd = d.C + node_off(1), *c3b = d.C + node_off(2), *cbj = d.C + node_off(3);
    const float stack = d.stack, bf = d.bf, dead = d.dead;
    const float jam_pot = __fadd_rn(__fmul_rn(2.0f, stack), dead);
    const float jam_net = __fsub_rn(jam_pot, stack);
    // eq * (jam_pot - stack) - (1 - eq) * bf * stack, evaluated left to right
    auto jam_value = [&](float eq) {
        return __fsub_rn(__fmul_rn(eq, jam_net), __fmul_rn(__fmul_rn(__fsub_rn(1.0f, eq), bf), stack));
    };
    const float* root = d.root;
    const float* A = d.allin;
    // BTN vs 3-bet jam
    c3b[cls] = __fmul_rn(-2.1f, bf);
    float m3 = 0.0f, eqc = 0.0f;
    for (int o = 0; o < NC; ++o) {
        const float r = __fmul_rn(root[o], sbd[2 * PAD + o]);
        m3 = __fadd_rn(m3, r);
        eqc = __fadd_rn(eqc, __fmul_rn(r, A[cls * NC + o]));
    }
    if (m3 > 1e-7f) eqc = __fdiv_rn(eqc, m3);
    c3b[PAD + cls] = jam_value(eqc);
    const float v3 = __fadd_rn(__fmul_rn(s3b[cls], c3b[cls]), __fmul_rn(s3b[PAD + cls], c3b[PAD + cls]));
    // BB vs min-raise
    cbd[cls] = __fmul_rn(-1.0f, bf);
    cbd[PAD + cls] = d.evbb[cls];
    float bf3 = 0.0f, bc3 = 0.0f, eqj = 0.0f;
    for (int o = 0; o < NC; ++o) {
        const float ro = __fmul_rn(root[o], sbr[PAD + o]);
        bf3 = __fadd_rn(bf3, __fmul_rn(ro, s3b[o]));
        bc3 = __fadd_rn(bc3, __fmul_rn(ro, s3b[PAD + o]));
        eqj = __fadd_rn(eqj, __fmul_rn(__fmul_rn(ro, s3b[PAD + o]), __fsub_rn(1.0f, A[o * NC + cls])));
    }
    if (bc3 > 1e-7f) eqj = __fdiv_rn(eqj, bc3);
    const float tot3 = __fadd_rn(__fadd_rn(bf3, bc3), 1e-9f);
    const float evsh = jam_value(eqj);
    cbd[2 * PAD + cls] = __fdiv_rn(__fadd_rn(__fmul_rn(bf3, __fadd_rn(dead, 2.1f)), __fmul_rn(bc3, evsh)), tot3);
    // BB vs open jam
    cbj[cls] = __fmul_rn(-1.0f, bf);
    float mj = 0.0f, eqo = 0.0f;
    for (int o = 0; o < NC; ++o) {
        const float r = __fmul_rn(root[o], sbr[2 * PAD + o]);
        mj = __fadd_rn(mj, r);
        eqo = __fadd_rn(eqo, __fmul_rn(r, __fsub_rn(1.0f, A[o * NC + cls])));
    }
    if (mj > 1e-7f) eqo = __fdiv_rn(eqo, mj);
    cbj[PAD + cls] = jam_value(eqo);
    // BTN root
    cbr[cls] = 0.0f;
    float fm = 0.0f, cm = 0.0f, jm = 0.0f;
    for (int o = 0; o < NC; ++o) {
        const float r = root[o];
        fm = __fadd_rn(fm, __fmul_rn(r, sbd[o]));
        cm = __fadd_rn(cm, __fmul_rn(r, sbd[PAD + o]));
        jm = __fadd_rn(jm, __fmul_rn(r, sbd[2 * PAD + o]));
    }
    const float tb = __fadd_rn(__fadd_rn(__fadd_rn(fm, cm), jm), 1e-9f);
    cbr[PAD + cls] = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(fm, dead), __fmul_rn(cm, d.evb[cls])), __fmul_rn(jm, v3)), tb);
    float fj = 0.0f, cj = 0.0f, eo = 0.0f;
    for (int o = 0; o < NC; ++o) {
        const float r = root[o];
        fj = __fadd_rn(fj, __fmul_rn(r, sbj[o]));
        cj = __fadd_rn(cj, __fmul_rn(r, sbj[PAD + o]));
        eo = __fadd_rn(eo, __fmul_rn(__fmul_rn(r, sbj[PAD + o]), A[cls * NC + o]));
    }
    const float toj = __fadd_rn(__fadd_rn(fj, cj), 1e-9f);
    if (cj > 1e-7f) eo = __fdiv_rn(eo, cj);
    const float evj = jam_value(eo);
    cbr[2 * PAD + cls] = __fdiv_rn(__fadd_rn(__fmul_rn(fj, dead), __fmul_rn(cj, evj)), toj);
}

// kernel_dcfr_step (:387-410) for the four nodes, then the next iteration.
__global__ void k_pf_dcfr(PfDev d) {
    const int cls = threadIdx.x, node = blockIdx.x;
    if (cls >= NC) return;
    const int t = *d.iter;
    const float wp = d.tab[2 * (t - 1)], ws = d.tab[2 * (t - 1) + 1];
    const int A = node_actions(node), off = node_off(node);
    float* R = d.R + off;
    float* G = d.G + off;
    float* S = d.S + off;
    const float* C = d.C + off;
    float v = 0.0f;
    for (int a = 0; a < A; ++a) v = __fadd_rn(v, __fmul_rn(G[a * PAD + cls], C[a * PAD + cls]));
    float pos = 0.0f, nxt[3] = {0.0f, 0.0f, 0.0f};
    for (int a = 0; a < A; ++a) {
        const int i = a * PAD + cls;
        const float nr = __fmul_rn(wp, fmaxf(0.0f, __fadd_rn(R[i], __fsub_rn(C[i], v))));
        R[i] = nr;
        pos = __fadd_rn(pos, nr);
        nxt[a] = nr;
        S[i] = __fadd_rn(S[i], __fmul_rn(__fmul_rn(ws, d.root[cls]), G[i]));
    }
    for (int a = 0; a < A; ++a) G[a * PAD + cls] = pos > 1e-7f ? __fdiv_rn(nxt[a], pos) : __fdiv_rn(1.0f, (float)A);
}

__global__ void k_pf_next(PfDev d) {
    if (threadIdx.x == 0) *d.iter += 1;
}

static int pf_iteration(const PfDev& d, cudaStream_t st) {
    k_pf_reach<<<1, PAD, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    k_pf_cosolve<<<NC, 128, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    k_pf_cfvs<<<1, PAD, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    k_pf_dcfr<<<4, PAD, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    k_pf_next<<<1, 32, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    return MTT_OK;
}

}  // namespace pf
}  // namespace mtt

extern "C" int mtt_pf_dcfr(const float* d_flop_weights, const float* d_class_mats, int32_t n_flops,
                           const float* d_allin, const mtt_pf_params* p, float* d_sums, float* d_sigma, void* stream) {
    if (!d_flop_weights || !d_class_mats || n_flops < 1 || !d_allin || !p || p->iters < 0 || !d_sums)
        return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    const int iters = std::max(p->iters, 1);
    std::vector<float> tab(2 * (size_t)iters);
    for (int t = 1; t <= iters; ++t) {   // host powf, as the reference's loop (:589-591)
        const float tf = (float)t;
        tab[2 * (t - 1)] = powf(tf, 1.5f) / (powf(tf, 1.5f) + 1.0f);
        tab[2 * (t - 1) + 1] = tf * tf;
    }
    float* buf = nullptr;
    int* d_iter = nullptr;
    const size_t nbuf = 2 * (size_t)iters + 4 * (size_t)STATE + 5 * (size_t)PAD;
    MTT_TRY_CUDA(cudaMallocAsync(&buf, sizeof(float) * nbuf, st));
    int s = cuda_status(cudaMallocAsync(&d_iter, sizeof(int), st));
    PfDev d{};
    d.fw = d_flop_weights; d.mats = d_class_mats; d.allin = d_allin;
    d.tab = buf;
    d.R = buf + 2 * (size_t)iters; d.G = d.R + STATE; d.S = d.G + STATE; d.C = d.S + STATE;
    d.root = d.C + STATE; d.rbc = d.root + PAD; d.rbb = d.rbc + PAD; d.evb = d.rbb + PAD; d.evbb = d.evb + PAD;
    d.iter = d_iter;
    d.nf = n_flops; d.stack = p->stack_bb; d.bf = p->bubble; d.dead = p->dead_pot;
    if (!s) s = cuda_status(cudaMemcpyAsync(buf, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
    if (!s) s = cuda_status(cudaMemsetAsync(d.evb, 0, sizeof(float) * 2 * PAD, st));
    if (!s) { k_pf_init<<<(STATE + 255) / 256, 256, 0, st>>>(d); s = cuda_status(cudaGetLastError()); }
    // one iteration captured as a graph, replayed p->iters times
    cudaGraphExec_t ge = nullptr;
    if (!s && p->iters > 0) {
        cudaStream_t cs;
        s = cuda_status(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        if (!s) {
            cudaGraph_t g = nullptr;
            s = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            if (!s) s = pf_iteration(d, cs);
            const int s2 = cuda_status(cudaStreamEndCapture(cs, &g));
            if (!s) s = s2;
            if (!s) s = cuda_status(cudaGraphInstantiate(&ge, g, 0));
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cs);
        }
        for (int t = 0; t < p->iters && !s; ++t) s = cuda_status(cudaGraphLaunch(ge, st));
    }
    if (!s) s = cuda_status(cudaMemcpyAsync(d_sums, d.S, sizeof(float) * STATE, cudaMemcpyDeviceToDevice, st));
    if (!s && d_sigma) s = cuda_status(cudaMemcpyAsync(d_sigma, d.G, sizeof(float) * STATE, cudaMemcpyDeviceToDevice, st));
    if (ge) {
        cudaStreamSynchronize(st);
        cudaGraphExecDestroy(ge);
    }
    cudaFreeAsync(buf, st);
    cudaFreeAsync(d_iter, st);
    return s;
}

extern "C" int mtt_pf_read_subset(const char* path, uint8_t* h_flops, float* h_weights, int32_t capacity, int32_t* n) {
    if (!n) return MTT_ERR_INVALID;
    const char* tries[2] = {path ? path : "data/mtt_subset.bin", path ? nullptr : "mtt_subset.bin"};
    FILE* fp = nullptr;
    for (const char* t : tries)
        if (t && (fp = fopen(t, "rb"))) break;
    if (!fp) return MTT_ERR_IO;
    uint32_t count = 0;
    int s = fread(&count, 4, 1, fp) == 1 ? MTT_OK : MTT_ERR_IO;
    if (!s && count > 100000u) s = MTT_ERR_IO;
    if (!s) *n = (int32_t)count;
    for (uint32_t i = 0; i < count && !s && h_flops; ++i) {
        uint8_t rec[8];
        if (fread(rec, 1, 8, fp) != 8) { s = MTT_ERR_IO; break; }
        if ((int32_t)i >= capacity) { s = MTT_ERR_INVALID; break; }
        h_flops[3 * i] = rec[0]; h_flops[3 * i + 1] = rec[1]; h_flops[3 * i + 2] = rec[2];
        if (rec[0] > 51 || rec[1] > 51 || rec[2] > 51) { s = MTT_ERR_IO; break; }
        if (h_weights) std::memcpy(&h_weights[i], rec + 4, 4);
    }
    fclose(fp);
    return s;
}
