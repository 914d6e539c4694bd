// solver.cu — batched heads-up CFR+/DCFR solver and its FP64 best response.
//
// Level-synchronous over the whole batch: every tree level of every subgame
// is one flat list of warp tasks (subgame, node, 32 groups of 4 hands), so a
// launch streams all subgames' nodes of that depth through HBM with float4
// accesses and no intra-kernel barriers.  An iteration is
//   [forward levels 0..D] [terminals] [backward levels D..0]   per pass,
// one pass per player with alternating updates (CFR+ as published) or one
// pass updating both (the reference kernels' simultaneous updates), captured
// once as a CUDA graph and replayed for every iteration; a device counter
// carries the iteration number into the kernels.
//
// Terminals are one warp each.  Fold values need the opponent's total and
// per-card reach mass; showdown values need one exclusive prefix scan of the
// opponent reach in rank order and in per-card rank order, from which wins,
// ties and losses with card removal are O(1) differences.  The scan is split
// over lanes by the opponent's hand count only, so results never depend on
// the launch configuration.
//
// Update rules follow the reference kernels: kernel_forward_sweep
// (honest_multistreet_solver.cu:88-126), kernel_evaluate_terminals
// (:128-196), kernel_backward_sweep (:198-249), kernel_4way_* (multiway_4way_
// engine.cu:41-83,219-257) and the DCFR weights of kernel_dcfr_step
// (preflop_grid_generator.cu:387-410, in the discount-then-add form).
#include <algorithm>
#include <atomic>
#include <functional>
#include <cmath>
#include <cstring>
#include <numeric>
#include <mutex>
#include <thread>
#include <vector>

#include "mtt_bulk.cuh"
#include "mtt_common.h"
#include "mtt_device.cuh"
#include "solver_impl.cuh"

namespace mtt {

int validate_tree(const mtt_node* nodes, int n, const int rows[2]);   // tree.cpp


// ====================================================================== device
__device__ __forceinline__ float4 f4(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
    return make_float4(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z), __fmul_rn(a.w, b.w));
}
// Starts a fetch of the line holding p into L2 (no register is written, so
// every row of a work item can be requested before its first use).
__device__ __forceinline__ void pf_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}

__device__ __forceinline__ float4 max04(float4 a) {
    return make_float4(fmaxf(a.x, 0.f), fmaxf(a.y, 0.f), fmaxf(a.z, 0.f), fmaxf(a.w, 0.f));
}
__device__ __forceinline__ float rm1(float pos, float sum, float invA) { return sum > 1e-7f ? __fdiv_rn(pos, sum) : invA; }
__device__ __forceinline__ float4 rm4(float4 pos, float4 sum, float invA) {
    return make_float4(rm1(pos.x, sum.x, invA), rm1(pos.y, sum.y, invA), rm1(pos.z, sum.z, invA),
                       rm1(pos.w, sum.w, invA));
}
__device__ __forceinline__ float4 fma4(float4 a, float4 b, float4 c) {
    return make_float4(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y), __fmaf_rn(a.z, b.z, c.z),
                       __fmaf_rn(a.w, b.w, c.w));
}
__device__ __forceinline__ float cfrplus1(float r, float inst) { return fmaxf(0.0f, __fadd_rn(r, inst)); }
__device__ __forceinline__ float dcfr1(float r, float inst, float dpos, float dneg) {
    return __fadd_rn(__fmul_rn(r, r > 0.0f ? dpos : dneg), inst);
}

struct Task {        // one warp: groups [g0, g0 + 32) of float4 hand groups at one node
    int node;        // global node index
    int sub;         // subgame
    int g0;
    int pad;
};

struct SolveDev {
    const SubDesc* desc;
    const DNode* nodes;
    const uint8_t* tabs;
    const uint16_t* hcards;
    const float* ranges;
    float* arena;
    float* R;
    float* S;
    double* darena;
    double* results;
    const float* iter_tab;
    int* iter;          // device iteration counter, 1-based
    int* err;           // bit 0: a bounded wait for a bulk copy gave up
    int algo, semantics;
    int span;           // float4 hand groups per sweep work item / 32 (hands per warp / 128)
};

#define HP(p) ((p) ? sd.Hp1 : sd.Hp0)
#define HH(p) ((p) ? sd.H1 : sd.H0)
#define OFF(p) ((p) ? sd.Hp0 : 0)
#define SRC(nd, p) ((p) ? (nd).reach_src1 : (nd).reach_src0)

__device__ __forceinline__ DNode load_node(const DNode* p) {
    DNode d;
    const uint4* s = reinterpret_cast<const uint4*>(p);
    uint4* o = reinterpret_cast<uint4*>(&d);
    o[0] = __ldg(s);
    o[1] = __ldg(s + 1);
    o[2] = __ldg(s + 2);
    return d;
}

__device__ __forceinline__ uint64_t hand_mask(uint16_t hc) {
    return hc == 0xFFFFu ? 0ull : ((1ull << (hc & 0xFF)) | (1ull << (hc >> 8)));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// ------------------------------------------------------------- terminals
struct TermInfo {
    int H[2], Hp[2];
    float pot, c[2];
    int type, wmask;
};

__device__ __forceinline__ TermInfo term_info(const SubDesc& sd, const DNode& nd) {
    TermInfo t;
    t.H[0] = sd.H0; t.H[1] = sd.H1; t.Hp[0] = sd.Hp0; t.Hp[1] = sd.Hp1;
    t.pot = nd.pot; t.c[0] = nd.c0; t.c[1] = nd.c1;
    t.type = nd.type; t.wmask = nd.wmask;
    return t;
}

// Shared scratch of one terminal CTA, in elements of the arithmetic type.
__host__ __device__ constexpr int term_scratch(int max_h) { return 4 * max_h + 96; }
constexpr int TT = 128;   // threads per terminal CTA (fixed: results never depend on it changing)

template <typename TA, int NT = TT>
__device__ __forceinline__ TA cta_sum(TA v, TA* wb, int tid) {
    v = warp_sum(v);
    if ((tid & 31) == 0) wb[tid >> 5] = v;
    __syncthreads();
    TA t = TA(0);
#pragma unroll
    for (int k = 0; k < NT / 32; ++k) t += wb[k];
    __syncthreads();
    return t;
}

// Values of player q at a terminal against opponent reach `ro` (H_o entries),
// written to out[0..Hp_q) (and out2), by one CTA of TT threads.  TI: stored
// reach type, TA: arithmetic type of the scan and differences, TO: stored
// value type.  The FP64 best response calls it with TA = double: win/tie/loss
// masses are differences of prefix sums, and a value that is exactly zero
// (all of the opponent's remaining mass blocked by the hand's cards) must
// come out as zero to the precision the regret-matching threshold (1e-7)
// can see.  The CFR sweeps use the fixed-point form below, which keeps that
// property with 4-byte scan elements.  X: the CTA's shared scratch (term_scratch
// elements), wb: NT/32 elements.  NT: threads of the CTA; the scan's chunks
// depend on it, so each caller fixes it.
template <typename TI, typename TA, typename TO, bool STAGED = false, int NT = TT>
__device__ void cta_terminal(const TermInfo& ti, const TabView& tv, int q, const TI* __restrict__ ro,
                             TO* __restrict__ out, TO* __restrict__ out2, TA* X, TA* wb, int semantics, int tid) {
    const int o = 1 - q;
    const int Ho = ti.H[o], Hq = ti.H[q], Hpq = ti.Hp[q];
    const uint16_t* co = tv.cl[o];
    const uint16_t* seg = tv.seg[o];
    const Entry* ent = tv.ent[q];
    const TA cq = (TA)ti.c[q];
    const TA pot = (TA)ti.pot;
    const TA gain = pot - cq, loss = -cq, tie = TA(0.5) * pot - cq;
    // opponent reach: already in shared memory (STAGED), else staged here with coalesced loads
    TA* Rd = X;
    TA* Xs = STAGED ? X : X + Ho + 8;   // scan region (3*Ho + 1) / fold: per-card order + card sums
    if (!STAGED) {
#pragma unroll 4
        for (int j = tid; j < Ho; j += NT) Rd[j] = (TA)ro[j];
        __syncthreads();
    }
    auto Rs = [&](int j) -> TA { return STAGED ? (TA)ro[j] : Rd[j]; };
    if (ti.type == MTT_NODE_FOLD) {
        const int winner = (ti.wmask == 1) ? 0 : 1;
        const TA payoff = (q == winner) ? gain : loss;
        TA part = TA(0);
        for (int j = tid; j < Ho; j += NT) part += Rs(j);
        const TA tot = cta_sum<TA, NT>(part, wb, tid);
        TA* Cs = Xs + 2 * Ho + 8;
#pragma unroll 4
        for (int e = tid; e < 2 * Ho; e += NT) Xs[e] = Rs(co[e]);
        __syncthreads();
        for (int c = tid; c < 52; c += NT) {
            TA sm = TA(0);
            for (int e = seg[c]; e < seg[c + 1]; ++e) sm += Xs[e];
            Cs[c] = sm;
        }
        __syncthreads();
        for (int h = tid; h < Hpq; h += NT) {
            TA v = TA(0);
            if (h < Hq) {
                const Entry et = ent[h];
                if (et.lt != 0xFFFFu) {
                    const TA ps = et.same >= 0 ? Rs(et.same) : TA(0);
                    const TA M = semantics ? tot : (tot - Cs[et.c1] - Cs[et.c2] + ps);
                    v = payoff * M;
                }
            }
            out[h] = (TO)v;
            if (out2) out2[h] = (TO)v;
        }
        __syncthreads();
        return;
    }
    // showdown: Xs = [reach in rank order | reach in per-card rank order], exclusive scan
    const uint16_t* so = tv.sorted[o];
    const int N = 3 * Ho;
#pragma unroll 4
    for (int k = tid; k < N; k += NT) Xs[k] = Rs(k < Ho ? so[k] : co[k - Ho]);
    __syncthreads();
    const int C = ((N + NT - 1) / NT) | 1;   // odd chunk: conflict-free strides
    const int s0 = min(tid * C, N), s1 = min(s0 + C, N);
    TA loc = TA(0);
    for (int k = s0; k < s1; ++k) loc += Xs[k];
    const int lane = tid & 31, wid = tid >> 5;
    TA inc = loc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const TA t = __shfl_up_sync(0xFFFFFFFFu, inc, off);
        if (lane >= off) inc += t;
    }
    TA run = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
    if (lane == 0) run = TA(0);
    if (lane == 31) wb[wid] = inc;
    __syncthreads();
    TA base = TA(0), total = TA(0);
#pragma unroll
    for (int k = 0; k < NT / 32; ++k) {
        if (k < wid) base += wb[k];
        total += wb[k];
    }
    run += base;
    for (int k = s0; k < s1; ++k) {
        const TA v = Xs[k];
        Xs[k] = run;
        run += v;
    }
    if (tid == 0) Xs[N] = total;
    __syncthreads();
    const TA Tt = Xs[Ho];
    for (int h = tid; h < Hpq; h += NT) {
        TA v = TA(0);
        if (h < Hq) {
            const Entry et = ent[h];
            if (et.lt != 0xFFFFu) {
                const int s1c = Ho + seg[et.c1], s2c = Ho + seg[et.c2];
                const TA b1 = Xs[s1c], b2 = Xs[s2c];
                const TA C1 = Xs[Ho + seg[et.c1 + 1]] - b1, C2 = Xs[Ho + seg[et.c2 + 1]] - b2;
 
                const TA ps = et.same >= 0 ? Rs(et.same) : TA(0);
                const TA W = Xs[et.lt] - (Xs[s1c + et.ltc1] - b1) - (Xs[s2c + et.ltc2] - b2);
                const TA LE = Xs[et.le] - (Xs[s1c + et.lec1] - b1) - (Xs[s2c + et.lec2] - b2);
                const TA Ti = LE - W + ps;
                if (!semantics) {
                    const TA L = Tt - C1 - C2 - LE;
                    v = gain * W + tie * Ti + loss * L;
                } else {
                    const TA Lr = Tt - W - Ti;   // blocked pairs count as P0 losses (honest:182-187)
                    v = (q == 0) ? (gain * W + tie * Ti + loss * Lr) : (gain * Lr + tie * Ti + loss * W);
                }
            }
        }
        out[h] = (TO)v;
        if (out2) out2[h] = (TO)v;
    }
    __syncthreads();
}

// Terminal values in 32-bit fixed point, for the CFR sweeps.  The opponent
// reach at one terminal is scaled by a power of two 2^k chosen from its own
// absolute sum S (S * 2^k < 2^29) and rounded to int32; every win / tie /
// loss mass is then a difference of exact integer prefix sums.  Integer sums
// do not depend on their order, so the scan's chunking cannot change a
// result, and a mass that is exactly zero stays exactly zero (the property
// the FP64 scan above exists for).  Every prefix sum over the three lists is
// at most 3 * (2^29 + H/2) < 2^31 in magnitude; the value combinations below
// are formed in unsigned (modular) arithmetic, exact because their true
// values are below 2^31.  Each reach value is off by at most half a unit,
// i.e. 2^-30 of S, far below FP32 resolution of S.  k is clamped to
// [-126, 126] so 2^k and 2^-k are normal floats; the clamp can only bite
// when S < 2^-97, where the values are below FP32 resolution of anything
// else in the solve.
//
// Per terminal the CTA (1) sums |reach| over the opponent's hands, (2)
// gathers, rounds and scans the opponent reach in scan order, each thread
// holding a chunk of C consecutive positions in registers (C odd, so the
// strided shared-memory accesses are conflict-free), (3) writes the
// exclusive prefix, and (4) forms each hand's value from two integer masses:
//   A = W + LE + same = 2 W + T   (twice the pot-share mass)
//   B = Tt - C1 - C2 + same       (opponent mass not blocked by the hand)
//   value = pot/2 * A - c * B     (= gain W + tie T + loss L)
// Folds scan only the per-card lists (each opponent hand sits in two of
// them, so their total is twice the opponent's mass) and use B.
struct FxScale { float f, inv; };

__device__ __forceinline__ FxScale fx_scale(float S) {
    // S < 2^e with e from S's exponent field (denormal or zero S: e = -126)
    const int E = (int)((__float_as_uint(S) >> 23) & 0xFFu);
    const int e = E == 0 ? -126 : E - 126;
    const int k = S > 0.f ? min(max(29 - e, -126), 126) : 0;
    FxScale s;
    s.f = __uint_as_float((uint32_t)(127 + k) << 23);
    s.inv = __uint_as_float((uint32_t)(127 - k) << 23);
    return s;
}

__device__ __forceinline__ int fx_round(float v, const FxScale& s) {
    return __float2int_rn(__fmul_rn(v, s.f));   // a power-of-two product is exact
}

// Steps (2)-(3) for chunks of C positions.  idx: the opponent's hand index of
// each scan position; X: N + 1 ints.  Returns the total.
template <int NT, int C>
__device__ __forceinline__ int fx_scan(const uint16_t* __restrict__ idx, const float* __restrict__ ro, int N,
                                       const FxScale& fs, int* X, int* wi, int tid) {
    const int lane = tid & 31, wid = tid >> 5;
    const int s0 = min(tid * C, N);
    int xv[C];
    int loc = 0;
    if (s0 + C <= N) {
#pragma unroll
        for (int j = 0; j < C; ++j) {
            xv[j] = fx_round(ro[idx[s0 + j]], fs);
            loc += xv[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < C; ++j) {
            xv[j] = s0 + j < N ? fx_round(ro[idx[s0 + j]], fs) : 0;
            loc += xv[j];
        }
    }
    int inc = loc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xFFFFFFFFu, inc, off);
        if (lane >= off) inc += t;
    }
    int run = inc - loc;
    if (lane == 31) wi[wid] = inc;
    __syncthreads();
    int total = 0;
#pragma unroll
    for (int k = 0; k < NT / 32; ++k) {
        const int w = wi[k];
        if (k < wid) run += w;
        total += w;
    }
    if (s0 + C <= N) {
#pragma unroll
        for (int j = 0; j < C; ++j) {
            X[s0 + j] = run;
            run += xv[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < C; ++j) {
            if (s0 + j < N) X[s0 + j] = run;
            run += xv[j];
        }
    }
    if (tid == 0) X[N] = total;
    __syncthreads();
    return total;
}

// This thread's share of the opponent's absolute mass sum |ro[j]|, j < Ho,
// reduced over its warp (valid in lane 0).  ro: 16-byte aligned.
template <int NT>
__device__ __forceinline__ float fx_abs_part(const float* __restrict__ ro, int Ho, int tid) {
    float part = 0.f;
    const float4* ro4 = reinterpret_cast<const float4*>(ro);
    for (int j = tid; j < (Ho >> 2); j += NT) {
        const float4 r = ro4[j];
        part += (fabsf(r.x) + fabsf(r.y)) + (fabsf(r.z) + fabsf(r.w));
    }
    if (tid < (Ho & 3)) part += fabsf(ro[(Ho & ~3) + tid]);
    return warp_sum(part);
}

// Per-card quantities of one scan, 52 entries each: the scan position of the
// card's list, twice the prefix at that position, and the list's mass.
struct FxCards {
    int pos[52];
    int b2[52];
    int mass[52];
};

// One terminal of a unit: where its values go and its payoff scalars.
struct FxItem {
    float* out;
    float pot, c0, c1;
    int type, wmask;
};

// The two integer masses of hand h (step 4); live = false for padding and
// for hands blocked by a dealt card (blocked = true).
struct FxHand {
    unsigned A, B;
    bool live, blocked;
};

template <int SEM>   // MTT_SEM_CORRECT or MTT_SEM_REFERENCE
struct FxEval {
    const Entry* ent;
    const FxCards* cd;
    const int* X;
    const float* ro;
    FxScale fs;
    unsigned Tt;
    int Hq, q;
    bool need_A;

    __device__ __forceinline__ FxHand hand(int h) const {
        FxHand x{0u, 0u, false, false};
        if (h >= Hq) return x;
        const Entry et = ent[h];
        if (et.lt == 0xFFFFu) { x.blocked = true; return x; }
        x.live = true;
        const unsigned ps = et.same >= 0 ? (unsigned)fx_round(ro[et.same], fs) : 0u;
        x.B = Tt - (unsigned)cd->mass[et.c1] - (unsigned)cd->mass[et.c2] + ps;
        if (need_A) {
            const int s1c = cd->pos[et.c1], s2c = cd->pos[et.c2];
            x.A = (unsigned)X[et.lt] + (unsigned)X[et.le] - (unsigned)X[s1c + et.ltc1] - (unsigned)X[s1c + et.lec1] -
                  (unsigned)X[s2c + et.ltc2] - (unsigned)X[s2c + et.lec2] + (unsigned)cd->b2[et.c1] +
                  (unsigned)cd->b2[et.c2] + ps;
        }
        return x;
    }

    // ga = pot/2 * 2^-k, gc = c * 2^-k, gp = fold payoff * 2^-k
    __device__ __forceinline__ float value(const FxHand& x, bool fold, float ga, float gc, float gp) const {
        if (!x.live) {
            // the reference's showdown (no card removal) still meets every
            // opponent with a hand a dealt card blocks: equity 0, so player 0
            // loses and player 1 (1 - eq) wins against the whole mass (A = 0)
            if (!(SEM && x.blocked && !fold)) return 0.f;
            return ga * (float)(int)(q == 0 ? 0u : 2u * Tt) - gc * (float)(int)Tt;
        }
        if (fold) return gp * (float)(int)(SEM ? Tt : x.B);
        if (!SEM) return ga * (float)(int)x.A - gc * (float)(int)x.B;
        // blocked pairs count as P0 losses (honest:182-187): B = Tt, and
        // player 1's pot share is 2 Lr + T = 2 Tt - A
        const unsigned Aq = q == 0 ? x.A : 2u * Tt - x.A;
        return ga * (float)(int)Aq - gc * (float)(int)Tt;
    }
};

// Steps (2)-(4) for player q at a unit of n_it (1 or 2) terminals that share
// the opponent reach ro (sibling terminals below a node where q acts: a fold
// and a call, whose opponent reach is the node's), staged in shared memory
// (16-byte aligned, zero past Ho up to a multiple of 4), whose absolute mass
// S the caller has reduced.  One scan serves the unit: over all three lists
// if it holds a showdown, else over the per-card lists.  X: 3 * Ho + 8 ints;
// wi: NT / 32.  Ends without a barrier: the caller's next barrier must come
// before X or ro is written again.
template <int NT, int SEM>
__device__ void cta_terminal_fx(const TermInfo& ti, const FxItem& it0, const FxItem& it1, int n_it, const TabView& tv, int q,
                                const float* __restrict__ ro, float S, int* X, int* wi, FxCards* cd, int tid) {
    static_assert(3 * 1326 <= 17 * NT, "scan chunks of at most 17 positions cover the largest hand count");
    const int o = 1 - q;
    const int Ho = ti.H[o], Hpq = ti.Hp[q];
    const bool need_A = it0.type != MTT_NODE_FOLD || (n_it > 1 && it1.type != MTT_NODE_FOLD);
    const int lo = need_A ? 0 : Ho;          // folds alone scan only the per-card lists
    const int N = 3 * Ho - lo;
    const uint16_t* idx = tv.sorted[o] + lo; // [rank order (Ho) | per-card lists (2 Ho)], contiguous
    const FxScale fs = fx_scale(S);
    const int C = ((N + NT - 1) / NT) | 1;
    int total;
    switch (C) {
        case 1: total = fx_scan<NT, 1>(idx, ro, N, fs, X, wi, tid); break;
        case 3: total = fx_scan<NT, 3>(idx, ro, N, fs, X, wi, tid); break;
        case 5: total = fx_scan<NT, 5>(idx, ro, N, fs, X, wi, tid); break;
        case 7: total = fx_scan<NT, 7>(idx, ro, N, fs, X, wi, tid); break;
        case 9: total = fx_scan<NT, 9>(idx, ro, N, fs, X, wi, tid); break;
        case 11: total = fx_scan<NT, 11>(idx, ro, N, fs, X, wi, tid); break;
        case 13: total = fx_scan<NT, 13>(idx, ro, N, fs, X, wi, tid); break;
        case 15: total = fx_scan<NT, 15>(idx, ro, N, fs, X, wi, tid); break;
        default: total = fx_scan<NT, 17>(idx, ro, N, fs, X, wi, tid); break;
    }
    const int cb = Ho - lo;                  // scan position of the per-card lists
    if (tid < 52) {
        const uint16_t* seg = tv.seg[o];
        const int p = cb + seg[tid];
        const int b = X[p];
        cd->pos[tid] = p;
        cd->b2[tid] = (int)(2u * (unsigned)b);
        cd->mass[tid] = X[cb + seg[tid + 1]] - b;
    }
    __syncthreads();
    FxEval<SEM> ev;
    ev.ent = tv.ent[q]; ev.cd = cd; ev.X = X; ev.ro = ro; ev.fs = fs;
    ev.Tt = (unsigned)(need_A ? X[Ho] : total >> 1);   // a fold scan's total is even: exact halving
    ev.Hq = ti.H[q]; ev.q = q; ev.need_A = need_A;
    float ga[2], gc[2], gp[2];
    bool fd[2];
    float* out[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const FxItem& it = (i == 1 && n_it > 1) ? it1 : it0;
        const float cq = q ? it.c1 : it.c0;
        ga[i] = __fmul_rn(__fmul_rn(0.5f, it.pot), fs.inv);
        gc[i] = __fmul_rn(cq, fs.inv);
        gp[i] = __fmul_rn((q == ((it.wmask == 1) ? 0 : 1)) ? it.pot - cq : -cq, fs.inv);
        fd[i] = it.type == MTT_NODE_FOLD;
        out[i] = it.out;
    }
    // two hands per step: their dependent shared-memory chains overlap
    for (int h = tid; h < Hpq; h += 2 * NT) {
        const FxHand x0 = ev.hand(h), x1 = ev.hand(h + NT);
        const bool in1 = h + NT < Hpq;
        out[0][h] = ev.value(x0, fd[0], ga[0], gc[0], gp[0]);
        if (in1) out[0][h + NT] = ev.value(x1, fd[0], ga[0], gc[0], gp[0]);
        if (n_it > 1) {
            out[1][h] = ev.value(x0, fd[1], ga[1], gc[1], gp[1]);
            if (in1) out[1][h + NT] = ev.value(x1, fd[1], ga[1], gc[1], gp[1]);
        }
    }
}

// ------------------------------------------------------------- solve kernels
// Work items carry absolute offsets so a warp needs one load before it
// streams: a sweep item is one node for one player, a warp loops over that
// player's float4 hand groups.
struct alignas(16) FwdItem {    // 64 B
    long long reach_in;   // arena float offset of the acting player's reach at the node
    long long child;      // arena float offset of child 0's part for that player
    long long rows;       // R/S float offset of the node's first regret row
    long long hc;         // hand-card offset of that player (chance items)
    int h4;               // float4 groups of that player
    int hs4;              // reach slot stride in float4
    int na;
    int flags;            // FI_REACH: write children's reach; FI_SUMS: add to S; FI_CHANCE
    int first;            // global index of child 0 (chance items read the dealt cards)
    int g0;               // first float4 group of this warp (lane l takes g0 + l)
    int sub;              // subgame
    int pad;
};
struct alignas(16) BwdItem {    // 64 B
    long long child;      // arena float offset (CFV region) of child 0's part for player q
    long long self;       // arena float offset (CFV region) of this node's part for q
    long long rows;       // R float offset of the node's first row (update items)
    long long hc;         // hand-card offset of q (chance items); q's reach at the node (BI_SUMS items)
    int h4;
    int hs4;
    int na;
    int flags;            // BI_UPDATE: q acts here (BI_SUMS: also add to S); BI_CHANCE; else sum of children;
                          // BI_NEG: q == 1 (sign of dEV0 in the differentiable pass)
    int first;            // global index of child 0 (chance items)
    float div;            // chance divisor
    int g0;               // first float4 group of this warp
    int sub;              // subgame
};
struct alignas(16) TermItem {   // 80 B
    long long ro[2];      // arena offsets of each player's reach at the terminal
    long long out[2];     // arena offsets (CFV region) of each player's values
    long long tab;        // byte offset of the showdown table variant
    float pot, c0, c1;
    int type_wmask;       // type | wmask << 8
    int H[2], Hp[2];
    int sub;              // subgame
    int pad[3];
};
static_assert(sizeof(FwdItem) == 64 && sizeof(BwdItem) == 64 && sizeof(TermItem) == 96, "item sizes");
enum { FI_REACH = 1, FI_SUMS = 2, FI_CHANCE = 4 };
enum { BI_UPDATE = 1, BI_SUMS = 2, BI_CHANCE = 4, BI_NEG = 8 };

__global__ void k_init(SolveDev a, int n_sub) {
    const int s = blockIdx.x;
    if (s == 0 && threadIdx.x == 0) { *a.iter = 1; *a.err = 0; }
    if (s >= n_sub) return;
    const SubDesc sd = a.desc[s];
    const long long n0 = (long long)sd.rows0 * sd.Hp0 / 4, n1 = (long long)sd.rows1 * sd.Hp1 / 4;
    float4* r0 = reinterpret_cast<float4*>(a.R + sd.rs_base0);
    float4* r1 = reinterpret_cast<float4*>(a.R + sd.rs_base1);
    float4* s0 = reinterpret_cast<float4*>(a.S + sd.rs_base0);
    float4* s1 = reinterpret_cast<float4*>(a.S + sd.rs_base1);
    for (long long i = threadIdx.x; i < n0; i += blockDim.x) { r0[i] = f4(0.f); s0[i] = f4(0.f); }
    for (long long i = threadIdx.x; i < n1; i += blockDim.x) { r1[i] = f4(0.f); s1[i] = f4(0.f); }
    const int HS4 = (sd.Hp0 + sd.Hp1) >> 2;
    const float4* rg = reinterpret_cast<const float4*>(a.ranges + sd.range_base);
    float4* rr = reinterpret_cast<float4*>(a.arena + sd.arena_base);
    for (int i = threadIdx.x; i < HS4; i += blockDim.x) rr[i] = rg[i];
}

__global__ void k_next_iter(SolveDev a) {
    if (threadIdx.x == 0) *a.iter += 1;
}

// Fixed-action-count paths of the sweeps: every row of the node is loaded
// before any is used (A independent 16-byte loads in flight per lane), with
// the same operations in the same order as the general loops below, so the
// results are bit-identical.
template <int A>
__device__ __forceinline__ void fwd_reach_fixed(const float4* __restrict__ Rb, const float4* __restrict__ rp,
                                                float4* __restrict__ ch, int H4, int HS4, int g) {
    float4 rk[A];
#pragma unroll
    for (int k = 0; k < A; ++k) rk[k] = max04(Rb[(size_t)k * H4 + g]);
    const float4 r = rp[g];
    float4 sum = f4(0.f);
#pragma unroll
    for (int k = 0; k < A; ++k) sum = add4(sum, rk[k]);
    const float invA = __fdiv_rn(1.0f, (float)A);
#pragma unroll
    for (int k = 0; k < A; ++k) ch[(size_t)k * HS4 + g] = mul4(r, rm4(rk[k], sum, invA));
}

template <int A>
__device__ __forceinline__ void bwd_sum_fixed(const float4* __restrict__ qc, float4* __restrict__ out, int HS4, int g) {
    float4 qk[A];
#pragma unroll
    for (int k = 0; k < A; ++k) qk[k] = qc[(size_t)k * HS4 + g];
    float4 so = f4(0.f);
#pragma unroll
    for (int k = 0; k < A; ++k) so = add4(so, qk[k]);
    out[g] = so;
}

// Forward sweep of one level: regret matching, children's reach and/or
// strategy sums (kernel_forward_sweep, honest_multistreet_solver.cu:88-126).
template <int ALGO, bool SUMS>
__device__ __forceinline__ void k_fwd_group(const SolveDev& a, const FwdItem& it, const int lane) {
    const float4* rp = reinterpret_cast<const float4*>(a.arena + it.reach_in);
    float4* ch = reinterpret_cast<float4*>(a.arena + it.child);
    const int A = it.na, H4 = it.h4, HS4 = it.hs4;
    if (it.flags & FI_CHANCE) {
        const uint16_t* hc = a.hcards + it.hc;
        const int g = it.g0 + lane;
        if (g < H4) {
            const float4 r = rp[g];
            const uint64_t m0 = hand_mask(hc[4 * g]), m1 = hand_mask(hc[4 * g + 1]);
            const uint64_t m2 = hand_mask(hc[4 * g + 2]), m3 = hand_mask(hc[4 * g + 3]);
            for (int k = 0; k < A; ++k) {
                const int card = a.nodes[it.first + k].dealt;
                float4 v = r;
                if ((m0 >> card) & 1ull) v.x = 0.f;
                if ((m1 >> card) & 1ull) v.y = 0.f;
                if ((m2 >> card) & 1ull) v.z = 0.f;
                if ((m3 >> card) & 1ull) v.w = 0.f;
                ch[(size_t)k * HS4 + g] = v;
            }
        }
        return;
    }
    const bool dr = it.flags & FI_REACH, ds = SUMS && (it.flags & FI_SUMS);
    const float4* Rb = reinterpret_cast<const float4*>(a.R + it.rows);
    float4* Sb = reinterpret_cast<float4*>(a.S + it.rows);
    if (dr && !ds) {
        const int g = it.g0 + lane;
        if (g >= H4) return;
        switch (A) {
            case 2: fwd_reach_fixed<2>(Rb, rp, ch, H4, HS4, g); return;
            case 3: fwd_reach_fixed<3>(Rb, rp, ch, H4, HS4, g); return;
            case 4: fwd_reach_fixed<4>(Rb, rp, ch, H4, HS4, g); return;
            case 5: fwd_reach_fixed<5>(Rb, rp, ch, H4, HS4, g); return;
            case 6: fwd_reach_fixed<6>(Rb, rp, ch, H4, HS4, g); return;
            default: break;
        }
    }
    const float invA = __fdiv_rn(1.0f, (float)A);
    float w_lin = 0.f, dstr = 0.f;
    if (ds && it.g0 + lane < H4)
        for (int k = 0; k < A; ++k) pf_l2(Sb + (size_t)k * H4 + it.g0 + lane);
    if (ds) {
        const float4 tb = *reinterpret_cast<const float4*>(a.iter_tab + 4 * (*a.iter - 1));
        w_lin = tb.x;
        dstr = tb.w;
    }
    constexpr bool dcfr = ALGO == MTT_ALGO_DCFR;
    // Regret rows are read twice (sum, then strategy); the second read hits
    // L1, which keeps registers low.
    const int g = it.g0 + lane;
    if (g < H4) {
        const float4 r = rp[g];
        float4 sum = f4(0.f);
        for (int k = 0; k < A; ++k) sum = add4(sum, max04(Rb[(size_t)k * H4 + g]));
        const float4 wr = mul4(r, f4(w_lin));
        for (int k = 0; k < A; ++k) {
            const float4 sg = rm4(max04(Rb[(size_t)k * H4 + g]), sum, invA);
            if (dr) ch[(size_t)k * HS4 + g] = mul4(r, sg);
            if (ds) {
                float4 sv = Sb[(size_t)k * H4 + g];
                sv = dcfr ? fma4(r, sg, mul4(sv, f4(dstr))) : fma4(wr, sg, sv);
                Sb[(size_t)k * H4 + g] = sv;
            }
        }
    }
}

// One warp per work item; the item covers span x 32 float4 hand groups.
// ALGO: the solve's a.algo; SUMS: the list may hold FI_SUMS items (without
// it, such items would pass reach only).  The reach-only kernel of the
// alternating passes took 0.734 ms per iteration on the 4,096-subgame river
// batch against 0.771 ms for the kernel that also handles strategy sums.
template <int SPAN, int ALGO, bool SUMS>
__global__ void __launch_bounds__(256, 5) k_fwd(SolveDev a, const FwdItem* __restrict__ items, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    const FwdItem it = items[w];      // work items are written once, before any solve
    grid_dep_trigger();
    grid_dep_wait();
#pragma unroll
    for (int s = 0; s < SPAN; ++s) {
        if (SPAN > 1 && it.g0 + 32 * s >= it.h4) break;
        k_fwd_group<ALGO, SUMS>(a, it, (threadIdx.x & 31) + 32 * s);
    }
}

// Terminals are processed in groups: consecutive terminals of one subgame
// that share a showdown table variant (all of a river subgame's terminals,
// or those below one river card of a turn subgame), at most TG_CHUNK per
// CTA.  The CTA stages the table blocks and the group's work items once, then
// walks its terminals with
// the opponent reach of terminal t+1 in flight (1-D bulk copy on the other
// stage's mbarrier) while terminal t is evaluated from shared memory.
constexpr int TG = 256;         // threads per terminal-group CTA (fixed: the scan chunks depend on it)
constexpr int TG_CHUNK = 16;    // terminals per group at most

struct alignas(16) TermGroup {  // 32 B
    long long tab;              // byte offset of the table variant
    int first, count;           // items [first, first + count) of the terminal list
    int H0, H1, Hp0, Hp1;
};
static_assert(sizeof(TermGroup) == 32, "TermGroup is 32 bytes");

// Shared-memory plan of a group for the updated players `upd` (bit q = q's
// values are computed).  One direction (upd = 1 << q) needs the opponent's
// index block, q's entry block and the opponent's reach; both directions
// need the whole variant and both reach vectors.
__host__ __device__ inline int tg_table_bytes(int H0, int H1, int upd) {
    if (upd == 3) return tab_variant_bytes(H0, H1);
    const int q = upd == 1 ? 0 : 1;
    const int Ho = q ? H0 : H1, Hq = q ? H1 : H0;
    return tab_idx_bytes(Ho) + tab_ent_bytes(Hq);
}
__host__ __device__ inline int tg_reach_bytes(int Hp0, int Hp1, int upd) {
    return upd == 3 ? 4 * (Hp0 + Hp1) : 4 * (upd == 1 ? Hp1 : Hp0);
}
__host__ __device__ inline int tg_scan_ints(int H0, int H1, int upd) {
    int m = 0;
    for (int q = 0; q < 2; ++q) {
        if (!((upd >> q) & 1)) continue;
        const int Ho = q ? H0 : H1;
        m = 3 * Ho + 8 > m ? 3 * Ho + 8 : m;
    }
    return m;
}
__host__ __device__ inline int tg_smem_bytes(int H0, int H1, int Hp0, int Hp1, int upd) {
    return tg_table_bytes(H0, H1, upd) + 2 * tg_reach_bytes(Hp0, Hp1, upd) + 4 * tg_scan_ints(H0, H1, upd) + 16;
}

// Terminal values of the updated players (kernel_evaluate_terminals,
// honest_multistreet_solver.cu:128-196), one terminal group per CTA.
// UPD: the updated players (bit q: q's values), 1, 2 or 3.  SEM: a.semantics,
// or -1 to branch on it at run time.
// One kernel per (UPD, SEM) lets the compiler fold the player and semantics
// choices: on the 4,096-subgame river batch the one-direction terminal pass
// took 2.70 ms per iteration against 2.89 ms with both chosen at run time.
// For UPD = 3 a fixed SEM spilled registers and was slower, so that kernel
// keeps the run-time branch (3.45 ms against 4.04 ms for the fully run-time
// kernel in the simultaneous-update mode).
template <int UPD, int SEM>
__global__ void __launch_bounds__(TG, 5) k_term(SolveDev a, const TermGroup* __restrict__ groups,
                                             const TermItem* items, int n) {
    constexpr int upd = UPD;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar[3];   // 0: table blocks, 1 + s: reach stage s
    __shared__ float wf[2][2][TG / 32];   // [terminal parity][updated player][warp]
    __shared__ int wi[TG / 32];
    __shared__ FxCards cards;
    __shared__ __align__(16) TermItem sitems[TG_CHUNK];   // the group's items, staged with the table
    const int gi = blockIdx.x, tid = threadIdx.x;
    if (gi >= n) return;
    const TermGroup g = groups[gi];
    const TermItem* const gitems = items;
    items = sitems - g.first;      // items[g.first + t] reads the staged copy below
    constexpr bool both = UPD == 3;
    constexpr int q1 = UPD == 2 ? 1 : 0;            // the updated player of a one-direction launch
    const uint32_t tb = (uint32_t)tg_table_bytes(g.H0, g.H1, upd);
    const uint32_t rbytes = (uint32_t)tg_reach_bytes(g.Hp0, g.Hp1, upd);
    uint8_t* T = smem;
    float* Rst0 = reinterpret_cast<float*>(smem + tb);
    float* Rst1 = reinterpret_cast<float*>(smem + tb + rbytes);
    int* X = reinterpret_cast<int*>(smem + tb + 2 * rbytes);   // tb, rbytes: multiples of 16
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init(&bar[2], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // thread 0 issues every copy; stage s of terminal t is reach vector(s) of items[first + t]
    auto issue_reach = [&](int t, int s) {
        const TermItem& it = gitems[g.first + t];   // the first one is issued before the staged copy lands
        float* dst = s ? Rst1 : Rst0;
        mbar_arrive_expect_tx(&bar[1 + s], rbytes);
        if (both) {
            bulk_g2s(dst, a.arena + it.ro[0], 4u * (uint32_t)g.Hp0, &bar[1 + s]);
            bulk_g2s(dst + g.Hp0, a.arena + it.ro[1], 4u * (uint32_t)g.Hp1, &bar[1 + s]);
        } else {
            bulk_g2s(dst, a.arena + it.ro[1 - q1], rbytes, &bar[1 + s]);
        }
    };
    if (tid == 0) {
        mbar_arrive_expect_tx(&bar[0], tb + (uint32_t)(sizeof(TermItem) * g.count));
        bulk_g2s(sitems, gitems + g.first, (uint32_t)(sizeof(TermItem) * g.count), &bar[0]);
        if (both) {
            bulk_g2s(T, a.tabs + g.tab, tb, &bar[0]);
        } else {
            const int o = 1 - q1;
            const int Ho = o ? g.H1 : g.H0;
            const uint32_t ib = (uint32_t)tab_idx_bytes(Ho);
            bulk_g2s(T, a.tabs + g.tab + tab_idx_off(o, g.H0), ib, &bar[0]);
            bulk_g2s(T + ib, a.tabs + g.tab + tab_ent_off(q1, g.H0, g.H1), tb - ib, &bar[0]);
        }
    }
    // tables and items are written once, before any solve; reach and values
    // belong to the previous kernels
    grid_dep_trigger();
    grid_dep_wait();
    if (tid == 0) issue_reach(0, 0);
    const bool okt = mbar_wait_bounded(&bar[0], 0u);
    if (__syncthreads_or(!okt)) {
        if (tid == 0) atomicOr(a.err, 1);
        (void)mbar_wait_bounded(&bar[1], 0u);    // the first reach copy may still be in flight
        return;
    }
    TabView tv;
    if (both) {
        tv = tab_view(T, g.H0, g.H1);
    } else {
        // one direction: both slots get the staged blocks (only the opponent's
        // index slot and q's entry slot are read), so no slot is chosen at run time
        const int Ho = q1 ? g.H0 : g.H1;
        const uint16_t *so, *co, *sg;
        tab_idx_view(T, Ho, &so, &co, &sg);
        const Entry* en = reinterpret_cast<const Entry*>(T + tab_idx_bytes(Ho));
        tv.sorted[0] = tv.sorted[1] = so;
        tv.cl[0] = tv.cl[1] = co;
        tv.seg[0] = tv.seg[1] = sg;
        tv.ent[0] = tv.ent[1] = en;
    }
    TermInfo ti;
    ti.H[0] = g.H0; ti.H[1] = g.H1; ti.Hp[0] = g.Hp0; ti.Hp[1] = g.Hp1;
    // opponent reach of player q inside a stage: player 1's part follows
    // player 0's in a two-direction stage
    auto opp = [&](const float* st, int q) -> const float* { return both ? (q == 0 ? st + g.Hp0 : st) : st; };
    // absolute opponent masses of the terminal staged in st, per updated
    // player, into wf[buf]; read after the next barrier
    auto mass_parts = [&](const float* st, int buf) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!((upd >> q) & 1)) continue;
            const float p = fx_abs_part<TG>(opp(st, q), q ? g.H0 : g.H1, tid);
            if ((tid & 31) == 0) wf[buf][q][tid >> 5] = p;
        }
    };
    uint32_t parity = 1u;   // bit s: phase of stage s's next wait (stage 0's first is done below)
    {
        const bool ok = mbar_wait_bounded(&bar[1], 0u);
        if (ok) mass_parts(Rst0, 0);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(a.err, 1);
            return;
        }
    }
    // Units: a terminal, or two adjacent ones (siblings) whose opponent reach
    // for the updated player is the same vector (one direction only).
    auto unit_len = [&](int t) -> int {
        if (both || t + 1 >= g.count) return 1;
        const int o = 1 - q1;
        return items[g.first + t + 1].ro[o] == items[g.first + t].ro[o] ? 2 : 1;
    };
    int t = 0, len = unit_len(0);
    for (int u = 0; t < g.count; ++u) {
        const int s = u & 1;
        const int tn = t + len;                  // the next unit's first terminal
        // stage s ^ 1 was last read by the previous unit, which ended on a barrier
        if (tid == 0 && tn < g.count) issue_reach(tn, s ^ 1);
        FxItem f0, f1;
        auto load_item = [&](FxItem& f, const TermItem& it) {
            f.pot = it.pot; f.c0 = it.c0; f.c1 = it.c1;
            f.type = it.type_wmask & 0xFF; f.wmask = (it.type_wmask >> 8) & 0xFF;
        };
        const TermItem& ia = items[g.first + t];
        const TermItem& ib = items[g.first + t + (len > 1 ? 1 : 0)];
        load_item(f0, ia);
        load_item(f1, ib);
        const float* st = s ? Rst1 : Rst0;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!((upd >> q) & 1)) continue;
            float S = 0.f;
#pragma unroll
            for (int k = 0; k < TG / 32; ++k) S += wf[s][q][k];
            f0.out = a.arena + ia.out[q];
            f1.out = a.arena + ib.out[q];
            if (both && q == 1) __syncthreads();   // player 0's values have been read out of X
            if constexpr (SEM >= 0)
                cta_terminal_fx<TG, SEM>(ti, f0, f1, len, tv, q, opp(st, q), S, X, wi, &cards, tid);
            else if (a.semantics)
                cta_terminal_fx<TG, MTT_SEM_REFERENCE>(ti, f0, f1, len, tv, q, opp(st, q), S, X, wi, &cards, tid);
            else
                cta_terminal_fx<TG, MTT_SEM_CORRECT>(ti, f0, f1, len, tv, q, opp(st, q), S, X, wi, &cards, tid);
        }
        // the next unit's reach and masses; the barrier also ends this unit
        const int lenn = tn < g.count ? unit_len(tn) : 0;
        bool ok = true;
        if (tn < g.count) {
            ok = mbar_wait_bounded(&bar[2 - s], (parity >> (s ^ 1)) & 1u);
            parity ^= 1u << (s ^ 1);
            if (ok) mass_parts(s ? Rst0 : Rst1, s ^ 1);
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(a.err, 1);
            return;
        }
        t = tn;
        len = lenn;
    }
}

// Backward sweep of one level for the updated players: counterfactual values
// and the CFR+/DCFR regret update (kernel_backward_sweep, honest:198-249).
template <int ALGO, bool SUMS>
__device__ __forceinline__ void k_bwd_group(const SolveDev& a, const BwdItem& it, const int lane) {
    const float4* qc = reinterpret_cast<const float4*>(a.arena + it.child);
    float4* out = reinterpret_cast<float4*>(a.arena + it.self);
    const int A = it.na, H4 = it.h4, HS4 = it.hs4;
    if (it.flags & BI_CHANCE) {
        const uint16_t* hc = a.hcards + it.hc;
        const float dv = a.semantics ? it.div + 2.0f : it.div;   // (N-2) in the reference's semantics
        const int g = it.g0 + lane;
        if (g < H4) {
            const uint64_t m0 = hand_mask(hc[4 * g]), m1 = hand_mask(hc[4 * g + 1]);
            const uint64_t m2 = hand_mask(hc[4 * g + 2]), m3 = hand_mask(hc[4 * g + 3]);
            float4 acc = f4(0.f);
            for (int k = 0; k < A; ++k) {
                const int card = a.nodes[it.first + k].dealt;
                const float4 cv = qc[(size_t)k * HS4 + g];
                if (!((m0 >> card) & 1ull)) acc.x = __fadd_rn(acc.x, cv.x);
                if (!((m1 >> card) & 1ull)) acc.y = __fadd_rn(acc.y, cv.y);
                if (!((m2 >> card) & 1ull)) acc.z = __fadd_rn(acc.z, cv.z);
                if (!((m3 >> card) & 1ull)) acc.w = __fadd_rn(acc.w, cv.w);
            }
            out[g] = make_float4(__fdiv_rn(acc.x, dv), __fdiv_rn(acc.y, dv), __fdiv_rn(acc.z, dv), __fdiv_rn(acc.w, dv));
        }
        return;
    }
    const int g = it.g0 + lane;
    if (g >= H4) return;
    if (!(it.flags & BI_UPDATE)) {
        switch (A) {
            case 2: bwd_sum_fixed<2>(qc, out, HS4, g); return;
            case 3: bwd_sum_fixed<3>(qc, out, HS4, g); return;
            case 4: bwd_sum_fixed<4>(qc, out, HS4, g); return;
            case 5: bwd_sum_fixed<5>(qc, out, HS4, g); return;
            case 6: bwd_sum_fixed<6>(qc, out, HS4, g); return;
            default: break;
        }
        {
            float4 so = f4(0.f);
            for (int k = 0; k < A; ++k) so = add4(so, qc[(size_t)k * HS4 + g]);
            out[g] = so;
        }
        return;
    }
    const float invA = __fdiv_rn(1.0f, (float)A);
    float4* Rb = reinterpret_cast<float4*>(a.R + it.rows);
    float dpos = 0.f, dneg = 0.f, w_lin = 0.f, dstr = 0.f;
    constexpr bool dcfr = ALGO == MTT_ALGO_DCFR;
    const bool ds = SUMS && (it.flags & BI_SUMS);
    for (int k = 0; k < A; ++k) {
        pf_l2(qc + (size_t)k * HS4 + g);
        if (ds) pf_l2(reinterpret_cast<const float4*>(a.S + it.rows) + (size_t)k * H4 + g);
    }
    if (dcfr || ds) {
        const float4 tb = *reinterpret_cast<const float4*>(a.iter_tab + 4 * (*a.iter - 1));
        dpos = tb.y;
        dneg = tb.z;
        w_lin = tb.x;
        dstr = tb.w;
    }
    // Rows and child values are re-read (L1 hits) instead of held in registers.
    {
        float4 sum = f4(0.f);
        for (int k = 0; k < A; ++k) sum = add4(sum, max04(Rb[(size_t)k * H4 + g]));
        float4 v = f4(0.f);
        if (ds) {
            // strategy sums of the acting player, from the same sigma and with
            // the same arithmetic as the forward sweep's FI_SUMS path
            const float4 r = reinterpret_cast<const float4*>(a.arena + it.hc)[g];
            const float4 wr = mul4(r, f4(w_lin));
            float4* Sb = reinterpret_cast<float4*>(a.S + it.rows);
            for (int k = 0; k < A; ++k) {
                const float4 sg = rm4(max04(Rb[(size_t)k * H4 + g]), sum, invA);
                v = fma4(sg, qc[(size_t)k * HS4 + g], v);
                float4 sv = Sb[(size_t)k * H4 + g];
                sv = dcfr ? fma4(r, sg, mul4(sv, f4(dstr))) : fma4(wr, sg, sv);
                Sb[(size_t)k * H4 + g] = sv;
            }
        } else {
            for (int k = 0; k < A; ++k)
                v = fma4(rm4(max04(Rb[(size_t)k * H4 + g]), sum, invA), qc[(size_t)k * HS4 + g], v);
        }
        out[g] = v;
        for (int k = 0; k < A; ++k) {
            const float4 rk = Rb[(size_t)k * H4 + g];
            const float4 qk = qc[(size_t)k * HS4 + g];
            float4 nr;
            if (dcfr) {
                nr.x = dcfr1(rk.x, __fsub_rn(qk.x, v.x), dpos, dneg);
                nr.y = dcfr1(rk.y, __fsub_rn(qk.y, v.y), dpos, dneg);
                nr.z = dcfr1(rk.z, __fsub_rn(qk.z, v.z), dpos, dneg);
                nr.w = dcfr1(rk.w, __fsub_rn(qk.w, v.w), dpos, dneg);
            } else {
                nr.x = cfrplus1(rk.x, __fsub_rn(qk.x, v.x));
                nr.y = cfrplus1(rk.y, __fsub_rn(qk.y, v.y));
                nr.z = cfrplus1(rk.z, __fsub_rn(qk.z, v.z));
                nr.w = cfrplus1(rk.w, __fsub_rn(qk.w, v.w));
            }
            Rb[(size_t)k * H4 + g] = nr;
        }
    }
}

// One warp per work item; the item covers span x 32 float4 hand groups.
// ALGO: the solve's a.algo (a kernel per algorithm: on the 4,096-subgame
// river batch the backward levels took 1.87 ms per iteration against 1.91 ms
// with the update rule chosen at run time; 64 registers a thread at four CTAs
// per SM, without the spills, took 1.94 ms).  SUMS: the list may hold
// BI_SUMS items (without it, such items would update regrets only).
template <int SPAN, int ALGO, bool SUMS>
__global__ void __launch_bounds__(256, 5) k_bwd(SolveDev a, const BwdItem* __restrict__ items, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    const BwdItem it = items[w];      // work items are written once, before any solve
    grid_dep_trigger();
    grid_dep_wait();
#pragma unroll
    for (int s = 0; s < SPAN; ++s) {
        if (SPAN > 1 && it.g0 + 32 * s >= it.h4) break;
        k_bwd_group<ALGO, SUMS>(a, it, (threadIdx.x & 31) + 32 * s);
    }
}

// ------------------------------------------------------------- depth-limit leaves
// A leaf (MTT_NODE_LEAF) ends a turn betting round that closed with chips
// behind; in the full game the river is dealt and played out.  Its values
// are built per river card c (48 rows per leaf) from both players' reach at
// the leaf with the combos holding c removed:
//  * the check-down value: the showdown of the pot at that reach, from the
//    turn subgame's table variant of c by the fixed-point terminal routine
//    (card removal, split ties), in chips;
//  * optionally the leaf network's correction: both reaches normalised to
//    ranges over the 1,326 combos and fed as in its training (each range
//    scaled by the 1,081 combos live on a river board, the 5-card board
//    one-hot, pot 1 and chips behind / pot); its output, in units of the
//    pot with both ranges summing to 1, times pot x the opponent's mass.
// Player q's value of hand h at the leaf is the sum over c not in h of those
// values, divided by the river chance divisor of the solver's semantics (44
// correct, 46 reference), as a river chance node of the full tree averages
// its children.  The check-down part always uses the correct semantics, the
// basis the network was trained on.
struct alignas(16) LeafItem {
    long long reach[2];   // arena float offsets of each player's reach at the leaf
    long long cfv[2];     // arena float offsets (value region) of each player's values at the leaf
    long long hc[2];      // hand-card offsets of each player
    long long tab;        // byte offset of the subgame's table variants (variant c = river card c)
    float pot, spr;       // chips in the pot; chips behind / pot
    int H[2], Hp[2];
    int row0;             // first row of the leaf
    int vsize;            // bytes per table variant
    uint8_t board[4];
    int sub;
};

constexpr int LEAF_RIVERS = 48;        // river cards after a 4-card board
constexpr int LEAF_IN = 2706, LEAF_OUT = 2652, LEAF_COMBOS = 1326;

__device__ __forceinline__ int combo_index(int a, int b) {   // a < b, lexicographic pairs
    return a * 51 - a * (a - 1) / 2 + (b - a - 1);
}

// The j-th card (ascending) not on the 4-card board.
__device__ __forceinline__ int leaf_river_card(const uint8_t* bd, int j) {
    int k = -1;
    for (int x = 0; x < 52; ++x) {
        if (x == bd[0] || x == bd[1] || x == bd[2] || x == bd[3]) continue;
        if (++k == j) return x;
    }
    return -1;
}

// Shared memory of k_leaf_showdown for one leaf and updated player q.
__host__ __device__ inline int leaf_sd_smem(int Ho, int Hq, int Hpo) {
    return tab_idx_bytes(Ho) + tab_ent_bytes(Hq) + 4 * Hpo + 4 * (3 * Ho + 8) + 16;
}

// One network row (leaf, river card) per CTA: features X [rows][2706] and
// reach masses M [rows][2].
__global__ void __launch_bounds__(256) k_leaf_rows(SolveDev a, const LeafItem* __restrict__ leaves, float* __restrict__ X,
                                                   float* __restrict__ M) {
    __shared__ float wsum[8];
    const int row = blockIdx.x, tid = threadIdx.x;
    const LeafItem L = leaves[row / LEAF_RIVERS];
    const int c = leaf_river_card(L.board, row % LEAF_RIVERS);
    float* x = X + (size_t)row * LEAF_IN;
    for (int i = tid; i < LEAF_IN; i += 256) x[i] = 0.0f;
    __syncthreads();
    for (int p = 0; p < 2; ++p) {
        const float* rp = a.arena + L.reach[p];
        const uint16_t* hc = a.hcards + L.hc[p];
        float part = 0.0f;
        for (int h = tid; h < L.H[p]; h += 256) {
            const int cc = hc[h];
            if ((cc & 0xFF) != c && (cc >> 8) != c) part += rp[h];
        }
        part = warp_sum(part);
        if ((tid & 31) == 0) wsum[tid >> 5] = part;
        __syncthreads();
        float tot = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) tot += wsum[k];
        __syncthreads();
        const float inv = tot > 0.0f ? 1.0f / tot : 0.0f;
        for (int h = tid; h < L.H[p]; h += 256) {
            const int cc = hc[h], c1 = cc & 0xFF, c2 = cc >> 8;
            if (c1 == c || c2 == c) continue;
            x[p * LEAF_COMBOS + combo_index(c1, c2)] = rp[h] * inv * 1081.0f;
        }
        if (tid == 0) M[2 * (size_t)row + p] = tot;
    }
    if (tid == 0) {
        for (int k = 0; k < 4; ++k) x[2 * LEAF_COMBOS + L.board[k]] = 1.0f;
        x[2 * LEAF_COMBOS + c] = 1.0f;
        x[2 * LEAF_COMBOS + 52] = 1.0f;       // pot / 100 with the pot scaled to 100
        x[2 * LEAF_COMBOS + 53] = L.spr;      // stack / 100 at that scale
    }
}

// Check-down values (chips) of one (leaf, river card) row per CTA for the
// updated players `upd`: SD[row][q][0..Hp_q), row stride 2 * sd_stride.
__global__ void __launch_bounds__(TG) k_leaf_showdown(SolveDev a, const LeafItem* __restrict__ leaves,
                                                      float* __restrict__ SD, int sd_stride, int upd) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ float wf[TG / 32];
    __shared__ int wi[TG / 32];
    __shared__ FxCards cards;
    const int row = blockIdx.x, tid = threadIdx.x;
    const LeafItem L = leaves[row / LEAF_RIVERS];
    const int c = leaf_river_card(L.board, row % LEAF_RIVERS);
    const uint8_t* var = a.tabs + L.tab + (size_t)c * L.vsize;
    for (int q = 0; q < 2; ++q) {
        if (!((upd >> q) & 1)) continue;
        const int o = 1 - q, Ho = L.H[o];
        const int ib = tab_idx_bytes(Ho), eb = tab_ent_bytes(L.H[q]);
        uint8_t* T = smem;
        const uint4* si = reinterpret_cast<const uint4*>(var + tab_idx_off(o, L.H[0]));
        const uint4* se = reinterpret_cast<const uint4*>(var + tab_ent_off(q, L.H[0], L.H[1]));
        for (int i = tid; i < ib / 16; i += TG) reinterpret_cast<uint4*>(T)[i] = si[i];
        for (int i = tid; i < eb / 16; i += TG) reinterpret_cast<uint4*>(T + ib)[i] = se[i];
        // opponent reach, without the combos the river card removes (zero past Ho)
        float* ro = reinterpret_cast<float*>(T + ib + eb);
        const float* rs = a.arena + L.reach[o];
        const uint16_t* hc = a.hcards + L.hc[o];
        for (int j = tid; j < L.Hp[o]; j += TG) {
            float r = 0.0f;
            if (j < Ho) {
                const int cc = hc[j];
                if ((cc & 0xFF) != c && (cc >> 8) != c) r = rs[j];
            }
            ro[j] = r;
        }
        int* X = reinterpret_cast<int*>(T + ib + eb + 4 * L.Hp[o]);
        __syncthreads();
        const float part = fx_abs_part<TG>(ro, Ho, tid);
        if ((tid & 31) == 0) wf[tid >> 5] = part;
        __syncthreads();
        float S = 0.0f;
#pragma unroll
        for (int k = 0; k < TG / 32; ++k) S += wf[k];
        TabView tv;
        const uint16_t *so, *co, *sg;
        tab_idx_view(T, Ho, &so, &co, &sg);
        tv.sorted[0] = tv.sorted[1] = so;
        tv.cl[0] = tv.cl[1] = co;
        tv.seg[0] = tv.seg[1] = sg;
        tv.ent[0] = tv.ent[1] = reinterpret_cast<const Entry*>(T + ib);
        TermInfo ti;
        ti.H[0] = L.H[0]; ti.H[1] = L.H[1]; ti.Hp[0] = L.Hp[0]; ti.Hp[1] = L.Hp[1];
        FxItem it;
        it.out = SD + ((size_t)row * 2 + q) * sd_stride;
        it.pot = L.pot; it.c0 = 0.5f * L.pot; it.c1 = 0.5f * L.pot;
        it.type = MTT_NODE_SHOWDOWN; it.wmask = 3;
        cta_terminal_fx<TG, MTT_SEM_CORRECT>(ti, it, it, 1, tv, q, ro, S, X, wi, &cards, tid);
        __syncthreads();   // the next player restages shared memory
    }
}

// Leaf values of the updated players `upd` from the check-down values SD
// and/or the network output Y with the masses M (either source may be null).
// One CTA per (leaf, 128 hands); each hand adds its 48 rivers in card order.
constexpr int LV_HANDS = 128;
__global__ void __launch_bounds__(LV_HANDS) k_leaf_values(SolveDev a, const LeafItem* __restrict__ leaves,
                                                          const float* __restrict__ SD, int sd_stride,
                                                          const float* __restrict__ Y, const float* __restrict__ M,
                                                          int upd, float div) {
    __shared__ int rc[LEAF_RIVERS];
    __shared__ float wm[2][LEAF_RIVERS];        // pot x the opponent's reach mass per river row
    const int tid = threadIdx.x;
    const LeafItem L = leaves[blockIdx.x];
    const int h = blockIdx.y * LV_HANDS + tid;
    if (tid < LEAF_RIVERS) {
        rc[tid] = leaf_river_card(L.board, tid);
        if (Y) {
            const size_t row = (size_t)L.row0 + tid;
            wm[0][tid] = __fmul_rn(L.pot, M[2 * row + 1]);   // q = 0 meets player 1's mass
            wm[1][tid] = __fmul_rn(L.pot, M[2 * row]);
        }
    }
    __syncthreads();
    for (int q = 0; q < 2; ++q) {
        if (!((upd >> q) & 1) || h >= L.Hp[q]) continue;
        float v = 0.0f;
        if (h < L.H[q]) {
            const int cc = a.hcards[L.hc[q] + h], c1 = cc & 0xFF, c2 = cc >> 8;
            const int id = q * LEAF_COMBOS + combo_index(c1, c2);
            float acc = 0.0f;
#pragma unroll 8
            for (int j = 0; j < LEAF_RIVERS; ++j) {
                if (rc[j] == c1 || rc[j] == c2) continue;
                const size_t row = (size_t)L.row0 + j;
                float y = SD ? SD[(row * 2 + q) * sd_stride + h] : 0.0f;
                if (Y) y = fmaf(wm[q][j], Y[row * LEAF_OUT + id], y);
                acc += y;
            }
            v = __fdiv_rn(acc, div);
        }
        a.arena[L.cfv[q] + h] = v;
    }
}

// ------------------------------------------------------------- differentiable EV
// Fixed strategies sigma = softmax(logits) per node and hand; the logits sit
// in the regret layout (a.R) and dEV0/dlogits is written in the same layout
// (a.S).  One forward pass (reach), the terminals of both players and one
// backward pass (counterfactual values and the adjoint of the softmax) give
// EV0 and all its gradients: dEV0/drange0 = cfv0 at the root, dEV0/drange1 =
// -cfv1 at the root (zero-sum payoffs), and for a node of player p
//   dEV0/dlogit_a(h) = sgn_p * reach_p(h) * sigma_a(h) * (cfv_p(child a, h) - cfv_p(node, h)),
// sgn_0 = +1, sgn_1 = -1.
__device__ __forceinline__ void softmax_groups(const float4* Lb, int H4, int g, int A, float4& mx, float4& den) {
    mx = Lb[g];
    for (int k = 1; k < A; ++k) {
        const float4 l = Lb[(size_t)k * H4 + g];
        mx = make_float4(fmaxf(mx.x, l.x), fmaxf(mx.y, l.y), fmaxf(mx.z, l.z), fmaxf(mx.w, l.w));
    }
    den = f4(0.f);
    for (int k = 0; k < A; ++k) {
        const float4 l = Lb[(size_t)k * H4 + g];
        den = add4(den, make_float4(expf(l.x - mx.x), expf(l.y - mx.y), expf(l.z - mx.z), expf(l.w - mx.w)));
    }
}
__device__ __forceinline__ float4 softmax_at(const float4* Lb, int H4, int g, int k, float4 mx, float4 den) {
    const float4 l = Lb[(size_t)k * H4 + g];
    return make_float4(__fdiv_rn(expf(l.x - mx.x), den.x), __fdiv_rn(expf(l.y - mx.y), den.y),
                       __fdiv_rn(expf(l.z - mx.z), den.z), __fdiv_rn(expf(l.w - mx.w), den.w));
}

__global__ void k_ev_init(SolveDev a, int n_sub) {
    const int s = blockIdx.x;
    if (s == 0 && threadIdx.x == 0) *a.err = 0;
    if (s >= n_sub) return;
    const SubDesc sd = a.desc[s];
    const int HS4 = (sd.Hp0 + sd.Hp1) >> 2;
    const float4* rg = reinterpret_cast<const float4*>(a.ranges + sd.range_base);
    float4* rr = reinterpret_cast<float4*>(a.arena + sd.arena_base);
    for (int i = threadIdx.x; i < HS4; i += blockDim.x) rr[i] = rg[i];
}

// Forward level: children's reach under softmax strategies; chance items as k_fwd.
__device__ __forceinline__ void k_ev_fwd_group(const SolveDev& a, const FwdItem& it, const int lane) {
    const float4* rp = reinterpret_cast<const float4*>(a.arena + it.reach_in);
    float4* ch = reinterpret_cast<float4*>(a.arena + it.child);
    const int A = it.na, H4 = it.h4, HS4 = it.hs4;
    const int g = it.g0 + lane;
    if (g >= H4) return;
    if (it.flags & FI_CHANCE) {
        const uint16_t* hc = a.hcards + it.hc;
        const float4 r = rp[g];
        const uint64_t m0 = hand_mask(hc[4 * g]), m1 = hand_mask(hc[4 * g + 1]);
        const uint64_t m2 = hand_mask(hc[4 * g + 2]), m3 = hand_mask(hc[4 * g + 3]);
        for (int k = 0; k < A; ++k) {
            const int card = a.nodes[it.first + k].dealt;
            float4 v = r;
            if ((m0 >> card) & 1ull) v.x = 0.f;
            if ((m1 >> card) & 1ull) v.y = 0.f;
            if ((m2 >> card) & 1ull) v.z = 0.f;
            if ((m3 >> card) & 1ull) v.w = 0.f;
            ch[(size_t)k * HS4 + g] = v;
        }
        return;
    }
    const float4* Lb = reinterpret_cast<const float4*>(a.R + it.rows);
    float4 mx, den;
    softmax_groups(Lb, H4, g, A, mx, den);
    const float4 r = rp[g];
    for (int k = 0; k < A; ++k) ch[(size_t)k * HS4 + g] = mul4(r, softmax_at(Lb, H4, g, k, mx, den));
}

// One warp per work item; the item covers span x 32 float4 hand groups.
template <int SPAN>
__global__ void __launch_bounds__(256) k_ev_fwd(SolveDev a, const FwdItem* __restrict__ items, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    const FwdItem it = items[w];
#pragma unroll
    for (int s = 0; s < SPAN; ++s) {
        if (SPAN > 1 && it.g0 + 32 * s >= it.h4) break;
        k_ev_fwd_group(a, it, (threadIdx.x & 31) + 32 * s);
    }
}

// Backward level: values of both players; the acting player's items also
// write the logit gradient.
__device__ __forceinline__ void k_ev_bwd_group(const SolveDev& a, const BwdItem& it, const int lane) {
    const float4* qc = reinterpret_cast<const float4*>(a.arena + it.child);
    float4* out = reinterpret_cast<float4*>(a.arena + it.self);
    const int A = it.na, H4 = it.h4, HS4 = it.hs4;
    const int g = it.g0 + lane;
    if (g >= H4) return;
    if (it.flags & BI_CHANCE) {
        const uint16_t* hc = a.hcards + it.hc;
        const float dv = it.div;
        const uint64_t m0 = hand_mask(hc[4 * g]), m1 = hand_mask(hc[4 * g + 1]);
        const uint64_t m2 = hand_mask(hc[4 * g + 2]), m3 = hand_mask(hc[4 * g + 3]);
        float4 acc = f4(0.f);
        for (int k = 0; k < A; ++k) {
            const int card = a.nodes[it.first + k].dealt;
            const float4 cv = qc[(size_t)k * HS4 + g];
            if (!((m0 >> card) & 1ull)) acc.x = __fadd_rn(acc.x, cv.x);
            if (!((m1 >> card) & 1ull)) acc.y = __fadd_rn(acc.y, cv.y);
            if (!((m2 >> card) & 1ull)) acc.z = __fadd_rn(acc.z, cv.z);
            if (!((m3 >> card) & 1ull)) acc.w = __fadd_rn(acc.w, cv.w);
        }
        out[g] = make_float4(__fdiv_rn(acc.x, dv), __fdiv_rn(acc.y, dv), __fdiv_rn(acc.z, dv), __fdiv_rn(acc.w, dv));
        return;
    }
    if (!(it.flags & BI_UPDATE)) {
        float4 so = f4(0.f);
        for (int k = 0; k < A; ++k) so = add4(so, qc[(size_t)k * HS4 + g]);
        out[g] = so;
        return;
    }
    const float4* Lb = reinterpret_cast<const float4*>(a.R + it.rows);
    float4* Gb = reinterpret_cast<float4*>(a.S + it.rows);
    float4 mx, den;
    softmax_groups(Lb, H4, g, A, mx, den);
    float4 v = f4(0.f);
    for (int k = 0; k < A; ++k) v = fma4(softmax_at(Lb, H4, g, k, mx, den), qc[(size_t)k * HS4 + g], v);
    out[g] = v;
    const float4 r = reinterpret_cast<const float4*>(a.arena + it.hc)[g];
    const float sgn = it.flags & BI_NEG ? -1.0f : 1.0f;
    const float4 sr = mul4(r, f4(sgn));
    for (int k = 0; k < A; ++k) {
        const float4 sg = softmax_at(Lb, H4, g, k, mx, den);
        const float4 d = make_float4(__fsub_rn(qc[(size_t)k * HS4 + g].x, v.x), __fsub_rn(qc[(size_t)k * HS4 + g].y, v.y),
                                     __fsub_rn(qc[(size_t)k * HS4 + g].z, v.z), __fsub_rn(qc[(size_t)k * HS4 + g].w, v.w));
        Gb[(size_t)k * H4 + g] = mul4(mul4(sr, sg), d);
    }
}

// One warp per work item; the item covers span x 32 float4 hand groups.
template <int SPAN>
__global__ void __launch_bounds__(256) k_ev_bwd(SolveDev a, const BwdItem* __restrict__ items, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    const BwdItem it = items[w];
#pragma unroll
    for (int s = 0; s < SPAN; ++s) {
        if (SPAN > 1 && it.g0 + 32 * s >= it.h4) break;
        k_ev_bwd_group(a, it, (threadIdx.x & 31) + 32 * s);
    }
}

// Root: EV0 = sum_h range0(h) cfv0(root, h) (accumulated in FP64), and the
// range gradients [cfv0 | -cfv1] in the packed range layout.
__global__ void __launch_bounds__(TT) k_ev_root(SolveDev a, int n_sub, float* __restrict__ ev,
                                               float* __restrict__ grad_ranges) {
    __shared__ double wb[TT / 32];
    const int s = blockIdx.x, tid = threadIdx.x;
    if (s >= n_sub) return;
    const SubDesc sd = a.desc[s];
    const int HS = sd.Hp0 + sd.Hp1;
    const float* cf = a.arena + sd.arena_base + (size_t)sd.n_nodes * HS;
    const float* rg = a.ranges + sd.range_base;
    double acc = 0.0;
    for (int h = tid; h < sd.H0; h += TT) acc += (double)rg[h] * (double)cf[h];
    for (int i = tid; i < HS; i += TT) grad_ranges[sd.range_base + i] = i < sd.Hp0 ? cf[i] : -cf[i];
    acc = cta_sum(acc, wb, tid);
    if (tid == 0) ev[s] = (float)acc;
}

// ------------------------------------------------------------- FP64 best response
// darena per subgame: reach | br | ev, each (n_nodes + 1) * HS doubles; the
// extra slot holds the compatible-mass values of the root.
__device__ __forceinline__ double avg_sigma(const float* Sb, int Hp, int k, int A, int h) {
    double sum = 0.0;
    for (int j = 0; j < A; ++j) sum += (double)Sb[(size_t)j * Hp + h];
    return sum > 0.0 ? (double)Sb[(size_t)k * Hp + h] / sum : 1.0 / (double)A;
}

__global__ void k_br_init(SolveDev a, const int* __restrict__ subs, int n_sub) {
    if ((int)blockIdx.x >= n_sub) return;
    const int s = subs[blockIdx.x];
    const SubDesc sd = a.desc[s];
    const int HS = sd.Hp0 + sd.Hp1;
    double* reach = a.darena + sd.darena_base;
    for (int i = threadIdx.x; i < HS; i += blockDim.x) reach[i] = (double)a.ranges[sd.range_base + i];
}

__global__ void __launch_bounds__(256) k_br_fwd(SolveDev a, const Task* __restrict__ tasks, int ntasks) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= ntasks) return;
    const Task tk = tasks[w];
    const SubDesc& sd = a.desc[tk.sub];
    const DNode nd = load_node(a.nodes + tk.node);
    const int g = tk.g0 + lane;
    const int HS = sd.Hp0 + sd.Hp1;
    double* reach = a.darena + sd.darena_base;
    if (nd.type == MTT_NODE_DECISION) {
        const int p = nd.player, A = nd.na, Hpp = HP(p);
        if (4 * g >= Hpp) return;
        const float* Sb = a.S + (p ? sd.rs_base1 : sd.rs_base0) + (size_t)nd.row * Hpp;
        const double* rp = reach + (size_t)SRC(nd, p) * HS + OFF(p);
        for (int i = 0; i < 4; ++i) {
            const int h = 4 * g + i;
            const double r = rp[h];
            for (int k = 0; k < A; ++k)
                reach[(size_t)(nd.first + k) * HS + OFF(p) + h] = r * avg_sigma(Sb, Hpp, k, A, h);
        }
    } else if (nd.type == MTT_NODE_CHANCE) {
        const DNode* nodes = a.nodes + sd.node_base;
        const uint16_t* hc = a.hcards + sd.hcard_base;
        for (int p = 0; p < 2; ++p) {
            if (4 * g >= HP(p)) continue;
            const double* rp = reach + (size_t)SRC(nd, p) * HS + OFF(p);
            for (int k = 0; k < nd.na; ++k) {
                const int card = nodes[nd.first + k].dealt;
                for (int i = 0; i < 4; ++i) {
                    const int h = 4 * g + i;
                    reach[(size_t)(nd.first + k) * HS + OFF(p) + h] =
                        ((hand_mask(hc[OFF(p) + h]) >> card) & 1ull) ? 0.0 : rp[h];
                }
            }
        }
    }
}

__global__ void __launch_bounds__(TT) k_br_term(SolveDev a, const int2* __restrict__ terms, int nterms) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ double wb[8];
    const int w = blockIdx.x;
    if (w >= nterms) return;
    const int2 tm = terms[w];
    const SubDesc& sd = a.desc[tm.y];
    const DNode nd = load_node(a.nodes + tm.x);
    const int nl = tm.x - (int)sd.node_base;
    const int HS = sd.Hp0 + sd.Hp1;
    const size_t reg = (size_t)(sd.n_nodes + 1) * HS;
    double* reach = a.darena + sd.darena_base;
    double* br = reach + reg;
    double* ev = br + reg;
    const TabView tv = tab_view(a.tabs + sd.tab_base + (size_t)nd.var * sd.tab_vsize, sd.H0, sd.H1);
    double* X = reinterpret_cast<double*>(smem);
    for (int q = 0; q < 2; ++q) {
        const int o = 1 - q;
        cta_terminal<double, double, double>(term_info(sd, nd), tv, q, reach + (size_t)SRC(nd, o) * HS + OFF(o),
                                             br + (size_t)nl * HS + OFF(q), ev + (size_t)nl * HS + OFF(q), X, wb,
                                             MTT_SEM_CORRECT, threadIdx.x);
    }
}

__global__ void __launch_bounds__(256) k_br_bwd(SolveDev a, const Task* __restrict__ tasks, int ntasks) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= ntasks) return;
    const Task tk = tasks[w];
    const SubDesc& sd = a.desc[tk.sub];
    const DNode nd = load_node(a.nodes + tk.node);
    const int nl = tk.node - (int)sd.node_base;
    const int g = tk.g0 + lane;
    const int HS = sd.Hp0 + sd.Hp1;
    const size_t reg = (size_t)(sd.n_nodes + 1) * HS;
    double* br = a.darena + sd.darena_base + reg;
    double* ev = br + reg;
    if (nd.type == MTT_NODE_DECISION) {
        const int p = nd.player, A = nd.na;
        for (int q = 0; q < 2; ++q) {
            const int Hpq = HP(q);
            if (4 * g >= Hpq) continue;
            const float* Sb = a.S + (p ? sd.rs_base1 : sd.rs_base0) + (size_t)nd.row * HP(p);
            for (int i = 0; i < 4; ++i) {
                const int h = 4 * g + i;
                double b = q == p ? -1e300 : 0.0, e = 0.0;
                for (int k = 0; k < A; ++k) {
                    const size_t c = (size_t)(nd.first + k) * HS + OFF(q) + h;
                    if (q == p) {
                        b = fmax(b, br[c]);
                        e += avg_sigma(Sb, HP(p), k, A, h) * ev[c];
                    } else {
                        b += br[c];
                        e += ev[c];
                    }
                }
                br[(size_t)nl * HS + OFF(q) + h] = b;
                ev[(size_t)nl * HS + OFF(q) + h] = e;
            }
        }
    } else if (nd.type == MTT_NODE_CHANCE) {
        const DNode* nodes = a.nodes + sd.node_base;
        const uint16_t* hc = a.hcards + sd.hcard_base;
        const double div = (double)(nd.nlive - 4);
        for (int q = 0; q < 2; ++q) {
            if (4 * g >= HP(q)) continue;
            for (int i = 0; i < 4; ++i) {
                const int h = 4 * g + i;
                const uint64_t m = hand_mask(hc[OFF(q) + h]);
                double sb = 0.0, se = 0.0;
                for (int k = 0; k < nd.na; ++k) {
                    const int card = nodes[nd.first + k].dealt;
                    if ((m >> card) & 1ull) continue;
                    const size_t c = (size_t)(nd.first + k) * HS + OFF(q) + h;
                    sb += br[c];
                    se += ev[c];
                }
                br[(size_t)nl * HS + OFF(q) + h] = sb / div;
                ev[(size_t)nl * HS + OFF(q) + h] = se / div;
            }
        }
    }
}

// One CTA per subgame: compatible range mass and the four root values.
__global__ void __launch_bounds__(TT) k_br_final(SolveDev a, const int* __restrict__ subs, int n_sub) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ double wb[8];
    const int tid = threadIdx.x;
    if ((int)blockIdx.x >= n_sub) return;
    const int s = subs[blockIdx.x];
    const SubDesc& sd = a.desc[s];
    const int HS = sd.Hp0 + sd.Hp1;
    const int nn = sd.n_nodes;
    const size_t reg = (size_t)(nn + 1) * HS;
    double* reach = a.darena + sd.darena_base;
    double* br = reach + reg;
    double* ev = br + reg;
    // Z: P0's hands against P1's range, a fold terminal with payoff 1
    DNode z{};
    z.type = MTT_NODE_FOLD;
    z.wmask = 1;
    z.pot = 1.0f;
    z.dealt = -1;
    const TabView tv = tab_view(a.tabs + sd.tab_base + (size_t)sd.var_none * sd.tab_vsize, sd.H0, sd.H1);
    double* X = reinterpret_cast<double*>(smem);
    double* zm = br + (size_t)nn * HS;
    cta_terminal<double, double, double>(term_info(sd, z), tv, 0, reach + OFF(1), zm, nullptr, X, wb,
                                         MTT_SEM_CORRECT, tid);
    double acc[5] = {0, 0, 0, 0, 0};
    for (int h = tid; h < sd.H0; h += TT) {
        const double r = reach[h];
        acc[0] += r * br[h];
        acc[2] += r * ev[h];
        acc[4] += r * zm[h];
    }
    for (int h = tid; h < sd.H1; h += TT) {
        const double r = reach[OFF(1) + h];
        acc[1] += r * br[OFF(1) + h];
        acc[3] += r * ev[OFF(1) + h];
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) acc[k] = cta_sum(acc[k], wb, tid);
    if (tid == 0) {
        const double Z = acc[4] > 0.0 ? acc[4] : 1.0;
        double* o = a.results + (size_t)s * 6;
        o[0] = acc[0] / Z;
        o[1] = acc[1] / Z;
        o[2] = acc[2] / Z;
        o[3] = acc[3] / Z;
        o[4] = acc[4];
        o[5] = 0.5 * (o[0] + o[1]) / (double)sd.pot;
    }
}

#undef HP
#undef HH
#undef OFF
#undef SRC

#include "solver_pack.cuh"

template <typename T>
struct LevelLists {                  // work lists per depth, concatenated on the device
    T* d = nullptr;
    long long cap = 0;               // allocated entries
    std::vector<long long> off;      // size levels + 1
};

// Host copies of every work list, built once per batch.  The continuation
// rounds of a gate-enforced solve upload the part that belongs to the
// subgames still above the exploitability target.
struct HostLists {
    std::vector<std::vector<FwdItem>> fi, fsim, fal[2];
    std::vector<std::vector<BwdItem>> bsim, bal[2];
    std::vector<std::vector<Task>> bf, bb;
    std::vector<TermItem> titems;    // by subgame, then table variant
    std::vector<int2> terms;
};

struct ListSet {
    LevelLists<FwdItem> f_init, f_sim, f_alt[2];
    LevelLists<BwdItem> b_sim, b_alt[2];
    LevelLists<Task> br_fwd, br_bwd;
    TermItem* titems = nullptr;
    long long titems_cap = 0;
    int2* terms = nullptr;
    long long terms_cap = 0;
    int n_terms = 0;
    TermGroup* tgroups = nullptr;
    long long tgroups_cap = 0;
    std::vector<int> tb_start, tb_count;             // terminal-group buckets: offset, size
    std::vector<int> tb_smem1, tb_smem3;             // shared bytes: one direction / both
    int* subs = nullptr;
    long long subs_cap = 0;
    int n_subs = 0;
};

}  // namespace mtt

using namespace mtt;

// ====================================================================== host driver
struct mtt_batch {
    int n = 0;
    // the streams this batch's work was issued on, each with an event
    // recorded after its last call; destroy waits on these, not the device
    std::vector<std::pair<cudaStream_t, cudaEvent_t>> used;
    SubDesc* d_desc = nullptr;
    DNode* d_nodes = nullptr;
    uint8_t* d_tabs = nullptr;
    uint16_t* d_hcards = nullptr;
    float* d_ranges = nullptr;
    float* d_arena = nullptr;
    float* d_R = nullptr;
    float* d_S = nullptr;
    double* d_darena = nullptr;
    double* d_results = nullptr;
    int* d_iter = nullptr;
    int* d_err = nullptr;             // bounded-wait error word of the staged kernels
    float* d_iter_tab = nullptr;
    int iter_cap = 0;
    int levels = 0;
    HostLists host;
    ListSet full, act;
    std::vector<SubDesc> desc;
    std::vector<int> iters_done;
    int max_h = 0;
    long long device_bytes = 0, iter_bytes = 0;
    int tuned_threads = 0;
    cudaGraphExec_t gexec = nullptr;   // one iteration over the full lists
    int gkernels = 0;                  // kernel nodes in gexec
    mtt_solve_params gparams{};
    int gthreads = 0;
    mutable long long launches = 0;    // kernels run for this batch (graph replays count every node)
    // depth-limit leaves (turn subgames built with river_leaves)
    std::vector<mtt::LeafItem> h_leaves;
    mtt::LeafItem* d_leaves = nullptr;
    int n_leaves = 0;
    bool leaf_ready = false;           // mtt_batch_set_leafnet was called
    mtt_leafnet* net = nullptr;
    bool leaf_residual = false;
    float *d_lx = nullptr, *d_ly = nullptr, *d_lm = nullptr, *d_lsd = nullptr;
    int leaf_sd_stride = 0;            // floats per (row, player) of d_lsd
    int leaf_smem = 0;                 // dynamic shared memory of k_leaf_showdown
    // schedule (mtt_batch_set_schedule / the autotuner): 32 x span float4
    // hand groups per sweep work item, at most tchunk terminals per CTA
    int span = 1;
    int tchunk = mtt::TG_CHUNK;
};

namespace mtt {
// Batch memory comes from a library-owned stream-ordered pool per device
// that keeps what batches free (no release threshold), so the next batch of
// a similar size allocates without the driver mapping fresh pages: a 22 GB
// batch created right after another was freed spent 0.3 s in cudaMalloc.
// mtt_trim_pool hands the kept memory back.  Allocations and frees are
// ordered on the legacy default stream; every free waits for the device
// first, as cudaFree does.
static cudaMemPool_t batch_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = p;
    }
    return pools[dev];
}

template <typename T>
static int dalloc(T** p, size_t count, long long& total) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaMemPool_t pool = batch_pool();
    if (pool) {
        MTT_TRY_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, 0));
        MTT_TRY_CUDA(cudaStreamSynchronize(0));
    } else {
        MTT_TRY_CUDA(cudaMalloc(reinterpret_cast<void**>(p), bytes));
    }
    total += (long long)bytes;
    return MTT_OK;
}

// Frees pool (or plain) allocations; the caller has waited for the device.
static void dfree(void* p) {
    if (p) cudaFreeAsync(p, 0);
}

static void free_set(ListSet& L) {
    dfree(L.f_init.d); dfree(L.f_sim.d); dfree(L.b_sim.d);
    for (int u = 0; u < 2; ++u) { dfree(L.f_alt[u].d); dfree(L.b_alt[u].d); }
    dfree(L.br_fwd.d); dfree(L.br_bwd.d); dfree(L.titems); dfree(L.terms); dfree(L.subs);
    dfree(L.tgroups);
}

// Waits for the batch's own work (the events of the streams it ran on; its
// uploads and allocations are synchronous on the legacy stream), not for the
// whole device: another host thread may be creating the next batch.  The
// frees are ordered on the legacy stream, after which the pool hands the
// memory out again.
static void free_batch(mtt_batch* b) {
    if (!b) return;
    for (auto& u : b->used) {
        cudaEventSynchronize(u.second);
        cudaEventDestroy(u.second);
    }
    b->used.clear();
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    dfree(b->d_desc); dfree(b->d_nodes); dfree(b->d_tabs); dfree(b->d_hcards);
    dfree(b->d_ranges); dfree(b->d_arena); dfree(b->d_R); dfree(b->d_S);
    dfree(b->d_darena); dfree(b->d_results); dfree(b->d_iter);
    dfree(b->d_iter_tab);
    dfree(b->d_err);
    dfree(b->d_leaves); dfree(b->d_lx); dfree(b->d_ly); dfree(b->d_lm); dfree(b->d_lsd);
    free_set(b->full);
    free_set(b->act);
    delete b;
}

// Record that work of the batch was issued on st (after the call's last launch).
static void note_stream(mtt_batch* b, cudaStream_t st) {
    for (auto& u : b->used)
        if (u.first == st) { cudaEventRecord(u.second, st); return; }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
        cudaStreamSynchronize(st);   // no event: wait here instead
        return;
    }
    cudaEventRecord(e, st);
    b->used.emplace_back(st, e);
}

template <typename T>
static int grow(T** d, long long* cap, long long need, long long& total) {
    if (need <= *cap && *d) return MTT_OK;
    if (*d) {
        MTT_TRY_CUDA(cudaDeviceSynchronize());
        dfree(*d);
    }
    *d = nullptr;
    *cap = 0;
    MTT_TRY(dalloc(d, (size_t)std::max(need, 1LL), total));
    *cap = std::max(need, 1LL);
    return MTT_OK;
}

// Upload the per-depth lists, keeping the entries whose subgame is active
// (all when `active` is null).
template <typename T, typename Keep>
static int upload_levels(LevelLists<T>& L, const std::vector<std::vector<T>>& lv, bool all, Keep keep,
                         long long& total) {
    L.off.assign(lv.size() + 1, 0);
    if (all) {   // every item: each level straight from its host vector
        for (size_t d = 0; d < lv.size(); ++d) L.off[d + 1] = L.off[d] + (long long)lv[d].size();
        MTT_TRY(grow(&L.d, &L.cap, L.off.back(), total));
        for (size_t d = 0; d < lv.size(); ++d)
            if (!lv[d].empty())
                MTT_TRY_CUDA(cudaMemcpy(L.d + L.off[d], lv[d].data(), sizeof(T) * lv[d].size(), cudaMemcpyHostToDevice));
        return MTT_OK;
    }
    std::vector<T> flat;
    for (size_t d = 0; d < lv.size(); ++d) {
        for (const T& x : lv[d])
            if (keep(x)) flat.push_back(x);
        L.off[d + 1] = (long long)flat.size();
    }
    MTT_TRY(grow(&L.d, &L.cap, (long long)flat.size(), total));
    if (!flat.empty()) MTT_TRY_CUDA(cudaMemcpy(L.d, flat.data(), sizeof(T) * flat.size(), cudaMemcpyHostToDevice));
    return MTT_OK;
}

static int build_set(mtt_batch* b, ListSet& L, const std::vector<char>* active, long long& total) {
    const HostLists& H = b->host;
    // the host lists hold one item per 32 float4 groups; a span of k keeps
    // every k-th (the kernels then walk 32 k groups per item)
    const int span = b->span;
    auto fkeep = [&](const FwdItem& x) { return (!active || (*active)[x.sub]) && (x.g0 / 32) % span == 0; };
    auto bkeep = [&](const BwdItem& x) { return (!active || (*active)[x.sub]) && (x.g0 / 32) % span == 0; };
    auto tkeep = [&](const Task& x) { return !active || (*active)[x.sub]; };
    const bool all_sweep = !active && span == 1;
    MTT_TRY(upload_levels(L.f_init, H.fi, all_sweep, fkeep, total));
    MTT_TRY(upload_levels(L.f_sim, H.fsim, all_sweep, fkeep, total));
    MTT_TRY(upload_levels(L.b_sim, H.bsim, all_sweep, bkeep, total));
    for (int u = 0; u < 2; ++u) {
        MTT_TRY(upload_levels(L.f_alt[u], H.fal[u], all_sweep, fkeep, total));
        MTT_TRY(upload_levels(L.b_alt[u], H.bal[u], all_sweep, bkeep, total));
    }
    MTT_TRY(upload_levels(L.br_fwd, H.bf, !active, tkeep, total));
    MTT_TRY(upload_levels(L.br_bwd, H.bb, !active, tkeep, total));
    std::vector<TermItem> ti;
    std::vector<int2> tm;
    std::vector<int> subs;
    for (const TermItem& t : H.titems) if (!active || (*active)[t.sub]) ti.push_back(t);
    for (const int2& t : H.terms) if (!active || (*active)[t.y]) tm.push_back(t);
    for (int i = 0; i < b->n; ++i) if (!active || (*active)[i]) subs.push_back(i);
    MTT_TRY(grow(&L.titems, &L.titems_cap, (long long)ti.size(), total));
    MTT_TRY(grow(&L.terms, &L.terms_cap, (long long)tm.size(), total));
    MTT_TRY(grow(&L.subs, &L.subs_cap, (long long)subs.size(), total));
    if (!ti.empty()) MTT_TRY_CUDA(cudaMemcpy(L.titems, ti.data(), sizeof(TermItem) * ti.size(), cudaMemcpyHostToDevice));
    if (!tm.empty()) MTT_TRY_CUDA(cudaMemcpy(L.terms, tm.data(), sizeof(int2) * tm.size(), cudaMemcpyHostToDevice));
    if (!subs.empty()) MTT_TRY_CUDA(cudaMemcpy(L.subs, subs.data(), sizeof(int) * subs.size(), cudaMemcpyHostToDevice));
    L.n_terms = (int)tm.size();
    L.n_subs = (int)subs.size();
    // Terminal groups: runs of items with the same subgame and table variant
    // (the host list is ordered that way), cut into chunks.  A CTA walks its
    // chunk's terminals one after another, so small batches (a single
    // subgame, the few still above the exploitability gate) get short chunks
    // and spread over the SMs: about 4 chunks per SM and CTA slot, TG_CHUNK
    // at most.
    int sm_count = 148;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
    }
    const long long slots = 4LL * 5 * std::max(sm_count, 1);   // 5 CTAs per SM
    const int chunk = (int)std::max(1LL, std::min<long long>(b->tchunk, (long long)ti.size() / slots));
    std::vector<TermGroup> gr;
    for (int i = 0; i < (int)ti.size();) {
        int j = i + 1;
        while (j < (int)ti.size() && j - i < chunk && ti[j].sub == ti[i].sub && ti[j].tab == ti[i].tab) ++j;
        TermGroup g{};
        g.tab = ti[i].tab;
        g.first = i;
        g.count = j - i;
        g.H0 = ti[i].H[0]; g.H1 = ti[i].H[1]; g.Hp0 = ti[i].Hp[0]; g.Hp1 = ti[i].Hp[1];
        gr.push_back(g);
        i = j;
    }
    // Buckets: ascending hand count, three equal-count launches whose shared
    // memory is sized by their largest group; inside a bucket the costliest
    // groups go first so that the last wave is made of short ones.  Groups
    // that all fit in one wave at the largest group's shared memory (a single
    // subgame, the few still above the exploitability gate) take one launch:
    // the buckets' launches run one after another, each as long as its
    // slowest CTA.
    std::stable_sort(gr.begin(), gr.end(), [](const TermGroup& x, const TermGroup& y) {
        return std::max(x.Hp0, x.Hp1) < std::max(y.Hp0, y.Hp1);
    });
    L.tb_start.clear(); L.tb_count.clear(); L.tb_smem1.clear(); L.tb_smem3.clear();
    int all1 = 0, all3 = 0;
    for (const TermGroup& g : gr) {
        all1 = std::max(all1, std::max(tg_smem_bytes(g.H0, g.H1, g.Hp0, g.Hp1, 1),
                                       tg_smem_bytes(g.H0, g.H1, g.Hp0, g.Hp1, 2)));
        all3 = std::max(all3, tg_smem_bytes(g.H0, g.H1, g.Hp0, g.Hp1, 3));
    }
    // CTAs per SM at a dynamic shared-memory size: 228 KB per SM, 4 KB a CTA
    // for its static shared memory and the system's reserve, 5 at most (registers)
    auto per_sm = [](int dyn) { return std::max(1, std::min(5, (228 * 1024) / (dyn + 4 * 1024))); };
    const long long wave = (long long)std::min(per_sm(all1), per_sm(all3)) * std::max(sm_count, 1);
    const int ng = (int)gr.size(), nb = ng < 3 || ng <= wave ? 1 : 3;
    for (int k = 0; k < nb; ++k) {
        const int lo = (int)((long long)ng * k / nb), hi = (int)((long long)ng * (k + 1) / nb);
        std::stable_sort(gr.begin() + lo, gr.begin() + hi, [](const TermGroup& x, const TermGroup& y) {
            return (long long)x.count * (x.H0 + x.H1) > (long long)y.count * (y.H0 + y.H1);
        });
        int need1 = 0, need3 = 0;
        for (int i = lo; i < hi; ++i) {
            const TermGroup& g = gr[i];
            need1 = std::max(need1, tg_smem_bytes(g.H0, g.H1, g.Hp0, g.Hp1, 1));
            need1 = std::max(need1, tg_smem_bytes(g.H0, g.H1, g.Hp0, g.Hp1, 2));
            need3 = std::max(need3, tg_smem_bytes(g.H0, g.H1, g.Hp0, g.Hp1, 3));
        }
        L.tb_start.push_back(lo);
        L.tb_count.push_back(hi - lo);
        L.tb_smem1.push_back(need1);
        L.tb_smem3.push_back(need3);
    }
    MTT_TRY(grow(&L.tgroups, &L.tgroups_cap, (long long)gr.size(), total));
    if (!gr.empty()) MTT_TRY_CUDA(cudaMemcpy(L.tgroups, gr.data(), sizeof(TermGroup) * gr.size(), cudaMemcpyHostToDevice));
    return MTT_OK;
}

// Per-iteration scalars (strategy-sum weight t^avg_power, DCFR positive and
// negative regret discounts, DCFR strategy-sum discount), computed on the
// host in double exactly as the oracle does.
static int fill_iter_table(mtt_batch* b, const mtt_solve_params& p, int iters, cudaStream_t st) {
    if (iters > b->iter_cap || !b->d_iter_tab) {
        if (b->d_iter_tab) { MTT_TRY_CUDA(cudaStreamSynchronize(st)); dfree(b->d_iter_tab); b->d_iter_tab = nullptr; }
        long long unused = 0;
        MTT_TRY(dalloc(&b->d_iter_tab, 4 * (size_t)std::max(iters, 1), unused));
        b->iter_cap = std::max(iters, 1);
        if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }   // captured the old table
    }
    std::vector<float> tab(4 * (size_t)std::max(iters, 1), 0.0f);
    for (int t = 1; t <= iters; ++t) {
        const double tm1 = (double)(t - 1);
        float* e = &tab[4 * (size_t)(t - 1)];
        e[0] = (float)std::pow((double)t, (double)p.avg_power);
        e[1] = (float)(std::pow(tm1, (double)p.alpha) / (std::pow(tm1, (double)p.alpha) + 1.0));
        e[2] = (float)(std::pow(tm1, (double)p.beta) / (std::pow(tm1, (double)p.beta) + 1.0));
        e[3] = (float)std::pow(tm1 / (double)t, (double)p.gamma);
    }
    // pageable source: the copy is staged before this returns
    MTT_TRY_CUDA(cudaMemcpyAsync(b->d_iter_tab, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
    return MTT_OK;
}

static SolveDev dev_args(const mtt_batch* b, const mtt_solve_params& p) {
    SolveDev a;
    a.desc = b->d_desc; a.nodes = b->d_nodes; a.tabs = b->d_tabs; a.hcards = b->d_hcards; a.ranges = b->d_ranges;
    a.arena = b->d_arena; a.R = b->d_R; a.S = b->d_S; a.darena = b->d_darena; a.results = b->d_results;
    a.iter_tab = b->d_iter_tab; a.iter = b->d_iter; a.err = b->d_err; a.algo = p.algo; a.semantics = p.semantics;
    a.span = b->span;
    return a;
}

static int term_xstride(const mtt_batch* b) { return term_scratch(b->max_h); }

// Launches after the first of a kernel class (forward levels, terminal
// groups, backward levels) are chained with programmatic stream
// serialization: their CTAs are scheduled during the previous launch's tail
// and read their work items before grid_dep_wait.  The first launch of each
// class is ordinary.  Chaining across classes as well measured 5% slower per
// iteration on the 4,096-subgame batch (backward CTAs then start on SMs still
// set up for the terminal kernel's shared memory); chaining within classes
// measured 0.3% faster.
// sums: the lists add to the strategy sums (simultaneous-update forward
// lists, alternating-update backward lists).
static int launch_levels_fwd(const mtt_batch* b, const SolveDev& a, const LevelLists<FwdItem>& L, int threads,
                             bool sums, cudaStream_t st) {
    const long long warps = threads / 32;
    bool chained = false;
    for (int d = 0; d < b->levels; ++d) {
        const long long n = L.off[d + 1] - L.off[d];
        if (n == 0) continue;
        using K = void (*)(SolveDev, const FwdItem*, int);
        const bool dc = a.algo == MTT_ALGO_DCFR;
        // reach-only lists do not depend on the update rule
        const K k = a.span == 2 ? (!sums ? k_fwd<2, MTT_ALGO_CFRPLUS, false>
                                   : dc  ? k_fwd<2, MTT_ALGO_DCFR, true>
                                         : k_fwd<2, MTT_ALGO_CFRPLUS, true>)
                                : (!sums ? k_fwd<1, MTT_ALGO_CFRPLUS, false>
                                   : dc  ? k_fwd<1, MTT_ALGO_DCFR, true>
                                         : k_fwd<1, MTT_ALGO_CFRPLUS, true>);
        MTT_TRY_CUDA(launch_pdl(k, (unsigned)((n + warps - 1) / warps), threads, 0, st, chained, a,
                                (const FwdItem*)(L.d + L.off[d]), (int)n));
        MTT_CHECK_LAUNCH();
        ++b->launches;
        chained = true;
    }
    return MTT_OK;
}

static int launch_levels_bwd(const mtt_batch* b, const SolveDev& a, const LevelLists<BwdItem>& L, int threads,
                             bool sums, cudaStream_t st) {
    const long long warps = threads / 32;
    bool chained = false;
    for (int d = b->levels - 1; d >= 0; --d) {
        const long long n = L.off[d + 1] - L.off[d];
        if (n == 0) continue;
        using K = void (*)(SolveDev, const BwdItem*, int);
        const bool dc = a.algo == MTT_ALGO_DCFR;
        static const K ks[2][2][2] = {   // [span - 1][dcfr][sums]
            {{k_bwd<1, MTT_ALGO_CFRPLUS, false>, k_bwd<1, MTT_ALGO_CFRPLUS, true>},
             {k_bwd<1, MTT_ALGO_DCFR, false>, k_bwd<1, MTT_ALGO_DCFR, true>}},
            {{k_bwd<2, MTT_ALGO_CFRPLUS, false>, k_bwd<2, MTT_ALGO_CFRPLUS, true>},
             {k_bwd<2, MTT_ALGO_DCFR, false>, k_bwd<2, MTT_ALGO_DCFR, true>}}};
        const K k = ks[a.span == 2 ? 1 : 0][dc ? 1 : 0][sums ? 1 : 0];
        MTT_TRY_CUDA(launch_pdl(k, (unsigned)((n + warps - 1) / warps), threads, 0, st, chained, a,
                                (const BwdItem*)(L.d + L.off[d]), (int)n));
        MTT_CHECK_LAUNCH();
        ++b->launches;
        chained = true;
    }
    return MTT_OK;
}

using TermKernel = void (*)(SolveDev, const TermGroup*, const TermItem*, int);
static TermKernel term_kernel(int upd, int semantics) {
    static const TermKernel k[2][3] = {
        {k_term<1, MTT_SEM_CORRECT>, k_term<2, MTT_SEM_CORRECT>, k_term<3, -1>},
        {k_term<1, MTT_SEM_REFERENCE>, k_term<2, MTT_SEM_REFERENCE>, k_term<3, -1>}};
    return k[semantics ? 1 : 0][upd - 1];
}

static int launch_term(const mtt_batch* b, const ListSet& L, const SolveDev& a, int upd, cudaStream_t st) {
    bool chained = false;
    for (size_t k = 0; k < L.tb_start.size(); ++k) {
        if (L.tb_count[k] == 0) continue;
        const int smem = upd == 3 ? L.tb_smem3[k] : L.tb_smem1[k];
        MTT_TRY_CUDA(launch_pdl(term_kernel(upd, a.semantics), (unsigned)L.tb_count[k], TG, smem, st, chained, a,
                                (const TermGroup*)(L.tgroups + L.tb_start[k]), (const TermItem*)L.titems,
                                L.tb_count[k]));
        MTT_CHECK_LAUNCH();
        ++b->launches;
        chained = true;
    }
    return MTT_OK;
}

// Depth-limit leaves of the updated players `upd`: the network's rows and
// forward pass (with a network), the check-down values (unless the network
// alone values them), then the leaf values.
static int launch_leaves(const mtt_batch* b, const SolveDev& a, int upd, cudaStream_t st) {
    if (!b->n_leaves) return MTT_OK;
    const int rows = LEAF_RIVERS * b->n_leaves;
    if (b->net) {
        k_leaf_rows<<<rows, 256, 0, st>>>(a, b->d_leaves, b->d_lx, b->d_lm);
        MTT_CHECK_LAUNCH();
        ++b->launches;
        MTT_TRY(mtt_leafnet_forward(b->net, b->d_lx, rows, b->d_ly, (void*)st));
        b->launches += 5;   // feature packing and four GEMMs
    }
    const bool cd = b->leaf_residual || !b->net;
    if (cd) {
        k_leaf_showdown<<<rows, TG, b->leaf_smem, st>>>(a, b->d_leaves, b->d_lsd, b->leaf_sd_stride, upd);
        MTT_CHECK_LAUNCH();
        ++b->launches;
    }
    const float div = (float)(LEAF_RIVERS - 4 + (a.semantics ? 2 : 0));
    const dim3 lv_grid((unsigned)b->n_leaves, (unsigned)((b->leaf_sd_stride + LV_HANDS - 1) / LV_HANDS));
    k_leaf_values<<<lv_grid, LV_HANDS, 0, st>>>(a, b->d_leaves, cd ? b->d_lsd : nullptr, b->leaf_sd_stride,
                                               b->net ? b->d_ly : nullptr, b->d_lm, upd, div);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    return MTT_OK;
}

// One CFR iteration: per pass forward levels, leaves, terminals, backward levels.
static int launch_iteration(const mtt_batch* b, const ListSet& L, const SolveDev& a, const mtt_solve_params& p,
                            int threads, cudaStream_t st) {
    if (p.alternate) {
        for (int u = 0; u < 2; ++u) {
            MTT_TRY(launch_levels_fwd(b, a, L.f_alt[u], threads, false, st));
            MTT_TRY(launch_leaves(b, a, 1 << u, st));
            MTT_TRY(launch_term(b, L, a, 1 << u, st));
            MTT_TRY(launch_levels_bwd(b, a, L.b_alt[u], threads, true, st));
        }
    } else {
        MTT_TRY(launch_levels_fwd(b, a, L.f_sim, threads, true, st));
        MTT_TRY(launch_leaves(b, a, 3, st));
        MTT_TRY(launch_term(b, L, a, 3, st));
        MTT_TRY(launch_levels_bwd(b, a, L.b_sim, threads, false, st));
    }
    k_next_iter<<<1, 32, 0, st>>>(a);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    return MTT_OK;
}

static int launch_br(const mtt_batch* b, const ListSet& L, const SolveDev& a, int threads, cudaStream_t st) {
    if (L.n_subs == 0) return MTT_OK;
    const long long warps = threads / 32;
    k_br_init<<<L.n_subs, 128, 0, st>>>(a, L.subs, L.n_subs);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    for (int d = 0; d < b->levels; ++d) {
        const long long n = L.br_fwd.off[d + 1] - L.br_fwd.off[d];
        if (n == 0) continue;
        k_br_fwd<<<(unsigned)((n + warps - 1) / warps), threads, 0, st>>>(a, L.br_fwd.d + L.br_fwd.off[d], (int)n);
        MTT_CHECK_LAUNCH();
        ++b->launches;
    }
    const size_t smem = sizeof(double) * (size_t)term_xstride(b);
    if (L.n_terms) {
        k_br_term<<<L.n_terms, TT, smem, st>>>(a, L.terms, L.n_terms);
        MTT_CHECK_LAUNCH();
        ++b->launches;
    }
    for (int d = b->levels - 1; d >= 0; --d) {
        const long long n = L.br_bwd.off[d + 1] - L.br_bwd.off[d];
        if (n == 0) continue;
        k_br_bwd<<<(unsigned)((n + warps - 1) / warps), threads, 0, st>>>(a, L.br_bwd.d + L.br_bwd.off[d], (int)n);
        MTT_CHECK_LAUNCH();
        ++b->launches;
    }
    k_br_final<<<L.n_subs, TT, smem, st>>>(a, L.subs, L.n_subs);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    return MTT_OK;
}

static int set_smem_attrs(const mtt_batch* b, const ListSet& L) {
    const size_t t = sizeof(double) * (size_t)term_xstride(b);
    if (t > 48 * 1024) {
        MTT_TRY_CUDA(cudaFuncSetAttribute(k_br_term, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t));
        MTT_TRY_CUDA(cudaFuncSetAttribute(k_br_final, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t));
    }
    int tmax = 0;
    for (int v : L.tb_smem1) tmax = std::max(tmax, v);
    for (int v : L.tb_smem3) tmax = std::max(tmax, v);
    if (tmax > 48 * 1024) {
        for (int sem = 0; sem < 2; ++sem)
            for (int upd = 1; upd <= 3; ++upd)
                MTT_TRY_CUDA(cudaFuncSetAttribute(term_kernel(upd, sem), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  tmax));
    }
    return MTT_OK;
}

static int check_params(const mtt_solve_params* p) {
    if (!p || p->iters < 0 || (p->algo != MTT_ALGO_CFRPLUS && p->algo != MTT_ALGO_DCFR) ||
        (p->semantics != MTT_SEM_CORRECT && p->semantics != MTT_SEM_REFERENCE) || p->alternate < 0 ||
        p->alternate > 1 || !(p->avg_power >= 0.0f && p->avg_power <= 8.0f) || !(p->target_expl >= 0.0f) ||
        p->max_iters < 0 || p->chunk_iters < 0)
        return MTT_ERR_INVALID;
    if (p->threads != 0 && p->threads != 64 && p->threads != 128 && p->threads != 256) return MTT_ERR_INVALID;
    return MTT_OK;
}

// Captures one iteration; *kernels = the kernel nodes it holds (captured
// launches do not run, so they are taken back out of the launch count).
static int capture_iteration(const mtt_batch* b, const ListSet& L, const SolveDev& a, const mtt_solve_params& p,
                             int threads, cudaGraphExec_t* out, int* kernels) {
    const long long before = b->launches;
    cudaStream_t cs;
    MTT_TRY_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    int s = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    if (!s) s = launch_iteration(b, L, a, p, threads, cs);
    const int s2 = cuda_status(cudaStreamEndCapture(cs, &g));
    if (!s) s = s2;
    if (!s) s = cuda_status(cudaGraphInstantiate(out, g, 0));
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    *kernels = (int)(b->launches - before);
    b->launches = before;
    return s;
}

static int run_iterations(mtt_batch* b, const ListSet& L, const SolveDev& a, const mtt_solve_params& p, int threads,
                          int iters, bool graph, bool cached, cudaStream_t st) {
    if (!graph) {
        for (int t = 0; t < iters; ++t) MTT_TRY(launch_iteration(b, L, a, p, threads, st));
        return MTT_OK;
    }
    if (cached) {
        // the graph reads the iteration table, refilled per solve, so only the launch shape matters
        const bool same = b->gexec && b->gthreads == threads && b->gparams.algo == p.algo &&
                          b->gparams.semantics == p.semantics && b->gparams.alternate == p.alternate;
        if (!same) {
            if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
            MTT_TRY(capture_iteration(b, L, a, p, threads, &b->gexec, &b->gkernels));
            b->gparams = p;
            b->gthreads = threads;
        }
        for (int t = 0; t < iters; ++t) {
            MTT_TRY_CUDA(cudaGraphLaunch(b->gexec, st));
            b->launches += b->gkernels;
        }
        return MTT_OK;
    }
    cudaGraphExec_t ge = nullptr;
    int kernels = 0;
    MTT_TRY(capture_iteration(b, L, a, p, threads, &ge, &kernels));
    int s = MTT_OK;
    for (int t = 0; t < iters && !s; ++t) {
        s = cuda_status(cudaGraphLaunch(ge, st));
        if (!s) b->launches += kernels;
    }
    cudaGraphExecDestroy(ge);
    return s;
}

static int run_solve(mtt_batch* b, const mtt_solve_params& p, cudaStream_t st, bool graph) {
    if (b->n_leaves && !b->leaf_ready) return MTT_ERR_INVALID;        // leaf values undefined
    if (b->n_leaves && p.exploitability) return MTT_ERR_UNSUPPORTED;  // no best response through leaves
    const int threads = p.threads ? p.threads : (b->tuned_threads ? b->tuned_threads : 256);
    const bool gate = p.exploitability && p.target_expl > 0.0f && p.max_iters > p.iters;
    const int chunk = p.chunk_iters > 0 ? p.chunk_iters : std::max(p.iters / 2, 1);
    MTT_TRY(set_smem_attrs(b, b->full));
    MTT_TRY(fill_iter_table(b, p, gate ? p.max_iters : p.iters, st));
    const SolveDev a = dev_args(b, p);
    k_init<<<b->n, 256, 0, st>>>(a, b->n);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    MTT_TRY(launch_levels_fwd(b, a, b->full.f_init, threads, false, st));
    MTT_TRY(run_iterations(b, b->full, a, p, threads, p.iters, graph, true, st));
    std::fill(b->iters_done.begin(), b->iters_done.end(), p.iters);
    if (p.exploitability) MTT_TRY(launch_br(b, b->full, a, threads, st));
    if (!gate) return MTT_OK;
    // Gate: subgames still above the target keep iterating, in chunks, on
    // work lists compacted to them, until they pass or reach max_iters.
    std::vector<double> res(6 * (size_t)b->n);
    int done = p.iters;
    long long scratch = 0;
    while (done < p.max_iters) {
        MTT_TRY_CUDA(cudaMemcpyAsync(res.data(), b->d_results, sizeof(double) * res.size(), cudaMemcpyDeviceToHost, st));
        MTT_TRY_CUDA(cudaStreamSynchronize(st));
        std::vector<char> active(b->n, 0);
        int n_act = 0;
        for (int i = 0; i < b->n; ++i)
            if (!(res[6 * (size_t)i + 5] <= (double)p.target_expl)) { active[i] = 1; ++n_act; }
        if (n_act == 0) break;
        MTT_TRY(build_set(b, b->act, &active, scratch));
        MTT_TRY(set_smem_attrs(b, b->act));
        const int it = std::min(chunk, p.max_iters - done);
        MTT_TRY(run_iterations(b, b->act, a, p, threads, it, graph, false, st));
        for (int i = 0; i < b->n; ++i) if (active[i]) b->iters_done[i] += it;
        done += it;
        MTT_TRY(launch_br(b, b->act, a, threads, st));
    }
    return MTT_OK;
}
// Compulsory bytes of one work item: every element it reads or writes,
// counted once (the second read of a regret row hits L1).  g: float4 groups
// the item's warp covers.
static double fwd_item_bytes(const FwdItem& it, int span) {
    if ((it.g0 / 32) % span) return 0.0;   // covered by the item span groups before it
    const double g = (double)std::min(32 * span, it.h4 - it.g0), row = 16.0 * g, A = it.na;
    if (it.flags & FI_CHANCE) return row * (1.0 + A) + 8.0 * g;       // reach, children, hand cards
    return row * (1.0 + A + ((it.flags & FI_REACH) ? A : 0.0) + ((it.flags & FI_SUMS) ? 2.0 * A : 0.0));
}
static double bwd_item_bytes(const BwdItem& it, int span) {
    if ((it.g0 / 32) % span) return 0.0;
    const double g = (double)std::min(32 * span, it.h4 - it.g0), row = 16.0 * g, A = it.na;
    if (it.flags & BI_CHANCE) return row * (A + 1.0) + 8.0 * g;       // children, value, hand cards
    if (!(it.flags & BI_UPDATE)) return row * (A + 1.0);
    // regret rows read and written, children read, value written; sums: reach and S rows
    return row * (3.0 * A + 1.0 + ((it.flags & BI_SUMS) ? 1.0 + 2.0 * A : 0.0));
}
// Terminal launch for the updated players `upd`: each group's table blocks,
// then per terminal the opponent reach read and the values written.
static double term_launch_bytes(const ListSet& L, const std::vector<TermGroup>& gr, const std::vector<TermItem>& ti,
                                int upd) {
    (void)L;
    double b = 0.0;
    for (const TermGroup& g : gr) {
        b += (double)tg_table_bytes(g.H0, g.H1, upd);
        for (int t = g.first; t < g.first + g.count; ++t)
            for (int q = 0; q < 2; ++q)
                if ((upd >> q) & 1) b += 4.0 * ((double)ti[t].Hp[1 - q] + (double)ti[t].Hp[q]);
    }
    return b;
}
}  // namespace mtt

static int mtt_batch_kernel_profile_impl(mtt_batch* b, const mtt_solve_params* prm, int32_t iters, double* h_ms,
                                        double* h_bytes, void* stream) {
    using namespace mtt;
    if (!b || !h_ms || !h_bytes || iters <= 0) return MTT_ERR_INVALID;
    if (b->n_leaves) return MTT_ERR_UNSUPPORTED;
    MTT_TRY(check_params(prm));
    const mtt_solve_params& p = *prm;
    cudaStream_t st = as_stream(stream);
    const int threads = p.threads ? p.threads : (b->tuned_threads ? b->tuned_threads : 256);
    const ListSet& L = b->full;
    MTT_TRY(set_smem_attrs(b, L));
    MTT_TRY(fill_iter_table(b, p, iters, st));
    const SolveDev a = dev_args(b, p);
    // per-iteration compulsory bytes of each kernel class, from the host lists
    const HostLists& HL = b->host;
    double bf = 0.0, bb = 0.0, bt = 0.0;
    std::vector<TermGroup> gr(L.tb_start.empty() ? 0 : (size_t)(L.tb_start.back() + L.tb_count.back()));
    if (!gr.empty())
        MTT_TRY_CUDA(cudaMemcpy(gr.data(), L.tgroups, sizeof(TermGroup) * gr.size(), cudaMemcpyDeviceToHost));
    if (p.alternate) {
        for (int u = 0; u < 2; ++u) {
            for (const auto& lv : HL.fal[u]) for (const FwdItem& it : lv) bf += fwd_item_bytes(it, b->span);
            for (const auto& lv : HL.bal[u]) for (const BwdItem& it : lv) bb += bwd_item_bytes(it, b->span);
            bt += term_launch_bytes(L, gr, HL.titems, 1 << u);
        }
    } else {
        for (const auto& lv : HL.fsim) for (const FwdItem& it : lv) bf += fwd_item_bytes(it, b->span);
        for (const auto& lv : HL.bsim) for (const BwdItem& it : lv) bb += bwd_item_bytes(it, b->span);
        bt += term_launch_bytes(L, gr, HL.titems, 3);
    }
    h_bytes[0] = bf; h_bytes[1] = bt; h_bytes[2] = bb;
    k_init<<<b->n, 256, 0, st>>>(a, b->n);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    MTT_TRY(launch_levels_fwd(b, a, L.f_init, threads, false, st));
    // one event before and after each kernel class of every pass
    const int passes = p.alternate ? 2 : 1, ne = 6 * passes;
    std::vector<cudaEvent_t> ev(ne, nullptr);
    int s = MTT_OK;
    for (int i = 0; i < ne && !s; ++i) s = cuda_status(cudaEventCreate(&ev[i]));
    double ms[3] = {0.0, 0.0, 0.0};
    for (int t = 0; t < iters && !s; ++t) {
        for (int u = 0; u < passes && !s; ++u) {
            cudaEvent_t* e = ev.data() + 6 * u;
            const LevelLists<FwdItem>& F = p.alternate ? L.f_alt[u] : L.f_sim;
            const LevelLists<BwdItem>& B = p.alternate ? L.b_alt[u] : L.b_sim;
            s = cuda_status(cudaEventRecord(e[0], st));
            if (!s) s = launch_levels_fwd(b, a, F, threads, !p.alternate, st);
            if (!s) s = cuda_status(cudaEventRecord(e[1], st));
            if (!s) s = cuda_status(cudaEventRecord(e[2], st));
            if (!s) s = launch_term(b, L, a, p.alternate ? 1 << u : 3, st);
            if (!s) s = cuda_status(cudaEventRecord(e[3], st));
            if (!s) s = cuda_status(cudaEventRecord(e[4], st));
            if (!s) s = launch_levels_bwd(b, a, B, threads, p.alternate != 0, st);
            if (!s) s = cuda_status(cudaEventRecord(e[5], st));
        }
        if (!s) {
            k_next_iter<<<1, 32, 0, st>>>(a);
            s = cuda_status(cudaGetLastError());
            ++b->launches;
        }
        if (!s) s = cuda_status(cudaStreamSynchronize(st));
        for (int u = 0; u < passes && !s; ++u) {
            for (int k = 0; k < 3 && !s; ++k) {
                float x = 0.f;
                s = cuda_status(cudaEventElapsedTime(&x, ev[6 * u + 2 * k], ev[6 * u + 2 * k + 1]));
                ms[k] += x;
            }
        }
    }
    for (cudaEvent_t e : ev) if (e) cudaEventDestroy(e);
    if (s) return s;
    std::fill(b->iters_done.begin(), b->iters_done.end(), iters);
    for (int k = 0; k < 3; ++k) h_ms[k] = ms[k] / iters;
    int err = 0;
    MTT_TRY_CUDA(cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    return err ? MTT_ERR_TIMEOUT : MTT_OK;
}

extern "C" int mtt_batch_kernel_profile(mtt_batch* b, const mtt_solve_params* prm, int32_t iters, double* h_ms,
                                        double* h_bytes, void* stream) {
    const int s = mtt_batch_kernel_profile_impl(b, prm, iters, h_ms, h_bytes, stream);
    if (b) note_stream(b, as_stream(stream));
    return s;
}

extern "C" int mtt_batch_create(const mtt_subgame* subs, int32_t n, mtt_batch** out) {
    if (!subs || n <= 0 || !out) return MTT_ERR_INVALID;
    *out = nullptr;
    std::vector<SubPack> packs(n);
    const int nthr = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 32));
    {
        std::vector<std::thread> th;
        for (int t = 0; t < nthr; ++t)
            th.emplace_back([&, t]() { for (int i = t; i < n; i += nthr) pack_one(subs[i], packs[i]); });
        for (auto& x : th) x.join();
    }
    for (int i = 0; i < n; ++i) if (packs[i].status) return packs[i].status;
    mtt_batch* b = new mtt_batch();
    b->n = n;
    b->iters_done.assign(n, 0);
    long long nodes = 0, arena = 0, rs = 0, tabs = 0, hcards = 0, ranges = 0, darena = 0, iter_bytes = 0;
    b->desc.resize(n);
    int levels = 0;
    for (int i = 0; i < n; ++i) {
        SubDesc d = packs[i].d;
        const long long HS = d.Hp0 + d.Hp1;
        d.node_base = nodes;
        d.arena_base = arena;
        d.rs_base0 = rs;
        d.rs_base1 = rs + (long long)d.rows0 * d.Hp0;
        d.tab_base = tabs;
        d.darena_base = darena;
        d.range_base = ranges;
        d.hcard_base = hcards;
        nodes += d.n_nodes;
        arena += 2LL * d.n_nodes * HS;
        rs += (long long)d.rows0 * d.Hp0 + (long long)d.rows1 * d.Hp1;
        tabs += (long long)packs[i].tab.size();
        darena += 3LL * (d.n_nodes + 1) * HS;
        ranges += HS;
        hcards += HS;
        b->max_h = std::max(b->max_h, std::max(d.Hp0, d.Hp1));
        for (int16_t dp : packs[i].depth) levels = std::max(levels, (int)dp + 1);
        b->desc[i] = d;
        // algorithmic bytes of one iteration (fp32): R and S read+write per
        // action-hand of the acting player; per node, reach written+read and
        // CFV written+read for both players
        iter_bytes += 16LL * ((long long)d.rows0 * d.H0 + (long long)d.rows1 * d.H1) +
                      16LL * (long long)d.n_nodes * (d.H0 + d.H1);
    }
    b->iter_bytes = iter_bytes;
    b->levels = levels;
    // FP64 best-response warp tasks, solver work items per level, terminal items
    HostLists& HL = b->host;
    auto init_lists = [levels](HostLists& L) {
        L.bf.assign(levels, {}); L.bb.assign(levels, {});
        L.fi.assign(levels, {}); L.fsim.assign(levels, {}); L.bsim.assign(levels, {});
        for (int u = 0; u < 2; ++u) { L.fal[u].assign(levels, {}); L.bal[u].assign(levels, {}); }
    };
    auto addT = [](std::vector<Task>& v, int node, int sub, int groups) {
        for (int g0 = 0; g0 < groups; g0 += 32) v.push_back(Task{node, sub, g0, 0});
    };
    // one subgame's work items, appended to L (and its leaves to lv)
    auto build_sub = [&](int i, HostLists& L, std::vector<LeafItem>& lv) {
        const SubDesc& d = b->desc[i];
        const long long HS = d.Hp0 + d.Hp1, nn = d.n_nodes;
        const int Hp[2] = {d.Hp0, d.Hp1}, Hh[2] = {d.H0, d.H1}, H4[2] = {d.Hp0 / 4, d.Hp1 / 4};
        const long long off[2] = {0, d.Hp0}, rsb[2] = {d.rs_base0, d.rs_base1};
        const long long reach0 = d.arena_base, cfv0 = d.arena_base + nn * HS;
        const int Hmax = std::max(H4[0], H4[1]);
        for (int k = 0; k < d.n_nodes; ++k) {
            const DNode& nd = packs[i].nodes[k];
            const int gn = (int)d.node_base + k, dp = packs[i].depth[k];
            const long long src[2] = {nd.reach_src0, nd.reach_src1};
            if (nd.type == MTT_NODE_DECISION) {
                const int p = nd.player;
                FwdItem f{};
                f.reach_in = reach0 + src[p] * HS + off[p];
                f.child = reach0 + (long long)nd.first * HS + off[p];
                f.rows = rsb[p] + (long long)nd.row * Hp[p];
                f.h4 = H4[p];
                f.hs4 = (int)(HS / 4);
                f.na = nd.na;
                f.sub = i;
                for (f.g0 = 0; f.g0 < f.h4; f.g0 += 32) {
                    f.flags = FI_REACH; L.fi[dp].push_back(f);
                    f.flags = FI_REACH | FI_SUMS; L.fsim[dp].push_back(f);
                    // alternating pass u: the opponent's nodes pass reach down; the
                    // acting player's strategy sums are added by its backward items
                    f.flags = FI_REACH; L.fal[1 - p][dp].push_back(f);
                }
                for (int q = 0; q < 2; ++q) {
                    BwdItem bw{};
                    bw.child = cfv0 + (long long)nd.first * HS + off[q];
                    bw.self = cfv0 + (long long)k * HS + off[q];
                    bw.rows = q == p ? f.rows : 0;
                    bw.h4 = H4[q];
                    bw.hs4 = (int)(HS / 4);
                    bw.na = nd.na;
                    bw.sub = i;
                    bw.hc = q == p ? f.reach_in : 0;
                    for (bw.g0 = 0; bw.g0 < bw.h4; bw.g0 += 32) {
                        bw.flags = q == p ? (BI_UPDATE | (q ? BI_NEG : 0)) : 0;
                        L.bsim[dp].push_back(bw);
                        if (q == p) bw.flags = BI_UPDATE | BI_SUMS;
                        L.bal[q][dp].push_back(bw);
                    }
                }
                addT(L.bf[dp], gn, i, H4[p]);
                addT(L.bb[dp], gn, i, Hmax);
            } else if (nd.type == MTT_NODE_CHANCE) {
                for (int p = 0; p < 2; ++p) {
                    FwdItem f{};
                    f.reach_in = reach0 + src[p] * HS + off[p];
                    f.child = reach0 + (long long)nd.first * HS + off[p];
                    f.hc = d.hcard_base + off[p];
                    f.h4 = H4[p];
                    f.hs4 = (int)(HS / 4);
                    f.na = nd.na;
                    f.flags = FI_CHANCE;
                    f.first = (int)d.node_base + nd.first;
                    f.sub = i;
                    for (f.g0 = 0; f.g0 < f.h4; f.g0 += 32) {
                        L.fi[dp].push_back(f);
                        L.fsim[dp].push_back(f);
                        L.fal[1 - p][dp].push_back(f);     // pass u recomputes the other player's reach
                    }
                    BwdItem bw{};
                    bw.child = cfv0 + (long long)nd.first * HS + off[p];
                    bw.self = cfv0 + (long long)k * HS + off[p];
                    bw.hc = d.hcard_base + off[p];
                    bw.h4 = H4[p];
                    bw.hs4 = (int)(HS / 4);
                    bw.na = nd.na;
                    bw.flags = BI_CHANCE;
                    bw.first = (int)d.node_base + nd.first;
                    bw.div = (float)(nd.nlive - 4);
                    bw.sub = i;
                    for (bw.g0 = 0; bw.g0 < bw.h4; bw.g0 += 32) {
                        L.bsim[dp].push_back(bw);
                        L.bal[p][dp].push_back(bw);
                    }
                }
                addT(L.bf[dp], gn, i, Hmax);
                addT(L.bb[dp], gn, i, Hmax);
            } else if (nd.type == MTT_NODE_LEAF) {
                LeafItem lf{};
                for (int p = 0; p < 2; ++p) {
                    lf.reach[p] = reach0 + src[p] * HS + off[p];
                    lf.cfv[p] = cfv0 + (long long)k * HS + off[p];
                    lf.hc[p] = d.hcard_base + off[p];
                    lf.H[p] = Hh[p];
                    lf.Hp[p] = Hp[p];
                }
                lf.pot = nd.pot;
                lf.spr = nd.pot > 0.0f ? subs[i].nodes[k].reserved / nd.pot : 0.0f;
                lf.row0 = 0;                          // set once the leaves are merged
                lf.tab = d.tab_base;
                lf.vsize = d.tab_vsize;
                lf.sub = i;
                for (int c = 0; c < 4; ++c) lf.board[c] = subs[i].board[c];
                lv.push_back(lf);
            } else {
                L.terms.push_back(make_int2(gn, i));
                TermItem t{};
                for (int p = 0; p < 2; ++p) {
                    t.ro[p] = reach0 + src[p] * HS + off[p];
                    t.out[p] = cfv0 + (long long)k * HS + off[p];
                    t.H[p] = Hh[p];
                    t.Hp[p] = Hp[p];
                }
                t.tab = d.tab_base + (long long)nd.var * d.tab_vsize;
                t.pot = nd.pot;
                t.c0 = nd.c0;
                t.c1 = nd.c1;
                t.type_wmask = nd.type | (nd.wmask << 8);
                t.sub = i;
                L.titems.push_back(t);
            }
        }
    };
    // subgames in contiguous chunks on host threads, merged in subgame order
    // (the same lists, in the same order, as one thread would build)
    const int nlt = std::max(1, std::min(n, std::min<int>((int)std::thread::hardware_concurrency(), 32)));
    std::vector<HostLists> part(nlt);
    std::vector<std::vector<LeafItem>> plv(nlt);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < nlt; ++t)
            th.emplace_back([&, t]() {
                init_lists(part[t]);
                const int lo = (int)((long long)n * t / nlt), hi = (int)((long long)n * (t + 1) / nlt);
                for (int i = lo; i < hi; ++i) build_sub(i, part[t], plv[t]);
                // terminals of one subgame and table variant are contiguous (terminal groups)
                std::stable_sort(part[t].titems.begin(), part[t].titems.end(),
                                 [](const TermItem& x, const TermItem& y) {
                                     return x.sub != y.sub ? x.sub < y.sub : x.tab < y.tab;
                                 });
            });
        for (auto& x : th) x.join();
    }
    init_lists(HL);
    auto merge = [&](auto get) {
        size_t k = 0;
        for (int t = 0; t < nlt; ++t) k += get(part[t]).size();
        auto& dst = get(HL);
        dst.reserve(k);
        for (int t = 0; t < nlt; ++t) dst.insert(dst.end(), get(part[t]).begin(), get(part[t]).end());
    };
    // every list is merged by its own job (distinct vectors), the jobs on the
    // host threads
    std::vector<std::function<void()>> jobs;
    auto add = [&](auto get) { jobs.emplace_back([&merge, get]() { merge(get); }); };
    for (int d = 0; d < levels; ++d) {
        add([d](HostLists& L) -> std::vector<Task>& { return L.bf[d]; });
        add([d](HostLists& L) -> std::vector<Task>& { return L.bb[d]; });
        add([d](HostLists& L) -> std::vector<FwdItem>& { return L.fi[d]; });
        add([d](HostLists& L) -> std::vector<FwdItem>& { return L.fsim[d]; });
        add([d](HostLists& L) -> std::vector<BwdItem>& { return L.bsim[d]; });
        for (int u = 0; u < 2; ++u) {
            add([d, u](HostLists& L) -> std::vector<FwdItem>& { return L.fal[u][d]; });
            add([d, u](HostLists& L) -> std::vector<BwdItem>& { return L.bal[u][d]; });
        }
    }
    add([](HostLists& L) -> std::vector<TermItem>& { return L.titems; });
    add([](HostLists& L) -> std::vector<int2>& { return L.terms; });
    {
        std::atomic<size_t> next{0};
        std::vector<std::thread> th;
        for (int t = 0; t < nlt; ++t)
            th.emplace_back([&]() {
                for (size_t j; (j = next.fetch_add(1)) < jobs.size();) jobs[j]();
            });
        for (auto& x : th) x.join();
    }
    for (int t = 0; t < nlt; ++t) b->h_leaves.insert(b->h_leaves.end(), plv[t].begin(), plv[t].end());
    for (size_t k = 0; k < b->h_leaves.size(); ++k) b->h_leaves[k].row0 = LEAF_RIVERS * (int)k;
    long long total = 0;
    int s = MTT_OK;
    if (!s) s = dalloc(&b->d_desc, n, total);
    if (!s) s = dalloc(&b->d_nodes, nodes, total);
    if (!s) s = dalloc(&b->d_tabs, tabs, total);
    if (!s) s = dalloc(&b->d_hcards, hcards, total);
    if (!s) s = dalloc(&b->d_ranges, ranges, total);
    if (!s) s = dalloc(&b->d_arena, arena, total);
    if (!s) s = dalloc(&b->d_R, rs, total);
    if (!s) s = dalloc(&b->d_S, rs, total);
    if (!s) s = dalloc(&b->d_darena, darena, total);
    if (!s) s = dalloc(&b->d_results, 6LL * n, total);
    if (!s) s = dalloc(&b->d_iter, 1, total);
    if (!s) s = dalloc(&b->d_err, 1, total);
    if (!s) s = cuda_status(cudaMemset(b->d_err, 0, sizeof(int)));
    if (!s) s = build_set(b, b->full, nullptr, total);
    b->n_leaves = (int)b->h_leaves.size();
    if (!s && b->n_leaves) {
        s = dalloc(&b->d_leaves, b->h_leaves.size(), total);
        if (!s) s = cuda_status(cudaMemcpy(b->d_leaves, b->h_leaves.data(), sizeof(LeafItem) * b->h_leaves.size(),
                                           cudaMemcpyHostToDevice));
    }
    if (s) { free_batch(b); return s; }
    b->device_bytes = total;
    {
        std::vector<DNode> hn(nodes);
        std::vector<uint8_t> ht(tabs);
        std::vector<uint16_t> hh(hcards);
        std::vector<float> hr(ranges);
        for (int i = 0; i < n; ++i) {
            const SubDesc& d = b->desc[i];
            std::copy(packs[i].nodes.begin(), packs[i].nodes.end(), hn.begin() + d.node_base);
            std::copy(packs[i].tab.begin(), packs[i].tab.end(), ht.begin() + d.tab_base);
            std::copy(packs[i].hcards.begin(), packs[i].hcards.end(), hh.begin() + d.hcard_base);
            std::copy(packs[i].range.begin(), packs[i].range.end(), hr.begin() + d.range_base);
        }
        s = cuda_status(cudaMemcpy(b->d_desc, b->desc.data(), sizeof(SubDesc) * n, cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemcpy(b->d_nodes, hn.data(), sizeof(DNode) * hn.size(), cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemcpy(b->d_tabs, ht.data(), ht.size(), cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemcpy(b->d_hcards, hh.data(), 2 * hh.size(), cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemcpy(b->d_ranges, hr.data(), 4 * hr.size(), cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemset(b->d_arena, 0, sizeof(float) * (size_t)std::max(arena, 1LL)));
        if (!s) s = cuda_status(cudaMemset(b->d_results, 0, sizeof(double) * 6 * (size_t)n));
    }
    if (s) { free_batch(b); return s; }
    *out = b;
    return MTT_OK;
}

extern "C" int mtt_batch_solve(mtt_batch* b, const mtt_solve_params* prm, void* stream) {
    if (!b) return MTT_ERR_INVALID;
    MTT_TRY(check_params(prm));
    const int s = run_solve(b, *prm, as_stream(stream), false);
    note_stream(b, as_stream(stream));
    return s;
}

extern "C" int mtt_batch_solve_graph(mtt_batch* b, const mtt_solve_params* prm, void* stream) {
    if (!b) return MTT_ERR_INVALID;
    MTT_TRY(check_params(prm));
    const int s = run_solve(b, *prm, as_stream(stream), true);
    note_stream(b, as_stream(stream));
    return s;
}

extern "C" int mtt_batch_results(mtt_batch* b, double* h_out, void* stream) {
    if (!b || !h_out) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    int err = 0;
    MTT_TRY_CUDA(cudaMemcpyAsync(h_out, b->d_results, sizeof(double) * 6 * (size_t)b->n, cudaMemcpyDeviceToHost, st));
    MTT_TRY_CUDA(cudaMemcpyAsync(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MTT_TRY_CUDA(cudaStreamSynchronize(st));
    return err ? MTT_ERR_TIMEOUT : MTT_OK;
}

extern "C" int mtt_batch_iterations(mtt_batch* b, int32_t* h_out) {
    if (!b || !h_out) return MTT_ERR_INVALID;
    std::copy(b->iters_done.begin(), b->iters_done.end(), h_out);
    return MTT_OK;
}

extern "C" int mtt_batch_read(mtt_batch* b, int32_t s, float* h_R0, float* h_R1, float* h_S0, float* h_S1,
                              float* h_cfv0, float* h_cfv1) {
    if (!b || s < 0 || s >= b->n) return MTT_ERR_INVALID;
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    const SubDesc& d = b->desc[s];
    auto rows_copy = [&](float* dst, const float* src, int rows, int H, int Hp) -> int {
        if (!dst || rows == 0) return MTT_OK;
        MTT_TRY_CUDA(cudaMemcpy2D(dst, sizeof(float) * H, src, sizeof(float) * Hp, sizeof(float) * H, rows,
                                  cudaMemcpyDeviceToHost));
        return MTT_OK;
    };
    MTT_TRY(rows_copy(h_R0, b->d_R + d.rs_base0, d.rows0, d.H0, d.Hp0));
    MTT_TRY(rows_copy(h_R1, b->d_R + d.rs_base1, d.rows1, d.H1, d.Hp1));
    MTT_TRY(rows_copy(h_S0, b->d_S + d.rs_base0, d.rows0, d.H0, d.Hp0));
    MTT_TRY(rows_copy(h_S1, b->d_S + d.rs_base1, d.rows1, d.H1, d.Hp1));
    const float* cf = b->d_arena + d.arena_base + (size_t)d.n_nodes * (d.Hp0 + d.Hp1);
    if (h_cfv0) MTT_TRY_CUDA(cudaMemcpy(h_cfv0, cf, sizeof(float) * d.H0, cudaMemcpyDeviceToHost));
    if (h_cfv1) MTT_TRY_CUDA(cudaMemcpy(h_cfv1, cf + d.Hp0, sizeof(float) * d.H1, cudaMemcpyDeviceToHost));
    return MTT_OK;
}

extern "C" int mtt_batch_read_vectors(mtt_batch* b, int32_t s, float* h_reach, float* h_cfv) {
    if (!b || s < 0 || s >= b->n) return MTT_ERR_INVALID;
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    const SubDesc& d = b->desc[s];
    const size_t HS = (size_t)d.Hp0 + d.Hp1, nn = (size_t)d.n_nodes;
    std::vector<float> arena(2 * nn * HS);
    MTT_TRY_CUDA(cudaMemcpy(arena.data(), b->d_arena + d.arena_base, sizeof(float) * arena.size(), cudaMemcpyDeviceToHost));
    std::vector<DNode> nodes(nn);
    MTT_TRY_CUDA(cudaMemcpy(nodes.data(), b->d_nodes + d.node_base, sizeof(DNode) * nn, cudaMemcpyDeviceToHost));
    const size_t W = (size_t)d.H0 + d.H1;
    for (size_t k = 0; k < nn; ++k) {
        for (int p = 0; p < 2; ++p) {
            const int H = p ? d.H1 : d.H0;
            const size_t off = p ? (size_t)d.Hp0 : 0, dst = k * W + (p ? (size_t)d.H0 : 0);
            const size_t src = (size_t)(p ? nodes[k].reach_src1 : nodes[k].reach_src0);
            if (h_reach) std::memcpy(h_reach + dst, arena.data() + src * HS + off, sizeof(float) * H);
            if (h_cfv) std::memcpy(h_cfv + dst, arena.data() + nn * HS + k * HS + off, sizeof(float) * H);
        }
    }
    return MTT_OK;
}

extern "C" int mtt_batch_root_values(mtt_batch* b, int32_t s, double* h_ev0, double* h_ev1, double* h_br0,
                                     double* h_br1) {
    if (!b || s < 0 || s >= b->n) return MTT_ERR_INVALID;
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    const SubDesc& d = b->desc[s];
    const size_t HS = (size_t)d.Hp0 + d.Hp1, reg = ((size_t)d.n_nodes + 1) * HS;
    const double* br = b->d_darena + d.darena_base + reg;
    const double* ev = br + reg;
    if (h_ev0) MTT_TRY_CUDA(cudaMemcpy(h_ev0, ev, sizeof(double) * d.H0, cudaMemcpyDeviceToHost));
    if (h_ev1) MTT_TRY_CUDA(cudaMemcpy(h_ev1, ev + d.Hp0, sizeof(double) * d.H1, cudaMemcpyDeviceToHost));
    if (h_br0) MTT_TRY_CUDA(cudaMemcpy(h_br0, br, sizeof(double) * d.H0, cudaMemcpyDeviceToHost));
    if (h_br1) MTT_TRY_CUDA(cudaMemcpy(h_br1, br + d.Hp0, sizeof(double) * d.H1, cudaMemcpyDeviceToHost));
    return MTT_OK;
}

extern "C" int mtt_batch_info(mtt_batch* b, int64_t* device_bytes, int64_t* iter_bytes) {
    if (!b) return MTT_ERR_INVALID;
    if (device_bytes) *device_bytes = b->device_bytes;
    if (iter_bytes) *iter_bytes = b->iter_bytes;
    return MTT_OK;
}

extern "C" int mtt_batch_layout(mtt_batch* b, int64_t* h_rows_off, int64_t* h_range_off, int64_t* total_rows,
                                int64_t* total_range) {
    if (!b) return MTT_ERR_INVALID;
    long long tr = 0, tg = 0;
    for (int i = 0; i < b->n; ++i) {
        const SubDesc& d = b->desc[i];
        if (h_rows_off) { h_rows_off[2 * i] = d.rs_base0; h_rows_off[2 * i + 1] = d.rs_base1; }
        if (h_range_off) h_range_off[i] = d.range_base;
        tr = std::max(tr, d.rs_base1 + (long long)d.rows1 * d.Hp1);
        tg = std::max(tg, d.range_base + (long long)(d.Hp0 + d.Hp1));
    }
    if (total_rows) *total_rows = tr;
    if (total_range) *total_range = tg;
    return MTT_OK;
}

extern "C" int mtt_trim_pool(void) {
    cudaMemPool_t pool = mtt::batch_pool();
    if (!pool) return MTT_ERR_CUDA;
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    MTT_TRY_CUDA(cudaMemPoolTrimTo(pool, 0));
    return MTT_OK;
}

extern "C" int mtt_batch_set_leafnet(mtt_batch* b, mtt_leafnet* net, int32_t flags) {
    using namespace mtt;
    if (!b || (flags & ~MTT_LEAF_VALUES_RESIDUAL) || !b->n_leaves) return MTT_ERR_INVALID;
    const long long rows = (long long)LEAF_RIVERS * b->n_leaves;
    if (net) {
        int32_t cap = 0;
        MTT_TRY(mtt_leafnet_capacity(net, &cap));
        if (rows > cap) return MTT_ERR_INVALID;
    }
    if (!b->d_lx) {
        int stride = 0, smem = 0;
        for (const LeafItem& lf : b->h_leaves) {
            stride = std::max(stride, std::max(lf.Hp[0], lf.Hp[1]));
            for (int q = 0; q < 2; ++q) smem = std::max(smem, leaf_sd_smem(lf.H[1 - q], lf.H[q], lf.Hp[1 - q]));
        }
        if (smem > 227 * 1024) return MTT_ERR_UNSUPPORTED;
        if (smem > 48 * 1024)
            MTT_TRY_CUDA(cudaFuncSetAttribute(k_leaf_showdown, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        long long total = 0;
        int s = dalloc(&b->d_lx, (size_t)rows * LEAF_IN, total);
        if (!s) s = dalloc(&b->d_ly, (size_t)rows * LEAF_OUT, total);
        if (!s) s = dalloc(&b->d_lm, (size_t)rows * 2, total);
        if (!s) s = dalloc(&b->d_lsd, (size_t)rows * 2 * stride, total);
        if (s) return s;
        b->leaf_sd_stride = stride;
        b->leaf_smem = smem;
        b->device_bytes += total;
    }
    b->net = net;
    b->leaf_residual = (flags & MTT_LEAF_VALUES_RESIDUAL) != 0;
    b->leaf_ready = true;
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }   // captured the old leaf launches
    return MTT_OK;
}

static int mtt_batch_ev_grad_impl(mtt_batch* b, const float* d_logits, const float* d_ranges, float* d_ev,
                                 float* d_grad_ranges, float* d_grad_logits, void* stream) {
    auto al16 = [](const void* p) { return p && ((uintptr_t)p & 15u) == 0; };
    if (!b || !al16(d_logits) || !al16(d_ranges) || !d_ev || !al16(d_grad_ranges) || !al16(d_grad_logits))
        return MTT_ERR_INVALID;
    if (b->n_leaves) return MTT_ERR_UNSUPPORTED;
    cudaStream_t st = as_stream(stream);
    mtt_solve_params p{};
    p.algo = MTT_ALGO_CFRPLUS;
    p.semantics = MTT_SEM_CORRECT;
    SolveDev a = dev_args(b, p);
    a.R = const_cast<float*>(d_logits);
    a.S = d_grad_logits;
    a.ranges = d_ranges;
    const ListSet& L = b->full;
    MTT_TRY(set_smem_attrs(b, L));
    k_ev_init<<<b->n, 256, 0, st>>>(a, b->n);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    const long long warps = 256 / 32;
    for (int d = 0; d < b->levels; ++d) {
        const long long n = L.f_init.off[d + 1] - L.f_init.off[d];
        if (n == 0) continue;
        if (a.span == 2) k_ev_fwd<2><<<(unsigned)((n + warps - 1) / warps), 256, 0, st>>>(a, L.f_init.d + L.f_init.off[d], (int)n);
        else k_ev_fwd<1><<<(unsigned)((n + warps - 1) / warps), 256, 0, st>>>(a, L.f_init.d + L.f_init.off[d], (int)n);
        MTT_CHECK_LAUNCH();
        ++b->launches;
    }
    MTT_TRY(launch_term(b, L, a, 3, st));
    for (int d = b->levels - 1; d >= 0; --d) {
        const long long n = L.b_sim.off[d + 1] - L.b_sim.off[d];
        if (n == 0) continue;
        if (a.span == 2) k_ev_bwd<2><<<(unsigned)((n + warps - 1) / warps), 256, 0, st>>>(a, L.b_sim.d + L.b_sim.off[d], (int)n);
        else k_ev_bwd<1><<<(unsigned)((n + warps - 1) / warps), 256, 0, st>>>(a, L.b_sim.d + L.b_sim.off[d], (int)n);
        MTT_CHECK_LAUNCH();
        ++b->launches;
    }
    k_ev_root<<<b->n, TT, 0, st>>>(a, b->n, d_ev, d_grad_ranges);
    MTT_CHECK_LAUNCH();
    ++b->launches;
    return MTT_OK;
}

extern "C" int mtt_batch_ev_grad(mtt_batch* b, const float* d_logits, const float* d_ranges, float* d_ev,
                                 float* d_grad_ranges, float* d_grad_logits, void* stream) {
    const int s = mtt_batch_ev_grad_impl(b, d_logits, d_ranges, d_ev, d_grad_ranges, d_grad_logits, stream);
    if (b) note_stream(b, as_stream(stream));
    return s;
}

extern "C" int mtt_batch_check(mtt_batch* b, void* stream) {
    if (!b) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    int err = 0;
    MTT_TRY_CUDA(cudaMemcpyAsync(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MTT_TRY_CUDA(cudaStreamSynchronize(st));
    return err ? MTT_ERR_TIMEOUT : MTT_OK;
}

extern "C" int mtt_batch_launch_count(mtt_batch* b, int64_t* launches) {
    if (!b || !launches) return MTT_ERR_INVALID;
    *launches = b->launches;
    return MTT_OK;
}

namespace mtt {
// Switch the batch to `span` x 32 float4 groups per sweep item and at most
// `chunk` terminals per CTA: the full work lists are rebuilt from the host
// lists and the cached iteration graph is dropped.
static int apply_schedule(mtt_batch* b, int span, int chunk) {
    if (span == b->span && chunk == b->tchunk) return MTT_OK;
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    b->span = span;
    b->tchunk = chunk;
    long long total = 0;
    MTT_TRY(build_set(b, b->full, nullptr, total));
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    return MTT_OK;
}
}  // namespace mtt

extern "C" int mtt_batch_set_schedule(mtt_batch* b, int32_t threads, int32_t hands_per_warp, int32_t term_chunk) {
    using namespace mtt;
    if (!b || (threads != 0 && threads != 64 && threads != 128 && threads != 256) ||
        (hands_per_warp != 128 && hands_per_warp != 256) || term_chunk < 1 || term_chunk > TG_CHUNK)
        return MTT_ERR_INVALID;
    MTT_TRY(apply_schedule(b, hands_per_warp / 128, term_chunk));
    b->tuned_threads = threads;
    return MTT_OK;
}

extern "C" int mtt_batch_schedule(mtt_batch* b, int32_t* threads, int32_t* hands_per_warp, int32_t* term_chunk) {
    if (!b) return MTT_ERR_INVALID;
    if (threads) *threads = b->tuned_threads ? b->tuned_threads : 256;
    if (hands_per_warp) *hands_per_warp = 128 * b->span;
    if (term_chunk) *term_chunk = b->tchunk;
    return MTT_OK;
}

static int mtt_batch_autotune_impl(mtt_batch* b, const mtt_solve_params* prm, void* stream, int32_t* threads) {
    using namespace mtt;
    if (!b) return MTT_ERR_INVALID;
    if (b->n_leaves && !b->leaf_ready) return MTT_ERR_INVALID;
    MTT_TRY(check_params(prm));
    cudaStream_t st = as_stream(stream);
    mtt_solve_params p = *prm;
    p.iters = std::min(std::max(prm->iters, 1), 8);
    p.exploitability = 0;
    p.target_expl = 0.0f;
    // every schedule: hands per warp item x terminals per CTA x sweep CTA size
    const int spans[2] = {1, 2}, chunks[2] = {8, 16}, cands[3] = {64, 128, 256};
    float best_ms = 1e30f;
    int best_t = 256, best_span = b->span, best_chunk = b->tchunk;
    cudaEvent_t e0, e1;
    MTT_TRY_CUDA(cudaEventCreate(&e0));
    MTT_TRY_CUDA(cudaEventCreate(&e1));
    int s = MTT_OK;
    for (int sp : spans) {
        for (int ch : chunks) {
            if (!s) s = apply_schedule(b, sp, ch);
            for (int c : cands) {
                p.threads = c;
                if (!s) s = run_solve(b, p, st, false);   // warm
                if (!s) s = cuda_status(cudaEventRecord(e0, st));
                if (!s) s = run_solve(b, p, st, false);
                if (!s) s = cuda_status(cudaEventRecord(e1, st));
                if (!s) s = cuda_status(cudaEventSynchronize(e1));
                float ms = 0.f;
                if (!s) s = cuda_status(cudaEventElapsedTime(&ms, e0, e1));
                if (!s && ms < best_ms) { best_ms = ms; best_t = c; best_span = sp; best_chunk = ch; }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!s) s = apply_schedule(b, best_span, best_chunk);
    if (s) return s;
    b->tuned_threads = best_t;
    if (threads) *threads = best_t;
    return MTT_OK;
}

extern "C" int mtt_batch_autotune(mtt_batch* b, const mtt_solve_params* prm, void* stream, int32_t* threads) {
    const int s = mtt_batch_autotune_impl(b, prm, stream, threads);
    if (b) note_stream(b, mtt::as_stream(stream));
    return s;
}

extern "C" int mtt_batch_destroy(mtt_batch* b) {
    if (!b) return MTT_ERR_INVALID;
    free_batch(b);
    return MTT_OK;
}
