// multiway.cu — four-player river CFR: tree builder, batched sweeps and
// rank-scan showdown terminals with ICM loss multipliers.
//
// The reference engine (multiway_4way_engine.cu:41-257) keeps every node's
// reach and values for 4 players over one shared combo axis and runs three
// kernels per depth: regret matching + child reach, terminal values, and the
// CFR+ backup with regret and strategy-sum updates of all four players at
// once.  Here a batch of subgames is swept level by level as in the
// heads-up solver: warp work items over (node, 32 float4 hand groups) with
// precomputed offsets, one CTA per terminal, one iteration captured as a
// CUDA graph.
//
// Terminal values (kernel_4way_evaluate_terminals, :85-217): with W_o the
// total reach of player o,
//   fold (one player w left): p == w: (pot - c_w) * prod_{o != p} W_o,
//                             else   -bf[p][w] c_p * prod_{o != p} W_o;
//   showdown, p folded earlier: -bf[p][p] c_p * prod_{o != p} W_o;
//   showdown, p still in, hand h:
//     reference semantics: F = prod over active o != p of the reach of o
//       strictly before h in the rank-position order (positions break ties),
//       value = ((pot - c_p) F - bf[p][p] c_p (prod W_o - F)) * prod_inactive W_o;
//     correct semantics: the hero's hand h removes its two cards from every
//       opponent's range (card removal) and hands of equal rank split the
//       pot: with W_o, L_o, E_o the reach of o over the hands that share no
//       card with h (in total, ranked below h, ranked equal to h),
//       value = (sum over subsets T of the active opponents of
//                prod_{T} E_o prod_{not T} L_o (pot / (1 + |T|) - c_p)
//                - bf[p][p] c_p (prod W_o - prod (L_o + E_o))) * prod_inactive W_o,
//       and fold values use the same W_o.  Opponents are not conditioned on
//       one another (two opponents' hands may share a card), the usual
//       approximation of multiway solvers; the exact game sums over disjoint
//       triples of opponent hands, which no per-hand scan gives.
//   The reference semantics remove no cards, as the reference does not.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <numeric>
#include <vector>

#include "mtt_bulk.cuh"
#include "mtt_common.h"
#include "mtt_device.cuh"

namespace mtt {
namespace mw {

constexpr int NP = MTT_MW_PLAYERS;
constexpr int MAXA = MTT_MW_MAX_ACTIONS;

// =================================================================== tree (host)
struct BState {
    float c[NP];        // chips in, including the dead-money share
    float behind[NP];   // chips left
    int in;             // players not folded
    int acted;          // players who acted since the last bet or raise
    int raises;
    int cur;            // first seat to look at for the next actor
    float level;        // highest commitment
};

static float pot_of(const BState& s) { return s.c[0] + s.c[1] + s.c[2] + s.c[3]; }

// Highest commitment reachable without side pots: the smallest total stack
// among the players still in.
static float level_cap(const BState& s) {
    float m = 1e30f;
    for (int p = 0; p < NP; ++p)
        if ((s.in >> p) & 1) m = std::min(m, s.c[p] + s.behind[p]);
    return m;
}

static bool needs_to_act(const BState& s, int p) {
    return ((s.in >> p) & 1) && s.behind[p] > 1e-6f && (!((s.acted >> p) & 1) || s.c[p] < s.level - 1e-6f);
}

static int build_tree(const mtt_mw_spec& sp, std::vector<mtt_mw_node>& out, int rows[NP], int* max_depth) {
    if (!(sp.pot >= 0.0f) || sp.n_bet_sizes < 1 || sp.n_bet_sizes > 2 || sp.raise_cap < 0 || sp.raise_cap > 4 ||
        !(sp.raise_size > 0.0f))
        return MTT_ERR_INVALID;
    for (int k = 0; k < sp.n_bet_sizes; ++k)
        if (!(sp.bet_sizes[k] > 0.0f)) return MTT_ERR_INVALID;
    for (int p = 0; p < NP; ++p)
        if (!(sp.stacks[p] >= 0.0f)) return MTT_ERR_INVALID;
    out.clear();
    for (int p = 0; p < NP; ++p) rows[p] = 0;
    struct Q { BState s; int idx; int depth; };
    std::deque<Q> q;
    BState root{};
    for (int p = 0; p < NP; ++p) { root.c[p] = sp.pot / NP; root.behind[p] = sp.stacks[p]; }
    root.in = 0xF;
    root.level = sp.pot / NP;
    out.push_back(mtt_mw_node{});
    q.push_back({root, 0, 0});
    int depth_max = 0;
    while (!q.empty()) {
        const Q cur = q.front();
        q.pop_front();
        const BState& s = cur.s;
        mtt_mw_node& nd = out[cur.idx];
        nd.pot_size = pot_of(s);
        for (int p = 0; p < NP; ++p) nd.committed[p] = s.c[p];
        depth_max = std::max(depth_max, cur.depth);
        if (__builtin_popcount(s.in) == 1) {
            nd.type = MTT_NODE_FOLD;
            nd.active_mask = (uint8_t)s.in;
            continue;
        }
        int p = -1;
        for (int k = 0; k < NP; ++k) {
            const int c = (s.cur + k) % NP;
            if (needs_to_act(s, c)) { p = c; break; }
        }
        if (p < 0) {
            nd.type = MTT_NODE_SHOWDOWN;
            nd.active_mask = (uint8_t)s.in;
            continue;
        }
        std::vector<BState> kids;
        const float cap = level_cap(s), pot = pot_of(s);
        BState b = s;
        b.cur = (p + 1) % NP;
        if (s.c[p] >= s.level - 1e-6f) {
            BState k0 = b;
            k0.acted |= 1 << p;
            kids.push_back(k0);                                 // check
            float last = s.level;
            for (int i = 0; i < sp.n_bet_sizes; ++i) {
                const float lv = std::min(s.c[p] + sp.bet_sizes[i] * pot, cap);
                if (lv <= last + 1e-4f) continue;                // collapsed into a smaller size or the cap
                BState k1 = b;
                k1.behind[p] -= lv - s.c[p];
                k1.c[p] = lv;
                k1.level = lv;
                k1.acted = 1 << p;
                kids.push_back(k1);
                last = lv;
            }
        } else {
            BState kf = b;
            kf.in &= ~(1 << p);
            kf.acted |= 1 << p;
            kids.push_back(kf);                                 // fold
            BState kc = b;
            kc.behind[p] -= s.level - s.c[p];
            kc.c[p] = s.level;
            kc.acted |= 1 << p;
            kids.push_back(kc);                                 // call
            if (s.raises < sp.raise_cap && s.level < cap - 1e-4f) {
                const float to_call = s.level - s.c[p];
                const float lv = std::min(s.c[p] + to_call + sp.raise_size * (pot + to_call), cap);
                if (lv > s.level + 1e-4f) {
                    BState kr = b;
                    kr.behind[p] -= lv - s.c[p];
                    kr.c[p] = lv;
                    kr.level = lv;
                    kr.acted = 1 << p;
                    kr.raises = s.raises + 1;
                    kids.push_back(kr);                         // raise
                }
            }
        }
        if ((int)kids.size() > MAXA) return MTT_ERR_UNSUPPORTED;
        nd.type = MTT_NODE_DECISION;
        nd.player = (uint8_t)p;
        nd.num_actions = (uint8_t)kids.size();
        nd.infoset_offset = rows[p];
        rows[p] += (int)kids.size();
        nd.children_offset = (int)out.size();
        for (const BState& k : kids) {
            q.push_back({k, (int)out.size(), cur.depth + 1});
            out.push_back(mtt_mw_node{});
        }
        if (out.size() > (1u << 20)) return MTT_ERR_UNSUPPORTED;
    }
    *max_depth = depth_max;
    return MTT_OK;
}

static int validate(const mtt_mw_node* nodes, int n, const int rows[NP]) {
    if (!nodes || n < 1) return MTT_ERR_INVALID;
    std::vector<int> used[NP];
    for (int p = 0; p < NP; ++p) used[p].assign(std::max(rows[p], 0), 0);
    std::vector<int> parents(n, 0);
    for (int i = 0; i < n; ++i) {
        const mtt_mw_node& d = nodes[i];
        if (d.type == MTT_NODE_DECISION) {
            if (d.player >= NP || d.num_actions < 1 || d.num_actions > MAXA) return MTT_ERR_INVALID;
            if (d.children_offset <= i || d.children_offset + d.num_actions > n) return MTT_ERR_INVALID;
            if (d.infoset_offset < 0 || d.infoset_offset + d.num_actions > rows[d.player]) return MTT_ERR_INVALID;
            for (int a = 0; a < d.num_actions; ++a) {
                if (used[d.player][d.infoset_offset + a]++) return MTT_ERR_INVALID;
                parents[d.children_offset + a]++;
            }
        } else if (d.type == MTT_NODE_FOLD) {
            if (__builtin_popcount(d.active_mask & 0xF) != 1) return MTT_ERR_INVALID;
        } else if (d.type == MTT_NODE_SHOWDOWN) {
            if (__builtin_popcount(d.active_mask & 0xF) < 2) return MTT_ERR_INVALID;
        } else {
            return MTT_ERR_INVALID;                         // no chance nodes in a river subgame
        }
        if (!(d.pot_size >= 0.0f)) return MTT_ERR_INVALID;
    }
    if (parents[0] != 0) return MTT_ERR_INVALID;
    for (int i = 1; i < n; ++i) if (parents[i] != 1) return MTT_ERR_INVALID;
    return MTT_OK;
}

// =================================================================== device layout
// One hand's positions in the card-removal scan [rank order (H) | per-card
// lists (2 H)], 16 bytes: lt / le, the first hand ranked >= / > it in rank
// order (its rank group); c1lt / c1le (c2lt / c2le), the same inside the list
// of hands holding its first (second) card, as absolute scan positions.
struct alignas(16) MwEntry {
    uint16_t lt, le;
    uint16_t c1lt, c1le;
    uint16_t c2lt, c2le;
    uint8_t c1, c2;
    uint16_t pad;
};
static_assert(sizeof(MwEntry) == 16, "MwEntry is 16 bytes");

struct alignas(16) MNode {      // 64 B
    uint8_t type, player, na, amask;
    int32_t first, row, pad0;
    int32_t src[NP];            // node whose reach slot holds player p's reach here
    float pot, c[NP];
    int32_t pad1[3];
};
static_assert(sizeof(MNode) == 64, "MNode is 64 bytes");

struct alignas(16) MDesc {
    long long node_base;        // into the MNode array
    long long arena_base;       // float offset: reach region [n_nodes][4][Hp], then the CFV region
    long long rs_base[NP];      // float offsets of R_p / S_p
    long long tab_base;         // u16 offset of [pos | gstart | gend] per hand, Hp each
    long long range_base;       // float offset of [4][Hp] root ranges
    long long ctab_base;        // u16 offset of the card-removal lists: [rank order H | per-card lists 2 H | seg 54]
    long long cent_base;        // u16 offset of the per-hand MwEntry records (16-byte aligned)
    int n_nodes, H, Hp, pad;
    int rows[NP];
    float bf[NP * NP];
};

struct alignas(16) MFwd {       // 64 B: one warp, one decision node, 32 float4 groups
    long long reach_in;         // arena offset of the actor's reach at the node
    long long child;            // arena offset of child 0's part of the actor
    long long rows;             // R/S offset of the node's first row
    int h4, hs4, na, g0;
    int sub, pad[5];
};
struct alignas(16) MBwd {       // 64 B
    long long child;            // CFV-region offset of child 0's part of player q
    long long self;             // CFV-region offset of this node's part of q
    long long rows;             // R/S offset (q acts here)
    long long reach;            // arena offset of q's reach at the node (q acts here)
    int h4, hs4, na, flags;     // flags: 1 = q acts here
    int g0, sub, pad[2];
};
static_assert(sizeof(MFwd) == 64 && sizeof(MBwd) == 64, "item sizes");

struct MwDev {
    const MDesc* desc;
    const MNode* nodes;
    const uint16_t* tabs;
    const float* ranges;
    float* arena;
    float* R;
    float* S;
    const float* iter_tab;
    int* iter;
    int algo, semantics;
};

enum { MODE_SOLVE = 0, MODE_AVG = 1 };

__device__ __forceinline__ float4 f4(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
    return make_float4(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z), __fmul_rn(a.w, b.w));
}
__device__ __forceinline__ float4 fma4(float4 a, float4 b, float4 c) {
    return make_float4(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y), __fmaf_rn(a.z, b.z, c.z),
                       __fmaf_rn(a.w, b.w, c.w));
}
__device__ __forceinline__ float4 max04(float4 a) {
    return make_float4(fmaxf(a.x, 0.f), fmaxf(a.y, 0.f), fmaxf(a.z, 0.f), fmaxf(a.w, 0.f));
}
__device__ __forceinline__ float rm1(float pos, float sum, float invA) { return sum > 1e-7f ? __fdiv_rn(pos, sum) : invA; }
__device__ __forceinline__ float avg1(float s, float sum, float invA) { return sum > 0.0f ? __fdiv_rn(s, sum) : invA; }

// sigma of action k for one float4 group: regret matching on R (threshold
// 1e-7, multiway_4way_engine.cu:52-62) or the normalised average S.
template <int MODE>
__device__ __forceinline__ float4 sigma_at(const float4* B, int H4, int g, int k, float4 sum, float invA) {
    const float4 v = B[(size_t)k * H4 + g];
    if (MODE == MODE_SOLVE) {
        const float4 p = max04(v);
        return make_float4(rm1(p.x, sum.x, invA), rm1(p.y, sum.y, invA), rm1(p.z, sum.z, invA), rm1(p.w, sum.w, invA));
    }
    return make_float4(avg1(v.x, sum.x, invA), avg1(v.y, sum.y, invA), avg1(v.z, sum.z, invA), avg1(v.w, sum.w, invA));
}
template <int MODE>
__device__ __forceinline__ float4 sigma_sum(const float4* B, int H4, int g, int A) {
    float4 s = f4(0.f);
    for (int k = 0; k < A; ++k) s = add4(s, MODE == MODE_SOLVE ? max04(B[(size_t)k * H4 + g]) : B[(size_t)k * H4 + g]);
    return s;
}

__global__ void k_mw_init(MwDev a, int n_sub, int zero_rs) {
    const int s = blockIdx.x;
    if (s == 0 && threadIdx.x == 0) *a.iter = 1;
    if (s >= n_sub) return;
    const MDesc d = a.desc[s];
    if (zero_rs) {
        for (int p = 0; p < NP; ++p) {
            const long long end = d.rs_base[p] + (long long)d.rows[p] * d.Hp;
            for (long long i = d.rs_base[p] + threadIdx.x; i < end; i += blockDim.x) { a.R[i] = 0.f; a.S[i] = 0.f; }
        }
    }
    float* rr = a.arena + d.arena_base;
    for (int i = threadIdx.x; i < NP * d.Hp; i += blockDim.x) rr[i] = a.ranges[d.range_base + i];
}

__global__ void k_mw_next_iter(MwDev a) {
    if (threadIdx.x == 0) *a.iter += 1;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_mw_fwd(MwDev a, const MFwd* __restrict__ items, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    const MFwd it = items[w];      // work items are written once, before any solve
    grid_dep_trigger();
    grid_dep_wait();
    const int g = it.g0 + lane;
    if (g >= it.h4) return;
    const int A = it.na, H4 = it.h4, HS4 = it.hs4;
    const float4* B = reinterpret_cast<const float4*>((MODE == MODE_SOLVE ? a.R : a.S) + it.rows);
    const float4* rp = reinterpret_cast<const float4*>(a.arena + it.reach_in);
    float4* ch = reinterpret_cast<float4*>(a.arena + it.child);
    const float invA = __fdiv_rn(1.0f, (float)A);
    const float4 sum = sigma_sum<MODE>(B, H4, g, A);
    const float4 r = rp[g];
    for (int k = 0; k < A; ++k) ch[(size_t)k * HS4 + g] = mul4(r, sigma_at<MODE>(B, H4, g, k, sum, invA));
}

template <int MODE>
__global__ void __launch_bounds__(256) k_mw_bwd(MwDev a, const MBwd* __restrict__ items, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    const MBwd it = items[w];      // work items are written once, before any solve
    grid_dep_trigger();
    grid_dep_wait();
    const int g = it.g0 + lane;
    if (g >= it.h4) return;
    const int A = it.na, H4 = it.h4, HS4 = it.hs4;
    const float4* qc = reinterpret_cast<const float4*>(a.arena + it.child);
    float4* out = reinterpret_cast<float4*>(a.arena + it.self);
    if (!(it.flags & 1)) {
        float4 so = f4(0.f);
        for (int k = 0; k < A; ++k) so = add4(so, qc[(size_t)k * HS4 + g]);
        out[g] = so;
        return;
    }
    float4* Rb = reinterpret_cast<float4*>(a.R + it.rows);
    float4* Sb = reinterpret_cast<float4*>(a.S + it.rows);
    const float4* B = MODE == MODE_SOLVE ? Rb : Sb;
    const float invA = __fdiv_rn(1.0f, (float)A);
    const float4 sum = sigma_sum<MODE>(B, H4, g, A);
    float4 v = f4(0.f);
    for (int k = 0; k < A; ++k) v = fma4(sigma_at<MODE>(B, H4, g, k, sum, invA), qc[(size_t)k * HS4 + g], v);
    out[g] = v;
    if (MODE != MODE_SOLVE) return;
    // kernel_4way_backward_cfr_plus (:219-257): regret update and strategy sum
    const float4 tb = *reinterpret_cast<const float4*>(a.iter_tab + 4 * (*a.iter - 1));
    const bool dcfr = a.algo == MTT_ALGO_DCFR;
    const float4 r = reinterpret_cast<const float4*>(a.arena + it.reach)[g];
    const float4 wr = mul4(r, f4(tb.x));
    for (int k = 0; k < A; ++k) {
        const float4 sg = sigma_at<MODE_SOLVE>(Rb, H4, g, k, sum, invA);
        const float4 rk = Rb[(size_t)k * H4 + g];
        const float4 qk = qc[(size_t)k * HS4 + g];
        float4 nr;
        if (dcfr) {
            nr.x = __fadd_rn(__fmul_rn(rk.x, rk.x > 0.f ? tb.y : tb.z), __fsub_rn(qk.x, v.x));
            nr.y = __fadd_rn(__fmul_rn(rk.y, rk.y > 0.f ? tb.y : tb.z), __fsub_rn(qk.y, v.y));
            nr.z = __fadd_rn(__fmul_rn(rk.z, rk.z > 0.f ? tb.y : tb.z), __fsub_rn(qk.z, v.z));
            nr.w = __fadd_rn(__fmul_rn(rk.w, rk.w > 0.f ? tb.y : tb.z), __fsub_rn(qk.w, v.w));
        } else {
            nr.x = fmaxf(0.f, __fadd_rn(rk.x, __fsub_rn(qk.x, v.x)));
            nr.y = fmaxf(0.f, __fadd_rn(rk.y, __fsub_rn(qk.y, v.y)));
            nr.z = fmaxf(0.f, __fadd_rn(rk.z, __fsub_rn(qk.z, v.z)));
            nr.w = fmaxf(0.f, __fadd_rn(rk.w, __fsub_rn(qk.w, v.w)));
        }
        float4 sv = Sb[(size_t)k * H4 + g];
        sv = dcfr ? fma4(r, sg, mul4(sv, f4(tb.w))) : fma4(wr, sg, sv);
        Rb[(size_t)k * H4 + g] = nr;
        Sb[(size_t)k * H4 + g] = sv;
    }
}

constexpr int MT = 256;   // threads per terminal CTA

__device__ __forceinline__ double mw_block_sum(double v, double* wb, int tid) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((tid & 31) == 0) wb[tid >> 5] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < MT / 32; ++k) t += wb[k];
    __syncthreads();
    return t;
}

// One terminal per CTA: every player's reach scattered into rank-position
// order and scanned (exclusive, FP64), then the values of all four players.
__global__ void __launch_bounds__(MT) k_mw_term(MwDev a, const int2* __restrict__ terms, int n) {
    extern __shared__ __align__(16) double xs[];     // [NP][Hp + 1]
    __shared__ double wb[MT / 32];
    __shared__ double tot[NP];
    const int t = blockIdx.x, tid = threadIdx.x;
    if (t >= n) return;
    const int node = terms[t].x, sub = terms[t].y;
    const MDesc d = a.desc[sub];
    const MNode nd = a.nodes[node];
    const int H = d.H, Hp = d.Hp, X = Hp + 1;
    const uint16_t* pos = a.tabs + d.tab_base;
    const uint16_t* gs = pos + Hp;
    const uint16_t* ge = gs + Hp;
    const long long HS = (long long)NP * Hp;
    const int k_local = node - (int)d.node_base;
    grid_dep_trigger();
    grid_dep_wait();
    for (int o = 0; o < NP; ++o) {
        const float* ro = a.arena + d.arena_base + (long long)nd.src[o] * HS + (long long)o * Hp;
        for (int h = tid; h < Hp; h += MT) xs[o * X + (h < H ? pos[h] : h)] = h < H ? (double)ro[h] : 0.0;
    }
    __syncthreads();
    // exclusive scans, one player at a time (chunked per thread, then across warps)
    for (int o = 0; o < NP; ++o) {
        double* x = xs + o * X;
        const int C = (Hp + MT - 1) / MT;
        const int s0 = min(tid * C, Hp), s1 = min(s0 + C, Hp);
        double loc = 0.0;
        for (int k = s0; k < s1; ++k) loc += x[k];
        const int lane = tid & 31, wid = tid >> 5;
        double inc = loc;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double v = __shfl_up_sync(0xFFFFFFFFu, inc, off);
            if (lane >= off) inc += v;
        }
        double run = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
        if (lane == 0) run = 0.0;
        if (lane == 31) wb[wid] = inc;
        __syncthreads();
        double base = 0.0, total = 0.0;
#pragma unroll
        for (int k = 0; k < MT / 32; ++k) {
            if (k < wid) base += wb[k];
            total += wb[k];
        }
        run += base;
        for (int k = s0; k < s1; ++k) {
            const double v = x[k];
            x[k] = run;
            run += v;
        }
        if (tid == 0) { x[Hp] = total; tot[o] = total; }
        __syncthreads();
    }
    const int am = nd.amask;
    float* outb = a.arena + d.arena_base + (long long)d.n_nodes * HS + (long long)k_local * HS;
    for (int h = tid; h < Hp; h += MT) {
        for (int p = 0; p < NP; ++p) {
            double v = 0.0;
            if (h < H) {
                double others = 1.0;
                for (int o = 0; o < NP; ++o) if (o != p) others *= tot[o];
                if (nd.type == MTT_NODE_FOLD) {
                    const int w = __ffs(am) - 1;
                    v = (p == w ? (double)nd.pot - (double)nd.c[p] : -(double)d.bf[p * NP + w] * (double)nd.c[p]) * others;
                } else if (!((am >> p) & 1)) {
                    v = -(double)d.bf[p * NP + p] * (double)nd.c[p] * others;
                } else {
                    const double gain = (double)nd.pot - (double)nd.c[p];
                    const double loss = -(double)d.bf[p * NP + p] * (double)nd.c[p];
                    double inact = 1.0, PW = 1.0;
                    int opp[NP - 1], no = 0;
                    for (int o = 0; o < NP; ++o) {
                        if (o == p) continue;
                        if ((am >> o) & 1) { PW *= tot[o]; opp[no++] = o; }
                        else inact *= tot[o];
                    }
                    if (a.semantics == MTT_SEM_REFERENCE) {
                        const int ps = pos[h];
                        double F = 1.0;
                        for (int i = 0; i < no; ++i) F *= xs[opp[i] * X + ps];
                        v = (gain * F + loss * (PW - F)) * inact;
                    } else {
                        const int s0 = gs[h], s1 = ge[h];
                        double L[NP - 1], E[NP - 1], LE = 1.0;
                        for (int i = 0; i < no; ++i) {
                            L[i] = xs[opp[i] * X + s0];
                            E[i] = xs[opp[i] * X + s1] - L[i];
                            LE *= L[i] + E[i];
                        }
                        double share = 0.0;
                        for (int T = 0; T < (1 << no); ++T) {
                            double pr = 1.0;
                            for (int i = 0; i < no; ++i) pr *= ((T >> i) & 1) ? E[i] : L[i];
                            share += pr * ((double)nd.pot / (1 + __popc(T)) - (double)nd.c[p]);
                        }
                        v = (share + loss * (PW - LE)) * inact;
                    }
                }
            }
            outb[(long long)p * Hp + h] = (float)v;
        }
    }
}

// The correct semantics' terminal, one terminal per CTA.  Each player's reach
// at the terminal is staged in shared memory (coalesced), scaled by a power of
// two 2^k_o with S_o 2^k_o < 2^29 for its absolute mass S_o and rounded to
// int32, then gathered into [rank order | per-card lists in rank order] (3 H
// positions) and scanned exclusively in integers.  Per hero hand h and
// opponent o, the masses of o's hands that share no card with h, ranked below
// (L), equal (E) and in total (W), are integer differences of that scan (the
// heads-up terminals' construction: the per-card lists of h's two cards are
// subtracted, the combo h itself, counted in both, added back once), exact
// and independent of the summation order, so a mass that is zero stays zero.
// Every prefix is below 3 (2^29 + H / 2) < 2^31; each reach value is off by at
// most 2^-30 S_o.  The payoffs are then formed in FP32 (the masses as
// float, relative error 2^-24; FP64 products measured within 3e-6 of these,
// and took 128 registers, two CTAs per SM, against 73 and three here).
__global__ void __launch_bounds__(MT, 3) k_mw_term_cr(MwDev a, const int2* __restrict__ terms, int n) {
    extern __shared__ __align__(16) int xsi[];       // [NP][3 H + 1] scans, then [NP][Hp] staged reach
    __shared__ int wbi[MT / 32];
    __shared__ float wsum[NP][MT / 32];
    __shared__ int2 ct[NP][52];                      // per player and card: scan at the list start, list mass
    __shared__ double inv_s[NP];                     // 2^-k_o
    const int t = blockIdx.x, tid = threadIdx.x;
    if (t >= n) return;
    const int node = terms[t].x, sub = terms[t].y;
    const MDesc d = a.desc[sub];
    const MNode nd = a.nodes[node];
    const int H = d.H, Hp = d.Hp, N = 3 * H, X = N + 1;
    const uint16_t* idx = a.tabs + d.ctab_base;
    const uint16_t* seg = idx + N;
    const MwEntry* ent = reinterpret_cast<const MwEntry*>(a.tabs + d.cent_base);
    const long long HS = (long long)NP * Hp;
    const int k_local = node - (int)d.node_base;
    float* rf = reinterpret_cast<float*>(xsi + NP * X);   // [NP][Hp] floats, then the same words as int
    int* ri = xsi + NP * X;
    const int lane = tid & 31, wid = tid >> 5;
    grid_dep_trigger();
    grid_dep_wait();
    // stage every player's reach (float4, coalesced) and its absolute mass
    for (int o = 0; o < NP; ++o) {
        const float4* src = reinterpret_cast<const float4*>(a.arena + d.arena_base + (long long)nd.src[o] * HS +
                                                            (long long)o * Hp);
        float4* dst = reinterpret_cast<float4*>(rf + o * Hp);
        float part = 0.f;
        for (int j = tid; j < (Hp >> 2); j += MT) {
            float4 v = src[j];
            const int h0 = 4 * j;
            if (h0 + 0 >= H) v.x = 0.f;
            if (h0 + 1 >= H) v.y = 0.f;
            if (h0 + 2 >= H) v.z = 0.f;
            if (h0 + 3 >= H) v.w = 0.f;
            dst[j] = v;
            part += (fabsf(v.x) + fabsf(v.y)) + (fabsf(v.z) + fabsf(v.w));
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, off);
        if (lane == 0) wsum[o][wid] = part;
    }
    __syncthreads();
    // the power-of-two scale of each player and the rounding to int32, in place
    for (int o = 0; o < NP; ++o) {
        float S = 0.f;
#pragma unroll
        for (int k = 0; k < MT / 32; ++k) S += wsum[o][k];
        const int E = (int)((__float_as_uint(S) >> 23) & 0xFFu);
        const int e = E == 0 ? -126 : E - 126;                       // S < 2^e
        const int kk = S > 0.f ? min(max(29 - e, -126), 126) : 0;
        const float f = __uint_as_float((uint32_t)(127 + kk) << 23);
        if (tid == 0) inv_s[o] = (double)__uint_as_float((uint32_t)(127 - kk) << 23);
        for (int j = tid; j < Hp; j += MT) ri[o * Hp + j] = __float2int_rn(__fmul_rn(rf[o * Hp + j], f));
    }
    __syncthreads();
    for (int o = 0; o < NP; ++o)
        for (int k = tid; k < N; k += MT) xsi[o * X + k] = ri[o * Hp + idx[k]];
    __syncthreads();
    const int C = (N + MT - 1) / MT;
    const int s0 = min(tid * C, N), s1 = min(s0 + C, N);
    for (int o = 0; o < NP; ++o) {
        int* x = xsi + o * X;
        int loc = 0;
        for (int k = s0; k < s1; ++k) loc += x[k];
        int inc = loc;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(0xFFFFFFFFu, inc, off);
            if (lane >= off) inc += v;
        }
        int run = inc - loc;
        if (lane == 31) wbi[wid] = inc;
        __syncthreads();
        int total = 0;
#pragma unroll
        for (int k = 0; k < MT / 32; ++k) {
            if (k < wid) run += wbi[k];
            total += wbi[k];
        }
        for (int k = s0; k < s1; ++k) {
            const int v = x[k];
            x[k] = run;
            run += v;
        }
        if (tid == 0) x[N] = total;
        __syncthreads();
    }
    for (int i = tid; i < NP * 52; i += MT) {
        const int o = i / 52, c = i - 52 * o;
        const int b0 = xsi[o * X + H + seg[c]];
        ct[o][c] = make_int2(b0, (int)((unsigned)xsi[o * X + H + seg[c + 1]] - (unsigned)b0));
    }
    __syncthreads();
    const int am = nd.amask;
    const bool fold = nd.type == MTT_NODE_FOLD;
    const int winner = __ffs(am) - 1;
    const float pot = nd.pot;
    float* outb = a.arena + d.arena_base + (long long)d.n_nodes * HS + (long long)k_local * HS;
    for (int h = tid; h < Hp; h += MT) {
        float L[NP], E[NP], W[NP];
#pragma unroll
        for (int o = 0; o < NP; ++o) { L[o] = 0.f; E[o] = 0.f; W[o] = 0.f; }
        if (h < H) {
            const MwEntry e = ent[h];
#pragma unroll
            for (int o = 0; o < NP; ++o) {
                const int* x = xsi + o * X;
                const int2 k1 = ct[o][e.c1], k2 = ct[o][e.c2];
                const unsigned rh = (unsigned)ri[o * Hp + h];
                const unsigned l = (unsigned)x[e.lt] - ((unsigned)x[e.c1lt] - (unsigned)k1.x) -
                                   ((unsigned)x[e.c2lt] - (unsigned)k2.x);
                const unsigned le = (unsigned)x[e.le] - ((unsigned)x[e.c1le] - (unsigned)k1.x) -
                                    ((unsigned)x[e.c2le] - (unsigned)k2.x) + rh;
                const unsigned w = (unsigned)x[H] - (unsigned)k1.y - (unsigned)k2.y + rh;
                const float sc = (float)inv_s[o];
                L[o] = (float)(int)l * sc;
                E[o] = (float)(int)(le - l) * sc;
                W[o] = (float)(int)w * sc;
            }
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            float v = 0.f;
            if (h < H) {
                float others = 1.f;
#pragma unroll
                for (int o = 0; o < NP; ++o) if (o != p) others *= W[o];
                const float cp = nd.c[p];
                if (fold) {
                    v = (p == winner ? pot - cp : -d.bf[p * NP + winner] * cp) * others;
                } else if (!((am >> p) & 1)) {
                    v = -d.bf[p * NP + p] * cp * others;
                } else {
                    // the opponents in seat order (slots 0..2); an inactive one
                    // contributes its total mass and never ties
                    float inact = 1.f, PW = 1.f, LE = 1.f;
#pragma unroll
                    for (int o = 0; o < NP; ++o) {
                        if (o == p) continue;
                        if ((am >> o) & 1) { PW *= W[o]; LE *= L[o] + E[o]; }
                        else inact *= W[o];
                    }
                    float share = 0.f;
#pragma unroll
                    for (int T = 0; T < 8; ++T) {
                        float pr = 1.f;
                        int nt = 0;
                        bool valid = true;
                        int slot = 0;
#pragma unroll
                        for (int o = 0; o < NP; ++o) {
                            if (o == p) continue;
                            const bool act = (am >> o) & 1;
                            const bool tie = (T >> slot) & 1;
                            ++slot;
                            if (!act) { valid = valid && !tie; continue; }
                            pr *= tie ? E[o] : L[o];
                            nt += tie ? 1 : 0;
                        }
                        if (valid) share += pr * (pot / (float)(1 + nt) - cp);
                    }
                    v = (share - d.bf[p * NP + p] * cp * (PW - LE)) * inact;
                }
            }
            outb[(long long)p * Hp + h] = v;
        }
    }
}

__global__ void __launch_bounds__(MT) k_mw_root(MwDev a, int n_sub, double* out) {
    __shared__ double wb[MT / 32];
    const int s = blockIdx.x, tid = threadIdx.x;
    if (s >= n_sub) return;
    const MDesc d = a.desc[s];
    const long long HS = (long long)NP * d.Hp;
    const float* cf = a.arena + d.arena_base + (long long)d.n_nodes * HS;
    for (int p = 0; p < NP; ++p) {
        double acc = 0.0;
        for (int h = tid; h < d.H; h += MT)
            acc += (double)a.ranges[d.range_base + (long long)p * d.Hp + h] * (double)cf[(long long)p * d.Hp + h];
        acc = mw_block_sum(acc, wb, tid);
        if (tid == 0) out[4 * s + p] = acc;
    }
}

}  // namespace mw
}  // namespace mtt

using namespace mtt;
using namespace mtt::mw;

struct mtt_mw_batch {
    int n = 0, levels = 0, Hmax = 0;
    MDesc* d_desc = nullptr;
    MNode* d_nodes = nullptr;
    uint16_t* d_tabs = nullptr;
    float* d_ranges = nullptr;
    float* d_arena = nullptr;
    float* d_R = nullptr;
    float* d_S = nullptr;
    int* d_iter = nullptr;
    float* d_iter_tab = nullptr;
    int iter_cap = 0;
    double* d_values = nullptr;
    MFwd* d_fwd = nullptr;
    MBwd* d_bwd = nullptr;
    int2* d_terms = nullptr;
    std::vector<long long> fwd_off, bwd_off;   // per level
    int n_terms = 0;
    std::vector<MDesc> desc;
    std::vector<int> rows;                      // 4 per subgame
    cudaGraphExec_t gexec = nullptr;
    int g_algo = -1, g_sem = -1;
    int last_sem = MTT_SEM_CORRECT;             // semantics of the last solve (used by the values pass)
};

namespace {
template <typename T>
int dalloc(T** p, size_t count) {
    return cuda_status(cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T)));
}

void free_mw(mtt_mw_batch* b) {
    if (!b) return;
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    cudaFree(b->d_desc); cudaFree(b->d_nodes); cudaFree(b->d_tabs); cudaFree(b->d_ranges); cudaFree(b->d_arena);
    cudaFree(b->d_R); cudaFree(b->d_S); cudaFree(b->d_iter); cudaFree(b->d_iter_tab); cudaFree(b->d_values);
    cudaFree(b->d_fwd); cudaFree(b->d_bwd); cudaFree(b->d_terms);
    delete b;
}

// Dynamic shared memory of k_mw_term_cr: four int32 scans of 3 H + 1
// positions and the four staged reach vectors.
size_t term_cr_smem(const mtt_mw_batch* b) {
    return sizeof(int) * (size_t)NP * (3 * (size_t)b->Hmax + 1) + sizeof(float) * (size_t)NP * (size_t)b->Hmax + 16;
}

MwDev mw_args(const mtt_mw_batch* b, int algo, int sem) {
    MwDev a;
    a.desc = b->d_desc; a.nodes = b->d_nodes; a.tabs = b->d_tabs; a.ranges = b->d_ranges; a.arena = b->d_arena;
    a.R = b->d_R; a.S = b->d_S; a.iter_tab = b->d_iter_tab; a.iter = b->d_iter; a.algo = algo; a.semantics = sem;
    return a;
}

int launch_sweep(const mtt_mw_batch* b, const MwDev& a, int mode, cudaStream_t st) {
    // every level and the terminals are launched with programmatic stream
    // serialization (the sweep's first level follows the iteration counter,
    // an ordinary launch).  A single subgame's launches are short, so the
    // next kernel's CTAs starting during the previous one's tail pays; the
    // batched solver chains only within a kernel class.
    bool chained = false;
    for (int d = 0; d < b->levels; ++d) {
        const long long n = b->fwd_off[d + 1] - b->fwd_off[d];
        if (!n) continue;
        const unsigned grid = (unsigned)((n + 7) / 8);
        const MFwd* items = b->d_fwd + b->fwd_off[d];
        if (mode == MODE_SOLVE) MTT_TRY_CUDA(launch_pdl(k_mw_fwd<MODE_SOLVE>, grid, 256, 0, st, chained, a, items, (int)n));
        else MTT_TRY_CUDA(launch_pdl(k_mw_fwd<MODE_AVG>, grid, 256, 0, st, chained, a, items, (int)n));
        MTT_CHECK_LAUNCH();
        chained = true;
    }
    if (b->n_terms) {
        if (a.semantics == MTT_SEM_CORRECT) {
            MTT_TRY_CUDA(launch_pdl(k_mw_term_cr, (unsigned)b->n_terms, MT, term_cr_smem(b), st, true, a,
                                    (const int2*)b->d_terms, b->n_terms));
        } else {
            const size_t smem = sizeof(double) * (size_t)NP * ((size_t)b->Hmax + 1);
            MTT_TRY_CUDA(launch_pdl(k_mw_term, (unsigned)b->n_terms, MT, smem, st, true, a, (const int2*)b->d_terms, b->n_terms));
        }
        MTT_CHECK_LAUNCH();
    }
    chained = true;
    for (int d = b->levels - 1; d >= 0; --d) {
        const long long n = b->bwd_off[d + 1] - b->bwd_off[d];
        if (!n) continue;
        const unsigned grid = (unsigned)((n + 7) / 8);
        const MBwd* items = b->d_bwd + b->bwd_off[d];
        if (mode == MODE_SOLVE) MTT_TRY_CUDA(launch_pdl(k_mw_bwd<MODE_SOLVE>, grid, 256, 0, st, chained, a, items, (int)n));
        else MTT_TRY_CUDA(launch_pdl(k_mw_bwd<MODE_AVG>, grid, 256, 0, st, chained, a, items, (int)n));
        MTT_CHECK_LAUNCH();
        chained = true;
    }
    return MTT_OK;
}

int launch_iteration(const mtt_mw_batch* b, const MwDev& a, cudaStream_t st) {
    MTT_TRY(launch_sweep(b, a, MODE_SOLVE, st));
    k_mw_next_iter<<<1, 32, 0, st>>>(a);
    MTT_CHECK_LAUNCH();
    return MTT_OK;
}

int set_term_smem(const mtt_mw_batch* b) {
    const size_t smem = sizeof(double) * (size_t)NP * ((size_t)b->Hmax + 1);
    if (smem > 48 * 1024)
        MTT_TRY_CUDA(cudaFuncSetAttribute(k_mw_term, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const size_t cr = term_cr_smem(b);
    if (cr > 48 * 1024)
        MTT_TRY_CUDA(cudaFuncSetAttribute(k_mw_term_cr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cr));
    return MTT_OK;
}
}  // namespace

extern "C" int mtt_mw_tree_build(const mtt_mw_spec* spec, mtt_mw_node* nodes, int32_t capacity, int32_t* n_nodes,
                                 int32_t rows[4], int32_t* max_depth) {
    if (!spec || !n_nodes || !rows) return MTT_ERR_INVALID;
    std::vector<mtt_mw_node> v;
    int r[NP] = {0, 0, 0, 0}, md = 0;
    MTT_TRY(build_tree(*spec, v, r, &md));
    *n_nodes = (int32_t)v.size();
    for (int p = 0; p < NP; ++p) rows[p] = r[p];
    if (max_depth) *max_depth = md;
    if (!nodes) return MTT_OK;
    if (capacity < (int32_t)v.size()) return MTT_ERR_INVALID;
    std::memcpy(nodes, v.data(), sizeof(mtt_mw_node) * v.size());
    return MTT_OK;
}

extern "C" int mtt_mw_batch_create(const mtt_mw_subgame* subs, int32_t n, mtt_mw_batch** out) {
    if (!subs || n <= 0 || !out) return MTT_ERR_INVALID;
    *out = nullptr;
    mtt_mw_batch* b = new mtt_mw_batch();
    b->n = n;
    std::vector<MNode> hn;
    std::vector<uint16_t> ht;
    std::vector<float> hr;
    std::vector<std::vector<MFwd>> fl;
    std::vector<std::vector<MBwd>> bl;
    std::vector<int2> tl;
    long long arena = 0, rs = 0;
    b->desc.resize(n);
    b->rows.resize(4 * (size_t)n);
    for (int s = 0; s < n; ++s) {
        const mtt_mw_subgame& g = subs[s];
        int rws[NP];
        for (int p = 0; p < NP; ++p) rws[p] = g.rows[p];
        int st = validate(g.nodes, g.n_nodes, rws);
        if (!st && (g.H < 1 || g.H > 1326 || !g.combos)) st = MTT_ERR_INVALID;
        for (int p = 0; p < NP && !st; ++p) if (!g.ranges[p]) st = MTT_ERR_INVALID;
        uint64_t bm = 0;
        for (int k = 0; k < 5 && !st; ++k) {
            if (g.board[k] >= 52 || ((bm >> g.board[k]) & 1)) st = MTT_ERR_INVALID;
            bm |= 1ull << g.board[k];
        }
        std::vector<uint16_t> cards(g.H);
        for (int h = 0; h < g.H && !st; ++h) {
            const int c = g.combos[h];
            if (c >= 1326 || (h && c <= g.combos[h - 1])) { st = MTT_ERR_INVALID; break; }
            int a = 0, r = c;
            while (r >= 51 - a) { r -= 51 - a; ++a; }
            const int c2 = a + 1 + r;
            if (((bm >> a) & 1) || ((bm >> c2) & 1)) { st = MTT_ERR_INVALID; break; }
            cards[h] = (uint16_t)(a | (c2 << 8));
        }
        if (st) { free_mw(b); return st; }
        MDesc d{};
        d.n_nodes = g.n_nodes;
        d.H = g.H;
        d.Hp = (g.H + 3) & ~3;
        const long long HS = (long long)NP * d.Hp;
        d.node_base = (long long)hn.size();
        d.arena_base = arena;
        d.tab_base = (long long)ht.size();
        d.range_base = (long long)hr.size();
        for (int p = 0; p < NP; ++p) { d.rs_base[p] = rs; rs += (long long)g.rows[p] * d.Hp; }
        for (int p = 0; p < NP; ++p) d.rows[p] = g.rows[p];
        for (int k = 0; k < 16; ++k) d.bf[k] = g.bubble[k];
        arena += 2LL * g.n_nodes * HS;
        b->Hmax = std::max(b->Hmax, d.Hp);
        // rank tables: score of every hand on the board, positions by ascending score
        std::vector<uint32_t> sc(g.H);
        for (int h = 0; h < g.H; ++h) {
            Planes pl; planes_clear(pl);
            for (int k = 0; k < 5; ++k) planes_add(pl, g.board[k]);
            planes_add(pl, cards[h] & 0xFF);
            planes_add(pl, cards[h] >> 8);
            sc[h] = score_planes(pl);
        }
        std::vector<int> ord(g.H);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return sc[x] < sc[y]; });
        std::vector<uint16_t> pos(d.Hp, 0), gsv(d.Hp, 0), gev(d.Hp, 0);
        for (int i = 0; i < g.H;) {
            int j = i;
            while (j < g.H && sc[ord[j]] == sc[ord[i]]) ++j;
            for (int k = i; k < j; ++k) { pos[ord[k]] = (uint16_t)k; gsv[ord[k]] = (uint16_t)i; gev[ord[k]] = (uint16_t)j; }
            i = j;
        }
        ht.insert(ht.end(), pos.begin(), pos.end());
        ht.insert(ht.end(), gsv.begin(), gsv.end());
        ht.insert(ht.end(), gev.begin(), gev.end());
        // card-removal lists: hands in rank order, then per card the hands
        // holding it in rank order, the list starts, and per hand its
        // positions in that 3 H scan (MwEntry; lt / le = its rank group)
        {
            const int H = g.H;
            std::vector<std::vector<uint16_t>> by(52);
            for (int i = 0; i < H; ++i) {
                const int h = ord[i];
                by[cards[h] & 0xFF].push_back((uint16_t)h);
                by[cards[h] >> 8].push_back((uint16_t)h);
            }
            std::vector<uint16_t> seg(54, 0), cl;
            for (int c = 0; c < 52; ++c) {
                seg[c] = (uint16_t)cl.size();
                cl.insert(cl.end(), by[c].begin(), by[c].end());
            }
            seg[52] = seg[53] = (uint16_t)cl.size();
            while (ht.size() % 8) ht.push_back(0);
            d.ctab_base = (long long)ht.size();
            for (int i = 0; i < H; ++i) ht.push_back((uint16_t)ord[i]);
            ht.insert(ht.end(), cl.begin(), cl.end());
            ht.insert(ht.end(), seg.begin(), seg.end());
            while (ht.size() % 8) ht.push_back(0);
            d.cent_base = (long long)ht.size();
            auto card_pos = [&](int c, uint32_t sv, bool upper) {
                int k = seg[c];
                const int end = seg[c + 1];
                while (k < end && (sc[cl[k]] < sv || (upper && sc[cl[k]] == sv))) ++k;
                return (uint16_t)(H + k);
            };
            for (int h = 0; h < H; ++h) {
                MwEntry e{};
                const int c1 = cards[h] & 0xFF, c2 = cards[h] >> 8;
                e.lt = gsv[h];
                e.le = gev[h];
                e.c1lt = card_pos(c1, sc[h], false);
                e.c1le = card_pos(c1, sc[h], true);
                e.c2lt = card_pos(c2, sc[h], false);
                e.c2le = card_pos(c2, sc[h], true);
                e.c1 = (uint8_t)c1;
                e.c2 = (uint8_t)c2;
                uint16_t w[8];
                std::memcpy(w, &e, sizeof(e));
                ht.insert(ht.end(), w, w + 8);
            }
        }
        for (int p = 0; p < NP; ++p)
            for (int h = 0; h < d.Hp; ++h) hr.push_back(h < g.H ? g.ranges[p][h] : 0.0f);
        // nodes with reach sources and depths
        std::vector<int> depth(g.n_nodes, 0);
        std::vector<MNode> loc(g.n_nodes);
        for (int k = 0; k < g.n_nodes; ++k) {
            const mtt_mw_node& x = g.nodes[k];
            MNode& m = loc[k];
            m.type = x.type; m.player = x.player; m.na = x.num_actions; m.amask = x.active_mask;
            m.first = x.children_offset; m.row = x.infoset_offset;
            m.pot = x.pot_size;
            for (int p = 0; p < NP; ++p) { m.c[p] = x.committed[p]; }
            if (k == 0) for (int p = 0; p < NP; ++p) m.src[p] = 0;
        }
        for (int k = 0; k < g.n_nodes; ++k) {
            const MNode& m = loc[k];
            if (m.type != MTT_NODE_DECISION) continue;
            for (int a = 0; a < m.na; ++a) {
                MNode& c = loc[m.first + a];
                depth[m.first + a] = depth[k] + 1;
                for (int p = 0; p < NP; ++p) c.src[p] = (p == m.player) ? m.first + a : m.src[p];
            }
        }
        int lv = 0;
        for (int k = 0; k < g.n_nodes; ++k) lv = std::max(lv, depth[k] + 1);
        if (lv > (int)fl.size()) { fl.resize(lv); bl.resize(lv); }
        b->levels = std::max(b->levels, lv);
        const int H4 = d.Hp / 4;
        for (int k = 0; k < g.n_nodes; ++k) {
            const MNode& m = loc[k];
            const int gn = (int)d.node_base + k;
            if (m.type == MTT_NODE_DECISION) {
                const int p = m.player;
                MFwd f{};
                f.reach_in = d.arena_base + (long long)m.src[p] * HS + (long long)p * d.Hp;
                f.child = d.arena_base + (long long)m.first * HS + (long long)p * d.Hp;
                f.rows = d.rs_base[p] + (long long)m.row * d.Hp;
                f.h4 = H4; f.hs4 = (int)(HS / 4); f.na = m.na; f.sub = s;
                for (f.g0 = 0; f.g0 < H4; f.g0 += 32) fl[depth[k]].push_back(f);
                const long long cfv0 = d.arena_base + (long long)g.n_nodes * HS;
                for (int q = 0; q < NP; ++q) {
                    MBwd w{};
                    w.child = cfv0 + (long long)m.first * HS + (long long)q * d.Hp;
                    w.self = cfv0 + (long long)k * HS + (long long)q * d.Hp;
                    w.rows = q == p ? f.rows : 0;
                    w.reach = q == p ? f.reach_in : 0;
                    w.h4 = H4; w.hs4 = (int)(HS / 4); w.na = m.na; w.flags = q == p ? 1 : 0; w.sub = s;
                    for (w.g0 = 0; w.g0 < H4; w.g0 += 32) bl[depth[k]].push_back(w);
                }
            } else {
                tl.push_back(make_int2(gn, s));
            }
        }
        hn.insert(hn.end(), loc.begin(), loc.end());
        b->desc[s] = d;
        for (int p = 0; p < NP; ++p) b->rows[4 * (size_t)s + p] = g.rows[p];
    }
    // flatten the level lists
    std::vector<MFwd> ff;
    std::vector<MBwd> bb;
    b->fwd_off.assign(b->levels + 1, 0);
    b->bwd_off.assign(b->levels + 1, 0);
    for (int d = 0; d < b->levels; ++d) {
        ff.insert(ff.end(), fl[d].begin(), fl[d].end());
        bb.insert(bb.end(), bl[d].begin(), bl[d].end());
        b->fwd_off[d + 1] = (long long)ff.size();
        b->bwd_off[d + 1] = (long long)bb.size();
    }
    b->n_terms = (int)tl.size();
    int s = MTT_OK;
    if (!s) s = dalloc(&b->d_desc, n);
    if (!s) s = dalloc(&b->d_nodes, hn.size());
    if (!s) s = dalloc(&b->d_tabs, ht.size());
    if (!s) s = dalloc(&b->d_ranges, hr.size());
    if (!s) s = dalloc(&b->d_arena, (size_t)arena);
    if (!s) s = dalloc(&b->d_R, (size_t)rs);
    if (!s) s = dalloc(&b->d_S, (size_t)rs);
    if (!s) s = dalloc(&b->d_iter, 1);
    if (!s) s = dalloc(&b->d_values, 4 * (size_t)n);
    if (!s) s = dalloc(&b->d_fwd, ff.size());
    if (!s) s = dalloc(&b->d_bwd, bb.size());
    if (!s) s = dalloc(&b->d_terms, tl.size());
    if (!s) s = cuda_status(cudaMemcpy(b->d_desc, b->desc.data(), sizeof(MDesc) * n, cudaMemcpyHostToDevice));
    if (!s) s = cuda_status(cudaMemcpy(b->d_nodes, hn.data(), sizeof(MNode) * hn.size(), cudaMemcpyHostToDevice));
    if (!s) s = cuda_status(cudaMemcpy(b->d_tabs, ht.data(), 2 * ht.size(), cudaMemcpyHostToDevice));
    if (!s) s = cuda_status(cudaMemcpy(b->d_ranges, hr.data(), 4 * hr.size(), cudaMemcpyHostToDevice));
    if (!s && !ff.empty()) s = cuda_status(cudaMemcpy(b->d_fwd, ff.data(), sizeof(MFwd) * ff.size(), cudaMemcpyHostToDevice));
    if (!s && !bb.empty()) s = cuda_status(cudaMemcpy(b->d_bwd, bb.data(), sizeof(MBwd) * bb.size(), cudaMemcpyHostToDevice));
    if (!s && !tl.empty()) s = cuda_status(cudaMemcpy(b->d_terms, tl.data(), sizeof(int2) * tl.size(), cudaMemcpyHostToDevice));
    if (!s) s = cuda_status(cudaMemset(b->d_arena, 0, sizeof(float) * (size_t)std::max(arena, 1LL)));
    if (s) { free_mw(b); return s; }
    *out = b;
    return MTT_OK;
}

extern "C" int mtt_mw_batch_solve(mtt_mw_batch* b, const mtt_solve_params* p, int32_t graph, void* stream) {
    if (!b || !p || p->iters < 0 || (p->algo != MTT_ALGO_CFRPLUS && p->algo != MTT_ALGO_DCFR) ||
        (p->semantics != MTT_SEM_CORRECT && p->semantics != MTT_SEM_REFERENCE) ||
        !(p->avg_power >= 0.0f && p->avg_power <= 8.0f))
        return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    const int iters = std::max(p->iters, 1);
    if (iters > b->iter_cap) {
        MTT_TRY_CUDA(cudaStreamSynchronize(st));
        cudaFree(b->d_iter_tab);
        b->d_iter_tab = nullptr;
        b->iter_cap = 0;
        MTT_TRY_CUDA(cudaMalloc(&b->d_iter_tab, sizeof(float) * 4 * (size_t)iters));
        b->iter_cap = iters;
        if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    }
    std::vector<float> tab(4 * (size_t)iters);
    for (int t = 1; t <= iters; ++t) {
        const double tm1 = (double)(t - 1);
        float* e = &tab[4 * (size_t)(t - 1)];
        e[0] = (float)std::pow((double)t, (double)p->avg_power);
        e[1] = (float)(std::pow(tm1, (double)p->alpha) / (std::pow(tm1, (double)p->alpha) + 1.0));
        e[2] = (float)(std::pow(tm1, (double)p->beta) / (std::pow(tm1, (double)p->beta) + 1.0));
        e[3] = (float)std::pow(tm1 / (double)t, (double)p->gamma);
    }
    MTT_TRY_CUDA(cudaMemcpyAsync(b->d_iter_tab, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
    MTT_TRY(set_term_smem(b));
    b->last_sem = p->semantics;
    const MwDev a = mw_args(b, p->algo, p->semantics);
    k_mw_init<<<b->n, 256, 0, st>>>(a, b->n, 1);
    MTT_CHECK_LAUNCH();
    if (!graph) {
        for (int t = 0; t < p->iters; ++t) MTT_TRY(launch_iteration(b, a, st));
        return MTT_OK;
    }
    if (!b->gexec || b->g_algo != p->algo || b->g_sem != p->semantics) {
        if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
        cudaStream_t cs;
        MTT_TRY_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t gr = nullptr;
        int s = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        if (!s) s = launch_iteration(b, a, cs);
        const int s2 = cuda_status(cudaStreamEndCapture(cs, &gr));
        if (!s) s = s2;
        if (!s) s = cuda_status(cudaGraphInstantiate(&b->gexec, gr, 0));
        if (gr) cudaGraphDestroy(gr);
        cudaStreamDestroy(cs);
        if (s) return s;
        b->g_algo = p->algo;
        b->g_sem = p->semantics;
    }
    for (int t = 0; t < p->iters; ++t) MTT_TRY_CUDA(cudaGraphLaunch(b->gexec, st));
    return MTT_OK;
}

extern "C" int mtt_mw_batch_values(mtt_mw_batch* b, double* h_out, void* stream) {
    if (!b || !h_out) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    MTT_TRY(set_term_smem(b));
    const MwDev a = mw_args(b, MTT_ALGO_CFRPLUS, b->last_sem);
    k_mw_init<<<b->n, 256, 0, st>>>(a, b->n, 0);
    MTT_CHECK_LAUNCH();
    MTT_TRY(launch_sweep(b, a, MODE_AVG, st));
    k_mw_root<<<b->n, MT, 0, st>>>(a, b->n, b->d_values);
    MTT_CHECK_LAUNCH();
    MTT_TRY_CUDA(cudaMemcpyAsync(h_out, b->d_values, sizeof(double) * 4 * (size_t)b->n, cudaMemcpyDeviceToHost, st));
    MTT_TRY_CUDA(cudaStreamSynchronize(st));
    return MTT_OK;
}

extern "C" int mtt_mw_batch_read(mtt_mw_batch* b, int32_t s, float* h_R[4], float* h_S[4], float* h_cfv) {
    if (!b || s < 0 || s >= b->n) return MTT_ERR_INVALID;
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    const MDesc& d = b->desc[s];
    for (int p = 0; p < NP; ++p) {
        const int rows = b->rows[4 * (size_t)s + p];
        if (!rows) continue;
        if (h_R && h_R[p])
            MTT_TRY_CUDA(cudaMemcpy2D(h_R[p], sizeof(float) * d.H, b->d_R + d.rs_base[p], sizeof(float) * d.Hp,
                                      sizeof(float) * d.H, rows, cudaMemcpyDeviceToHost));
        if (h_S && h_S[p])
            MTT_TRY_CUDA(cudaMemcpy2D(h_S[p], sizeof(float) * d.H, b->d_S + d.rs_base[p], sizeof(float) * d.Hp,
                                      sizeof(float) * d.H, rows, cudaMemcpyDeviceToHost));
    }
    if (h_cfv) {
        const float* cf = b->d_arena + d.arena_base + (long long)d.n_nodes * NP * d.Hp;
        MTT_TRY_CUDA(cudaMemcpy2D(h_cfv, sizeof(float) * d.H, cf, sizeof(float) * d.Hp, sizeof(float) * d.H, NP,
                                  cudaMemcpyDeviceToHost));
    }
    return MTT_OK;
}

extern "C" int mtt_mw_batch_destroy(mtt_mw_batch* b) {
    if (!b) return MTT_ERR_INVALID;
    cudaDeviceSynchronize();
    free_mw(b);
    return MTT_OK;
}
