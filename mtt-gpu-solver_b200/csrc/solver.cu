// solver.cu — batched heads-up CFR+/DCFR solver and its FP64 best response.
//
// One persistent kernel solves every subgame of a batch: each CTA pulls the
// next subgame (largest first) from an atomic work queue and runs all
// iterations on it.  Inside a CTA each thread owns fixed groups of 4 hands
// (float4), so the forward sweep (regret matching, reach, strategy sums) and
// the backward sweep (counterfactual values, regret update) walk the tree
// node by node with NO barriers: a thread only ever reads values it wrote.
// Only terminals mix hands; they are evaluated CTA-wide with one exclusive
// prefix scan per terminal over the opponent reach in rank order and in
// per-card rank order, from which wins, ties and losses with card removal
// are O(1) differences (no 1326x1326 matrices).
//
// Update rules follow the reference kernels: kernel_forward_sweep
// (honest_multistreet_solver.cu:88-126), kernel_backward_sweep (:198-249),
// kernel_4way_* (multiway_4way_engine.cu:41-83,219-257) and the DCFR weights
// of kernel_dcfr_step (preflop_grid_generator.cu:387-410, in the
// discount-then-add form).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "mtt_common.h"
#include "mtt_device.cuh"
#include "solver_impl.cuh"

namespace mtt {

int validate_tree(const mtt_node* nodes, int n, const int rows[2]);   // tree.cpp

// Table variant of a terminal: river subgames have one board; turn subgames
// one per dealt river card plus index 52 for nodes before the chance layer
// (folds there need card lists only, no ranks).
__host__ __device__ __forceinline__ int tab_variant(int river, int dealt) {
    return river ? 0 : (dealt < 0 ? 52 : dealt);
}

// ====================================================================== device
__device__ __forceinline__ float4 f4(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
    return make_float4(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z), __fmul_rn(a.w, b.w));
}
__device__ __forceinline__ float4 max04(float4 a) { return make_float4(fmaxf(a.x, 0.f), fmaxf(a.y, 0.f), fmaxf(a.z, 0.f), fmaxf(a.w, 0.f)); }
__device__ __forceinline__ float rm1(float pos, float sum, float invA) { return sum > 1e-7f ? __fdiv_rn(pos, sum) : invA; }
__device__ __forceinline__ float4 rm4(float4 pos, float4 sum, float invA) {
    return make_float4(rm1(pos.x, sum.x, invA), rm1(pos.y, sum.y, invA), rm1(pos.z, sum.z, invA), rm1(pos.w, sum.w, invA));
}
__device__ __forceinline__ float4 fma4(float4 a, float4 b, float4 c) {
    return make_float4(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y), __fmaf_rn(a.z, b.z, c.z), __fmaf_rn(a.w, b.w, c.w));
}
__device__ __forceinline__ float cfrplus1(float r, float inst) { return fmaxf(0.0f, __fadd_rn(r, inst)); }
__device__ __forceinline__ float dcfr1(float r, float inst, float dpos, float dneg) {
    return __fadd_rn(__fmul_rn(r, r > 0.0f ? dpos : dneg), inst);
}

struct BatchDev {
    const SubDesc* desc;
    int n_sub;
    const int* order;
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
    int iters, algo, semantics;
    int* queue;
};

// per-player selects (runtime-indexed local arrays would live in local memory)
#define HP(p) ((p) ? sd.Hp1 : sd.Hp0)
#define OFF(p) ((p) ? sd.Hp0 : 0)
#define RP(p) (a.R + ((p) ? sd.rs_base1 : sd.rs_base0))
#define SP(p) (a.S + ((p) ? sd.rs_base1 : sd.rs_base0))

// exclusive scan of x[0..n) in place, x[n] = total; all threads of the CTA
template <typename T>
__device__ void block_scan_excl(T* x, int n, T* wbuf, int tid, int B) {
    const int C = (n + B - 1) / B;
    const int s = min(tid * C, n), e = min(s + C, n);
    T loc = T(0);
    for (int k = s; k < e; ++k) loc += x[k];
    const int lane = tid & 31, wid = tid >> 5, nw = B >> 5;
    T inc = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += t;
    }
    T exc = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
    if (lane == 0) exc = T(0);
    if (lane == 31) wbuf[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T w = lane < nw ? wbuf[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= o) wi += t;
        }
        T we = __shfl_up_sync(0xFFFFFFFFu, wi, 1);
        if (lane == 0) we = T(0);
        if (lane < nw) wbuf[lane] = we;
        if (lane == nw - 1) wbuf[32] = wi;
    }
    __syncthreads();
    T run = wbuf[wid] + exc;
    for (int k = s; k < e; ++k) {
        const T v = x[k];
        x[k] = run;
        run += v;
    }
    if (tid == 0) x[n] = wbuf[32];
    __syncthreads();
}

template <typename T>
__device__ T block_sum(T v, T* wbuf, int tid, int B) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    const int lane = tid & 31, wid = tid >> 5, nw = B >> 5;
    __syncthreads();
    if (lane == 0) wbuf[wid] = v;
    __syncthreads();
    T r = T(0);
    if (wid == 0) {
        r = lane < nw ? wbuf[lane] : T(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xFFFFFFFFu, r, o);
        if (lane == 0) wbuf[32] = r;
    }
    __syncthreads();
    r = wbuf[32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ DNode load_node(const DNode* p) {
    DNode d;
    const uint4* s = reinterpret_cast<const uint4*>(p);
    uint4* o = reinterpret_cast<uint4*>(&d);
    o[0] = __ldg(s);
    o[1] = __ldg(s + 1);
    o[2] = __ldg(s + 2);
    return d;
}

// Terminal values of both players at `node` into val (and val2 if given):
// val[node*HS + off_q + h].  Reach of both players staged in sm_r.
template <typename T>
__device__ void eval_terminal(const SubDesc& sd, const DNode& nd, int node, const TabView& tv,
                              const T* reach, T* val, T* val2, int HS, int semantics, T* sm_r, T* sm_x,
                              T* wbuf, int tid, int B) {
    const int H[2] = {sd.H0, sd.H1};
    const int Hp[2] = {sd.Hp0, sd.Hp1};
    const int off[2] = {0, sd.Hp0};
    const int src[2] = {nd.reach_src0, nd.reach_src1};
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const T* r = reach + (size_t)src[p] * HS + OFF(p);
        T* d = sm_r + (p ? H[0] : 0);
        for (int j = tid; j < H[p]; j += B) d[j] = r[j];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int o = 1 - q, Ho = H[o];
        const int base = q ? 3 * H[1] : 0;
        const T* ro = sm_r + (o ? H[0] : 0);
        const uint16_t* so = tv.sorted[o];
        const uint16_t* co = tv.cl[o];
        for (int i = tid; i < Ho; i += B) sm_x[base + i] = ro[so[i]];
        for (int e = tid; e < 2 * Ho; e += B) sm_x[base + Ho + e] = ro[co[e]];
    }
    __syncthreads();
    block_scan_excl<T>(sm_x, 3 * (H[0] + H[1]), wbuf, tid, B);
    const bool fold = nd.type == MTT_NODE_FOLD;
    const int winner = (nd.wmask == 1) ? 0 : 1;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int o = 1 - q, Ho = H[o];
        const T* E = sm_x + (q ? 3 * H[1] : 0);
        const T e0 = E[0];
        const T Tt = E[Ho] - e0;
        const T* ro = sm_r + (o ? H[0] : 0);
        const uint16_t* seg = tv.seg[o];
        const Entry* ent = tv.ent[q];
        const T cq = (T)(q ? nd.c1 : nd.c0);
        const T pot = (T)nd.pot;
        const T gain = pot - cq, loss = -cq, tie = T(0.5) * pot - cq;
        const T payoff = (q == winner) ? gain : loss;
        T* out = val + (size_t)node * HS + off[q];
        T* out2 = val2 ? val2 + (size_t)node * HS + off[q] : nullptr;
        for (int h = tid; h < Hp[q]; h += B) {
            T v = T(0);
            if (h < H[q]) {
                const Entry et = ent[h];
                if (et.lt != 0xFFFFu) {
                    const int s1 = Ho + seg[et.c1], s2 = Ho + seg[et.c2];
                    const T b1 = E[s1], b2 = E[s2];
                    const T C1 = E[Ho + seg[et.c1 + 1]] - b1, C2 = E[Ho + seg[et.c2 + 1]] - b2;
                    const T ps = et.same >= 0 ? ro[et.same] : T(0);
                    if (fold) {
                        const T M = semantics ? Tt : (Tt - C1 - C2 + ps);
                        v = payoff * M;
                    } else {
                        const T W = (E[et.lt] - e0) - (E[s1 + et.ltc1] - b1) - (E[s2 + et.ltc2] - b2);
                        const T LE = (E[et.le] - e0) - (E[s1 + et.lec1] - b1) - (E[s2 + et.lec2] - b2);
                        const T Ti = LE - W + ps;
                        if (!semantics) {
                            const T L = Tt - C1 - C2 - LE;
                            v = gain * W + tie * Ti + loss * L;
                        } else {
                            const T Lr = Tt - W - Ti;   // blocked pairs count as P0 losses
                            v = (q == 0) ? (gain * W + tie * Ti + loss * Lr) : (gain * Lr + tie * Ti + loss * W);
                        }
                    }
                }
            }
            out[h] = v;
            if (out2) out2[h] = v;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ uint64_t hand_mask(uint16_t hc) {
    return hc == 0xFFFFu ? 0ull : ((1ull << (hc & 0xFF)) | (1ull << (hc >> 8)));
}

template <typename T>
__device__ __forceinline__ T blocked_zero(uint16_t hc, int card, T v) {
    return (hand_mask(hc) >> card) & 1ull ? T(0) : v;
}

// ------------------------------------------------------------------ solve
__device__ void solve_one(const BatchDev& a, const SubDesc& sd, uint8_t* smem, int tid, int B) {
    const int nn = sd.n_nodes;
    const int HS = sd.Hp0 + sd.Hp1, HS4 = HS >> 2;
    float* reach = a.arena + sd.arena_base;
    float* cfv = reach + (size_t)nn * HS;
    const DNode* nodes = a.nodes + sd.node_base;
    const uint16_t* hc = a.hcards + sd.hcard_base;
    const int Hsum = sd.H0 + sd.H1;
    float* sm_r = reinterpret_cast<float*>(smem);
    float* sm_x = sm_r + ((Hsum + 3) & ~3);
    float* wbuf = sm_x + ((3 * Hsum + 1 + 3) & ~3);
    const float div = (float)(a.semantics ? sd.n_live - 2 : sd.n_live - 4);

    // zero regrets and strategy sums, load root reach
    {
        const long long n0 = (long long)sd.rows0 * sd.Hp0 / 4, n1 = (long long)sd.rows1 * sd.Hp1 / 4;
        float4* r0 = reinterpret_cast<float4*>(RP(0));
        float4* r1 = reinterpret_cast<float4*>(RP(1));
        float4* s0 = reinterpret_cast<float4*>(SP(0));
        float4* s1 = reinterpret_cast<float4*>(SP(1));
        for (long long i = tid; i < n0; i += B) { r0[i] = f4(0.f); s0[i] = f4(0.f); }
        for (long long i = tid; i < n1; i += B) { r1[i] = f4(0.f); s1[i] = f4(0.f); }
        const float4* rg = reinterpret_cast<const float4*>(a.ranges + sd.range_base);
        float4* rr = reinterpret_cast<float4*>(reach);
        for (int i = tid; i < HS4; i += B) rr[i] = rg[i];
    }
    __syncthreads();

    for (int t = 1; t <= a.iters; ++t) {
        const float4 it = *reinterpret_cast<const float4*>(a.iter_tab + 4 * (t - 1));
        const float w = it.x, dpos = it.y, dneg = it.z, dstr = it.w;
        // ---------------- forward: regret matching, reach, strategy sums
        for (int n = 0; n < nn; ++n) {
            const DNode nd = load_node(nodes + n);
            if (nd.type == MTT_NODE_DECISION) {
                const int p = nd.player, A = nd.na, H4 = HP(p) >> 2;
                const float invA = __fdiv_rn(1.0f, (float)A);
                const float4* rp = reinterpret_cast<const float4*>(reach + (size_t)(p ? nd.reach_src1 : nd.reach_src0) * HS + OFF(p));
                float4* ch = reinterpret_cast<float4*>(reach + (size_t)nd.first * HS + OFF(p));
                const float4* Rb = reinterpret_cast<const float4*>(RP(p) + (size_t)nd.row * HP(p));
                float4* Sb = reinterpret_cast<float4*>(SP(p) + (size_t)nd.row * HP(p));
                for (int g = tid; g < H4; g += B) {
                    const float4 r = rp[g];
                    float4 pos[MAXA];
                    float4 sum = f4(0.f);
#pragma unroll
                    for (int k = 0; k < MAXA; ++k)
                        if (k < A) { pos[k] = max04(Rb[(size_t)k * H4 + g]); sum = add4(sum, pos[k]); }
                    const float4 wr = mul4(r, f4(w));
#pragma unroll
                    for (int k = 0; k < MAXA; ++k)
                        if (k < A) {
                            const float4 sg = rm4(pos[k], sum, invA);
                            ch[(size_t)k * HS4 + g] = mul4(r, sg);
                            float4 sv = Sb[(size_t)k * H4 + g];
                            sv = a.algo == MTT_ALGO_DCFR ? fma4(r, sg, mul4(sv, f4(dstr))) : fma4(wr, sg, sv);
                            Sb[(size_t)k * H4 + g] = sv;
                        }
                }
            } else if (nd.type == MTT_NODE_CHANCE) {
                for (int k = 0; k < nd.na; ++k) {
                    const int card = nodes[nd.first + k].dealt;
#pragma unroll
                    for (int p = 0; p < 2; ++p) {
                        const int H4 = HP(p) >> 2;
                        const float4* rp = reinterpret_cast<const float4*>(reach + (size_t)(p ? nd.reach_src1 : nd.reach_src0) * HS + OFF(p));
                        float4* ch = reinterpret_cast<float4*>(reach + (size_t)(nd.first + k) * HS + OFF(p));
                        const uint16_t* hcp = hc + OFF(p);
                        for (int g = tid; g < H4; g += B) {
                            float4 r = rp[g];
                            r.x = blocked_zero(hcp[4 * g + 0], card, r.x);
                            r.y = blocked_zero(hcp[4 * g + 1], card, r.y);
                            r.z = blocked_zero(hcp[4 * g + 2], card, r.z);
                            r.w = blocked_zero(hcp[4 * g + 3], card, r.w);
                            ch[g] = r;
                        }
                    }
                }
            }
        }
        __syncthreads();
        // ---------------- terminals
        for (int n = 0; n < nn; ++n) {
            const DNode nd = load_node(nodes + n);
            if (nd.type != MTT_NODE_FOLD && nd.type != MTT_NODE_SHOWDOWN) continue;
            const int v = tab_variant(sd.river, nd.dealt);
            const TabView tv = tab_view(a.tabs + sd.tab_base + (size_t)v * sd.tab_vsize, sd.H0, sd.H1);
            eval_terminal<float>(sd, nd, n, tv, reach, cfv, nullptr, HS, a.semantics, sm_r, sm_x, wbuf, tid, B);
        }
        // ---------------- backward: values and regrets
        for (int n = nn - 1; n >= 0; --n) {
            const DNode nd = load_node(nodes + n);
            if (nd.type == MTT_NODE_DECISION) {
                const int p = nd.player, o = 1 - p, A = nd.na;
                const int H4 = HP(p) >> 2, H4o = HP(o) >> 2;
                const float invA = __fdiv_rn(1.0f, (float)A);
                float4* Rb = reinterpret_cast<float4*>(RP(p) + (size_t)nd.row * HP(p));
                const float4* qc = reinterpret_cast<const float4*>(cfv + (size_t)nd.first * HS + OFF(p));
                float4* outp = reinterpret_cast<float4*>(cfv + (size_t)n * HS + OFF(p));
                for (int g = tid; g < H4; g += B) {
                    // only the regrets stay in registers; the child values
                    // are re-read (an L1 hit) for the update
                    float4 rr[MAXA];
                    float4 sum = f4(0.f);
#pragma unroll
                    for (int k = 0; k < MAXA; ++k)
                        if (k < A) {
                            rr[k] = Rb[(size_t)k * H4 + g];
                            sum = add4(sum, max04(rr[k]));
                        }
                    float4 v = f4(0.f);
#pragma unroll
                    for (int k = 0; k < MAXA; ++k)
                        if (k < A) v = fma4(rm4(max04(rr[k]), sum, invA), qc[(size_t)k * HS4 + g], v);
                    outp[g] = v;
#pragma unroll
                    for (int k = 0; k < MAXA; ++k)
                        if (k < A) {
                            const float4 qk = qc[(size_t)k * HS4 + g];
                            float4 nr;
                            if (a.algo == MTT_ALGO_DCFR) {
                                nr.x = dcfr1(rr[k].x, __fsub_rn(qk.x, v.x), dpos, dneg);
                                nr.y = dcfr1(rr[k].y, __fsub_rn(qk.y, v.y), dpos, dneg);
                                nr.z = dcfr1(rr[k].z, __fsub_rn(qk.z, v.z), dpos, dneg);
                                nr.w = dcfr1(rr[k].w, __fsub_rn(qk.w, v.w), dpos, dneg);
                            } else {
                                nr.x = cfrplus1(rr[k].x, __fsub_rn(qk.x, v.x));
                                nr.y = cfrplus1(rr[k].y, __fsub_rn(qk.y, v.y));
                                nr.z = cfrplus1(rr[k].z, __fsub_rn(qk.z, v.z));
                                nr.w = cfrplus1(rr[k].w, __fsub_rn(qk.w, v.w));
                            }
                            Rb[(size_t)k * H4 + g] = nr;
                        }
                }
                const float4* oc = reinterpret_cast<const float4*>(cfv + (size_t)nd.first * HS + OFF(o));
                float4* outo = reinterpret_cast<float4*>(cfv + (size_t)n * HS + OFF(o));
                for (int g = tid; g < H4o; g += B) {
                    float4 so = f4(0.f);
                    for (int k = 0; k < A; ++k) so = add4(so, oc[(size_t)k * HS4 + g]);
                    outo[g] = so;
                }
            } else if (nd.type == MTT_NODE_CHANCE) {
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const int H4 = HP(p) >> 2;
                    const uint16_t* hcp = hc + OFF(p);
                    float4* outp = reinterpret_cast<float4*>(cfv + (size_t)n * HS + OFF(p));
                    for (int g = tid; g < H4; g += B) {
                        const uint64_t m0 = hand_mask(hcp[4 * g]), m1 = hand_mask(hcp[4 * g + 1]);
                        const uint64_t m2 = hand_mask(hcp[4 * g + 2]), m3 = hand_mask(hcp[4 * g + 3]);
                        float4 acc = f4(0.f);
                        for (int k = 0; k < nd.na; ++k) {
                            const int card = nodes[nd.first + k].dealt;
                            const float4 cv = reinterpret_cast<const float4*>(cfv + (size_t)(nd.first + k) * HS + OFF(p))[g];
                            if (!((m0 >> card) & 1ull)) acc.x = __fadd_rn(acc.x, cv.x);
                            if (!((m1 >> card) & 1ull)) acc.y = __fadd_rn(acc.y, cv.y);
                            if (!((m2 >> card) & 1ull)) acc.z = __fadd_rn(acc.z, cv.z);
                            if (!((m3 >> card) & 1ull)) acc.w = __fadd_rn(acc.w, cv.w);
                        }
                        outp[g] = make_float4(__fdiv_rn(acc.x, div), __fdiv_rn(acc.y, div), __fdiv_rn(acc.z, div),
                                              __fdiv_rn(acc.w, div));
                    }
                }
            }
        }
        // The next forward sweep touches only this thread's own hands and
        // the terminal phase starts behind a barrier, so none is needed here.
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256, 2) k_batch_solve(BatchDev a) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ int s_item;
    const int tid = threadIdx.x, B = blockDim.x;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.queue, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= a.n_sub) return;
        const int s = a.order ? a.order[item] : item;
        const SubDesc sd = a.desc[s];
        solve_one(a, sd, smem, tid, B);
    }
}

// ------------------------------------------------------------- FP64 best response
__device__ void br_one(const BatchDev& a, const SubDesc& sd, int s, uint8_t* smem, int tid, int B) {
    const int nn = sd.n_nodes;
    const int HS = sd.Hp0 + sd.Hp1;
    const size_t reg = (size_t)(nn + 1) * HS;
    double* reach = a.darena + sd.darena_base;
    double* br = reach + reg;
    double* ev = br + reg;
    const DNode* nodes = a.nodes + sd.node_base;
    const uint16_t* hc = a.hcards + sd.hcard_base;
    const int Hsum = sd.H0 + sd.H1;
    double* sm_r = reinterpret_cast<double*>(smem);
    double* sm_x = sm_r + Hsum + 1;
    double* wbuf = sm_x + 3 * Hsum + 2;
    const double div = (double)(sd.n_live - 4);

    for (int i = tid; i < HS; i += B) reach[i] = (double)a.ranges[sd.range_base + i];
    __syncthreads();
    // forward with the average strategies
    for (int n = 0; n < nn; ++n) {
        const DNode nd = load_node(nodes + n);
        if (nd.type == MTT_NODE_DECISION) {
            const int p = nd.player, A = nd.na;
            const double* rp = reach + (size_t)(p ? nd.reach_src1 : nd.reach_src0) * HS + OFF(p);
            const float* Sb = SP(p) + (size_t)nd.row * HP(p);
            for (int h = tid; h < HP(p); h += B) {
                double sum = 0.0;
                for (int k = 0; k < A; ++k) sum += (double)Sb[(size_t)k * HP(p) + h];
                const double r = rp[h];
                for (int k = 0; k < A; ++k) {
                    const double sg = sum > 0.0 ? (double)Sb[(size_t)k * HP(p) + h] / sum : 1.0 / (double)A;
                    reach[(size_t)(nd.first + k) * HS + OFF(p) + h] = r * sg;
                }
            }
        } else if (nd.type == MTT_NODE_CHANCE) {
            for (int k = 0; k < nd.na; ++k) {
                const int card = nodes[nd.first + k].dealt;
                for (int p = 0; p < 2; ++p) {
                    const double* rp = reach + (size_t)(p ? nd.reach_src1 : nd.reach_src0) * HS + OFF(p);
                    double* ch = reach + (size_t)(nd.first + k) * HS + OFF(p);
                    for (int h = tid; h < HP(p); h += B) ch[h] = blocked_zero(hc[OFF(p) + h], card, rp[h]);
                }
            }
        }
    }
    __syncthreads();
    for (int n = 0; n < nn; ++n) {
        const DNode nd = load_node(nodes + n);
        if (nd.type != MTT_NODE_FOLD && nd.type != MTT_NODE_SHOWDOWN) continue;
        const int v = tab_variant(sd.river, nd.dealt);
        const TabView tv = tab_view(a.tabs + sd.tab_base + (size_t)v * sd.tab_vsize, sd.H0, sd.H1);
        eval_terminal<double>(sd, nd, n, tv, reach, br, ev, HS, MTT_SEM_CORRECT, sm_r, sm_x, wbuf, tid, B);
    }
    for (int n = nn - 1; n >= 0; --n) {
        const DNode nd = load_node(nodes + n);
        if (nd.type == MTT_NODE_DECISION) {
            const int p = nd.player, o = 1 - p, A = nd.na;
            const float* Sb = SP(p) + (size_t)nd.row * HP(p);
            for (int h = tid; h < HP(p); h += B) {
                double sum = 0.0;
                for (int k = 0; k < A; ++k) sum += (double)Sb[(size_t)k * HP(p) + h];
                double best = -1e300, e = 0.0;
                for (int k = 0; k < A; ++k) {
                    const size_t c = (size_t)(nd.first + k) * HS + OFF(p) + h;
                    const double sg = sum > 0.0 ? (double)Sb[(size_t)k * HP(p) + h] / sum : 1.0 / (double)A;
                    best = fmax(best, br[c]);
                    e += sg * ev[c];
                }
                br[(size_t)n * HS + OFF(p) + h] = best;
                ev[(size_t)n * HS + OFF(p) + h] = e;
            }
            for (int h = tid; h < HP(o); h += B) {
                double sb = 0.0, se = 0.0;
                for (int k = 0; k < A; ++k) {
                    const size_t c = (size_t)(nd.first + k) * HS + OFF(o) + h;
                    sb += br[c];
                    se += ev[c];
                }
                br[(size_t)n * HS + OFF(o) + h] = sb;
                ev[(size_t)n * HS + OFF(o) + h] = se;
            }
        } else if (nd.type == MTT_NODE_CHANCE) {
            for (int p = 0; p < 2; ++p)
                for (int h = tid; h < HP(p); h += B) {
                    const uint64_t m = hand_mask(hc[OFF(p) + h]);
                    double sb = 0.0, se = 0.0;
                    for (int k = 0; k < nd.na; ++k) {
                        const int card = nodes[nd.first + k].dealt;
                        if ((m >> card) & 1ull) continue;
                        const size_t c = (size_t)(nd.first + k) * HS + OFF(p) + h;
                        sb += br[c];
                        se += ev[c];
                    }
                    br[(size_t)n * HS + OFF(p) + h] = sb / div;
                    ev[(size_t)n * HS + OFF(p) + h] = se / div;
                }
        }
    }
    // compatible range mass: a fold-like terminal with payoff 1 for P0 at the root
    {
        DNode z{};
        z.type = MTT_NODE_FOLD;
        z.wmask = 1;
        z.pot = 1.0f;
        z.reach_src0 = 0;
        z.reach_src1 = 0;
        z.dealt = -1;
        const TabView tv = tab_view(a.tabs + sd.tab_base + (size_t)tab_variant(sd.river, -1) * sd.tab_vsize,
                                    sd.H0, sd.H1);
        eval_terminal<double>(sd, z, nn, tv, reach, br, nullptr, HS, MTT_SEM_CORRECT, sm_r, sm_x, wbuf, tid, B);
    }
    double acc[5] = {0, 0, 0, 0, 0};
    for (int h = tid; h < sd.H0; h += B) {
        const double r = reach[h];
        acc[0] += r * br[h];
        acc[2] += r * ev[h];
        acc[4] += r * br[(size_t)nn * HS + h];
    }
    for (int h = tid; h < sd.H1; h += B) {
        const double r = reach[sd.Hp0 + h];
        acc[1] += r * br[sd.Hp0 + h];
        acc[3] += r * ev[sd.Hp0 + h];
    }
    double tot[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) tot[k] = block_sum<double>(acc[k], wbuf, tid, B);
    if (tid == 0) {
        const double Z = tot[4] > 0.0 ? tot[4] : 1.0;
        double* o = a.results + (size_t)s * 6;
        o[0] = tot[0] / Z;
        o[1] = tot[1] / Z;
        o[2] = tot[2] / Z;
        o[3] = tot[3] / Z;
        o[4] = tot[4];
        o[5] = 0.5 * (o[0] + o[1]) / (double)sd.pot;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_batch_br(BatchDev a) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ int s_item;
    const int tid = threadIdx.x, B = blockDim.x;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.queue + 1, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= a.n_sub) return;
        const int s = a.order ? a.order[item] : item;
        const SubDesc sd = a.desc[s];
        br_one(a, sd, s, smem, tid, B);
    }
}

// ====================================================================== host
struct SubPack {
    std::vector<DNode> nodes;
    std::vector<uint8_t> tab;
    std::vector<uint16_t> hcards;
    std::vector<float> range;
    SubDesc d{};
    int status = MTT_OK;
};

static int pad4(int h) { return (h + 3) & ~3; }

static void build_variant(const uint8_t* board, int nboard, int dealt, const int H[2],
                          const std::vector<uint16_t> cards[2], const std::vector<uint16_t> combos[2], uint8_t* out) {
    std::vector<uint32_t> sc[2];
    for (int p = 0; p < 2; ++p) {
        sc[p].resize(H[p]);
        for (int h = 0; h < H[p]; ++h) {
            const int c1 = cards[p][h] & 0xFF, c2 = cards[p][h] >> 8;
            if (dealt >= 0 && (c1 == dealt || c2 == dealt)) { sc[p][h] = 0u; continue; }
            Planes pl; planes_clear(pl);
            for (int k = 0; k < nboard; ++k) planes_add(pl, board[k]);
            if (dealt >= 0) planes_add(pl, dealt);
            planes_add(pl, c1);
            planes_add(pl, c2);
            sc[p][h] = score_planes(pl);
        }
    }
    TabView tv = tab_view(out, H[0], H[1]);
    std::vector<uint16_t> sorted[2], cl[2], seg[2];
    std::vector<uint32_t> ssc[2], clsc[2];
    for (int p = 0; p < 2; ++p) {
        sorted[p].resize(H[p]);
        std::iota(sorted[p].begin(), sorted[p].end(), (uint16_t)0);
        std::stable_sort(sorted[p].begin(), sorted[p].end(), [&](uint16_t x, uint16_t y) { return sc[p][x] < sc[p][y]; });
        ssc[p].resize(H[p]);
        for (int i = 0; i < H[p]; ++i) ssc[p][i] = sc[p][sorted[p][i]];
        // per card lists in rank order
        std::vector<std::vector<uint16_t>> by(52);
        for (int i = 0; i < H[p]; ++i) {
            const uint16_t h = sorted[p][i];
            by[cards[p][h] & 0xFF].push_back(h);
            by[cards[p][h] >> 8].push_back(h);
        }
        seg[p].assign(54, 0);
        cl[p].clear();
        for (int c = 0; c < 52; ++c) {
            seg[p][c] = (uint16_t)cl[p].size();
            for (uint16_t h : by[c]) cl[p].push_back(h);
        }
        seg[p][52] = seg[p][53] = (uint16_t)cl[p].size();
        clsc[p].resize(cl[p].size());
        for (size_t e = 0; e < cl[p].size(); ++e) clsc[p][e] = sc[p][cl[p][e]];
        std::memcpy(const_cast<uint16_t*>(tv.sorted[p]), sorted[p].data(), 2 * (size_t)H[p]);
        std::memcpy(const_cast<uint16_t*>(tv.cl[p]), cl[p].data(), 2 * cl[p].size());
        std::memcpy(const_cast<uint16_t*>(tv.seg[p]), seg[p].data(), 2 * 54);
    }
    for (int q = 0; q < 2; ++q) {
        const int o = 1 - q;
        Entry* ent = const_cast<Entry*>(tv.ent[q]);
        for (int h = 0; h < H[q]; ++h) {
            Entry e{};
            const int c1 = cards[q][h] & 0xFF, c2 = cards[q][h] >> 8;
            e.c1 = (uint8_t)c1;
            e.c2 = (uint8_t)c2;
            if (dealt >= 0 && (c1 == dealt || c2 == dealt)) {
                e.lt = e.le = 0xFFFFu;
                e.same = -1;
                ent[h] = e;
                continue;
            }
            const uint32_t s = sc[q][h];
            e.lt = (uint16_t)(std::lower_bound(ssc[o].begin(), ssc[o].end(), s) - ssc[o].begin());
            e.le = (uint16_t)(std::upper_bound(ssc[o].begin(), ssc[o].end(), s) - ssc[o].begin());
            auto seg_pos = [&](int c, bool upper) {
                auto b = clsc[o].begin() + seg[o][c], en = clsc[o].begin() + seg[o][c + 1];
                return (uint8_t)((upper ? std::upper_bound(b, en, s) : std::lower_bound(b, en, s)) - b);
            };
            e.ltc1 = seg_pos(c1, false);
            e.lec1 = seg_pos(c1, true);
            e.ltc2 = seg_pos(c2, false);
            e.lec2 = seg_pos(c2, true);
            const uint16_t cid = combos[q][h];
            auto it = std::lower_bound(combos[o].begin(), combos[o].end(), cid);
            e.same = (it != combos[o].end() && *it == cid) ? (int16_t)(it - combos[o].begin()) : (int16_t)-1;
            ent[h] = e;
        }
    }
}

static void combo_cards(int id, int& c1, int& c2) {
    int a = 0, row = 51, k = id;
    while (k >= row) { k -= row; ++a; --row; }
    c1 = a;
    c2 = a + 1 + k;
}

static void pack_one(const mtt_subgame& g, SubPack& sp) {
    sp.status = MTT_OK;
    int rows[2] = {g.rows[0], g.rows[1]};
    if (!g.nodes || g.n_nodes <= 0 || (g.nboard != 5 && g.nboard != 4)) { sp.status = MTT_ERR_INVALID; return; }
    int st = validate_tree(g.nodes, g.n_nodes, rows);
    if (st) { sp.status = st; return; }
    uint64_t bm = 0;
    for (int k = 0; k < g.nboard; ++k) {
        if (g.board[k] > 51 || ((bm >> g.board[k]) & 1ull)) { sp.status = MTT_ERR_INVALID; return; }
        bm |= 1ull << g.board[k];
    }
    const int H[2] = {g.H[0], g.H[1]};
    std::vector<uint16_t> combos[2], cards[2];
    for (int p = 0; p < 2; ++p) {
        if (H[p] < 1 || H[p] > 1326 || !g.combos[p] || !g.ranges[p]) { sp.status = MTT_ERR_INVALID; return; }
        combos[p].assign(g.combos[p], g.combos[p] + H[p]);
        cards[p].resize(H[p]);
        for (int h = 0; h < H[p]; ++h) {
            const int id = combos[p][h];
            if (id >= 1326 || (h > 0 && combos[p][h - 1] >= id)) { sp.status = MTT_ERR_INVALID; return; }
            int c1, c2;
            combo_cards(id, c1, c2);
            if (((bm >> c1) & 1ull) || ((bm >> c2) & 1ull)) { sp.status = MTT_ERR_INVALID; return; }
            const float r = g.ranges[p][h];
            if (!(r >= 0.0f) || !std::isfinite(r)) { sp.status = MTT_ERR_INVALID; return; }
            cards[p][h] = (uint16_t)(c1 | (c2 << 8));
        }
    }
    const int nn = g.n_nodes;
    const int Hp[2] = {pad4(H[0]), pad4(H[1])};
    // nodes
    sp.nodes.assign(nn, DNode{});
    std::vector<int> rsrc0(nn, 0), rsrc1(nn, 0), dealt(nn, -1);
    for (int i = 0; i < nn; ++i) {
        const mtt_node& m = g.nodes[i];
        DNode& d = sp.nodes[i];
        d.type = m.type;
        d.player = m.player;
        d.na = (m.type == MTT_NODE_DECISION || m.type == MTT_NODE_CHANCE) ? m.num_actions : 0;
        d.wmask = m.active_mask;
        d.first = m.children_offset;
        d.row = m.infoset_offset;
        d.pot = m.pot_size;
        d.c0 = m.committed[0];
        d.c1 = m.committed[1];
        if (m.type == MTT_NODE_DECISION && m.num_actions > MAXA) { sp.status = MTT_ERR_UNSUPPORTED; return; }
        if (m.type == MTT_NODE_CHANCE && g.nboard != 4) { sp.status = MTT_ERR_INVALID; return; }
    }
    for (int i = 0; i < nn; ++i) {
        const mtt_node& m = g.nodes[i];
        if (m.type == MTT_NODE_DECISION) {
            for (int k = 0; k < m.num_actions; ++k) {
                const int c = m.children_offset + k;
                rsrc0[c] = m.player == 0 ? c : rsrc0[i];
                rsrc1[c] = m.player == 1 ? c : rsrc1[i];
                dealt[c] = dealt[i];
            }
        } else if (m.type == MTT_NODE_CHANCE) {
            for (int k = 0; k < m.num_actions; ++k) {
                const int c = m.children_offset + k;
                rsrc0[c] = c;
                rsrc1[c] = c;
                dealt[c] = g.nodes[c].turn_idx;
                if (dealt[c] < 0 || dealt[c] > 51 || ((bm >> dealt[c]) & 1ull)) { sp.status = MTT_ERR_INVALID; return; }
            }
        }
    }
    for (int i = 0; i < nn; ++i) {
        sp.nodes[i].reach_src0 = rsrc0[i];
        sp.nodes[i].reach_src1 = rsrc1[i];
        sp.nodes[i].dealt = (int16_t)dealt[i];
        // a turn subgame cannot reach a showdown before the river is dealt
        if (g.nboard == 4 && g.nodes[i].type == MTT_NODE_SHOWDOWN && dealt[i] < 0) { sp.status = MTT_ERR_INVALID; return; }
    }
    // tables
    const int vsize = tab_variant_bytes(H[0], H[1]);
    const int nvar = g.nboard == 5 ? 1 : 53;
    sp.tab.assign((size_t)vsize * nvar, 0);
    if (g.nboard == 5) {
        build_variant(g.board, 5, -1, H, cards, combos, sp.tab.data());
    } else {
        for (int c = 0; c < 52; ++c) {
            if ((bm >> c) & 1ull) continue;
            build_variant(g.board, 4, c, H, cards, combos, sp.tab.data() + (size_t)vsize * c);
        }
        build_variant(g.board, 4, -1, H, cards, combos, sp.tab.data() + (size_t)vsize * 52);
    }
    sp.hcards.assign((size_t)Hp[0] + Hp[1], 0xFFFFu);
    sp.range.assign((size_t)Hp[0] + Hp[1], 0.0f);
    for (int h = 0; h < H[0]; ++h) { sp.hcards[h] = cards[0][h]; sp.range[h] = g.ranges[0][h]; }
    for (int h = 0; h < H[1]; ++h) { sp.hcards[Hp[0] + h] = cards[1][h]; sp.range[Hp[0] + h] = g.ranges[1][h]; }
    SubDesc& d = sp.d;
    d.n_nodes = nn;
    d.H0 = H[0]; d.H1 = H[1];
    d.Hp0 = Hp[0]; d.Hp1 = Hp[1];
    d.rows0 = rows[0]; d.rows1 = rows[1];
    d.tab_vsize = vsize;
    d.n_live = 52 - g.nboard;
    d.river = g.nboard == 5 ? 1 : 0;
    d.pot = g.nodes[0].pot_size;
}

}  // namespace mtt

using namespace mtt;

struct mtt_batch {
    int n = 0;
    int device = 0;
    SubDesc* d_desc = nullptr;
    int* d_order = nullptr;
    DNode* d_nodes = nullptr;
    uint8_t* d_tabs = nullptr;
    uint16_t* d_hcards = nullptr;
    float* d_ranges = nullptr;
    float* d_arena = nullptr;
    float* d_R = nullptr;
    float* d_S = nullptr;
    double* d_darena = nullptr;
    double* d_results = nullptr;
    int* d_queue = nullptr;
    float* d_iter = nullptr;        // iteration weights of direct solves
    int iter_cap = 0;
    float* d_iter_graph = nullptr;  // owned by the captured graph
    std::vector<SubDesc> desc;
    int max_hsum = 0;
    long long device_bytes = 0;
    long long iter_bytes = 0;
    int tuned_threads = 0;
    // graph cache
    cudaGraphExec_t gexec = nullptr;
    mtt_solve_params gparams{};
    cudaStream_t gstream = nullptr;
};

namespace mtt {
template <typename T>
static int dalloc(T** p, size_t count, long long& total) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    MTT_TRY_CUDA(cudaMalloc(reinterpret_cast<void**>(p), bytes));
    total += (long long)bytes;
    return MTT_OK;
}

static void free_batch(mtt_batch* b) {
    if (!b) return;
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    cudaFree(b->d_desc); cudaFree(b->d_order); cudaFree(b->d_nodes); cudaFree(b->d_tabs);
    cudaFree(b->d_hcards); cudaFree(b->d_ranges); cudaFree(b->d_arena); cudaFree(b->d_R);
    cudaFree(b->d_S); cudaFree(b->d_darena); cudaFree(b->d_results); cudaFree(b->d_queue);
    cudaFree(b->d_iter);
    cudaFree(b->d_iter_graph);
    delete b;
}

// Per-iteration scalars (t, DCFR positive/negative regret discounts and the
// strategy-sum discount), computed on the host in double exactly as the oracle does.
static int fill_iter_table(float** dst, int* cap, const mtt_solve_params& p, cudaStream_t st) {
    if (p.iters > *cap || !*dst) {
        if (*dst) { MTT_TRY_CUDA(cudaStreamSynchronize(st)); cudaFree(*dst); *dst = nullptr; }
        MTT_TRY_CUDA(cudaMalloc(dst, sizeof(float) * 4 * (size_t)std::max(p.iters, 1)));
        *cap = std::max(p.iters, 1);
    }
    std::vector<float> tab(4 * (size_t)std::max(p.iters, 1), 0.0f);
    for (int t = 1; t <= p.iters; ++t) {
        const double tm1 = (double)(t - 1);
        float* e = &tab[4 * (size_t)(t - 1)];
        e[0] = (float)t;
        e[1] = (float)(std::pow(tm1, (double)p.alpha) / (std::pow(tm1, (double)p.alpha) + 1.0));
        e[2] = (float)(std::pow(tm1, (double)p.beta) / (std::pow(tm1, (double)p.beta) + 1.0));
        e[3] = (float)std::pow(tm1 / (double)t, (double)p.gamma);
    }
    MTT_TRY_CUDA(cudaMemcpyAsync(*dst, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
    // pageable source: the copy is staged before returning, so `tab` may go
    return MTT_OK;
}

static size_t solve_smem(const mtt_batch* b) { return sizeof(float) * (size_t)(4 * b->max_hsum + 64); }
static size_t br_smem(const mtt_batch* b) { return sizeof(double) * (size_t)(4 * b->max_hsum + 64); }

static BatchDev dev_args(const mtt_batch* b, const mtt_solve_params& p, const float* iter_tab) {
    BatchDev a;
    a.desc = b->d_desc; a.n_sub = b->n; a.order = b->d_order; a.nodes = b->d_nodes; a.tabs = b->d_tabs;
    a.hcards = b->d_hcards; a.ranges = b->d_ranges; a.arena = b->d_arena; a.R = b->d_R; a.S = b->d_S;
    a.darena = b->d_darena; a.results = b->d_results; a.iter_tab = iter_tab; a.iters = p.iters;
    a.algo = p.algo; a.semantics = p.semantics; a.queue = b->d_queue;
    return a;
}

static int grid_for(const void* kernel, int threads, size_t smem, int n, int* grid) {
    int dev = 0, sms = 0, per = 0;
    MTT_TRY_CUDA(cudaGetDevice(&dev));
    MTT_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MTT_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
    if (per < 1) return MTT_ERR_UNSUPPORTED;
    *grid = std::min(n, sms * per);
    return MTT_OK;
}

static int launch_solve(mtt_batch* b, const mtt_solve_params& p, int threads, cudaStream_t st, const float* iter_tab) {
    const size_t sm1 = solve_smem(b), sm2 = br_smem(b);
    if (sm1 > 48 * 1024) MTT_TRY_CUDA(cudaFuncSetAttribute(k_batch_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    if (sm2 > 48 * 1024) MTT_TRY_CUDA(cudaFuncSetAttribute(k_batch_br, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    int g1 = 0, g2 = 0;
    MTT_TRY(grid_for((const void*)k_batch_solve, threads, sm1, b->n, &g1));
    const BatchDev a = dev_args(b, p, iter_tab);
    MTT_TRY_CUDA(cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(int), st));
    k_batch_solve<<<g1, threads, sm1, st>>>(a);
    MTT_CHECK_LAUNCH();
    if (p.exploitability) {
        MTT_TRY(grid_for((const void*)k_batch_br, threads, sm2, b->n, &g2));
        k_batch_br<<<g2, threads, sm2, st>>>(a);
        MTT_CHECK_LAUNCH();
    }
    return MTT_OK;
}

static int check_params(const mtt_solve_params* p) {
    if (!p || p->iters < 0 || (p->algo != MTT_ALGO_CFRPLUS && p->algo != MTT_ALGO_DCFR) ||
        (p->semantics != MTT_SEM_CORRECT && p->semantics != MTT_SEM_REFERENCE))
        return MTT_ERR_INVALID;
    if (p->threads != 0 && p->threads != 64 && p->threads != 128 && p->threads != 256) return MTT_ERR_INVALID;
    return MTT_OK;
}
}  // namespace mtt

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
    cudaGetDevice(&b->device);
    long long nodes = 0, arena = 0, rs = 0, tabs = 0, hcards = 0, ranges = 0, darena = 0;
    b->desc.resize(n);
    long long iter_bytes = 0;
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
        b->max_hsum = std::max(b->max_hsum, d.H0 + d.H1);
        b->desc[i] = d;
        // algorithmic bytes of one iteration (fp32): R,S read+write per
        // action-hand of the acting player; per node, reach written+read and
        // CFV written+read for both players
        iter_bytes += 16LL * ((long long)d.rows0 * d.H0 + (long long)d.rows1 * d.H1) +
                      16LL * (long long)d.n_nodes * (d.H0 + d.H1);
    }
    b->iter_bytes = iter_bytes;
    long long total = 0;
    int s = MTT_OK;
    if (!s) s = dalloc(&b->d_desc, n, total);
    if (!s) s = dalloc(&b->d_order, n, total);
    if (!s) s = dalloc(&b->d_nodes, nodes, total);
    if (!s) s = dalloc(&b->d_tabs, tabs, total);
    if (!s) s = dalloc(&b->d_hcards, hcards, total);
    if (!s) s = dalloc(&b->d_ranges, ranges, total);
    if (!s) s = dalloc(&b->d_arena, arena, total);
    if (!s) s = dalloc(&b->d_R, rs, total);
    if (!s) s = dalloc(&b->d_S, rs, total);
    if (!s) s = dalloc(&b->d_darena, darena, total);
    if (!s) s = dalloc(&b->d_results, 6LL * n, total);
    if (!s) s = dalloc(&b->d_queue, 2, total);
    if (s) { free_batch(b); return s; }
    b->device_bytes = total;
    // gather host arrays and upload
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
        // largest subgames first (longest-processing-time order for the work queue)
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            const SubDesc& a = b->desc[x];
            const SubDesc& c = b->desc[y];
            return (long long)a.n_nodes * (a.Hp0 + a.Hp1) > (long long)c.n_nodes * (c.Hp0 + c.Hp1);
        });
        s = cuda_status(cudaMemcpy(b->d_desc, b->desc.data(), sizeof(SubDesc) * n, cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemcpy(b->d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
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
    cudaStream_t st = as_stream(stream);
    const int threads = prm->threads ? prm->threads : (b->tuned_threads ? b->tuned_threads : 128);
    MTT_TRY(fill_iter_table(&b->d_iter, &b->iter_cap, *prm, st));
    return launch_solve(b, *prm, threads, st, b->d_iter);
}

extern "C" int mtt_batch_solve_graph(mtt_batch* b, const mtt_solve_params* prm, void* stream) {
    if (!b) return MTT_ERR_INVALID;
    MTT_TRY(check_params(prm));
    cudaStream_t st = as_stream(stream);
    const bool same = b->gexec && std::memcmp(&b->gparams, prm, sizeof(*prm)) == 0;
    if (!same) {
        if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
        const int threads = prm->threads ? prm->threads : (b->tuned_threads ? b->tuned_threads : 128);
        int gcap = 0;
        if (b->d_iter_graph) { MTT_TRY_CUDA(cudaStreamSynchronize(st)); cudaFree(b->d_iter_graph); b->d_iter_graph = nullptr; }
        MTT_TRY(fill_iter_table(&b->d_iter_graph, &gcap, *prm, st));
        MTT_TRY_CUDA(cudaStreamSynchronize(st));
        // kernel attributes are set outside capture
        const size_t sm1 = solve_smem(b), sm2 = br_smem(b);
        if (sm1 > 48 * 1024) MTT_TRY_CUDA(cudaFuncSetAttribute(k_batch_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
        if (sm2 > 48 * 1024) MTT_TRY_CUDA(cudaFuncSetAttribute(k_batch_br, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
        cudaStream_t cs;
        MTT_TRY_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        int s = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        if (!s) s = launch_solve(b, *prm, threads, cs, b->d_iter_graph);
        const int s2 = cuda_status(cudaStreamEndCapture(cs, &graph));
        if (!s) s = s2;
        if (!s) s = cuda_status(cudaGraphInstantiate(&b->gexec, graph, 0));
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (s) { b->gexec = nullptr; return s; }
        b->gparams = *prm;
    }
    MTT_TRY_CUDA(cudaGraphLaunch(b->gexec, st));
    return MTT_OK;
}

extern "C" int mtt_batch_results(mtt_batch* b, double* h_out, void* stream) {
    if (!b || !h_out) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    MTT_TRY_CUDA(cudaMemcpyAsync(h_out, b->d_results, sizeof(double) * 6 * (size_t)b->n, cudaMemcpyDeviceToHost, st));
    MTT_TRY_CUDA(cudaStreamSynchronize(st));
    return MTT_OK;
}

extern "C" int mtt_batch_read(mtt_batch* b, int32_t s, float* h_R0, float* h_R1, float* h_S0, float* h_S1,
                              float* h_cfv0, float* h_cfv1) {
    if (!b || s < 0 || s >= b->n) return MTT_ERR_INVALID;
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    const SubDesc& d = b->desc[s];
    auto rows_copy = [&](float* dst, const float* src, int rows, int H, int Hp) -> int {
        if (!dst) return MTT_OK;
        if (rows == 0) return MTT_OK;
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

extern "C" int mtt_batch_info(mtt_batch* b, int64_t* device_bytes, int64_t* iter_bytes) {
    if (!b) return MTT_ERR_INVALID;
    if (device_bytes) *device_bytes = b->device_bytes;
    if (iter_bytes) *iter_bytes = b->iter_bytes;
    return MTT_OK;
}

extern "C" int mtt_batch_autotune(mtt_batch* b, const mtt_solve_params* prm, void* stream, int32_t* threads) {
    if (!b) return MTT_ERR_INVALID;
    MTT_TRY(check_params(prm));
    cudaStream_t st = as_stream(stream);
    mtt_solve_params p = *prm;
    p.iters = std::min(std::max(prm->iters, 1), 16);
    p.exploitability = 0;
    MTT_TRY(fill_iter_table(&b->d_iter, &b->iter_cap, p, st));
    const int cands[3] = {64, 128, 256};
    float best_ms = 1e30f;
    int best = 128;
    cudaEvent_t e0, e1;
    MTT_TRY_CUDA(cudaEventCreate(&e0));
    MTT_TRY_CUDA(cudaEventCreate(&e1));
    int s = MTT_OK;
    for (int c : cands) {
        if (!s) s = launch_solve(b, p, c, st, b->d_iter);   // warm
        if (!s) s = cuda_status(cudaEventRecord(e0, st));
        if (!s) s = launch_solve(b, p, c, st, b->d_iter);
        if (!s) s = cuda_status(cudaEventRecord(e1, st));
        if (!s) s = cuda_status(cudaEventSynchronize(e1));
        float ms = 0.f;
        if (!s) s = cuda_status(cudaEventElapsedTime(&ms, e0, e1));
        if (!s && ms < best_ms) { best_ms = ms; best = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s) return s;
    b->tuned_threads = best;
    if (threads) *threads = best;
    return MTT_OK;
}

extern "C" int mtt_batch_destroy(mtt_batch* b) {
    if (!b) return MTT_ERR_INVALID;
    cudaDeviceSynchronize();
    free_batch(b);
    return MTT_OK;
}
