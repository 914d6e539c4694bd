// subset.cu — flop-subset selection by non-negative orthogonal matching
// pursuit (scripts/optimize_subset.py:29-50), all steps on one device.
//
// Column j of the problem matrix A is the feature vector of flop j: row j of
// mtt_ev_dump_1755.bin read as [ncols][nfeat] f32, so every column read is one
// contiguous, coalesced row.  The whole matrix (9.5 MB for the dump) stays in
// L2 across the steps; nothing returns to the host between steps.
//
//   target      b = A colw / sum(colw), FP64                (optimize_subset.py:32)
//   per step s = 0 .. nselect - 1                            (optimize_subset.py:40-47)
//     k_ss_corr   corr_j = <A_j, r> / |A_j| for every unselected column j,
//                 one warp per column, and a (max, first index) per CTA
//     k_ss_gram   the argmax t (the first maximum, as numpy's argmax) and the
//                 Gram row G[s][0..s] = <A_t, A_sel[q]>, h[s] = <A_t, b>, one
//                 warp per dot
//     k_ss_nnls   one CTA: the non-negative least-squares weights x of the
//                 selected columns, then the residual r = b - A_sel x
//   output      x * ncols / sum(x)                           (optimize_subset.py:50)
//
// The weights come from Lawson and Hanson's active-set method ("Solving Least
// Squares Problems", SIAM 1995, ch. 23), the algorithm of the reference's
// scipy.optimize.nnls, here on the normal equations G x = h with an FP64
// L D L^T factor of the passive block, started from the previous step's
// weights instead of from zero.  A full-column-rank NNLS problem has one
// solution, so both choices change rounding only: about cond(A_sel)^2 * 2^-53
// relative, 2e-12 for the 100 flops the shipped dump selects (condition
// number 120).  The correlations are formed in FP64 from the f32 features and
// the FP64 norm, where the reference divides the features by their f32 norm
// in f32 first; the two differ by about 1e-7 relative, while the best and the
// second-best correlation of every step on the shipped dump are at least
// 8.4e-5 apart.  Every reduction runs in a fixed order: results are the same
// on every run.
//
// The refit is a chain of short dependent steps on one SM: the factor takes
// one barrier per passive column, and the triangular solves run on one warp
// with each lane's rows in registers, one shuffle per row.
#include <cfloat>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "mtt_common.h"

namespace mtt {
namespace ss {

constexpr int kCorrWarps = 8;          // columns per k_ss_corr CTA
constexpr int kStepThreads = 512;      // k_ss_nnls CTA
constexpr int kStepWarps = kStepThreads / 32;
constexpr int kTargetChunks = 32;      // column chunks of the target's partial sums

constexpr int kErrRank = 1;            // a passive block was not positive definite
constexpr int kErrIters = 2;           // more than 3 n passive-set solves in one subproblem
constexpr int kErrNoCandidate = 4;     // no finite correlation left (non-finite input)

struct SsDev {
    const float* A;       // [ncols][nfeat]
    const double* colw;   // [ncols]
    int ncols, nfeat, nsel;
    int ncorr;            // k_ss_corr CTAs
    double* b;            // [nfeat] target
    double* r;            // [nfeat] residual
    double* nrm;          // [ncols] column norms (1 for a zero column)
    double* bpart;        // [kTargetChunks][nfeat]
    double* part_v;       // [ncorr] per-CTA best correlation
    int* part_i;          // [ncorr] its column
    uint8_t* taken;       // [ncols] selected columns
    double* G;            // packed lower Gram matrix of the selected columns, selection order
    double* h;            // [nsel] <A_sel[p], b>
    double* x;            // [nsel] current weights
    int* sel;             // [nsel]
    int* err;
    int32_t* out_idx;
    double* out_w;
};

__host__ __device__ __forceinline__ int tri(int i) { return i * (i + 1) / 2; }

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// (max, first index) merge: a larger value wins, an equal value goes to the
// lower index; NaN never wins.
__device__ __forceinline__ void amax_merge(double& v, int& i, double v2, int i2) {
    if (v2 > v || (v2 == v && i2 < i)) { v = v2; i = i2; }
}

__device__ __forceinline__ void warp_amax(double& v, int& i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        const int i2 = __shfl_xor_sync(0xFFFFFFFFu, i, o);
        amax_merge(v, i, v2, i2);
    }
}

// <a, y> over n features (a: f32 column, y: FP64), this lane's share; VEC: a
// and n allow float4 loads (16-byte aligned, n % 4 == 0).
template <bool VEC>
__device__ __forceinline__ double lane_dot(const float* __restrict__ a, const double* __restrict__ y, int n, int lane) {
    double s = 0.0;
    if (VEC) {
        const float4* a4 = reinterpret_cast<const float4*>(a);
        const double2* y2 = reinterpret_cast<const double2*>(y);
#pragma unroll 4
        for (int q = lane; q < (n >> 2); q += 32) {
            const float4 v = __ldg(a4 + q);
            const double2 u0 = __ldg(y2 + 2 * q), u1 = __ldg(y2 + 2 * q + 1);
            s = fma((double)v.x, u0.x, s);
            s = fma((double)v.y, u0.y, s);
            s = fma((double)v.z, u1.x, s);
            s = fma((double)v.w, u1.y, s);
        }
    } else {
        for (int q = lane; q < n; q += 32) s = fma((double)__ldg(a + q), __ldg(y + q), s);
    }
    return s;
}

// <a, c> of two f32 columns in FP64 (each product is exact in FP64).
template <bool VEC>
__device__ __forceinline__ double lane_dot_ff(const float* __restrict__ a, const float* __restrict__ c, int n, int lane) {
    double s = 0.0;
    if (VEC) {
        const float4* a4 = reinterpret_cast<const float4*>(a);
        const float4* c4 = reinterpret_cast<const float4*>(c);
#pragma unroll 4
        for (int q = lane; q < (n >> 2); q += 32) {
            const float4 u = __ldg(a4 + q), v = __ldg(c4 + q);
            s = fma((double)u.x, (double)v.x, s);
            s = fma((double)u.y, (double)v.y, s);
            s = fma((double)u.z, (double)v.z, s);
            s = fma((double)u.w, (double)v.w, s);
        }
    } else {
        for (int q = lane; q < n; q += 32) s = fma((double)__ldg(a + q), (double)__ldg(c + q), s);
    }
    return s;
}

// Column norms, one warp per column (optimize_subset.py:36-37).
template <bool VEC>
__global__ void __launch_bounds__(256) k_ss_norms(SsDev d) {
    const int lane = threadIdx.x & 31;
    const int j = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (j >= d.ncols) return;
    const float* a = d.A + (size_t)j * d.nfeat;
    const double ss = warp_sum_d(lane_dot_ff<VEC>(a, a, d.nfeat, lane));
    if (lane == 0) {
        d.nrm[j] = ss > 0.0 ? sqrt(ss) : 1.0;
        d.taken[j] = 0;
    }
}

// Partial target sums over one chunk of columns: bpart[c][i] = sum_j colw[j] A[j][i].
__global__ void __launch_bounds__(256) k_ss_target_part(SsDev d) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (i >= d.nfeat) return;
    const int lo = (int)((long long)d.ncols * c / kTargetChunks), hi = (int)((long long)d.ncols * (c + 1) / kTargetChunks);
    double s = 0.0;
#pragma unroll 8
    for (int j = lo; j < hi; ++j) s = fma(__ldg(d.colw + j), (double)__ldg(d.A + (size_t)j * d.nfeat + i), s);
    d.bpart[(size_t)c * d.nfeat + i] = s;
}

// b = sum of the partials / sum(colw) (optimize_subset.py:32); r = b (:35).
__global__ void __launch_bounds__(256) k_ss_target(SsDev d) {
    __shared__ double ws[8];
    double w = 0.0;
    for (int j = threadIdx.x; j < d.ncols; j += 256) w += d.colw[j];
    w = warp_sum_d(w);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = w;
    __syncthreads();
    double W = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) W += ws[k];
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= d.nfeat) return;
    double s = 0.0;
    for (int c = 0; c < kTargetChunks; ++c) s += d.bpart[(size_t)c * d.nfeat + i];
    const double b = s / W;
    d.b[i] = b;
    d.r[i] = b;
}

// corr_j = <A_j, r> / |A_j| for unselected j (optimize_subset.py:41-43) and
// the CTA's (max, first index).
template <bool VEC>
__global__ void __launch_bounds__(kCorrWarps * 32) k_ss_corr(SsDev d) {
    __shared__ double wv[kCorrWarps];
    __shared__ int wi[kCorrWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int j = blockIdx.x * kCorrWarps + w;
    double v = -INFINITY;
    int idx = INT_MAX;
    if (j < d.ncols && !d.taken[j] && !*d.err) {
        const double s = warp_sum_d(lane_dot<VEC>(d.A + (size_t)j * d.nfeat, d.r, d.nfeat, lane));
        v = s / d.nrm[j];
        idx = j;
    }
    if (lane == 0) { wv[w] = v; wi[w] = idx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bv = wv[0];
        int bi = wi[0];
        for (int k = 1; k < kCorrWarps; ++k) amax_merge(bv, bi, wv[k], wi[k]);
        d.part_v[blockIdx.x] = bv;
        d.part_i[blockIdx.x] = bi;
    }
}

// The (max, first index) of the k_ss_corr partials, reduced by one CTA of
// NT threads (every thread gets it); -1 when no finite correlation is left.
template <int NT>
__device__ __forceinline__ int ss_argmax_partials(const SsDev& d) {
    __shared__ double av[NT / 32];
    __shared__ int ai[NT / 32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    double v = -INFINITY;
    int i = INT_MAX;
    for (int k = tid; k < d.ncorr; k += NT) amax_merge(v, i, d.part_v[k], d.part_i[k]);
    warp_amax(v, i);
    if (lane == 0) { av[w] = v; ai[w] = i; }
    __syncthreads();
    double bv = av[0];
    int bi = ai[0];
#pragma unroll
    for (int k = 1; k < NT / 32; ++k) amax_merge(bv, bi, av[k], ai[k]);
    return (bv > -INFINITY && bi < d.ncols) ? bi : -1;
}

// Step s, part 1 (optimize_subset.py:44-45): the selected column t and its
// Gram row G[s][0..s] = <A_t, A_sel[q]> (q < s), <A_t, A_t>, and
// h[s] = <A_t, b>: one warp per dot, s + 2 dots.
template <bool VEC>
__global__ void __launch_bounds__(256) k_ss_gram(SsDev d, int s) {
    if (*d.err) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int t = ss_argmax_partials<256>(d);
    if (t < 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(d.err, kErrNoCandidate);
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d.sel[s] = t;
        d.taken[t] = 1;
    }
    const int q = blockIdx.x * 8 + w;
    if (q > s + 1) return;
    const float* At = d.A + (size_t)t * d.nfeat;
    double v;
    if (q <= s) {
        const int c = q < s ? d.sel[q] : t;
        v = warp_sum_d(lane_dot_ff<VEC>(At, d.A + (size_t)c * d.nfeat, d.nfeat, lane));
    } else {
        v = warp_sum_d(lane_dot<VEC>(At, d.b, d.nfeat, lane));
    }
    if (lane == 0) {
        if (q <= s) d.G[tri(s) + q] = v;
        else d.h[s] = v;
    }
}

// Shared memory of k_ss_nnls for subproblems of up to K <= 128 columns.
struct StepSmem {
    double* G;      // tri(K): packed lower Gram matrix of the selected columns
    double* F;      // tri(K): LDL^T factor of the passive block, list order (see ss_factor)
    double* h;      // K
    double* x;      // K: current weights
    double* z;      // K: passive-set solution, list order
    double* y;      // K: D^-1 L'^-1 h_P, list order
    double* dual;   // K
    double* invd;   // K: 1 / pivot
    int* plist;     // K: the passive set in the order it was built
    int* inP;       // K: 1 for a passive column
    int* misc;      // [0] passive count, [1] pivot flag, [3] outcome
    static size_t bytes(int K) { return sizeof(double) * (2 * (size_t)tri(K) + 6 * (size_t)K) + sizeof(int) * (2 * (size_t)K + 8); }
    __device__ void carve(void* base, int K) {
        double* p = reinterpret_cast<double*>(base);
        G = p; p += tri(K);
        F = p; p += tri(K);
        h = p; p += K;
        x = p; p += K;
        z = p; p += K;
        y = p; p += K;
        dual = p; p += K;
        invd = p; p += K;
        plist = reinterpret_cast<int*>(p);
        inP = plist + K;
        misc = inP + K;
    }
};

__device__ __forceinline__ double gsym(const double* G, int i, int j) { return i >= j ? G[tri(i) + j] : G[tri(j) + i]; }

// The register of a warp-distributed vector (row i = lane + 32 g) that holds row k.
__device__ __forceinline__ double pick4(double v0, double v1, double v2, double v3, int k) {
    const int g = k >> 5;
    return g == 0 ? v0 : (g == 1 ? v1 : (g == 2 ? v2 : v3));
}

// G_PP = L' D L'^T for the passive list P (np >= 1) by right-looking
// elimination, one barrier per column.  F holds, on and below the diagonal,
// the eliminated matrix: F(i, k) = L'(i, k) d_k and F(k, k) = d_k; invd[k] =
// 1 / d_k, computed by the thread that finishes pivot k.  Returns false, in
// every thread, when a pivot is not positive (a rank-deficient block).
__device__ bool ss_factor(StepSmem& m, int np) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int* P = m.plist;
    for (int i = w; i < np; i += kStepWarps)
        for (int k = lane; k <= i; k += 32) m.F[tri(i) + k] = gsym(m.G, P[i], P[k]);
    __syncthreads();
    if (tid == 0) {
        const double d0 = m.F[0];
        m.misc[1] = d0 > 0.0 ? 0 : 1;
        m.invd[0] = 1.0 / d0;
    }
    __syncthreads();
    for (int j = 0; j + 1 < np; ++j) {
        const double ivj = m.invd[j];
        const double* Fj = m.F + j;   // column j: Fj[tri(k)] = F(k, j)
        // row i = j + 1 + w + 16 r; warp 0 owns row j + 1 and lane 0 its diagonal
        for (int i = j + 1 + w; i < np; i += kStepWarps) {
            double* Fi = m.F + tri(i);
            const double lij = Fi[j] * ivj;
            for (int k = j + 1 + lane; k <= i; k += 32) Fi[k] = fma(-lij, Fj[tri(k)], Fi[k]);
            if (i == j + 1 && lane == 0) {
                const double dd = Fi[i];
                if (!(dd > 0.0)) m.misc[1] = 1;
                m.invd[i] = 1.0 / dd;
            }
        }
        __syncthreads();
    }
    return m.misc[1] == 0;
}

// z = G_PP^-1 h_P from the factor, on one warp: L' u = h_P, y = D^-1 u,
// L'^T z = y.  Each lane holds rows lane + 32 mm in registers; a step
// broadcasts one finished row with a shuffle.
__device__ __forceinline__ void ss_solve_warp(StepSmem& m, int np, int lane) {
    const int* P = m.plist;
    const int i0 = lane, i1 = lane + 32, i2 = lane + 64, i3 = lane + 96;
    double u0 = i0 < np ? m.h[P[i0]] : 0.0, u1 = i1 < np ? m.h[P[i1]] : 0.0;
    double u2 = i2 < np ? m.h[P[i2]] : 0.0, u3 = i3 < np ? m.h[P[i3]] : 0.0;
    for (int k = 0; k < np; ++k) {
        const double yk = __shfl_sync(0xFFFFFFFFu, pick4(u0, u1, u2, u3, k), k & 31) * m.invd[k];
        if (lane == (k & 31)) m.y[k] = yk;
        if (i0 > k && i0 < np) u0 = fma(-m.F[tri(i0) + k], yk, u0);
        if (i1 > k && i1 < np) u1 = fma(-m.F[tri(i1) + k], yk, u1);
        if (i2 > k && i2 < np) u2 = fma(-m.F[tri(i2) + k], yk, u2);
        if (i3 > k && i3 < np) u3 = fma(-m.F[tri(i3) + k], yk, u3);
    }
    __syncwarp();
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;   // sum over k > i of F(k, i) z_k
    for (int k = np - 1; k >= 0; --k) {
        const double own = m.y[k] - m.invd[k] * pick4(a0, a1, a2, a3, k);   // z_k on its lane
        const double zk = __shfl_sync(0xFFFFFFFFu, own, k & 31);
        if (lane == (k & 31)) m.z[k] = zk;
        const double* Fk = m.F + tri(k);
        if (i0 < k) a0 = fma(Fk[i0], zk, a0);
        if (i1 < k) a1 = fma(Fk[i1], zk, a1);
        if (i2 < k) a2 = fma(Fk[i2], zk, a2);
        if (i3 < k) a3 = fma(Fk[i3], zk, a3);
    }
    __syncwarp();
}

// Step s, part 2 (optimize_subset.py:46-47): the non-negative least-squares
// weights of the selected columns (Lawson-Hanson on G x = h, started from the
// previous step's weights), then the residual r = b - A_sel x.
template <bool VEC>
__global__ void __launch_bounds__(kStepThreads) k_ss_nnls(SsDev d, int s) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (*d.err) return;
    StepSmem m;
    m.carve(smem_raw, d.nsel);
    const int n = s + 1;
    for (int k = tid; k < tri(n); k += kStepThreads) m.G[k] = d.G[k];
    for (int k = tid; k < n; k += kStepThreads) {
        m.h[k] = d.h[k];
        m.x[k] = k < s ? d.x[k] : 0.0;
    }
    __syncthreads();
    // the passive set starts as the previous weights' support
    if (w == 0) {
        int base = 0;
        for (int c = 0; c < n; c += 32) {
            const int i = c + lane;
            const bool in = i < n && m.x[i] > 0.0;
            if (i < n) m.inP[i] = in;
            const unsigned bal = __ballot_sync(0xFFFFFFFFu, in);
            if (in) m.plist[base + __popc(bal & ((1u << lane) - 1u))] = i;
            base += __popc(bal);
        }
        if (lane == 0) {
            m.misc[0] = base;
            m.misc[3] = 0;
        }
    }
    double hmax = 0.0;
    for (int i = 0; i < n; ++i) hmax = fmax(hmax, fabs(m.h[i]));
    const double tol = 1e-10 * hmax;   // dual tolerance, far inside the shipped dump's 2.6e-6 margin
    int solves = 0;
    bool fail = false;
    __syncthreads();
    for (;;) {
        // dual d_i = h_i - sum_k G_ik x_k, one warp per row
        for (int i = w; i < n; i += kStepWarps) {
            double sacc = 0.0;
            for (int k = lane; k < n; k += 32) sacc = fma(gsym(m.G, i, k), m.x[k], sacc);
            sacc = warp_sum_d(sacc);
            if (lane == 0) m.dual[i] = m.h[i] - sacc;
        }
        __syncthreads();
        if (w == 0) {
            // the free index with the largest dual above tol (the first on ties) joins P
            double bv = tol;
            int best = INT_MAX;
            for (int i = lane; i < n; i += 32)
                if (!m.inP[i] && m.dual[i] > bv) { bv = m.dual[i]; best = i; }
            warp_amax(bv, best);
            if (lane == 0) {
                if (best == INT_MAX) {
                    m.misc[3] = 1;
                } else {
                    m.plist[m.misc[0]++] = best;
                    m.inP[best] = 1;
                }
            }
        }
        __syncthreads();
        if (m.misc[3] == 1) break;
        // inner loop: solve on P, step back towards the solution while a weight is not positive
        for (;;) {
            if (++solves > 3 * n) {
                if (tid == 0) atomicOr(d.err, kErrIters);
                fail = true;
                break;
            }
            const int np = m.misc[0];
            if (!ss_factor(m, np)) {
                if (tid == 0) atomicOr(d.err, kErrRank);
                fail = true;
                break;
            }
            if (w == 0) {
                ss_solve_warp(m, np, lane);
                // outcome: 2 = z is the solution, 0 = stepped back, 3 = z holds a NaN
                bool pos = true;
                for (int a = lane; a < np; a += 32) pos &= m.z[a] > 0.0;
                pos = __all_sync(0xFFFFFFFFu, pos);
                if (pos) {
                    for (int a = lane; a < np; a += 32) m.x[m.plist[a]] = m.z[a];
                    if (lane == 0) m.misc[3] = 2;
                } else {
                    // the largest step from x towards z that keeps x >= 0 (first minimum in list order)
                    double al = INFINITY;
                    int qa = INT_MAX;
                    for (int a = lane; a < np; a += 32) {
                        const double za = m.z[a];
                        if (za <= 0.0) {
                            const double xa = m.x[m.plist[a]];
                            const double c = xa / (xa - za);
                            if (c < al) { al = c; qa = a; }
                        }
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const double al2 = __shfl_xor_sync(0xFFFFFFFFu, al, o);
                        const int qa2 = __shfl_xor_sync(0xFFFFFFFFu, qa, o);
                        if (al2 < al || (al2 == al && qa2 < qa)) { al = al2; qa = qa2; }
                    }
                    if (qa == INT_MAX) {
                        if (lane == 0) m.misc[3] = 3;
                    } else {
                        for (int a = lane; a < np; a += 32) {
                            const int i = m.plist[a];
                            m.x[i] = fma(al, m.z[a] - m.x[i], m.x[i]);
                        }
                        __syncwarp();
                        if (lane == 0) m.x[m.plist[qa]] = 0.0;
                        __syncwarp();
                        // keep the positive weights, in order
                        int base = 0;
                        for (int c = 0; c < np; c += 32) {
                            const int a = c + lane;
                            const int i = a < np ? m.plist[a] : -1;
                            const bool keep = i >= 0 && m.x[i] > 0.0;
                            const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
                            __syncwarp();
                            if (keep) {
                                m.plist[base + __popc(bal & ((1u << lane) - 1u))] = i;
                            } else if (i >= 0) {
                                m.x[i] = 0.0;
                                m.inP[i] = 0;
                            }
                            base += __popc(bal);
                            __syncwarp();
                        }
                        if (lane == 0) {
                            m.misc[0] = base;
                            m.misc[3] = base == 0 ? 2 : 0;   // an empty passive set is its own solution
                        }
                    }
                }
            }
            __syncthreads();
            const int outcome = m.misc[3];
            __syncthreads();
            if (outcome == 3) {
                if (tid == 0) atomicOr(d.err, kErrRank);
                fail = true;
                break;
            }
            if (outcome == 2) {
                if (tid == 0) m.misc[3] = 0;
                break;
            }
        }
        __syncthreads();
        if (fail) return;
    }
    // the residual r = b - A_sel x over the passive columns (the weights off
    // the passive set are zero), and the weights for the next step; the
    // passive columns' rows and weights are staged where inP and z were
    const int np = m.misc[0];
    for (int a = tid; a < np; a += kStepThreads) {
        m.inP[a] = d.sel[m.plist[a]];
        m.z[a] = m.x[m.plist[a]];
    }
    __syncthreads();
    if (VEC) {
        const double2* b2 = reinterpret_cast<const double2*>(d.b);
        double2* r2 = reinterpret_cast<double2*>(d.r);
        for (int qv = tid; qv < (d.nfeat >> 2); qv += kStepThreads) {
            double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
#pragma unroll 8
            for (int a = 0; a < np; ++a) {
                const float4 u = __ldg(reinterpret_cast<const float4*>(d.A + (size_t)m.inP[a] * d.nfeat) + qv);
                const double xa = m.z[a];
                v0 = fma((double)u.x, xa, v0);
                v1 = fma((double)u.y, xa, v1);
                v2 = fma((double)u.z, xa, v2);
                v3 = fma((double)u.w, xa, v3);
            }
            const double2 bl = b2[2 * qv], bh = b2[2 * qv + 1];
            r2[2 * qv] = make_double2(bl.x - v0, bl.y - v1);
            r2[2 * qv + 1] = make_double2(bh.x - v2, bh.y - v3);
        }
    } else {
        for (int i = tid; i < d.nfeat; i += kStepThreads) {
            double v = 0.0;
#pragma unroll 8
            for (int a = 0; a < np; ++a) v = fma((double)__ldg(d.A + (size_t)m.inP[a] * d.nfeat + i), m.z[a], v);
            d.r[i] = d.b[i] - v;
        }
    }
    for (int k = tid; k < n; k += kStepThreads) d.x[k] = m.x[k];
    // after the last step: the weights normalised to sum ncols (optimize_subset.py:49-50)
    if (s + 1 == d.nsel) {
        double sum = 0.0;
        for (int p = 0; p < n; ++p) sum += m.x[p];   // every thread, the same order
        const double f = (double)d.ncols / sum;
        for (int p = tid; p < n; p += kStepThreads) {
            d.out_idx[p] = d.sel[p];
            d.out_w[p] = m.x[p] * f;
        }
    }
}

template <bool VEC>
int run(SsDev& d, cudaStream_t st) {
    const size_t smem = StepSmem::bytes(d.nsel);
    MTT_TRY_CUDA(cudaFuncSetAttribute(k_ss_nnls<VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_ss_norms<VEC><<<ceil_div(d.ncols, 8), 256, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    k_ss_target_part<<<dim3(ceil_div(d.nfeat, 256), kTargetChunks), 256, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    k_ss_target<<<ceil_div(d.nfeat, 256), 256, 0, st>>>(d);
    MTT_CHECK_LAUNCH();
    for (int s = 0; s < d.nsel; ++s) {
        k_ss_corr<VEC><<<d.ncorr, kCorrWarps * 32, 0, st>>>(d);
        MTT_CHECK_LAUNCH();
        k_ss_gram<VEC><<<ceil_div(s + 2, 8), 256, 0, st>>>(d, s);
        MTT_CHECK_LAUNCH();
        k_ss_nnls<VEC><<<1, kStepThreads, smem, st>>>(d, s);
        MTT_CHECK_LAUNCH();
    }
    return MTT_OK;
}


}  // namespace ss
}  // namespace mtt

extern "C" int mtt_subset_nnomp(const float* d_cols, int32_t ncols, int32_t nfeat, const double* d_colw,
                                int32_t nselect, int32_t* d_idx, double* d_w, void* stream) {
    using namespace mtt;
    using namespace mtt::ss;
    if (!d_cols || !d_colw || !d_idx || !d_w || ncols < 1 || nfeat < 1 || nselect < 1 || nselect > ncols ||
        nselect > MTT_SUBSET_MAX_SELECT)
        return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    SsDev d{};
    d.A = d_cols; d.colw = d_colw;
    d.ncols = ncols; d.nfeat = nfeat; d.nsel = nselect;
    d.ncorr = ceil_div(ncols, kCorrWarps);
    d.out_idx = d_idx; d.out_w = d_w;
    // one workspace: doubles first, then ints, then bytes
    const size_t nd = 2 * (size_t)nfeat + (size_t)ncols + (size_t)kTargetChunks * nfeat + (size_t)d.ncorr +
                      (size_t)tri(nselect) + 2 * (size_t)nselect;
    const size_t ni = (size_t)d.ncorr + (size_t)nselect + 4;
    const size_t bytes = sizeof(double) * nd + sizeof(int) * ni + (size_t)ncols;
    unsigned char* ws = nullptr;
    MTT_TRY_CUDA(cudaMallocAsync(&ws, bytes, st));
    double* p = reinterpret_cast<double*>(ws);
    d.b = p; p += nfeat;
    d.r = p; p += nfeat;
    d.nrm = p; p += ncols;
    d.bpart = p; p += (size_t)kTargetChunks * nfeat;
    d.part_v = p; p += d.ncorr;
    d.G = p; p += tri(nselect);
    d.h = p; p += nselect;
    d.x = p; p += nselect;
    int* q = reinterpret_cast<int*>(p);
    d.part_i = q; q += d.ncorr;
    d.sel = q; q += nselect;
    d.err = q; q += 4;
    d.taken = reinterpret_cast<uint8_t*>(q);
    int s = cuda_status(cudaMemsetAsync(d.err, 0, sizeof(int), st));
    if (!s) s = cuda_status(cudaMemsetAsync(d.x, 0, sizeof(double) * nselect, st));
    const bool vec = (nfeat % 4 == 0) && (reinterpret_cast<uintptr_t>(d_cols) % 16 == 0);
    if (!s) s = vec ? run<true>(d, st) : run<false>(d, st);
    int herr = 0;
    if (!s) s = cuda_status(cudaMemcpyAsync(&herr, d.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (!s) s = cuda_status(cudaStreamSynchronize(st));
    cudaFreeAsync(ws, st);
    if (!s && herr) s = (herr & kErrNoCandidate) ? MTT_ERR_INVALID : MTT_ERR_UNSUPPORTED;
    return s;
}

extern "C" int mtt_subset_write(const char* bin_path, const char* txt_path, const uint8_t* h_flops3, const double* h_w,
                                int32_t n) {
    if (n < 0 || (n > 0 && (!h_flops3 || !h_w))) return MTT_ERR_INVALID;
    for (int32_t i = 0; i < 3 * n; ++i)
        if (h_flops3[i] > 51) return MTT_ERR_INVALID;
    if (bin_path) {
        FILE* f = std::fopen(bin_path, "wb");
        if (!f) return MTT_ERR_IO;
        const uint32_t cnt = (uint32_t)n;
        bool ok = std::fwrite(&cnt, 4, 1, f) == 1;
        for (int32_t i = 0; i < n && ok; ++i) {
            unsigned char rec[8] = {h_flops3[3 * i], h_flops3[3 * i + 1], h_flops3[3 * i + 2], 0};
            const float w = (float)h_w[i];   // round to nearest, as struct.pack("f")
            std::memcpy(rec + 4, &w, 4);
            ok = std::fwrite(rec, 1, 8, f) == 8;
        }
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) return MTT_ERR_IO;
    }
    if (txt_path) {
        FILE* f = std::fopen(txt_path, "w");
        if (!f) return MTT_ERR_IO;
        static const char kRanks[] = "23456789TJQKA", kSuits[] = "cdhs";
        bool ok = true;
        for (int32_t i = 0; i < n && ok; ++i) {
            char name[7];
            for (int k = 0; k < 3; ++k) {
                name[2 * k] = kRanks[h_flops3[3 * i + k] / 4];
                name[2 * k + 1] = kSuits[h_flops3[3 * i + k] % 4];
            }
            name[6] = 0;
            ok = std::fprintf(f, "%s:%.4f\n", name, h_w[i]) > 0;
        }
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) return MTT_ERR_IO;
    }
    return MTT_OK;
}
