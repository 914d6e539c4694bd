// gemm.cu — BF16 GEMM on the 5th-generation tensor cores (tcgen05) for the
// leaf network: C[M x N] = epilogue(A[M x K] * B[N x K]^T), A and B row-major
// (K contiguous), FP32 accumulation in tensor memory.
//
// One 128 x 256 output tile per CTA of 576 threads:
//   warp 0      one thread streams 128 x 64 tiles of A and 256 x 64 of B into a 4-stage
//               shared-memory ring with 2-D TMA loads (128-byte swizzle),
//               completing on the stage's "full" mbarrier;
//   warp 1      allocates 256 TMEM columns; one thread issues
//               tcgen05.mma (M=128, N=256, K=16, kind::f16, BF16 in, FP32
//               accumulate) four times per stage and commits each stage back
//               to its "empty" mbarrier, then commits the accumulator;
//   warps 2..17 read the accumulator with tcgen05.ld (warp w owns TMEM lanes
//               32*(w%4) .. +31 = output rows; warps 2-5 take columns 0-63,
//               6-9 the next 64, and so on), add the bias, apply ReLU or a
//               ReLU mask, convert, and stage 32-row boxes in the (now idle)
//               operand ring for TMA stores; an output whose rows are not
//               16-byte aligned goes through a padded transpose tile instead,
//               one row of 32 columns per store instruction.
// Every mbarrier wait is bounded; a wait that gives up sets *err, the
// producer still waits (bounded) for its own copies and the allocating warp
// frees the TMEM before the CTA leaves.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "mtt_bulk.cuh"
#include "mtt_common.h"

namespace mtt {
namespace gemm {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4, THREADS = 576;
constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;   // tiles (1024-aligned) + barriers
constexpr uint32_t TMEM_COLS = BN;   // one FP32 column per output column

enum { F_RELU = 1, F_OUT_BF16 = 2, F_MASK = 4 };

// Shared-memory matrix descriptor of a K-major operand tile written by TMA
// with 128-byte swizzle: rows of 128 B, 8-row groups 1024 B apart (stride
// byte offset), leading byte offset 16 B (unused for swizzled K-major),
// descriptor version 1, layout type 2 = SWIZZLE_128B.
__device__ __forceinline__ uint64_t smem_desc(const void* p) {
    const uint64_t a = (uint64_t)(smem_addr(p) >> 4) & 0x3FFFull;
    return a | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor of kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    const uint32_t m0 = 0u, m1 = 0u, m2 = 0u, m3 = 0u;   // no output lanes disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2), "r"(m3)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive accumulator columns of this warp's 32 TMEM lanes (lane =
// row); complete after tmem_ld_wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// TMA store of one staged box (this CTA's shared memory -> global) through a
// 3-D map, in this thread's bulk group.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y, int z) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map), "r"(x),
                 "r"(y), "r"(z), "r"(smem_addr(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Output paths of the epilogue.
enum { OUT_DIRECT = 0, OUT_TMA_C = 1, OUT_TMA_WS = 2 };

__global__ void __launch_bounds__(THREADS, 1)
k_gemm_bf16(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
            const __grid_constant__ CUtensorMap tc, int out_mode, void* __restrict__ C,
            int M, int N, int K, int ldc, const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask,
            int ldm, int flags, int* __restrict__ err, int kps, float* __restrict__ ws, int ldw) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* accum = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
    int* s_fail = reinterpret_cast<int*>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    // split z of gridDim.z takes k-tiles [kt0, kt0 + KT); with ws its raw
    // FP32 partial tile goes to ws + z M N (row stride N) for k_gemm_reduce
    const int kt0 = (int)blockIdx.z * kps;
    const int KT = min((K + BK - 1) / BK - kt0, kps);
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(accum, 1);
        *s_fail = 0;
        mbar_fence_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // launched with programmatic stream serialization: the set-up above ran
    // while the previous kernel drained; its outputs (A, B, C) are ours now
    grid_dep_trigger();
    grid_dep_wait();

    if (warp == 0 && lane == 0) {
        // producer: stage s of k-tile kt; the stage is free once the MMAs of
        // k-tile kt - STAGES have completed (their commit to empty[s])
        int kt = 0;
        for (; kt < KT; ++kt) {
            const int s = kt % STAGES;
            if (kt >= STAGES && !mbar_wait_bounded(&empty[s], (uint32_t)((kt / STAGES - 1) & 1))) {
                atomicOr(err, 1);
                *s_fail = 1;
                break;
            }
            uint8_t* st = smem + s * STAGE_BYTES;
            mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
            tma_load_2d(st, &ta, (kt0 + kt) * BK, m0, &full[s]);
            tma_load_2d(st + A_BYTES, &tb, (kt0 + kt) * BK, n0, &full[s]);
        }
        // our own copies have landed before the CTA can leave
        for (int j = (kt > STAGES ? kt - STAGES : 0); j < kt; ++j)
            (void)mbar_wait_bounded(&full[j % STAGES], (uint32_t)((j / STAGES) & 1));
    } else if (warp == 1 && lane == 0) {
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % STAGES;
            if (!mbar_wait_bounded(&full[s], (uint32_t)((kt / STAGES) & 1))) {
                atomicOr(err, 1);
                *s_fail = 1;
                break;
            }
            tc_fence_after();
            const uint8_t* st = smem + s * STAGE_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
                umma_bf16(tmem, smem_desc(st + kk * 32), smem_desc(st + A_BYTES + kk * 32), (kt | kk) ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        umma_commit(accum);   // fires when every MMA issued above has completed
    } else if (warp >= 2) {
        const bool ok = mbar_wait_bounded(accum, 0u);
        __syncwarp();
        tc_fence_after();
        if (!ok) atomicOr(err, 1);
        const int lg = warp & 3;                     // TMEM lanes 32*lg .. 32*lg+31
        const int c_lo = ((warp - 2) >> 2) * (BN / 4), c_hi = c_lo + BN / 4;   // this warp's 64 columns
        const int r0 = m0 + 32 * lg;
        const bool live = ok && !*(volatile int*)s_fail;
        if (out_mode != OUT_DIRECT) {
            // Each lane holds one output row.  A box is 32 rows x 128 bytes
            // (32 FP32 or 64 BF16 columns), staged in the now idle operand
            // ring with the 128-byte swizzle (16-byte chunk j of row r at
            // chunk j ^ (r & 7): one store instruction fills 4 banks-wide
            // wavefronts) and written by one TMA store; two boxes per warp
            // alternate so that filling one overlaps the other's store.
            const bool to_bf16 = out_mode == OUT_TMA_C && (flags & F_OUT_BF16);
            const int groups = to_bf16 ? 2 : 1;                  // 32-column TMEM groups per box
            uint8_t* stage = smem + (size_t)(warp - 2) * 8192;
            const int row = r0 + lane;
            int k = 0;
#pragma unroll 1
            for (int c = c_lo; c < c_hi; c += 32 * groups, ++k) {
                uint8_t* box = stage + (k & 1) * 4096;
                if (lane == 0) bulk_wait_read_1();                // the store that last read this box is done
                __syncwarp();
                bool any = false;
#pragma unroll 1
                for (int g = 0; g < groups; ++g) {
                    const int cg = c + 32 * g;
                    uint32_t r[32];
                    tmem_ld16(tmem + ((uint32_t)(32 * lg) << 16) + (uint32_t)cg, r);
                    tmem_ld16(tmem + ((uint32_t)(32 * lg) << 16) + (uint32_t)(cg + 16), r + 16);
                    tmem_ld_wait();
                    if (!live || n0 + cg >= N || r0 >= M) continue;   // warp-uniform
                    any = true;
                    if (out_mode == OUT_TMA_C) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int col = n0 + cg + j;
                            float v = __uint_as_float(r[j]);
                            if (bias) v += col < N ? __ldg(bias + col) : 0.0f;
                            if ((flags & F_RELU) && v < 0.0f) v = 0.0f;
                            if ((flags & F_MASK) && row < M && col < N &&
                                !(__bfloat162float(mask[(size_t)row * ldm + col]) > 0.0f))
                                v = 0.0f;
                            r[j] = __float_as_uint(v);
                        }
                    }
                    if (to_bf16) {   // 32 columns = 64 bytes = chunks 4 g .. 4 g + 3
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            uint32_t w[4];
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const __nv_bfloat162 h = __floats2bfloat162_rn(__uint_as_float(r[8 * q + 2 * e]),
                                                                               __uint_as_float(r[8 * q + 2 * e + 1]));
                                w[e] = *reinterpret_cast<const uint32_t*>(&h);
                            }
                            const int ch = (4 * g + q) ^ (lane & 7);
                            *reinterpret_cast<uint4*>(box + lane * 128 + ch * 16) = make_uint4(w[0], w[1], w[2], w[3]);
                        }
                    } else {         // 32 columns = 128 bytes = chunks 0 .. 7
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int ch = q ^ (lane & 7);
                            *reinterpret_cast<uint4*>(box + lane * 128 + ch * 16) =
                                make_uint4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
                        }
                    }
                }
                if (!any) continue;                                   // warp-uniform
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tma_store_3d(&tc, box, n0 + c, r0, out_mode == OUT_TMA_WS ? (int)blockIdx.z : 0);
                    bulk_commit();
                }
            }
            if (lane == 0) bulk_wait_all();
            __syncwarp();
        } else {
        // this warp's 32 x 33 transpose tile in the (now idle) operand ring
        float* P = reinterpret_cast<float*>(smem) + (warp - 2) * 32 * 33;
#pragma unroll 1
        for (int c = c_lo; c < c_hi; c += 32) {
            uint32_t r[32];
            tmem_ld16(tmem + ((uint32_t)(32 * lg) << 16) + (uint32_t)c, r);
            tmem_ld16(tmem + ((uint32_t)(32 * lg) << 16) + (uint32_t)(c + 16), r + 16);
            tmem_ld_wait();
            if (!live || n0 + c >= N || r0 >= M) continue;   // warp-uniform
#pragma unroll
            for (int j = 0; j < 32; ++j) P[lane * 33 + j] = __uint_as_float(r[j]);   // (row lane, column j)
            __syncwarp();
            const int col = n0 + c + lane;
            const bool cin = col < N;
            if (ws) {   // a split's raw partial sums
                float* W = ws + (size_t)blockIdx.z * M * ldw;
#pragma unroll 4
                for (int i = 0; i < 32; ++i) {
                    const int row = r0 + i;
                    if (row >= M) break;
                    if (cin) W[(size_t)row * ldw + col] = P[i * 33 + lane];
                }
                __syncwarp();
                continue;
            }
            const float b = (bias && cin) ? bias[col] : 0.0f;
#pragma unroll 4
            for (int i = 0; i < 32; ++i) {
                const int row = r0 + i;
                if (row >= M) break;
                float v = P[i * 33 + lane];
                if (bias) v += b;
                if ((flags & F_RELU) && v < 0.0f) v = 0.0f;
                if (cin) {
                    if ((flags & F_MASK) && !(__bfloat162float(mask[(size_t)row * ldm + col]) > 0.0f)) v = 0.0f;
                    if (flags & F_OUT_BF16) reinterpret_cast<__nv_bfloat16*>(C)[(size_t)row * ldc + col] = __float2bfloat16_rn(v);
                    else reinterpret_cast<float*>(C)[(size_t)row * ldc + col] = v;
                }
            }
            __syncwarp();
        }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Sum of the splits' partial tiles in split order, then the epilogue of the
// single-pass kernel (bias, ReLU, ReLU mask, BF16 or FP32 store).
__global__ void __launch_bounds__(256) k_gemm_reduce(const float* __restrict__ ws, int ldw, int splits,
                                                     void* __restrict__ C, int M, int N, int ldc,
                                                     const float* __restrict__ bias,
                                                     const __nv_bfloat16* __restrict__ mask, int ldm, int flags) {
    grid_dep_wait();   // the splits' partial tiles
    grid_dep_trigger();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)M * N) return;
    const int row = (int)(i / N), col = (int)(i % N);
    const size_t w = (size_t)row * ldw + col;
    float v = ws[w];
    for (int z = 1; z < splits; ++z) v += ws[(size_t)z * M * ldw + w];
    if (bias) v += bias[col];
    if ((flags & F_RELU) && v < 0.0f) v = 0.0f;
    if ((flags & F_MASK) && !(__bfloat162float(mask[(size_t)row * ldm + col]) > 0.0f)) v = 0.0f;
    if (flags & F_OUT_BF16) reinterpret_cast<__nv_bfloat16*>(C)[(size_t)row * ldc + col] = __float2bfloat16_rn(v);
    else reinterpret_cast<float*>(C)[(size_t)row * ldc + col] = v;
}

// Host: the driver's tensor-map encoder, found once through the runtime.
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;

static int encoder(PFN_cuTensorMapEncodeTiled_v12000* out) {
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return MTT_ERR_UNSUPPORTED;
    *out = g_encode;
    return MTT_OK;
}

// 2-D map of a row-major bf16 matrix [rows x cols] with leading dimension ld,
// box 64 (cols) x box_rows (rows), 128-byte swizzle, zero fill outside.
// 3-D map of an output [z][rows][cols] with row stride ld elements of esize
// bytes: boxes of 32 rows x 128 bytes, 128-byte swizzle (the epilogue's
// staging layout).  ld * esize must be a multiple of 16.
static int make_out_map(CUtensorMap* map, void* base, CUtensorMapDataType dt, int esize, int rows, int cols, int ld,
                        int z) {
    PFN_cuTensorMapEncodeTiled_v12000 enc;
    MTT_TRY(encoder(&enc));
    const cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)z};
    const cuuint64_t strides[2] = {(cuuint64_t)ld * esize, (cuuint64_t)rows * ld * esize};
    const cuuint32_t box[3] = {(cuuint32_t)(128 / esize), 32, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(map, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MTT_OK : MTT_ERR_INVALID;
}

static int make_map(CUtensorMap* map, const void* base, int rows, int cols, int ld, int box_rows) {
    PFN_cuTensorMapEncodeTiled_v12000 enc;
    MTT_TRY(encoder(&enc));
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MTT_OK : MTT_ERR_INVALID;
}

// The kernel's shared-memory opt-in, set once per device (a per-call
// cudaFuncSetAttribute costs host time on every launch).
static std::mutex g_attr_mu;
static bool g_attr_done[64] = {};

static int smem_attr_once() {
    int dev = 0;
    MTT_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return MTT_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_attr_mu);
    if (!g_attr_done[dev]) {
        MTT_TRY_CUDA(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        g_attr_done[dev] = true;
    }
    return MTT_OK;
}

// Split-K: a grid of fewer tiles than about the SM count, over at least 8
// k-tiles of 64, is cut along K into splits of at least 4 k-tiles, so that
// tiles x splits comes near the SM count; each split writes its partial tile
// to ws and k_gemm_reduce adds them in split order.  Without ws (or with too
// small a ws) the GEMM runs in one pass.
static int choose_splits(int M, int N, int K, int ldw, size_t ws_floats, int* kps) {
    const int tiles = ((N + BN - 1) / BN) * ((M + BM - 1) / BM);
    const int KT = (K + BK - 1) / BK;
    *kps = KT;
    if (!ws_floats || tiles >= 100 || KT < 8) return 1;
    int splits = std::min(std::max(148 / tiles, 1), KT / 4);
    while (splits > 1 && (size_t)splits * M * ldw > ws_floats) --splits;
    if (splits <= 1) return 1;
    *kps = (KT + splits - 1) / splits;
    return (KT + *kps - 1) / *kps;
}

static int launch(const void* A, int lda, const void* B, int ldb, void* C, int ldc, int M, int N, int K,
                  const float* bias, const void* mask, int ldm, int flags, int* d_err, cudaStream_t st,
                  float* ws, size_t ws_floats) {
    if (M <= 0 || N <= 0 || K <= 0) return M == 0 || N == 0 ? MTT_OK : MTT_ERR_INVALID;
    if (!A || !B || !C || !d_err || (lda % 8) || (ldb % 8) || lda < K || ldb < K || ldc < N) return MTT_ERR_INVALID;
    if (((uintptr_t)A & 15) || ((uintptr_t)B & 15)) return MTT_ERR_INVALID;
    if ((flags & F_MASK) && (!mask || ldm < N)) return MTT_ERR_INVALID;
    CUtensorMap ta, tb;
    MTT_TRY(make_map(&ta, A, M, K, lda, BM));
    MTT_TRY(make_map(&tb, B, N, K, ldb, BN));
    MTT_TRY(smem_attr_once());
    int kps = 0;
    const int ldw = (N + 3) & ~3;                  // workspace rows of 16-byte multiples
    const int splits = choose_splits(M, N, K, ldw, ws_floats, &kps);
    // the output path: TMA stores of staged boxes when the destination rows
    // are 16-byte aligned, else per-lane stores
    CUtensorMap tc;
    std::memset(&tc, 0, sizeof(tc));
    int out_mode = OUT_DIRECT;
    if (splits > 1) {
        if (!((uintptr_t)ws & 15) &&
            make_out_map(&tc, ws, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, M, N, ldw, splits) == MTT_OK)
            out_mode = OUT_TMA_WS;
    } else {
        const bool obf = flags & F_OUT_BF16;
        const int es = obf ? 2 : 4;
        if (!((uintptr_t)C & 15) && ((size_t)ldc * es) % 16 == 0 &&
            make_out_map(&tc, C, obf ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, es, M, N, ldc,
                         1) == MTT_OK)
            out_mode = OUT_TMA_C;
    }
    const dim3 grid((unsigned)((N + BN - 1) / BN), (unsigned)((M + BM - 1) / BM), (unsigned)splits);
    // both kernels wait in grid_dep_wait before touching global memory, so a
    // programmatic launch only lets their set-up overlap the previous kernel
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = grid;
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SMEM_BYTES;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MTT_TRY_CUDA(cudaLaunchKernelEx(&cfg, k_gemm_bf16, ta, tb, tc, out_mode, C, M, N, K, ldc, bias,
                                    reinterpret_cast<const __nv_bfloat16*>(mask), ldm, flags, d_err, kps,
                                    splits > 1 ? ws : nullptr, ldw));
    MTT_CHECK_LAUNCH();
    if (splits > 1) {
        const long long n = (long long)M * N;
        MTT_TRY_CUDA(launch_pdl(k_gemm_reduce, (unsigned)((n + 255) / 256), 256u, 0, st, true, (const float*)ws, ldw,
                                splits, C, M, N, ldc, bias, reinterpret_cast<const __nv_bfloat16*>(mask), ldm,
                                flags));
        MTT_CHECK_LAUNCH();
    }
    return MTT_OK;
}

}  // namespace gemm

int gemm_bf16(const void* A, int lda, const void* B, int ldb, void* C, int ldc, int M, int N, int K,
              const float* bias, const void* mask, int ldm, int flags, int* d_err, cudaStream_t st, float* ws,
              size_t ws_floats) {
    return gemm::launch(A, lda, B, ldb, C, ldc, M, N, K, bias, mask, ldm, flags, d_err, st, ws, ws_floats);
}

}  // namespace mtt

extern "C" int mtt_gemm_bf16(const void* d_A, int32_t lda, const void* d_B, int32_t ldb, void* d_C, int32_t ldc,
                             int32_t M, int32_t N, int32_t K, const float* d_bias, const void* d_mask, int32_t ldm,
                             int32_t flags, int32_t* d_err, void* stream) {
    return mtt::gemm_bf16(d_A, lda, d_B, ldb, d_C, ldc, M, N, K, d_bias, d_mask, ldm, flags, d_err,
                          mtt::as_stream(stream), nullptr, 0);
}

extern "C" int mtt_gemm_bf16_ws(const void* d_A, int32_t lda, const void* d_B, int32_t ldb, void* d_C, int32_t ldc,
                                int32_t M, int32_t N, int32_t K, const float* d_bias, const void* d_mask, int32_t ldm,
                                int32_t flags, int32_t* d_err, float* d_ws, int64_t ws_floats, void* stream) {
    if (ws_floats < 0 || (ws_floats > 0 && !d_ws)) return MTT_ERR_INVALID;
    return mtt::gemm_bf16(d_A, lda, d_B, ldb, d_C, ldc, M, N, K, d_bias, d_mask, ldm, flags, d_err,
                          mtt::as_stream(stream), d_ws, d_ws ? (size_t)ws_floats : 0);
}
