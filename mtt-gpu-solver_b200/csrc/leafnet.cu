// leafnet.cu — the leaf network for depth-limited solving: an MLP that maps a
// river subgame (two 1,326-combo ranges, 52-card board one-hot, pot, stack;
// 2,706 features) through three ReLU layers of 1,024 to the two players'
// 1,326 counterfactual values (2,652 outputs, in units of the pot).
//
// Weights are kept in FP32 (Adam state alongside) and mirrored in BF16, both
// as W [out][in] and as W^T [in][out], so that every product of the forward
// and backward passes is one C = A * B^T call of the tcgen05 GEMM:
//   forward   H_l = relu(H_{l-1} W_l^T + b_l)              A = H_{l-1}, B = W_l
//   backward  dH_{l-1} = (dH_l W_l) * [H_{l-1} > 0]         A = dH_l,    B = W_l^T
//             dW_l = dH_l^T H_{l-1}                         A = dH_l^T,  B = H_{l-1}^T
// The transposes of the activations are written by a tiled transpose
// kernel; bias gradients are column sums; the loss is the masked mean
// squared error.  Feature width is padded to 2,752 and the output width to
// 2,688 (multiples of 64 and 128) with zeros.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "mtt_common.h"
#include "mtt_device.cuh"

namespace mtt {
int gemm_bf16(const void* A, int lda, const void* B, int ldb, void* C, int ldc, int M, int N, int K,
              const float* bias, const void* mask, int ldm, int flags, int* d_err, cudaStream_t st, float* ws,
              size_t ws_floats);

namespace leaf {

constexpr int IN = MTT_LEAF_IN, HID = MTT_LEAF_HIDDEN, OUT = MTT_LEAF_OUT;
constexpr int INP = 2752, OUTP = 2688;       // padded widths
constexpr int NL = 4;
constexpr int DIN[NL] = {INP, HID, HID, HID};
constexpr int DOUT[NL] = {HID, HID, HID, OUTP};
enum { F_RELU = 1, F_OUT_BF16 = 2, F_MASK = 4 };

typedef __nv_bfloat16 bf16;

__global__ void k_pack_features(const float* __restrict__ x, int M, bf16* __restrict__ X0) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)M * INP) return;
    const int r = (int)(i / INP), c = (int)(i % INP);
    X0[i] = __float2bfloat16_rn(c < IN ? x[(size_t)r * IN + c] : 0.0f);
}

// out[c][r] = in[r][c] for a rows x cols bf16 matrix (row strides ldi, ldo).
__global__ void k_transpose(const bf16* __restrict__ in, int rows, int cols, int ldi, bf16* __restrict__ out, int ldo) {
    __shared__ bf16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        t[k][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * ldi + c] : __float2bfloat16_rn(0.0f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[(size_t)c * ldo + r] = t[threadIdx.x][k];
    }
}

// Masked MSE: loss partials per block (summed on the host in FP64) and
// dY = 2 w (Y - T) / n_valid as bf16, zero in the padding columns.
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ W, int M,
                      float inv_n, bf16* __restrict__ dY, double* __restrict__ partial) {
    __shared__ double s[256];
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)M * OUTP;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / OUTP), c = (int)(i % OUTP);
        float g = 0.0f;
        if (c < OUT) {
            const size_t o = (size_t)r * OUT + c;
            const float w = W ? W[o] : 1.0f;
            const float d = Y[i] - T[o];
            acc += (double)w * (double)d * (double)d;
            g = 2.0f * w * d * inv_n;
        }
        dY[i] = __float2bfloat16_rn(g);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// db[c] = sum over rows of dY[r][c], in a fixed order: a CTA of 32 x 32
// threads takes 32 columns; thread (x, y) sums rows y, y + 32, ... of column
// x (each warp reads 64 consecutive bytes of a row), then the 32 partial sums
// of a column are added in slice order.
constexpr int CS_COLS = 32, CS_SLICES = 32;
__global__ void __launch_bounds__(CS_COLS * CS_SLICES) k_colsum(const bf16* __restrict__ dY, int M, int N, int ld,
                                                               float* __restrict__ db) {
    __shared__ float part[CS_SLICES][CS_COLS + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int c = blockIdx.x * CS_COLS + tx;
    float acc = 0.0f;
    if (c < N) {
#pragma unroll 8
        for (int r = ty; r < M; r += CS_SLICES) acc += __bfloat162float(dY[(size_t)r * ld + c]);
    }
    part[ty][tx] = acc;
    __syncthreads();
    if (ty == 0 && c < N) {
        float t = 0.0f;
#pragma unroll
        for (int k = 0; k < CS_SLICES; ++k) t += part[k][tx];
        db[c] = t;
    }
}

// Adam on FP32 masters; refreshes the BF16 copy W [rows][cols] (and, in a
// second kernel, W^T).  Padding rows/columns stay zero.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       bf16* __restrict__ wb, const unsigned char* __restrict__ live) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (live && !live[i]) { wb[i] = __float2bfloat16_rn(0.0f); return; }
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_adam_bias(float* __restrict__ b, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int n, int n_live, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i >= n_live) { b[i] = 0.0f; return; }
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    b[i] = b[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct Layer {
    float *w = nullptr, *b = nullptr, *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr;
    float *gw = nullptr, *gb = nullptr;
    bf16 *wb = nullptr, *wt = nullptr;       // W [out][in] and W^T [in][out]
    unsigned char* live = nullptr;           // 1 where (out, in) is inside the unpadded shape
    int in = 0, out = 0, in_live = 0, out_live = 0;
};

}  // namespace leaf
}  // namespace mtt

using namespace mtt;
using namespace mtt::leaf;

struct mtt_leafnet {
    Layer L[NL];
    int cap = 0;
    bf16 *X0 = nullptr, *H[3] = {nullptr, nullptr, nullptr}, *dY = nullptr, *dH[3] = {nullptr, nullptr, nullptr};
    bf16 *T1 = nullptr, *T2 = nullptr;       // transposes: gradient (A operand) and activation (B operand)
    float* Y = nullptr;
    double* partial = nullptr;
    int* err = nullptr;
    float* ws = nullptr;                     // split-K partial tiles of the GEMMs with few output tiles
    long long step = 0;
};

namespace {
constexpr int MSE_BLOCKS = 592;
constexpr size_t WS_FLOATS = 8u << 20;      // 32 MB: four 1,024 x 1,024 splits, or ten of 240 x 2,688

template <typename T>
int dmalloc(T** p, size_t n) {
    return cuda_status(cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)));
}

void free_net(mtt_leafnet* n) {
    if (!n) return;
    for (Layer& l : n->L) {
        cudaFree(l.w); cudaFree(l.b); cudaFree(l.mw); cudaFree(l.vw); cudaFree(l.mb); cudaFree(l.vb);
        cudaFree(l.gw); cudaFree(l.gb); cudaFree(l.wb); cudaFree(l.wt); cudaFree(l.live);
    }
    cudaFree(n->X0); cudaFree(n->dY); cudaFree(n->T1); cudaFree(n->T2); cudaFree(n->Y); cudaFree(n->partial);
    cudaFree(n->err); cudaFree(n->ws);
    for (int k = 0; k < 3; ++k) { cudaFree(n->H[k]); cudaFree(n->dH[k]); }
    delete n;
}

int transpose(const bf16* in, int rows, int cols, int ldi, bf16* out, int ldo, cudaStream_t st) {
    const dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
    k_transpose<<<grid, dim3(32, 8), 0, st>>>(in, rows, cols, ldi, out, ldo);
    MTT_CHECK_LAUNCH();
    return MTT_OK;
}

// BF16 mirrors (W and W^T) of layer l from its FP32 master.
int refresh_bf16(mtt_leafnet* n, int l, cudaStream_t st);

__global__ void k_to_bf16(const float* __restrict__ w, long long n, bf16* __restrict__ o) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = __float2bfloat16_rn(w[i]);
}

int refresh_bf16(mtt_leafnet* n, int l, cudaStream_t st) {
    Layer& L = n->L[l];
    const long long cnt = (long long)L.out * L.in;
    k_to_bf16<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(L.w, cnt, L.wb);
    MTT_CHECK_LAUNCH();
    return transpose(L.wb, L.out, L.in, L.in, L.wt, L.out, st);
}

int forward(mtt_leafnet* n, const float* d_x, int M, cudaStream_t st) {
    if (M < 1 || M > n->cap) return MTT_ERR_INVALID;
    const long long cnt = (long long)M * INP;
    k_pack_features<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(d_x, M, n->X0);
    MTT_CHECK_LAUNCH();
    const bf16* in = n->X0;
    for (int l = 0; l < 3; ++l) {
        MTT_TRY(gemm_bf16(in, DIN[l], n->L[l].wb, DIN[l], n->H[l], HID, M, HID, DIN[l], n->L[l].b, nullptr, 0,
                          F_RELU | F_OUT_BF16, n->err, st, n->ws, WS_FLOATS));
        in = n->H[l];
    }
    return gemm_bf16(in, HID, n->L[3].wb, HID, n->Y, OUTP, M, OUTP, HID, n->L[3].b, nullptr, 0, 0, n->err, st, n->ws,
                     WS_FLOATS);
}

// Gradients of the masked MSE into L[l].gw / gb; *h_loss = the loss.
int backward(mtt_leafnet* n, const float* d_y, const float* d_w, int M, double n_valid, double* h_loss,
             cudaStream_t st) {
    k_mse<<<MSE_BLOCKS, 256, 0, st>>>(n->Y, d_y, d_w, M, (float)(1.0 / n_valid), n->dY, n->partial);
    MTT_CHECK_LAUNCH();
    const bf16* acts[4] = {n->X0, n->H[0], n->H[1], n->H[2]};   // input of layer l
    const bf16* g = n->dY;                                       // gradient at the output of layer l
    int gw = OUTP;
    for (int l = NL - 1; l >= 0; --l) {
        Layer& L = n->L[l];
        // dW = g^T * act: A = g^T [out][M], B = act^T [in][M]
        MTT_TRY(transpose(g, M, gw, gw, n->T1, M, st));
        MTT_TRY(transpose(acts[l], M, DIN[l], DIN[l], n->T2, M, st));
        MTT_TRY(gemm_bf16(n->T1, M, n->T2, M, L.gw, L.in, L.out, L.in, M, nullptr, nullptr, 0, 0, n->err, st, n->ws,
                          WS_FLOATS));
        k_colsum<<<(unsigned)((L.out + CS_COLS - 1) / CS_COLS), dim3(CS_COLS, CS_SLICES), 0, st>>>(g, M, L.out, gw, L.gb);
        MTT_CHECK_LAUNCH();
        if (l == 0) break;
        // dH_{l-1} = (g * W) masked by H_{l-1} > 0: A = g [M][out], B = W^T [in][out]
        bf16* dh = n->dH[l - 1];
        MTT_TRY(gemm_bf16(g, gw, L.wt, L.out, dh, HID, M, HID, L.out, nullptr, acts[l], HID, F_MASK | F_OUT_BF16,
                          n->err, st, n->ws, WS_FLOATS));
        g = dh;
        gw = HID;
    }
    if (h_loss) {
        std::vector<double> part(MSE_BLOCKS);
        MTT_TRY_CUDA(cudaMemcpyAsync(part.data(), n->partial, sizeof(double) * MSE_BLOCKS, cudaMemcpyDeviceToHost, st));
        MTT_TRY_CUDA(cudaStreamSynchronize(st));
        double s = 0.0;
        for (double v : part) s += v;
        *h_loss = s / n_valid;
    }
    return MTT_OK;
}
}  // namespace

extern "C" int mtt_leafnet_create(int32_t batch_cap, uint64_t seed, int32_t flags, mtt_leafnet** out) {
    if (!out || batch_cap < 1 || batch_cap > (1 << 20) || (batch_cap % 8)) return MTT_ERR_INVALID;
    *out = nullptr;
    mtt_leafnet* n = new mtt_leafnet();
    n->cap = batch_cap;
    int s = MTT_OK;
    const int in_live[NL] = {IN, HID, HID, HID}, out_live[NL] = {HID, HID, HID, OUT};
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    auto urand = [&]() {   // splitmix64 -> uniform (0, 1)
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return ((double)(z >> 11) + 0.5) / 9007199254740992.0;
    };
    for (int l = 0; l < NL && !s; ++l) {
        Layer& L = n->L[l];
        L.in = DIN[l]; L.out = DOUT[l]; L.in_live = in_live[l]; L.out_live = out_live[l];
        const size_t cnt = (size_t)L.in * L.out;
        std::vector<float> w(cnt, 0.0f);
        std::vector<unsigned char> live(cnt, 0);
        // He initialisation; the output layer starts at zero when asked
        const double sd = (l == NL - 1 && (flags & MTT_LEAF_ZERO_OUTPUT)) ? 0.0 : std::sqrt(2.0 / (double)L.in_live);
        for (int o = 0; o < L.out_live; ++o)
            for (int i = 0; i < L.in_live; ++i) {
                const double u1 = urand(), u2 = urand();
                w[(size_t)o * L.in + i] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
                live[(size_t)o * L.in + i] = 1;
            }
        if (!s) s = dmalloc(&L.w, cnt);
        if (!s) s = dmalloc(&L.mw, cnt);
        if (!s) s = dmalloc(&L.vw, cnt);
        if (!s) s = dmalloc(&L.gw, cnt);
        if (!s) s = dmalloc(&L.wb, cnt);
        if (!s) s = dmalloc(&L.wt, cnt);
        if (!s) s = dmalloc(&L.live, cnt);
        if (!s) s = dmalloc(&L.b, L.out);
        if (!s) s = dmalloc(&L.mb, L.out);
        if (!s) s = dmalloc(&L.vb, L.out);
        if (!s) s = dmalloc(&L.gb, L.out);
        if (!s) s = cuda_status(cudaMemcpy(L.w, w.data(), 4 * cnt, cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemcpy(L.live, live.data(), cnt, cudaMemcpyHostToDevice));
        if (!s) s = cuda_status(cudaMemset(L.mw, 0, 4 * cnt));
        if (!s) s = cuda_status(cudaMemset(L.vw, 0, 4 * cnt));
        if (!s) s = cuda_status(cudaMemset(L.b, 0, 4 * (size_t)L.out));
        if (!s) s = cuda_status(cudaMemset(L.mb, 0, 4 * (size_t)L.out));
        if (!s) s = cuda_status(cudaMemset(L.vb, 0, 4 * (size_t)L.out));
    }
    const size_t M = (size_t)batch_cap;
    if (!s) s = dmalloc(&n->X0, M * INP);
    for (int k = 0; k < 3 && !s; ++k) {
        s = dmalloc(&n->H[k], M * HID);
        if (!s) s = dmalloc(&n->dH[k], M * HID);
    }
    if (!s) s = dmalloc(&n->dY, M * OUTP);
    if (!s) s = dmalloc(&n->T1, M * OUTP);
    if (!s) s = dmalloc(&n->T2, M * INP);
    if (!s) s = dmalloc(&n->Y, M * OUTP);
    if (!s) s = dmalloc(&n->partial, MSE_BLOCKS);
    if (!s) s = dmalloc(&n->err, 1);
    if (!s) s = dmalloc(&n->ws, WS_FLOATS);
    if (!s) s = cuda_status(cudaMemset(n->err, 0, sizeof(int)));
    for (int l = 0; l < NL && !s; ++l) s = refresh_bf16(n, l, nullptr);
    if (!s) s = cuda_status(cudaDeviceSynchronize());
    if (s) { free_net(n); return s; }
    *out = n;
    return MTT_OK;
}

extern "C" int mtt_leafnet_forward(mtt_leafnet* n, const float* d_x, int32_t M, float* d_y, void* stream) {
    if (!n || !d_x || !d_y) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    MTT_TRY(forward(n, d_x, M, st));
    MTT_TRY_CUDA(cudaMemcpy2DAsync(d_y, sizeof(float) * OUT, n->Y, sizeof(float) * OUTP, sizeof(float) * OUT, M,
                                   cudaMemcpyDeviceToDevice, st));
    return MTT_OK;
}

extern "C" int mtt_leafnet_capacity(mtt_leafnet* n, int32_t* cap) {
    if (!n || !cap) return MTT_ERR_INVALID;
    *cap = n->cap;
    return MTT_OK;
}

extern "C" int mtt_leafnet_gradients(mtt_leafnet* n, const float* d_x, const float* d_y, const float* d_w, int32_t M,
                                     double* h_loss, void* stream) {
    if (!n || !d_x || !d_y || (M % 8)) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    MTT_TRY(forward(n, d_x, M, st));
    return backward(n, d_y, d_w, M, (double)M * OUT, h_loss, st);
}

extern "C" int mtt_leafnet_train_step(mtt_leafnet* n, const float* d_x, const float* d_y, const float* d_w, int32_t M,
                                      float lr, double* h_loss, void* stream) {
    if (!n || !d_x || !d_y || (M % 8) || !(lr > 0.0f)) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    MTT_TRY(forward(n, d_x, M, st));
    MTT_TRY(backward(n, d_y, d_w, M, (double)M * OUT, h_loss, st));
    n->step += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = (float)(1.0 - std::pow(0.9, (double)n->step)), c2 = (float)(1.0 - std::pow(0.999, (double)n->step));
    for (int l = 0; l < NL; ++l) {
        Layer& L = n->L[l];
        const long long cnt = (long long)L.in * L.out;
        k_adam<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(L.w, L.mw, L.vw, L.gw, cnt, lr, b1, b2, eps, c1, c2, L.wb,
                                                             L.live);
        MTT_CHECK_LAUNCH();
        k_adam_bias<<<(unsigned)((L.out + 255) / 256), 256, 0, st>>>(L.b, L.mb, L.vb, L.gb, L.out, L.out_live, lr, b1,
                                                                     b2, eps, c1, c2);
        MTT_CHECK_LAUNCH();
        MTT_TRY(transpose(L.wb, L.out, L.in, L.in, L.wt, L.out, st));
    }
    return MTT_OK;
}

// Parameters of layer l: w [out][in] (padded shape), b [out]; either may be NULL.
extern "C" int mtt_leafnet_params(mtt_leafnet* n, int32_t layer, float* h_w, float* h_b, float* h_gw, float* h_gb,
                                  int32_t* shape) {
    if (!n || layer < 0 || layer >= NL) return MTT_ERR_INVALID;
    const Layer& L = n->L[layer];
    MTT_TRY_CUDA(cudaDeviceSynchronize());
    if (shape) { shape[0] = L.out; shape[1] = L.in; }
    const size_t cnt = (size_t)L.in * L.out;
    if (h_w) MTT_TRY_CUDA(cudaMemcpy(h_w, L.w, 4 * cnt, cudaMemcpyDeviceToHost));
    if (h_b) MTT_TRY_CUDA(cudaMemcpy(h_b, L.b, 4 * (size_t)L.out, cudaMemcpyDeviceToHost));
    if (h_gw) MTT_TRY_CUDA(cudaMemcpy(h_gw, L.gw, 4 * cnt, cudaMemcpyDeviceToHost));
    if (h_gb) MTT_TRY_CUDA(cudaMemcpy(h_gb, L.gb, 4 * (size_t)L.out, cudaMemcpyDeviceToHost));
    return MTT_OK;
}

extern "C" int mtt_leafnet_check(mtt_leafnet* n) {
    if (!n) return MTT_ERR_INVALID;
    int e = 0;
    MTT_TRY_CUDA(cudaMemcpy(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost));
    return e ? MTT_ERR_TIMEOUT : MTT_OK;
}

extern "C" int mtt_leafnet_destroy(mtt_leafnet* n) {
    if (!n) return MTT_ERR_INVALID;
    cudaDeviceSynchronize();
    free_net(n);
    return MTT_OK;
}

// ------------------------------------------------------------ check-down leaves
// The leaf estimate without a network: both players check the river down.
// Value of combo h of player p in units of the pot, with both players having
// put in half of it: 0.5 * sum over the opponent's combos j that share no
// card with h or the board of r_opp(j) * sign(score(h) - score(j)).  One CTA
// per subgame; every opponent combo is read by all lanes at once (broadcast
// from shared memory), and each hand sums its opponents in the same order, so
// the result is deterministic.
namespace mtt {
namespace leaf {
constexpr int NCOMBO = 1326;

__global__ void __launch_bounds__(256) k_checkdown(const uint8_t* __restrict__ boards, const float* __restrict__ r0,
                                                   const float* __restrict__ r1, int n, float* __restrict__ out) {
    __shared__ uint16_t key[NCOMBO];
    __shared__ unsigned long long msk[NCOMBO];
    __shared__ float ro[NCOMBO];
    const int b = blockIdx.x;
    if (b >= n) return;
    const uint8_t* bd = boards + 5 * (size_t)b;
    uint64_t bm = 0;
    for (int k = 0; k < 5; ++k) bm |= 1ull << bd[k];
    for (int h = threadIdx.x; h < NCOMBO; h += blockDim.x) {
        int c1 = 0, r = h, row = 51;
        while (r >= row) { r -= row; ++c1; --row; }
        const int c2 = c1 + 1 + r;
        const uint64_t m = (1ull << c1) | (1ull << c2);
        msk[h] = m;
        uint16_t k = 0xFFFFu;                     // combos touching the board take no part
        if (!(m & bm)) {
            Planes p; planes_clear(p);
            for (int i = 0; i < 5; ++i) planes_add(p, bd[i]);
            planes_add(p, c1); planes_add(p, c2);
            k = (uint16_t)key_planes(p);
        }
        key[h] = k;
    }
    for (int dir = 0; dir < 2; ++dir) {
        __syncthreads();
        const float* rg = (dir == 0 ? r1 : r0) + (size_t)b * NCOMBO;   // the opponent's range
        for (int j = threadIdx.x; j < NCOMBO; j += blockDim.x) ro[j] = key[j] == 0xFFFFu ? 0.0f : rg[j];
        __syncthreads();
        float* o = out + ((size_t)b * 2 + dir) * NCOMBO;
        for (int h = threadIdx.x; h < NCOMBO; h += blockDim.x) {
            const uint16_t kh = key[h];
            float acc = 0.0f;
            if (kh != 0xFFFFu) {
                const uint64_t mh = msk[h];
                for (int j = 0; j < NCOMBO; ++j) {
                    const uint16_t kj = key[j];
                    const float w = (msk[j] & mh) ? 0.0f : ro[j];
                    acc += kh > kj ? w : (kh < kj ? -w : 0.0f);
                }
            }
            o[h] = 0.5f * acc;
        }
    }
}
}  // namespace leaf
}  // namespace mtt

extern "C" int mtt_checkdown_values(const uint8_t* d_boards, const float* d_range0, const float* d_range1, int32_t n,
                                    float* d_out, void* stream) {
    if (n < 0 || (n > 0 && (!d_boards || !d_range0 || !d_range1 || !d_out))) return MTT_ERR_INVALID;
    if (n == 0) return MTT_OK;
    mtt::leaf::k_checkdown<<<n, 256, 0, as_stream(stream)>>>(d_boards, d_range0, d_range1, n, d_out);
    MTT_CHECK_LAUNCH();
    return MTT_OK;
}
