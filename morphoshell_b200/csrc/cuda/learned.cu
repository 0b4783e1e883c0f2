// Coordinate network for the learned warm start (ms_mlp_* in
// include/morphoshell_gpu.h): a SiLU MLP trained and evaluated on the GPU
// with the tcgen05 BF16 GEMM of tc_gemm.cuh (FP32 accumulation), FP32
// master weights and Adam.
//
// Layer l maps K_l inputs to N_l outputs: Z_l = H_{l-1} W_l^T + b_l,
// H_l = SiLU(Z_l) on hidden layers, the last layer linear.  Widths are
// padded: inputs to a multiple of 16, the output to 16.  Backward for a
// batch of B rows (padded to a multiple of 128, padding rows carry zero
// gradient):
//   dY     = 2 (Y - T) / (rows * out)               (mean squared error)
//   dW_l   = dZ_l^T H_{l-1}                          GEMM, K = B, split-K
//   db_l   = column sums of dZ_l
//   dZ_l-1 = (dZ_l W_l) * SiLU'(Z_l-1)               GEMM with fused epilogue
// The transposed operands (dZ^T, H^T, W^T) are materialised by a transpose
// kernel so that every GEMM is A[M x K] * B[N x K]^T with K contiguous.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../../include/morphoshell_gpu.h"
#include "tc_gemm.cuh"

using namespace msb;

namespace {

constexpr int kMaxLayers = 8;

__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, int rows,
                                 int cols, int ld_in, int ld_out) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        tile[i][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * ld_in + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[(size_t)c * ld_out + r] = tile[threadIdx.x][i];
    }
}

// Rows idx[row0 .. row0+B) of the data set into a padded bf16 batch; rows
// past n_rows are zero.
__global__ void k_gather(const float* __restrict__ X, const float* __restrict__ T, const long long* __restrict__ idx,
                         long long row0, long long n_rows, int in_dim, int in_pad, int out_dim, int B,
                         __nv_bfloat16* __restrict__ Xb, float* __restrict__ Tb) {
    const int r = blockIdx.x;
    const long long src_row = row0 + r;
    const bool valid = src_row < n_rows;
    const long long s = valid ? (idx ? idx[src_row] : src_row) : 0;
    for (int c = threadIdx.x; c < in_pad; c += blockDim.x)
        Xb[(size_t)r * in_pad + c] = __float2bfloat16(valid && c < in_dim ? X[s * in_dim + c] : 0.0f);
    if (T)
        for (int c = threadIdx.x; c < out_dim; c += blockDim.x) Tb[(size_t)r * out_dim + c] = valid ? T[s * out_dim + c] : 0.0f;
}

// dY (bf16, [B][out_pad]) and per-block partial sums of the squared error.
__global__ void k_loss_grad(const float* __restrict__ Y, const float* __restrict__ T, int B, int valid_rows, int out_dim,
                            int out_pad, double scale, __nv_bfloat16* __restrict__ dY, double* __restrict__ part) {
    __shared__ double red[256];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B * out_pad; i += gridDim.x * blockDim.x) {
        const int r = i / out_pad, c = i % out_pad;
        float g = 0.0f;
        if (r < valid_rows && c < out_dim) {
            const float d = Y[(size_t)r * out_pad + c] - T[(size_t)r * out_dim + c];
            acc += (double)d * (double)d;
            g = (float)(2.0 * scale * d);
        }
        dY[i] = __float2bfloat16(g);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Sum of the split-K partials [S][Mp][ldp] into out[M][N] (+= when accumulate).
__global__ void k_splitk_sum(const float* __restrict__ part, int S, int Mp, int ldp, int M, int N,
                             float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M * N) return;
    const int m = i / N, n = i % N;
    float s = 0.0f;
    for (int k = 0; k < S; ++k) s += part[((size_t)k * Mp + m) * ldp + n];
    out[i] = s;
}

// Column sums of a bf16 [B][N] matrix (bias gradients) in two fixed-order
// passes: block (x, y) sums columns 32x .. 32x+31 over rows
// [y R, (y+1) R) into part[y][c] (8 row lanes, then the lanes in order),
// then one thread per column adds the partials in order.
constexpr int kColChunks = 64;

__global__ void k_colsum_part(const __nv_bfloat16* __restrict__ D, int B, int N, float* __restrict__ part) {
    __shared__ float acc[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    const int R = (B + kColChunks - 1) / kColChunks;
    const int r0 = blockIdx.y * R, r1 = min(B, r0 + R);
    float s = 0.0f;
    if (c < N)
        for (int r = r0 + threadIdx.y; r < r1; r += 8) s += __bfloat162float(D[(size_t)r * N + c]);
    acc[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < N) {
        float t = acc[0][threadIdx.x];
        for (int k = 1; k < 8; ++k) t += acc[k][threadIdx.x];
        part[(size_t)blockIdx.y * N + c] = t;
    }
}

__global__ void k_colsum_final(const float* __restrict__ part, int N, int n_valid, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_valid) return;
    float s = 0.0f;
    for (int k = 0; k < kColChunks; ++k) s += part[(size_t)k * N + c];
    out[c] = s;
}

// acc[0] += sum of the loss partials (one thread, fixed order).
__global__ void k_loss_accumulate(const double* __restrict__ part, int n, double* __restrict__ acc) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += part[i];
    acc[0] += s;
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// FP32 master weights [N][K] -> bf16 [Np][K] (rows past N zero) and its
// transpose [K][Np].
__global__ void k_weights_bf16(const float* __restrict__ W, int N, int K, int Np, __nv_bfloat16* __restrict__ Wb,
                               __nv_bfloat16* __restrict__ Wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Np * K) return;
    const int n = i / K, k = i % K;
    const __nv_bfloat16 v = __float2bfloat16(n < N ? W[(size_t)n * K + k] : 0.0f);
    Wb[i] = v;
    Wt[(size_t)k * Np + n] = v;
}

struct Layer {
    int K, N, Np;            // inputs, outputs, outputs padded (16 for the last layer)
    size_t w_off, b_off;     // offsets into the flat parameter vector
    __nv_bfloat16 *Wb, *Wt;  // [Np][K], [K][Np]
};

}  // namespace

struct ms_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    int in_dim = 0, in_pad = 0, out_dim = 0, width = 0, nl = 0;
    Layer L[kMaxLayers];
    size_t n_params = 0;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    long long adam_t = 0;
    // batch work space (rows = cap)
    int cap = 0;
    __nv_bfloat16 *Xb = nullptr, *XbT = nullptr;
    __nv_bfloat16 *Z[kMaxLayers] = {}, *H[kMaxLayers] = {}, *HT[kMaxLayers] = {};
    __nv_bfloat16 *dZ = nullptr, *dZ2 = nullptr, *dZT = nullptr;
    float *Y = nullptr, *Tb = nullptr, *part = nullptr;
    double* loss_part = nullptr;
    double* loss_acc = nullptr;   // [1] running sum over an epoch
    float* colpart = nullptr;     // [kColChunks][width] bias-gradient partials
    size_t part_cap = 0;
    int* err = nullptr;
    // data set
    float *dX = nullptr, *dT = nullptr;
    long long n_rows = 0;
    long long* d_idx = nullptr;
    std::vector<void*> allocs;
    std::string last_error;
};

namespace {

ms_status mfail(ms_mlp* h, ms_status st, const std::string& msg) {
    if (h) h->last_error = msg;
    return st;
}

#define ML_CUDA(h, call)                                                                                  \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            return mfail(h, e_ == cudaErrorMemoryAllocation ? MS_ERR_OUT_OF_MEMORY : MS_ERR_CUDA,         \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                             \
    } while (0)

#define ML_TRY(expr)                  \
    do {                              \
        ms_status st_ = (expr);       \
        if (st_ != MS_OK) return st_; \
    } while (0)

template <typename T>
ms_status malloc_dev(ms_mlp* h, T** p, size_t count) {
    void* q = nullptr;
    ML_CUDA(h, cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    h->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return MS_OK;
}

template <int BN, int EPI>
cudaError_t launch_gemm(const tc::GemmArgs& a, int splits, cudaStream_t st) {
    static bool attr_set = false;
    constexpr int smem = tc::gemm_smem_bytes<BN>();
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(tc::k_gemm<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    dim3 grid(a.M / tc::kBM, a.N / BN, splits);
    tc::k_gemm<BN, EPI><<<grid, tc::kThreads, smem, st>>>(a);
    return cudaGetLastError();
}

// C = A B^T with the widest tile that divides N.
cudaError_t gemm(const tc::GemmArgs& a, int epi, int splits, cudaStream_t st) {
    if (a.N % 128 == 0) {
        if (epi == tc::EPI_F32) return launch_gemm<128, tc::EPI_F32>(a, splits, st);
        if (epi == tc::EPI_BIAS_SILU) return launch_gemm<128, tc::EPI_BIAS_SILU>(a, splits, st);
        return launch_gemm<128, tc::EPI_DSILU>(a, splits, st);
    }
    if (a.N % 32 == 0) {
        if (epi == tc::EPI_F32) return launch_gemm<32, tc::EPI_F32>(a, splits, st);
        if (epi == tc::EPI_BIAS_SILU) return launch_gemm<32, tc::EPI_BIAS_SILU>(a, splits, st);
        return launch_gemm<32, tc::EPI_DSILU>(a, splits, st);
    }
    if (a.N % 16 == 0) {
        if (epi == tc::EPI_F32) return launch_gemm<16, tc::EPI_F32>(a, splits, st);
        if (epi == tc::EPI_BIAS_SILU) return launch_gemm<16, tc::EPI_BIAS_SILU>(a, splits, st);
        return launch_gemm<16, tc::EPI_DSILU>(a, splits, st);
    }
    return cudaErrorInvalidValue;
}

ms_status ensure_batch(ms_mlp* h, int rows) {
    if (rows <= h->cap) return MS_OK;
    const int B = rows;
    ML_TRY(malloc_dev(h, &h->Xb, (size_t)B * h->in_pad));
    ML_TRY(malloc_dev(h, &h->XbT, (size_t)h->in_pad * B));
    for (int l = 0; l < h->nl; ++l) {
        const int Np = h->L[l].Np;
        ML_TRY(malloc_dev(h, &h->Z[l], (size_t)B * Np));
        ML_TRY(malloc_dev(h, &h->H[l], (size_t)B * Np));
        ML_TRY(malloc_dev(h, &h->HT[l], (size_t)Np * B));
    }
    ML_TRY(malloc_dev(h, &h->dZ, (size_t)B * h->width));
    ML_TRY(malloc_dev(h, &h->dZ2, (size_t)B * h->width));
    ML_TRY(malloc_dev(h, &h->dZT, (size_t)std::max(h->width, 128) * B));
    ML_CUDA(h, cudaMemset(h->dZT, 0, sizeof(__nv_bfloat16) * (size_t)std::max(h->width, 128) * B));
    ML_TRY(malloc_dev(h, &h->Y, (size_t)B * 16));
    ML_TRY(malloc_dev(h, &h->Tb, (size_t)B * h->out_dim));
    ML_TRY(malloc_dev(h, &h->loss_part, 1024));
    ML_TRY(malloc_dev(h, &h->loss_acc, 1));
    ML_TRY(malloc_dev(h, &h->colpart, (size_t)kColChunks * std::max(h->width, 16)));
    h->cap = rows;
    return MS_OK;
}

ms_status ensure_part(ms_mlp* h, size_t count) {
    if (count <= h->part_cap) return MS_OK;
    ML_TRY(malloc_dev(h, &h->part, count));
    h->part_cap = count;
    return MS_OK;
}

ms_status refresh_bf16(ms_mlp* h) {
    for (int l = 0; l < h->nl; ++l) {
        const Layer& y = h->L[l];
        const int n = y.Np * y.K;
        k_weights_bf16<<<(n + 255) / 256, 256, 0, h->stream>>>(h->p + y.w_off, y.N, y.K, y.Np, y.Wb, y.Wt);
    }
    ML_CUDA(h, cudaGetLastError());
    return MS_OK;
}

// Forward pass over the rows already in h->Xb (B rows, a multiple of 128).
ms_status forward(ms_mlp* h, int B) {
    const __nv_bfloat16* in = h->Xb;
    int K = h->in_pad;
    for (int l = 0; l < h->nl; ++l) {
        const Layer& y = h->L[l];
        tc::GemmArgs a{};
        a.A = in;
        a.B = y.Wb;
        a.M = B;
        a.N = y.Np;
        a.K = K;
        a.lda = K;
        a.ldb = K;
        a.k_split = K;
        a.bias = h->p + y.b_off;
        a.ldc = y.Np;
        a.err = h->err;
        const bool last = l == h->nl - 1;
        if (last) {
            a.Cf = h->Y;
            // bias of the padded output columns: the vector has Np entries
            ML_CUDA(h, gemm(a, tc::EPI_F32, 1, h->stream));
        } else {
            a.Z = h->Z[l];
            a.H = h->H[l];
            ML_CUDA(h, gemm(a, tc::EPI_BIAS_SILU, 1, h->stream));
        }
        in = h->H[l];
        K = y.Np;
    }
    return MS_OK;
}

void transpose(const __nv_bfloat16* in, __nv_bfloat16* out, int rows, int cols, int ld_in, int ld_out,
               cudaStream_t st) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    k_transpose_bf16<<<grid, dim3(32, 8), 0, st>>>(in, out, rows, cols, ld_in, ld_out);
}

// Backward pass after forward() and the loss gradient in h->dZ (as
// [B][16]); gradients into h->g.
ms_status backward(ms_mlp* h, int B) {
    // Split K = B into chunks of 512 rows.
    const int chunk = 512;
    const int S = (B + chunk - 1) / chunk;
    __nv_bfloat16* dZcur = h->dZ;  // [B][Np_l]
    __nv_bfloat16* dZnext = h->dZ2;
    for (int l = h->nl - 1; l >= 0; --l) {
        const Layer& y = h->L[l];
        const __nv_bfloat16* Hin = l > 0 ? h->H[l - 1] : h->Xb;
        const int Kin = y.K;
        // dW_l = dZ_l^T H_{l-1}
        const int Mp = std::max(y.Np, 128);
        transpose(dZcur, h->dZT, B, y.Np, y.Np, B, h->stream);
        __nv_bfloat16* HinT = l > 0 ? h->HT[l - 1] : h->XbT;
        transpose(Hin, HinT, B, Kin, Kin, B, h->stream);
        ML_TRY(ensure_part(h, (size_t)S * Mp * Kin));
        tc::GemmArgs a{};
        a.A = h->dZT;
        a.B = HinT;
        a.M = Mp;
        a.N = Kin;
        a.K = B;
        a.lda = B;
        a.ldb = B;
        a.k_split = chunk;
        a.Cf = h->part;
        a.ldc = Kin;
        a.err = h->err;
        ML_CUDA(h, gemm(a, tc::EPI_F32, S, h->stream));
        const int nw = y.N * Kin;
        k_splitk_sum<<<(nw + 255) / 256, 256, 0, h->stream>>>(h->part, S, Mp, Kin, y.N, Kin, h->g + y.w_off);
        k_colsum_part<<<dim3((y.Np + 31) / 32, kColChunks), dim3(32, 8), 0, h->stream>>>(dZcur, B, y.Np,
                                                                                         h->colpart);
        k_colsum_final<<<(y.N + 127) / 128, 128, 0, h->stream>>>(h->colpart, y.Np, y.N, h->g + y.b_off);
        ML_CUDA(h, cudaGetLastError());
        if (l == 0) break;
        // dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1})
        tc::GemmArgs b{};
        b.A = dZcur;
        b.B = y.Wt;
        b.M = B;
        b.N = Kin;
        b.K = y.Np;
        b.lda = y.Np;
        b.ldb = y.Np;
        b.k_split = y.Np;
        b.Z = h->Z[l - 1];
        b.H = dZnext;
        b.ldc = Kin;
        b.err = h->err;
        ML_CUDA(h, gemm(b, tc::EPI_DSILU, 1, h->stream));
        std::swap(dZcur, dZnext);
    }
    return MS_OK;
}

// Loss and dY of the rows in h->Tb; returns the sum of squared errors via
// the partials (read after the stream synchronises).
ms_status loss_grad(ms_mlp* h, int B, int valid) {
    const double scale = 1.0 / ((double)std::max(valid, 1) * h->out_dim);
    k_loss_grad<<<256, 256, 0, h->stream>>>(h->Y, h->Tb, B, valid, h->out_dim, 16, scale, h->dZ, h->loss_part);
    ML_CUDA(h, cudaGetLastError());
    return MS_OK;
}

ms_status check_err(ms_mlp* h) {
    int e = 0;
    ML_CUDA(h, cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return mfail(h, MS_ERR_TIMEOUT, "tensor-core GEMM wait timed out");
    return MS_OK;
}

int round_up(long long n, int q) { return (int)((n + q - 1) / q * q); }

}  // namespace

extern "C" {

ms_status ms_mlp_create(int32_t in_dim, int32_t width, int32_t hidden_layers, int32_t out_dim, uint64_t seed,
                        int32_t device, ms_mlp** out) {
    if (!out) return MS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (in_dim <= 0 || in_dim > 256 || out_dim <= 0 || out_dim > 16 || width <= 0 || width % 128 ||
        width > 512 || hidden_layers < 1 || hidden_layers + 1 > kMaxLayers)
        return MS_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MS_ERR_NO_DEVICE;
    if (device >= ndev) return MS_ERR_INVALID_ARGUMENT;
    if (device >= 0) cudaSetDevice(device);
    ms_mlp* h = new ms_mlp();
    cudaGetDevice(&h->device);
    auto bail = [&](ms_status st) {
        ms_mlp_destroy(h);
        return st;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(MS_ERR_CUDA);
    h->in_dim = in_dim;
    h->in_pad = (in_dim + 15) / 16 * 16;
    h->out_dim = out_dim;
    h->width = width;
    h->nl = hidden_layers + 1;
    size_t off = 0;
    for (int l = 0; l < h->nl; ++l) {
        Layer& y = h->L[l];
        y.K = l == 0 ? h->in_pad : width;
        y.N = l == h->nl - 1 ? out_dim : width;
        y.Np = l == h->nl - 1 ? 16 : width;
        y.w_off = off;
        off += (size_t)y.N * y.K;
        y.b_off = off;
        off += (size_t)y.Np;  // padded bias (entries past N stay zero)
    }
    h->n_params = off;
    ms_status st;
    if ((st = malloc_dev(h, &h->p, off)) || (st = malloc_dev(h, &h->g, off)) || (st = malloc_dev(h, &h->m1, off)) ||
        (st = malloc_dev(h, &h->m2, off)) || (st = malloc_dev(h, &h->err, 1)))
        return bail(st);
    for (int l = 0; l < h->nl; ++l) {
        Layer& y = h->L[l];
        if ((st = malloc_dev(h, &y.Wb, (size_t)y.Np * y.K)) || (st = malloc_dev(h, &y.Wt, (size_t)y.K * y.Np)))
            return bail(st);
    }
    // Initial weights: normal with variance 1 / fan_in (inputs past in_dim
    // get zero weights), zero biases.
    std::vector<float> p(off, 0.0f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < h->nl; ++l) {
        const Layer& y = h->L[l];
        const int fan_in = l == 0 ? in_dim : width;
        std::normal_distribution<float> nd(0.0f, 1.0f / std::sqrt((float)fan_in));
        for (int n = 0; n < y.N; ++n)
            for (int k = 0; k < y.K; ++k) p[y.w_off + (size_t)n * y.K + k] = (l == 0 && k >= in_dim) ? 0.0f : nd(rng);
    }
    if (cudaMemcpy(h->p, p.data(), off * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(h->g, 0, off * sizeof(float)) != cudaSuccess || cudaMemset(h->m1, 0, off * sizeof(float)) ||
        cudaMemset(h->m2, 0, off * sizeof(float)) || cudaMemset(h->err, 0, sizeof(int)))
        return bail(MS_ERR_CUDA);
    if ((st = refresh_bf16(h))) return bail(st);
    *out = h;
    return MS_OK;
}

void ms_mlp_destroy(ms_mlp* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* q : h->allocs) cudaFree(q);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

const char* ms_mlp_last_error(const ms_mlp* h) { return h ? h->last_error.c_str() : "null network"; }

ms_status ms_mlp_num_params(const ms_mlp* h, int64_t* n) {
    if (!h || !n) return MS_ERR_INVALID_ARGUMENT;
    *n = (int64_t)h->n_params;
    return MS_OK;
}

ms_status ms_mlp_get_params(ms_mlp* h, float* params) {
    if (!h || !params) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    ML_CUDA(h, cudaStreamSynchronize(h->stream));
    ML_CUDA(h, cudaMemcpy(params, h->p, h->n_params * sizeof(float), cudaMemcpyDeviceToHost));
    return MS_OK;
}

ms_status ms_mlp_set_params(ms_mlp* h, const float* params) {
    if (!h || !params) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    ML_CUDA(h, cudaStreamSynchronize(h->stream));
    ML_CUDA(h, cudaMemcpy(h->p, params, h->n_params * sizeof(float), cudaMemcpyHostToDevice));
    h->adam_t = 0;
    ML_CUDA(h, cudaMemset(h->m1, 0, h->n_params * sizeof(float)));
    ML_CUDA(h, cudaMemset(h->m2, 0, h->n_params * sizeof(float)));
    ML_TRY(refresh_bf16(h));
    return MS_OK;
}

ms_status ms_mlp_forward(ms_mlp* h, const float* x, int64_t n, float* y) {
    if (!h || !x || !y || n <= 0) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int B = round_up(std::min<int64_t>(n, 65536), 128);
    ML_TRY(ensure_batch(h, B));
    float* dx;
    ML_CUDA(h, cudaMalloc(&dx, sizeof(float) * (size_t)n * h->in_dim));
    std::vector<float> yb((size_t)B * 16);
    ms_status rc = MS_OK;
    if (cudaMemcpy(dx, x, sizeof(float) * (size_t)n * h->in_dim, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = mfail(h, MS_ERR_CUDA, "upload");
    for (long long r0 = 0; r0 < n && rc == MS_OK; r0 += B) {
        const int rows = (int)std::min<long long>(B, n - r0);
        k_gather<<<B, 64, 0, h->stream>>>(dx, nullptr, nullptr, r0, n, h->in_dim, h->in_pad, h->out_dim, B, h->Xb,
                                          nullptr);
        rc = forward(h, B);
        if (rc != MS_OK) break;
        if (cudaMemcpyAsync(yb.data(), h->Y, sizeof(float) * (size_t)B * 16, cudaMemcpyDeviceToHost, h->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess) {
            rc = mfail(h, MS_ERR_CUDA, "forward");
            break;
        }
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < h->out_dim; ++c) y[(r0 + r) * h->out_dim + c] = yb[(size_t)r * 16 + c];
    }
    cudaFree(dx);
    if (rc == MS_OK) rc = check_err(h);
    return rc;
}

ms_status ms_mlp_loss_grad(ms_mlp* h, const float* x, const float* t, int64_t n, double* loss, float* grads) {
    if (!h || !x || !t || n <= 0 || n > 65536) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int B = round_up(n, 128);
    ML_TRY(ensure_batch(h, B));
    float *dx, *dt;
    ML_CUDA(h, cudaMalloc(&dx, sizeof(float) * (size_t)n * h->in_dim));
    if (cudaMalloc(&dt, sizeof(float) * (size_t)n * h->out_dim) != cudaSuccess) {
        cudaFree(dx);
        return mfail(h, MS_ERR_OUT_OF_MEMORY, "cudaMalloc");
    }
    ms_status rc = MS_OK;
    if (cudaMemcpy(dx, x, sizeof(float) * (size_t)n * h->in_dim, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dt, t, sizeof(float) * (size_t)n * h->out_dim, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = mfail(h, MS_ERR_CUDA, "upload");
    if (rc == MS_OK) {
        k_gather<<<B, 64, 0, h->stream>>>(dx, dt, nullptr, 0, n, h->in_dim, h->in_pad, h->out_dim, B, h->Xb, h->Tb);
        rc = forward(h, B);
    }
    if (rc == MS_OK) rc = loss_grad(h, B, (int)n);
    if (rc == MS_OK) rc = backward(h, B);
    std::vector<double> part(256);
    if (rc == MS_OK &&
        (cudaMemcpyAsync(part.data(), h->loss_part, 256 * sizeof(double), cudaMemcpyDeviceToHost, h->stream) !=
             cudaSuccess ||
         cudaStreamSynchronize(h->stream) != cudaSuccess))
        rc = mfail(h, MS_ERR_CUDA, "loss_grad");
    cudaFree(dx);
    cudaFree(dt);
    if (rc == MS_OK) rc = check_err(h);
    if (rc != MS_OK) return rc;
    double s = 0.0;
    for (double v : part) s += v;
    if (loss) *loss = s / ((double)n * h->out_dim);
    if (grads) ML_CUDA(h, cudaMemcpy(grads, h->g, h->n_params * sizeof(float), cudaMemcpyDeviceToHost));
    return MS_OK;
}

ms_status ms_mlp_set_data(ms_mlp* h, const float* x, const float* t, int64_t n) {
    if (!h || !x || !t || n <= 0) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    ML_CUDA(h, cudaStreamSynchronize(h->stream));
    if (h->dX) {
        cudaFree(h->dX);
        cudaFree(h->dT);
        cudaFree(h->d_idx);
        h->allocs.erase(std::remove_if(h->allocs.begin(), h->allocs.end(),
                                       [&](void* q) { return q == h->dX || q == h->dT || q == h->d_idx; }),
                        h->allocs.end());
        h->dX = h->dT = nullptr;
        h->d_idx = nullptr;
    }
    ML_TRY(malloc_dev(h, &h->dX, (size_t)n * h->in_dim));
    ML_TRY(malloc_dev(h, &h->dT, (size_t)n * h->out_dim));
    ML_TRY(malloc_dev(h, &h->d_idx, (size_t)n));
    ML_CUDA(h, cudaMemcpy(h->dX, x, sizeof(float) * (size_t)n * h->in_dim, cudaMemcpyHostToDevice));
    ML_CUDA(h, cudaMemcpy(h->dT, t, sizeof(float) * (size_t)n * h->out_dim, cudaMemcpyHostToDevice));
    h->n_rows = n;
    return MS_OK;
}

ms_status ms_mlp_train(ms_mlp* h, int32_t epochs, int32_t batch, double lr, uint64_t seed, float* epoch_loss) {
    if (!h || epochs <= 0 || batch <= 0 || !(lr > 0.0)) return MS_ERR_INVALID_ARGUMENT;
    if (!h->dX) return mfail(h, MS_ERR_INVALID_ARGUMENT, "no training data (ms_mlp_set_data)");
    cudaSetDevice(h->device);
    const int B = round_up(std::min<long long>(batch, h->n_rows), 128);
    ML_TRY(ensure_batch(h, B));
    const long long n = h->n_rows;
    std::vector<long long> perm(n);
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ++ep) {
        for (long long i = 0; i < n; ++i) perm[i] = i;
        std::shuffle(perm.begin(), perm.end(), rng);
        ML_CUDA(h, cudaMemcpyAsync(h->d_idx, perm.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, h->stream));
        ML_CUDA(h, cudaMemsetAsync(h->loss_acc, 0, sizeof(double), h->stream));
        for (long long r0 = 0; r0 < n; r0 += B) {
            const int rows = (int)std::min<long long>(B, n - r0);
            k_gather<<<B, 64, 0, h->stream>>>(h->dX, h->dT, h->d_idx, r0, n, h->in_dim, h->in_pad, h->out_dim, B,
                                              h->Xb, h->Tb);
            ML_TRY(forward(h, B));
            ML_TRY(loss_grad(h, B, rows));
            ML_TRY(backward(h, B));
            h->adam_t += 1;
            const float c1 = 1.0f - std::pow(b1, (float)h->adam_t), c2 = 1.0f - std::pow(b2, (float)h->adam_t);
            k_adam<<<(unsigned)((h->n_params + 255) / 256), 256, 0, h->stream>>>(h->p, h->g, h->m1, h->m2,
                                                                                (long long)h->n_params, (float)lr,
                                                                                b1, b2, eps, c1, c2);
            ML_TRY(refresh_bf16(h));
            k_loss_accumulate<<<1, 1, 0, h->stream>>>(h->loss_part, 256, h->loss_acc);
        }
        double ep_sum = 0.0;
        ML_CUDA(h, cudaMemcpyAsync(&ep_sum, h->loss_acc, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        ML_CUDA(h, cudaStreamSynchronize(h->stream));
        ML_TRY(check_err(h));
        if (epoch_loss) epoch_loss[ep] = (float)(ep_sum / ((double)n * h->out_dim));
    }
    return MS_OK;
}

void* ms_mlp_stream(ms_mlp* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"
