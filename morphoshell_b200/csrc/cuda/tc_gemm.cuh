// BF16 GEMM on the 5th-generation tensor cores (tcgen05) with the
// accumulator in tensor memory, for the warm-start network's layers.
//
//   C[M x N] = A[M x K] * B[N x K]^T      A, B row-major bf16 (K contiguous),
//                                         FP32 accumulation in TMEM
//
// One CTA of 128 threads computes a 128 x BN tile.  All threads stage
// 128 x 64 and BN x 64 operand tiles into shared memory with 16-byte
// cp.async copies, in the canonical K-major no-swizzle layout of the MMA's
// shared-memory descriptors (8-row x 16-byte core matrices: consecutive
// 8-row groups 128 B apart, the two 16-byte K halves of a K=16 step
// `rows/8 * 128` B apart), kStages stages deep: while the tensor cores work
// on one stage the next two are in flight.  Thread 0 issues tcgen05.mma
// (M = 128, N = BN, K = 16) four times per stage and commits them to the
// stage's mbarrier, which frees the stage for its refill; the epilogue reads
// the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 =
// rows) and applies a fused bias / activation.  Every mbarrier wait is
// bounded: on timeout the kernel records an error and still frees its
// tensor memory.
#pragma once

#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace msb {
namespace tc {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kThreads = 128;
constexpr int kStages = 3;  // shared-memory stages of the K loop

enum Epilogue {
    EPI_F32 = 0,        // Cf = acc (+ bias[n])
    EPI_BIAS_SILU = 1,  // Z = acc + bias[n] (bf16), H = SiLU(Z) (bf16)
    EPI_DSILU = 2,      // H = acc * SiLU'(Z[m][n]) (bf16), Z read
};

struct GemmArgs {
    const __nv_bfloat16* A;  // [M][lda]
    const __nv_bfloat16* B;  // [N][ldb]
    int M, N, K;             // M % 128 == 0, N % BN == 0, K % 16 == 0
    int lda, ldb;
    int k_split;             // K range of one CTA (multiple of 16); blockIdx.z picks the range
    const float* bias;       // [N] or null
    float* Cf;               // [splits][M][ldc] (EPI_F32)
    __nv_bfloat16* Z;        // [M][ldc]
    __nv_bfloat16* H;        // [M][ldc]
    int ldc;
    int* err;                // set to 1 when a wait times out
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle (layout type 0),
// descriptor version 1, base offset 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int n) {
    return (1u << 4)                          // C format F32
           | (1u << 7)                        // A format BF16
           | (1u << 10)                       // B format BF16
           | ((uint32_t)(n >> 3) << 17)       // N / 8
           | ((uint32_t)(kBM >> 4) << 24);    // M / 16
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete, for at most about
// a second of SM clock; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > 2000000000LL) return false;
    }
    return true;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Stage a rows x 64 tile (row-major source, leading dimension ld elements)
// into the canonical layout at `dst`; rows is a multiple of 8, k_valid (a
// multiple of 8) columns are copied, the rest of the 64 are zero.
template <int ROWS>
__device__ __forceinline__ void stage_tile(uint32_t dst, const __nv_bfloat16* src, int ld, int k_valid,
                                           unsigned char* dst_generic) {
    constexpr int kChunks = ROWS * (kBK / 8);
    constexpr uint32_t kLBO = ROWS / 8 * 128;
#pragma unroll 4
    for (int c = threadIdx.x; c < kChunks; c += kThreads) {
        const int row = c % ROWS, kc = c / ROWS;
        const uint32_t off = kc * kLBO + (row >> 3) * 128 + (row & 7) * 16;
        if (kc * 8 < k_valid) {
            cp_async16(dst + off, src + (size_t)row * ld + kc * 8);
        } else {
            *reinterpret_cast<uint4*>(dst_generic + off) = make_uint4(0, 0, 0, 0);
        }
    }
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kThreads, 1) k_gemm(const GemmArgs g) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int kABytes = kBM * kBK * 2, kBBytes = BN * kBK * 2;
    constexpr int kStage = kABytes + kBBytes;
    constexpr uint32_t kCols = BN < 32 ? 32 : BN;  // TMEM columns (power of two >= 32)
    __shared__ uint64_t bar[kStages];
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_split, ke = min(g.K, kb + g.k_split);

    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; ++i) mbar_init(&bar[i], 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = instr_desc_bf16(BN);
    const uint32_t base = smem_u32(smem);
    const int nk = (ke - kb + kBK - 1) / kBK;

    // K step kt lives in slot kt % kStages; the j-th commit to a slot's
    // mbarrier is step kStages j + slot, so step kt's MMAs are done when the
    // phase of parity (kt / kStages) & 1 of bar[kt % kStages] completes.
    auto load = [&](int kt) {
        const int s = kt % kStages;
        const int k0 = kb + kt * kBK;
        const int kv = min(kBK, ke - k0);
        const uint32_t sa = base + s * kStage, sb = sa + kABytes;
        stage_tile<kBM>(sa, g.A + (size_t)m0 * g.lda + k0, g.lda, kv, smem + s * kStage);
        stage_tile<BN>(sb, g.B + (size_t)n0 * g.ldb + k0, g.ldb, kv, smem + s * kStage + kABytes);
    };
    // Prologue: steps 0 .. kStages-2 in flight (one copy group each, empty
    // groups past the end keep the count uniform).
#pragma unroll
    for (int p = 0; p < kStages - 1; ++p) {
        if (p < nk) load(p);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    int last = -1;  // last step whose MMAs were committed
    for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % kStages;
        // kStages-1+kt groups committed; step kt's is the (kStages-2)-th newest.
        asm volatile("cp.async.wait_group %0;" ::"n"(kStages - 2) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int kv = min(kBK, ke - (kb + kt * kBK));
            const uint32_t sa = base + s * kStage, sb = sa + kABytes;
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j) {
                if (j * 16 < kv) {
                    const uint64_t ad = smem_desc(sa + 2 * j * (kBM / 8 * 128), kBM / 8 * 128, 128);
                    const uint64_t bd = smem_desc(sb + 2 * j * (BN / 8 * 128), BN / 8 * 128, 128);
                    mma_bf16(tmem, ad, bd, idesc, (kt > 0 || j > 0) ? 1u : 0u);
                }
            }
            mma_commit(&bar[s]);
        }
        last = kt;
        // Refill: step kt+kStages-1 goes into the slot step kt-1 used, once
        // that step's MMAs are done (step kt's are already queued behind).
        const int nxt = kt + kStages - 1;
        if (nxt < nk) {
            int ok = 1;
            if (kt >= 1) ok = mbar_wait_bounded(&bar[(kt - 1) % kStages], ((kt - 1) / kStages) & 1) ? 1 : 0;
            if (!__syncthreads_and(ok)) {
                if (threadIdx.x == 0) failed = 1;
                break;
            }
            load(nxt);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    // The last commit covers every earlier MMA.
    if (last >= 0) {
        const bool ok = mbar_wait_bounded(&bar[last % kStages], (last / kStages) & 1);
        if (!ok && threadIdx.x == 0) failed = 1;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (failed) {
        if (threadIdx.x == 0) atomicExch(g.err, 1);
    } else {
        const int row = m0 + warp * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(trow + c0, r);
            const int col = n0 + c0;
            if constexpr (EPI == EPI_F32) {
                float* out = g.Cf + (size_t)blockIdx.z * g.M * g.ldc + (size_t)row * g.ldc + col;
#pragma unroll
                for (int j = 0; j < 16; j += 4) {
                    float4 v = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                                           __uint_as_float(r[j + 3]));
                    if (g.bias) {
                        v.x += g.bias[col + j];
                        v.y += g.bias[col + j + 1];
                        v.z += g.bias[col + j + 2];
                        v.w += g.bias[col + j + 3];
                    }
                    *reinterpret_cast<float4*>(out + j) = v;
                }
            } else if constexpr (EPI == EPI_BIAS_SILU) {
                __align__(16) __nv_bfloat16 zb[16], hb[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float z = __uint_as_float(r[j]) + (g.bias ? g.bias[col + j] : 0.0f);
                    const __nv_bfloat16 zq = __float2bfloat16(z);
                    zb[j] = zq;
                    hb[j] = __float2bfloat16(silu(__bfloat162float(zq)));
                }
                uint4* zo = reinterpret_cast<uint4*>(g.Z + (size_t)row * g.ldc + col);
                uint4* ho = reinterpret_cast<uint4*>(g.H + (size_t)row * g.ldc + col);
                zo[0] = reinterpret_cast<const uint4*>(zb)[0];
                zo[1] = reinterpret_cast<const uint4*>(zb)[1];
                ho[0] = reinterpret_cast<const uint4*>(hb)[0];
                ho[1] = reinterpret_cast<const uint4*>(hb)[1];
            } else {
                __align__(16) __nv_bfloat16 zb[16], hb[16];
                const uint4* zi = reinterpret_cast<const uint4*>(g.Z + (size_t)row * g.ldc + col);
                reinterpret_cast<uint4*>(zb)[0] = zi[0];
                reinterpret_cast<uint4*>(zb)[1] = zi[1];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    hb[j] = __float2bfloat16(__uint_as_float(r[j]) * dsilu(__bfloat162float(zb[j])));
                uint4* ho = reinterpret_cast<uint4*>(g.H + (size_t)row * g.ldc + col);
                ho[0] = reinterpret_cast<const uint4*>(hb)[0];
                ho[1] = reinterpret_cast<const uint4*>(hb)[1];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

template <int BN>
constexpr int gemm_smem_bytes() {
    return kStages * (kBM * kBK * 2 + BN * kBK * 2);
}

}  // namespace tc
}  // namespace msb
