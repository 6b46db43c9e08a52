// Batched control-matrix MVM on the 5th-generation tensor cores (tcgen05).
//
// For nbatch instances sharing one BF16 or FP8 control matrix the MVM is a
// GEMM: part[ks][b][row] = sum_{k in slab ks} M[row][k] g[b][k].  One CTA of
// 128 threads owns 128 rows x one K slab; per chunk of 64 columns it stages
// the M tile (FP8 widened to BF16, exact) and the gradient tile in shared
// memory in the K-major core-matrix layout (8 rows x 16 bytes per core
// matrix), and one thread issues tcgen05.mma (M=128, N = batch tile, K=16)
// accumulating in TMEM.  The gradients enter as three BF16 terms
// g = hi + mid + lo (each the BF16 rounding of what the previous terms left),
// so the products carry FP32-level accuracy in g; only M's storage type
// rounds.  The epilogue reads the accumulators with tcgen05.ld (warp w owns
// TMEM lanes 32w..32w+31 = rows) and writes the split-K partials.
//
// Every wait on the MMA-completion mbarrier is bounded: on timeout the CTA
// records an error, waits once more (bounded) and still frees its TMEM.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mb {

constexpr int kTcRows = 128;     // UMMA M
constexpr int kTcK = 64;         // columns per shared-memory chunk (4 MMAs of K=16)
constexpr int kTcThreads = 128;  // 4 warps, one per TMEM lane quarter
constexpr int kTcTerms = 3;      // BF16 terms of the gradients

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no-swizzle shared-memory matrix descriptor (sm_100): start
// address, leading byte offset (between core matrices adjacent in K), stride
// byte offset (between core matrices adjacent in M/N), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major,
// M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

// Byte offset of element (r, k) of a [rows x 64] K-major tile: core matrix
// (r/8, k/8) at ((r/8)*8 + k/8)*128 bytes, row r%8 at 16*(r%8).
__device__ __forceinline__ uint32_t tile_off(int r, int kgrp) { return (uint32_t)(((r >> 3) * 8 + kgrp) * 128 + (r & 7) * 16); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int DT>
struct TcA;  // the M tile: 16 bytes of a row (global) -> BF16 core-matrix rows
template <>
struct TcA<MB_MVM_BF16> {
    using T = __nv_bfloat16;
    static constexpr int kVec = 8;  // elements per 16-byte load
    __device__ static void stage(const uint4 &q, char *tile, int r, int kgrp) {
        *reinterpret_cast<uint4 *>(tile + tile_off(r, kgrp)) = q;
    }
};
template <>
struct TcA<MB_MVM_FP8> {
    using T = __nv_fp8_e4m3;
    static constexpr int kVec = 16;
    __device__ static void stage(const uint4 &q, char *tile, int r, int kgrp) {
        const __nv_fp8x2_e4m3 *h = reinterpret_cast<const __nv_fp8x2_e4m3 *>(&q);
        uint32_t w[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const float2 f = static_cast<float2>(h[i]);
            const __nv_bfloat162 b = __floats2bfloat162_rn(f.x, f.y);  // exact: E4M3 fits BF16
            w[i] = *reinterpret_cast<const uint32_t *>(&b);
        }
        *reinterpret_cast<uint4 *>(tile + tile_off(r, kgrp)) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4 *>(tile + tile_off(r, kgrp + 1)) = make_uint4(w[4], w[5], w[6], w[7]);
    }
};

// grid: (ceil(nact/128), nks, ceil(nbatch/N)); block kTcThreads; dynamic
// shared memory: A tile (16 KB) + kTcTerms gradient tiles (N*128 bytes each).
template <int DT, int N>
__global__ void __launch_bounds__(kTcThreads)
k_mvm_tc(const typename TcA<DT>::T *__restrict__ M, long ldm, const float *__restrict__ g, long ngrad,
         float *__restrict__ part, int nact, int nbatch, int kslab, int *__restrict__ err) {
    static_assert(N == 16 || N == 32 || N == 64, "batch tile");
    constexpr int NCOL = N < 32 ? 32 : N;  // TMEM columns (power of 2, >= 32)
    using A = TcA<DT>;
    extern __shared__ __align__(128) char tcsm[];
    char *ta = tcsm;                                // [128 x 64] BF16
    char *tb = tcsm + kTcRows * kTcK * 2;           // kTcTerms x [N x 64] BF16
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_tmem;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row0 = blockIdx.x * kTcRows;
    const long k0 = (long)blockIdx.y * kslab;
    const int kn = (int)((ngrad - k0) < kslab ? (ngrad - k0) : kslab);
    const int b0 = blockIdx.z * N;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&s_tmem)), "r"(NCOL) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t bar_a = smem_addr(&bar);
    bool ok = true;
    uint32_t phase = 0;
    const int nchunk = (kn + kTcK - 1) / kTcK;
    for (int ch = 0; ch < nchunk; ch++) {
        const int kc = ch * kTcK;
        if (ch > 0) {  // the previous chunk's MMAs have read the tiles
            ok = ok && mbar_wait(bar_a, phase);
            phase ^= 1;
        }
        // M tile: row r, 16-byte group u (A::kVec elements); zero past the matrix
        constexpr int UPR = kTcK / A::kVec;  // 16-byte loads per row
        for (int q = threadIdx.x; q < kTcRows * UPR; q += blockDim.x) {
            const int r = q / UPR, u = q - r * UPR;
            const int row = row0 + r, col = kc + u * A::kVec;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (row < nact && col < kn) v = *reinterpret_cast<const uint4 *>(M + (size_t)row * ldm + k0 + col);
            A::stage(v, ta, r, u * A::kVec / 8);
        }
        // gradient tiles: instance n, 8 columns per item, split into three BF16 terms
        for (int q = threadIdx.x; q < N * (kTcK / 8); q += blockDim.x) {
            const int n = q >> 3, kg = q & 7;
            const int b = b0 + n;
            float v[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const long col = k0 + kc + kg * 8 + e;
                v[e] = (b < nbatch && kc + kg * 8 + e < kn) ? g[(size_t)b * ngrad + col] : 0.f;
            }
#pragma unroll
            for (int t = 0; t < kTcTerms; t++) {
                uint32_t w[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
                    const float2 back = __bfloat1622float2(h);
                    v[2 * e] -= back.x;
                    v[2 * e + 1] -= back.y;
                    w[e] = *reinterpret_cast<const uint32_t *>(&h);
                }
                *reinterpret_cast<uint4 *>(tb + t * (N * kTcK * 2) + tile_off(n, kg)) =
                    make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t idesc = umma_idesc_bf16(N);
            const uint32_t abase = smem_addr(ta), bbase = smem_addr(tb);
#pragma unroll
            for (int s = 0; s < kTcK / 16; s++) {
                const uint64_t ad = umma_desc(abase + s * 256, 128, 1024);
#pragma unroll
                for (int t = 0; t < kTcTerms; t++) {
                    const uint64_t bd = umma_desc(bbase + t * (N * kTcK * 2) + s * 256, 128, 1024);
                    const uint32_t acc = (ch > 0 || s > 0 || t > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(bar_a) : "memory");
        }
    }
    if (nchunk > 0) {
        ok = ok && mbar_wait(bar_a, phase);
        if (!ok) {
            if (lane == 0) atomicExch(err, 1);
            mbar_wait(bar_a, phase);  // bounded, before the accumulators are freed
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w reads TMEM lanes 32w.. (rows), N columns (instances)
    if (ok && nchunk > 0) {
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        const int row = row0 + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < nact)
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int b = b0 + c0 + j;
                    if (b < nbatch) part[((size_t)blockIdx.y * nbatch + b) * nact + row] = __uint_as_float(r[j]);
                }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(NCOL) : "memory");
}

}  // namespace mb
