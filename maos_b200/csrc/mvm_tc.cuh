// Batched control-matrix MVM on the 5th-generation tensor cores (tcgen05).
//
// For nbatch instances sharing one BF16 or FP8 control matrix the MVM is a
// GEMM: part[ks][b][row] = sum_{k in slab ks} M[row][k] g[b][k], with M the
// A operand (UMMA M = 128 rows) and the gradients the B operand, accumulated
// in FP32 in tensor memory.
//
// Layout in HBM.  M is stored pre-tiled: tile (row block rb, chunk c) holds
// rows 128rb.. and columns 64c.. contiguously, already in the order the
// tensor core reads from shared memory (K-major, no swizzle, 8-row x
// 16-byte core matrices): a BF16 tile is 16 KB (core matrix (r/8, k/8) at
// ((r/8)*8 + k/8)*128 bytes), an FP8 tile 8 KB (core matrix (r/8, k/16) at
// ((r/8)*4 + k/16)*128 bytes); row r%8 of a core matrix is at 16*(r%8).
//
// Gradients.  The tensor core multiplies like types only, so the FP32
// gradients are split once per call into terms of M's type, stacked as the
// rows of one B tile per (batch tile, chunk):
//   BF16 M (kind::f16): k_gsplit writes g = hi + lo, lo the BF16 rounding of
//     g - hi, 16 significant bits; each product carries a relative error of
//     at most 2^-17 from g, 500 times below the BF16 rounding of M (2^-8).
//     Both terms accumulate into the same TMEM columns.
//   FP8 M (kind::f8f6f4): k_gsplit8 writes four E4M3 terms per instance,
//     g = sum_t 2^(e-4t) q_t + r_4, 2^e the power of two that maps the
//     instance's max|g| (k_gmax) to at most 448; |r_4| <= 2^-16 max|g|
//     elementwise and the decomposition is otherwise exact.  Row t*N + n of
//     the B tile is term t of instance n, one MMA (N = 4 x batch tile) per
//     K-step writes each term to its own TMEM columns, and the epilogue
//     forms sum_t 2^(e-4t) acc_t.  The matrix is read by the tensor core as
//     stored: no widening pass.
// Every pipeline stage is therefore two contiguous bulk copies
// (cp.async.bulk, completing on an mbarrier by byte count): no tensor map,
// no per-element address arithmetic, no shared-memory bank conflicts.
//
// CTA (rb, ks, z): 128 threads, 128 rows x one K slab x one batch tile, with
// warp roles that meet only on mbarriers:
//   warp 0, lane 0: copies.  Keeps all S stages in flight; a stage is
//     refilled as soon as the MMAs that read it completed ("empty").
//   warp 1, lane 0: MMAs.  Per 64-column chunk, the K-steps (4 of K=16 for
//     BF16 times 2 terms, 2 of K=32 for FP8) of tcgen05.mma into TMEM,
//     committed to the stage's "empty" barrier.
// The epilogue reads the accumulators with tcgen05.ld (warp w reaches TMEM
// lanes 32w.. = rows) and writes the split-K partials.
//
// Every mbarrier wait is bounded.  On a timeout a thread raises the CTA's
// abort flag, every role stops issuing, the copy thread waits (bounded) for
// the copies it issued, one thread waits (bounded) for the MMAs issued, and
// the tensor memory is still freed; the error flag tells the host.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mb {

constexpr int kTcRows = 128;     // UMMA M
constexpr int kTcK = 64;         // columns per chunk
constexpr int kTcThreads = 128;  // copy warp, MMA warp; all four warps read the accumulators
constexpr int kTcTerms = 2;      // BF16 terms of the gradients
constexpr int kTcTermsFp8 = 4;   // E4M3 terms of the gradients
constexpr int kTcTileBf16 = kTcRows * kTcK * 2;  // bytes of a BF16 M tile
constexpr int kTcTileFp8 = kTcRows * kTcK;       // bytes of an FP8 M tile

__host__ __device__ constexpr int tc_a_bytes(int dt) { return dt == MB_MVM_BF16 ? kTcTileBf16 : kTcTileFp8; }
// Gradient tile of a batch tile of n: 2 BF16 terms x n x 64 x 2 bytes, or
// 4 E4M3 terms x n x 64 bytes; the same size for both.
__host__ __device__ constexpr int tc_b_bytes(int n) { return kTcTerms * n * kTcK * 2; }
// Pipeline depth: batch tiles of 16 and 32 keep two CTAs per SM (at most
// about 110 KB each); the 64 tile runs one CTA per SM with a deeper ring.
__host__ __device__ constexpr int tc_stages(int dt, int n) {
    return dt == MB_MVM_BF16 ? (n <= 16 ? 5 : n <= 32 ? 4 : 5) : (n <= 16 ? 8 : n <= 32 ? 6 : 8);
}
__host__ __device__ constexpr int tc_smem_bytes(int dt, int n) {
    return tc_stages(dt, n) * (tc_a_bytes(dt) + tc_b_bytes(n));
}
// TMEM columns (a power of two, at least 32): one per instance of the tile,
// times the four terms for FP8.
__host__ __device__ constexpr int tc_tmem_cols(int dt, int n) {
    return dt == MB_MVM_BF16 ? (n < 32 ? 32 : n) : kTcTermsFp8 * n;
}

// Byte offset of the 16-byte row holding columns 8*kgrp.. of row r in a
// BF16 [rows x 64] K-major core-matrix tile.
__host__ __device__ __forceinline__ uint32_t tile_off(int r, int kgrp) {
    return (uint32_t)(((r >> 3) * 8 + kgrp) * 128 + (r & 7) * 16);
}
// Byte offset of element (r, k) in an 8-bit [rows x 64] K-major
// core-matrix tile: core matrix (r/8, k/16), 16-byte row r%8.
__host__ __device__ __forceinline__ uint32_t tc_fp8_off(int r, int k) {
    return (uint32_t)((((r >> 3) * 4 + (k >> 4)) * 8 + (r & 7)) * 16 + (k & 15));
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no-swizzle shared-memory matrix descriptor (sm_100): start
// address, leading byte offset (between core matrices adjacent in K), stride
// byte offset (between core matrices adjacent in M/N), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor (kind::f16 and kind::f8f6f4): D FP32, A and B of
// M's type (BF16 = 1 in kind::f16, E4M3 = 0 in kind::f8f6f4), both K-major,
// M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc(int dt, int n) {
    return (1u << 4) | (dt == MB_MVM_BF16 ? (1u << 7) | (1u << 10) : 0u) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(kTcRows >> 4) << 24);
}

// Bounded parity wait; gives up early once a thread of the CTA has raised
// the abort hint.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, const volatile int *abort = nullptr) {
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
        if (abort && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}

// One stage: the M tile and the three gradient-term tiles, both landing on
// the stage's full barrier.
__device__ __forceinline__ void tc_load_stage(uint32_t bar, uint32_t sa, const void *ga, int abytes, uint32_t sb,
                                              const void *gb, int bbytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(abytes + bbytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(sa), "l"(ga), "r"(abytes), "r"(bar) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(sb), "l"(gb), "r"(bbytes), "r"(bar) : "memory");
}

// The MMAs of one 64-column chunk: 4 K-steps of 16 times kTcTerms gradient terms.
__device__ __forceinline__ void tc_mma_chunk(uint32_t tmem, uint32_t abase, uint32_t bbase, int term_bytes,
                                             uint32_t idesc, bool first) {
#pragma unroll
    for (int s = 0; s < kTcK / 16; s++) {
        const uint64_t ad = umma_desc(abase + s * 256, 128, 1024);
#pragma unroll
        for (int t = 0; t < kTcTerms; t++) {
            const uint64_t bd = umma_desc(bbase + t * term_bytes + s * 256, 128, 1024);
            const uint32_t acc = (!first || s > 0 || t > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
        }
    }
}

// The MMAs of one 64-column FP8 chunk: 2 K-steps of 32, each one MMA over
// the stacked terms (the B tile's 4N rows).
__device__ __forceinline__ void tc_mma_chunk_fp8(uint32_t tmem, uint32_t abase, uint32_t bbase, uint32_t idesc,
                                                 bool first) {
#pragma unroll
    for (int s = 0; s < kTcK / 32; s++) {
        const uint64_t ad = umma_desc(abase + s * 256, 128, 512);
        const uint64_t bd = umma_desc(bbase + s * 256, 128, 512);
        const uint32_t acc = (!first || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}"
            :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
    }
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar)
                 : "memory");
}

// Gradients -> kTcTerms BF16 terms in per-(batch tile, chunk) core-matrix tiles.
// gs: [nz][nch][kTcTerms][N x 64] BF16, zero past nbatch and ngrad.  One
// thread per 8 columns of one instance; consecutive threads write
// consecutive 16-byte rows.
template <int N>
__global__ void __launch_bounds__(256)
k_gsplit(const float *__restrict__ g, long ngrad, int nbatch, long nch, int nz, char *__restrict__ gs) {
    const long item = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= (long)nz * nch * N * 8) return;
    // item = ((z*nch + c)*(N/8) + n/8)*64 + kg*8 + n%8
    const int r8 = (int)(item & 7), kg = (int)((item >> 3) & 7);
    const long rest = item >> 6;
    const int ng = (int)(rest % (N / 8));
    const long zc = rest / (N / 8);
    const long c = zc % nch;
    const int n = ng * 8 + r8, b = (int)(zc / nch) * N + n;
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const long col = c * kTcK + kg * 8 + e;
        v[e] = (b < nbatch && col < ngrad) ? g[(size_t)b * ngrad + col] : 0.f;
    }
    char *base = gs + (size_t)zc * tc_b_bytes(N);
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
        *reinterpret_cast<uint4 *>(base + t * (N * kTcK * 2) + tile_off(n, kg)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// FP8 gradient terms.  The scale of term t of an instance is 2^(e - 4t),
// with e the smallest exponent for which max|g| / 2^e <= 448 (the E4M3
// maximum).  Rounding to E4M3 (3 mantissa bits) leaves at most 2^-4 of each
// value, so the residual that term t + 1 receives, divided by its scale,
// is again at most 448: the terms never saturate, and after four terms
// |g - sum_t 2^(e-4t) q_t| <= 2^-16 max|g| elementwise.  e is clamped so that
// every scale is a normal FP32 number.
__device__ __forceinline__ int tc_fp8_exp(unsigned maxbits) {
    const float m = __uint_as_float(maxbits);
    if (!(m > 0.f) || m > 3.0e38f) return 0;
    int e;
    const float f = frexpf(m, &e);                // m = f 2^e, f in [0.5, 1)
    const int k = f <= 0.875f ? e - 9 : e - 8;    // m / 2^k <= 448 = 0.875 2^9
    return k < -110 ? -110 : k > 120 ? 120 : k;
}
__device__ __forceinline__ float tc_pow2(int k) { return __int_as_float((127 + k) << 23); }

// Largest |g| of each instance, as the bits of a non-negative float (which
// order as unsigned integers); gmax zeroed before.  grid: (blocks, nbatch).
__global__ void __launch_bounds__(256)
k_gmax(const float *__restrict__ g, long ngrad, unsigned *__restrict__ gmax) {
    const int b = blockIdx.y;
    float m = 0.f;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < ngrad; i += (long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(g[(size_t)b * ngrad + i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, red[w]);
        atomicMax(gmax + b, __float_as_uint(m));
    }
}

// Gradients -> kTcTermsFp8 E4M3 terms in per-(batch tile, chunk) [4N x 64]
// tiles, row t*N + n = term t of instance n (zero past nbatch and ngrad).
// One thread per 16 columns of one instance; consecutive threads write
// consecutive 16-byte rows.
template <int N>
__global__ void __launch_bounds__(256)
k_gsplit8(const float *__restrict__ g, long ngrad, int nbatch, long nch, int nz, const unsigned *__restrict__ gmax,
          char *__restrict__ gs) {
    const long item = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= (long)nz * nch * N * 4) return;
    // item = ((z*nch + c)*(N/8) + n/8)*32 + kq*8 + n%8
    const int r8 = (int)(item & 7), kq = (int)((item >> 3) & 3);
    const long rest = item >> 5;
    const int ng = (int)(rest % (N / 8));
    const long zc = rest / (N / 8);
    const long c = zc % nch;
    const int n = ng * 8 + r8, b = (int)(zc / nch) * N + n;
    float v[16];
#pragma unroll
    for (int e = 0; e < 16; e++) {
        const long col = c * kTcK + kq * 16 + e;
        v[e] = (b < nbatch && col < ngrad) ? g[(size_t)b * ngrad + col] : 0.f;
    }
    const int k = b < nbatch ? tc_fp8_exp(gmax[b]) : 0;
    char *tile = gs + (size_t)zc * tc_b_bytes(N);
#pragma unroll
    for (int t = 0; t < kTcTermsFp8; t++) {
        const float sc = tc_pow2(k - 4 * t), inv = tc_pow2(4 * t - k);
        uint32_t w[4];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const __nv_fp8x2_storage_t q =
                __nv_cvt_float2_to_fp8x2(make_float2(v[2 * e] * inv, v[2 * e + 1] * inv), __NV_SATFINITE, __NV_E4M3);
            const float2 back = __half22float2(__half2(__nv_cvt_fp8x2_to_halfraw2(q, __NV_E4M3)));
            v[2 * e] -= sc * back.x;  // exact: power-of-two scale, residual below the value
            v[2 * e + 1] -= sc * back.y;
            if (e & 1) w[e >> 1] |= (uint32_t)q << 16;
            else w[e >> 1] = (uint32_t)q;
        }
        *reinterpret_cast<uint4 *>(tile + tc_fp8_off(t * N + n, kq * 16)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// grid: (row blocks, K slabs, batch tiles); block kTcThreads; dynamic shared
// memory tc_smem_bytes(DT, N).  Mt: pre-tiled M ([row blocks][nch] tiles of
// tc_a_bytes(DT)); gs: the gradient terms (k_gsplit or k_gsplit8); gmax:
// each instance's max|g| (FP8 only: the terms' scales); each slab is `cps`
// chunks.
template <int DT, int N>
__global__ void __launch_bounds__(kTcThreads)
k_mvm_tc(const char *__restrict__ Mt, const char *__restrict__ gs, const unsigned *__restrict__ gmax, long nch,
         int cps, float *__restrict__ part, int nact, int nbatch, int *__restrict__ err) {
    static_assert(N == 16 || N == 32 || N == 64, "batch tile");
    constexpr bool kFp8 = DT != MB_MVM_BF16;
    constexpr int NCOL = tc_tmem_cols(DT, N);
    constexpr int S = tc_stages(DT, N);
    constexpr int AB = tc_a_bytes(DT), BB = tc_b_bytes(N), SB = AB + BB;
    constexpr uint32_t idesc = umma_idesc(DT, kFp8 ? kTcTermsFp8 * N : N);
    extern __shared__ __align__(128) char tcsm[];
    __shared__ __align__(8) uint64_t full[S], empty[S], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_mmas;
    __shared__ volatile int s_abort;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rb = blockIdx.x, ks = blockIdx.y, z = blockIdx.z;
    const long c0 = (long)ks * cps;
    const int nchunk = (int)((nch - c0) < cps ? (nch - c0) : cps);
    const char *ga = Mt + ((size_t)rb * nch + c0) * AB;
    const char *gb = gs + ((size_t)z * nch + c0) * BB;
    const uint32_t sbase = smem_addr(tcsm);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&s_tmem)), "r"(NCOL) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 32) {
        for (int i = 0; i < S; i++) {
            mbar_init(smem_addr(&full[i]), 1);
            mbar_init(smem_addr(&empty[i]), 1);
        }
        mbar_init(smem_addr(&done), 1);
        s_abort = 0;
        s_mmas = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (warp == 0) {
        if (lane == 0) {  // copies
            auto load = [&](int c) {
                const int st = c % S;
                tc_load_stage(smem_addr(&full[st]), sbase + st * SB, ga + (size_t)c * AB, AB, sbase + st * SB + AB,
                              gb + (size_t)c * BB, BB);
            };
            int issued = 0;
            for (; issued < nchunk && issued < S; issued++) load(issued);
            for (; issued < nchunk; issued++) {
                const int c = issued - S;  // the chunk that last used this stage
                if (!mbar_wait(smem_addr(&empty[c % S]), (uint32_t)((c / S) & 1), &s_abort)) {
                    s_abort = 1;
                    break;
                }
                load(issued);
            }
            // every copy this thread issued has landed before the CTA can exit
            for (int c = issued - S < 0 ? 0 : issued - S; c < issued; c++)
                mbar_wait(smem_addr(&full[c % S]), (uint32_t)((c / S) & 1));
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {  // MMAs
            int mmas = 0;
            for (int ch = 0; ch < nchunk; ch++) {
                const int st = ch % S;
                if (!mbar_wait(smem_addr(&full[st]), (uint32_t)((ch / S) & 1), &s_abort)) {
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if constexpr (kFp8)
                    tc_mma_chunk_fp8(tmem, sbase + st * SB, sbase + st * SB + AB, idesc, ch == 0);
                else
                    tc_mma_chunk(tmem, sbase + st * SB, sbase + st * SB + AB, N * kTcK * 2, idesc, ch == 0);
                tc_commit(smem_addr(&empty[st]));
                mmas = ch + 1;
            }
            s_mmas = mmas;
            tc_commit(smem_addr(&done));  // tracks every MMA this thread issued
        }
        __syncwarp();
    }
    // one thread waits for the MMAs (bounded, twice before the accumulators
    // are freed); the rest of the CTA waits at the barrier, not on the mbarrier
    bool bad = false;
    if (threadIdx.x == 0) {
        bad = !mbar_wait(smem_addr(&done), 0);
        if (bad) mbar_wait(smem_addr(&done), 0);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    const bool skip = __syncthreads_or(bad) || s_abort || s_mmas < nchunk;
    if (skip && threadIdx.x == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w reads TMEM lanes 32w.. (rows); column j (BF16) or
    // t*N + j (FP8 term t) is instance z*N + j
    if (!skip && nchunk > 0) {
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        const int row = rb * kTcRows + warp * 32 + lane;
#pragma unroll
        for (int cc = 0; cc < N; cc += 16) {
            int ke[16];  // FP8: instance exponents
#pragma unroll
            for (int j = 0; j < 16; j++) ke[j] = (kFp8 && z * N + cc + j < nbatch) ? tc_fp8_exp(gmax[z * N + cc + j]) : 0;
            float y[16];
#pragma unroll
            for (int j = 0; j < 16; j++) y[j] = 0.f;
#pragma unroll
            for (int t = 0; t < (kFp8 ? kTcTermsFp8 : 1); t++) {
                uint32_t r[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                      "=r"(r[14]), "=r"(r[15])
                    : "r"(taddr + (uint32_t)(t * N + cc)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; j++) y[j] += (kFp8 ? tc_pow2(ke[j] - 4 * t) : 1.f) * __uint_as_float(r[j]);
            }
            if (row < nact)
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int b = z * N + cc + j;
                    if (b < nbatch) part[((size_t)ks * nbatch + b) * nact + row] = y[j];
                }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(NCOL) : "memory");
}

}  // namespace mb
