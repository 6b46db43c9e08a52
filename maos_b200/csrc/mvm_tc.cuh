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
//     instance's max|g| to at most 448; |r_4| <= 2^-16 max|g|
//     elementwise and the decomposition is otherwise exact.  Row t*N + n of
//     the B tile is term t of instance n, one MMA (N = 4 x batch tile) per
//     K-step writes each term to its own TMEM columns, and the epilogue
//     forms sum_t 2^(e-4t) acc_t.  The matrix is read by the tensor core as
//     stored: no widening pass.
// Every pipeline stage is therefore two contiguous bulk copies
// (cp.async.bulk, completing on an mbarrier by byte count): no tensor map,
// no per-element address arithmetic, no shared-memory bank conflicts.
//
// Persistent stream-K CTAs (k_mvm_tc): 192 threads each, as many as are
// resident; the (batch tile, row block, chunk) units are cut into P equal
// contiguous ranges, one per CTA, so there is no tail wave and each ring is
// filled once.  Warp roles meet only on mbarriers:
//   warp 0, lane 0: copies.  Keeps all S stages in flight across row-block
//     boundaries; a stage is refilled as soon as the MMAs that read it
//     completed ("empty").
//   warp 1, lane 0: MMAs.  Per 64-column chunk, the K-steps (4 of K=16 for
//     BF16 times 2 terms, 2 of K=32 for FP8) of tcgen05.mma into one of two
//     TMEM accumulators, committed to the stage's "empty" barrier.
//   warps 2-5: epilogue.  Read an accumulator with tcgen05.ld (warp w reaches
//     TMEM lanes 32(w%4).. = rows) while the next row block accumulates in
//     the other, and finish the split-K sum in the kernel (the CTA that
//     completes a row block adds its pieces in fixed order).
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
constexpr int kTcThreads = 192;  // copy warp, MMA warp, 4 epilogue warps
constexpr int kTcTerms = 2;      // BF16 terms of the gradients
constexpr int kTcTermsFp8 = 4;   // E4M3 terms of the gradients
constexpr int kTcTileBf16 = kTcRows * kTcK * 2;  // bytes of a BF16 M tile
constexpr int kTcTileFp8 = kTcRows * kTcK;       // bytes of an FP8 M tile
constexpr int kSplitCta = 8;     // CTAs (one cluster) splitting one instance's gradients (FP8)

__host__ __device__ constexpr int tc_a_bytes(int dt) { return dt == MB_MVM_BF16 ? kTcTileBf16 : kTcTileFp8; }
// Gradient tile of a batch tile of n: 2 BF16 terms x n x 64 x 2 bytes, or
// 4 E4M3 terms x n x 64 bytes; the same size for both.
__host__ __device__ constexpr int tc_b_bytes(int n) { return kTcTerms * n * kTcK * 2; }
// Chunks per pipeline stage.  A CTA's stages follow one another at about
// half a microsecond whatever their size (measured on B200: 12, 24 and
// 48 KB stages of one CTA per SM streamed at 0.33, 0.60 and 0.74 of HBM), so
// a stage carries 32 KB of M: two BF16 or four FP8 consecutive tiles, one
// copy each side.
__host__ __device__ constexpr int tc_unit_chunks(int dt) { return dt == MB_MVM_BF16 ? 2 : 4; }
__host__ __device__ constexpr int tc_stage_bytes(int dt, int n) { return tc_unit_chunks(dt) * (tc_a_bytes(dt) + tc_b_bytes(n)); }
// Shared memory of the ring: BF16 with batch tiles of 16 and 32 runs two
// CTAs per SM (100 KB each: 0.89 / 0.82 of HBM against 0.74 / 0.71 with one
// 196 KB ring); the other cases one CTA per SM with a 196 KB ring.
__host__ __device__ constexpr int tc_ring_budget(int dt, int n) { return dt == MB_MVM_BF16 && n <= 32 ? 102400 : 200704; }
// Pipeline depth: as many stages as the budget holds, 2 to 8.
__host__ __device__ constexpr int tc_stages(int dt, int n) {
    return tc_ring_budget(dt, n) / tc_stage_bytes(dt, n) < 2 ? 2
           : tc_ring_budget(dt, n) / tc_stage_bytes(dt, n) > 8 ? 8
                                                                : tc_ring_budget(dt, n) / tc_stage_bytes(dt, n);
}
__host__ __device__ constexpr int tc_smem_bytes(int dt, int n) { return tc_stages(dt, n) * tc_stage_bytes(dt, n); }
// TMEM columns of one accumulator: one per instance of the tile, times the
// four terms for FP8.  Two accumulators alternate (the epilogue of one row
// block overlaps the MMAs of the next); the allocation is a power of two.
__host__ __device__ constexpr int tc_acc_cols(int dt, int n) { return dt == MB_MVM_BF16 ? n : kTcTermsFp8 * n; }
__host__ __device__ constexpr int tc_tmem_cols(int dt, int n) {
    return 2 * tc_acc_cols(dt, n) <= 32 ? 32 : 2 * tc_acc_cols(dt, n);
}

// Stream-K partition: work unit u = (z*nrb + rb)*nchu + cu (batch tile z, row
// block rb, unit cu of tc_unit_chunks consecutive chunks, nchu units per
// row); CTA i of P takes units [iW/P, (i+1)W/P).  A segment (z, rb) is cut
// into pieces, one per CTA that meets it.
__host__ __device__ __forceinline__ long tc_unit_lo(long i, long W, long P) { return i * W / P; }
// The CTA that holds unit u.
__host__ __device__ __forceinline__ long tc_unit_cta(long u, long W, long P) { return ((u + 1) * P - 1) / W; }
// Most pieces any segment of nchu units has (every CTA holds at least W/P units).
__host__ __device__ __forceinline__ int tc_max_pieces(long nchu, long W, long P) {
    const long q = W / P;
    return (int)((nchu + q - 1) / q + 1);
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
// One bulk copy completing on `bar` (whose expected bytes were set before).
__device__ __forceinline__ void tc_copy(uint32_t bar, uint32_t sdst, const void *gsrc, int bytes) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(sdst), "l"(gsrc), "r"(bytes), "r"(bar) : "memory");
}
__device__ __forceinline__ void tc_expect(uint32_t bar, int bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}
// The kernel that precedes k_mvm_tc on the stream (the gradient split) may
// let it start early (programmatic dependent launch); this waits until that
// kernel has completed and its writes are visible.  A no-op otherwise.
__device__ __forceinline__ void tc_wait_prior() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void tc_release_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

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
// consecutive 16-byte rows.  Also zeroes the stream-K arrival counters.
template <int N>
__global__ void __launch_bounds__(256)
k_gsplit(const float *__restrict__ g, long ngrad, int nbatch, long nch, int nz, char *__restrict__ gs,
         int *__restrict__ cnt, int ncnt) {
    tc_release_dependents();  // k_mvm_tc may start its M copies now
    const long item = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long i = item; i < ncnt; i += (long)gridDim.x * blockDim.x) cnt[i] = 0;  // stream-K arrival counters
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

__device__ __forceinline__ void cl_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cl_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

// Gradients -> kTcTermsFp8 E4M3 terms in per-(batch tile, chunk) [4N x 64]
// tiles, row t*N + n = term t of instance n, and each instance's scale
// exponent kexp[b].  One cluster of kSplitCta CTAs per live instance (grid
// (kSplitCta, nbatch)): each CTA takes the largest |g| over its share of the
// columns, the cluster combines them through distributed shared memory, and
// every CTA then writes the terms of its share (one thread per 16 columns).
// Dynamic shared memory: 64 bytes per 16-column group of the largest share
// when `stage` (the share is then read from HBM once).  Rows of padded
// instances and columns past ngrad are never written (the buffer is zeroed
// once).  Also zeroes the stream-K arrival counters.
template <int N>
__global__ void __cluster_dims__(kSplitCta, 1, 1) __launch_bounds__(256)
k_gsplit8(const float *__restrict__ g, long ngrad, long nch, int *__restrict__ kexp, char *__restrict__ gs,
          int *__restrict__ cnt, int ncnt, bool stage) {
    tc_release_dependents();  // k_mvm_tc may start its M copies now
    __shared__ float red[8];
    __shared__ float s_max;
    __shared__ int s_k;
    extern __shared__ float gsh[];
    const int part = blockIdx.x, b = blockIdx.y, z = b / N, n = b % N;
    {
        const long tid = ((long)b * kSplitCta + part) * blockDim.x + threadIdx.x;
        for (long i = tid; i < ncnt; i += (long)gridDim.y * kSplitCta * blockDim.x) cnt[i] = 0;
    }
    const long ngr = nch * 4;  // 16-column groups
    const long g0 = part * ngr / kSplitCta, g1 = (part + 1) * ngr / kSplitCta;
    const float *gb = g + (size_t)b * ngrad;
    float m = 0.f;
    const long e1 = g1 * 16 < ngrad ? g1 * 16 : ngrad;
    for (long e = g0 * 16 + threadIdx.x; e < g1 * 16; e += blockDim.x) {
        const float v = e < e1 ? gb[e] : 0.f;
        if (stage) gsh[e - g0 * 16] = v;
        m = fmaxf(m, fabsf(v));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, red[w]);
        s_max = m;
    }
    cl_arrive();
    cl_wait();  // every rank's maximum is in its shared memory
    if (threadIdx.x < 32) {
        float t = 0.f;
        if (threadIdx.x < kSplitCta) {
            const unsigned la = (unsigned)__cvta_generic_to_shared(&s_max);
            unsigned ra;
            asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(la), "r"((unsigned)threadIdx.x));
            asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(t) : "r"(ra) : "memory");
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = fmaxf(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) {
            s_k = tc_fp8_exp(__float_as_uint(t));
            if (part == 0) kexp[b] = s_k;
        }
    }
    __syncthreads();
    cl_arrive();  // done reading the other ranks
    const int k = s_k;
    for (long gi = g0 + threadIdx.x; gi < g1; gi += blockDim.x) {
        float v[16];
        if (stage) {
            const float4 *sp = reinterpret_cast<const float4 *>(gsh + (gi - g0) * 16);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float4 f = sp[e];
                v[4 * e] = f.x;
                v[4 * e + 1] = f.y;
                v[4 * e + 2] = f.z;
                v[4 * e + 3] = f.w;
            }
        } else {
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const long col = gi * 16 + e;
                v[e] = col < ngrad ? gb[col] : 0.f;
            }
        }
        char *tile = gs + ((size_t)z * nch + (gi >> 2)) * tc_b_bytes(N);
        const int kq = (int)(gi & 3);
#pragma unroll
        for (int t = 0; t < kTcTermsFp8; t++) {
            const float sc = tc_pow2(k - 4 * t), inv = tc_pow2(4 * t - k);
            uint32_t w[4];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const __nv_fp8x2_storage_t q = __nv_cvt_float2_to_fp8x2(
                    make_float2(v[2 * e] * inv, v[2 * e + 1] * inv), __NV_SATFINITE, __NV_E4M3);
                const float2 back = __half22float2(__half2(__nv_cvt_fp8x2_to_halfraw2(q, __NV_E4M3)));
                v[2 * e] -= sc * back.x;  // exact: power-of-two scale, residual below the value
                v[2 * e + 1] -= sc * back.y;
                if (e & 1) w[e >> 1] |= (uint32_t)q << 16;
                else w[e >> 1] = (uint32_t)q;
            }
            *reinterpret_cast<uint4 *>(tile + tc_fp8_off(t * N + n, kq * 16)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    cl_wait();  // no rank exits while another may still read its maximum
}

// Bounded parity wait that sleeps between polls (for threads off the
// critical path, so they do not compete with the copy and MMA threads for
// the mbarrier unit); at most about half a second.
__device__ __forceinline__ bool mbar_wait_sleep(uint32_t bar, uint32_t phase, const volatile int *abort) {
    for (int i = 0; i < (1 << 21); i++) {
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
        __nanosleep(200);
    }
    return false;
}

// Persistent stream-K GEMM.  grid: P CTAs (at most the resident count);
// block kTcThreads; dynamic shared memory tc_smem_bytes(DT, N).  CTA i
// streams units [iW/P, (i+1)W/P) (tc_unit_lo) through one ring of S stages
// that runs on across row blocks; each piece of a segment (z, rb) is
// accumulated in one of two TMEM accumulators and read out by the four
// epilogue warps while the MMAs of the next piece proceed.
//   Mt: pre-tiled M ([nrb][nch] tiles of tc_a_bytes(DT)); gs: the gradient
//   terms; kexp: FP8 scale exponents per instance; rscale: FP8 row scales.
// A segment met by one CTA is written to out directly.  Otherwise each piece
// goes to part[(seg*maxp + j)][N][128] (j = the piece's index in the
// segment), and the CTA that completes the segment (arrival counter cnt[seg])
// adds the pieces in index order, so the result does not depend on which
// CTA arrives last, and resets the counter.
template <int DT, int N>
__global__ void __launch_bounds__(kTcThreads)
k_mvm_tc(const char *__restrict__ Mt, const char *__restrict__ gs, const int *__restrict__ kexp,
         const float *__restrict__ rscale, int nrb, long nch, long W, int P, int maxp, float *__restrict__ part,
         int *__restrict__ cnt, float *__restrict__ out, int nact, int nbatch, int *__restrict__ err) {
    static_assert(N == 16 || N == 32 || N == 64, "batch tile");
    constexpr bool kFp8 = DT != MB_MVM_BF16;
    constexpr int ACC = tc_acc_cols(DT, N);
    constexpr int NCOL = tc_tmem_cols(DT, N);
    constexpr int S = tc_stages(DT, N);
    constexpr int U = tc_unit_chunks(DT);
    constexpr int AB = tc_a_bytes(DT), BB = tc_b_bytes(N), SB = U * (AB + BB);  // stage: U A tiles, then U B tiles
    constexpr uint32_t idesc = umma_idesc(DT, kFp8 ? kTcTermsFp8 * N : N);
    extern __shared__ __align__(128) char tcsm[];
    __shared__ __align__(8) uint64_t full[S], empty[S], tfull[2], tempty[2], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_mmas, s_units;
    __shared__ int s_last[2];
    __shared__ volatile int s_abort;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long nchu = (nch + U - 1) / U;  // units per segment
    const long ci = blockIdx.x;
    const long lo = tc_unit_lo(ci, W, P), hi = tc_unit_lo(ci + 1, W, P);
    const int nunit = (int)(hi - lo);
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
        for (int i = 0; i < 2; i++) {
            mbar_init(smem_addr(&tfull[i]), 1);
            mbar_init(smem_addr(&tempty[i]), 4);  // one arrival per epilogue warp
        }
        mbar_init(smem_addr(&done), 1);
        s_abort = 0;
        s_mmas = 0;
        s_units = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (warp == 0) {
        if (lane == 0) {  // copies: the ring runs on across segments
            auto unit = [&](int q, long &a_off, long &b_off, int &nc) {
                const long u = lo + q;
                const long seg = u / nchu, c = (u - seg * nchu) * U;
                const long z = seg / nrb, rb = seg - z * nrb;
                nc = (int)(nch - c < U ? nch - c : U);
                a_off = (rb * nch + c) * AB;
                b_off = (z * nch + c) * BB;
            };
            // the first stages' M tiles go out before the gradient terms exist
            // (M does not depend on the split kernel), their terms after it
            const int npre = nunit < S ? nunit : S;
            for (int q0 = 0; q0 < npre; q0++) {
                long ao, bo;
                int nc;
                unit(q0, ao, bo, nc);
                tc_expect(smem_addr(&full[q0]), nc * (AB + BB));
                tc_copy(smem_addr(&full[q0]), sbase + q0 * SB, Mt + ao, nc * AB);
            }
            tc_wait_prior();
            for (int q0 = 0; q0 < npre; q0++) {
                long ao, bo;
                int nc;
                unit(q0, ao, bo, nc);
                tc_copy(smem_addr(&full[q0]), sbase + q0 * SB + U * AB, gs + bo, nc * BB);
            }
            int q = npre;
            for (; q < nunit; q++) {
                const long u = lo + q;
                const long seg = u / nchu, c = (u - seg * nchu) * U;
                const long z = seg / nrb, rb = seg - z * nrb;
                const int nc = (int)(nch - c < U ? nch - c : U);  // consecutive tiles, one copy each side
                const int st = q % S;
                if (q >= S && !mbar_wait(smem_addr(&empty[st]), (uint32_t)((q / S - 1) & 1), &s_abort)) {
                    s_abort = 1;
                    break;
                }
                tc_load_stage(smem_addr(&full[st]), sbase + st * SB, Mt + ((size_t)rb * nch + c) * AB, nc * AB,
                              sbase + st * SB + U * AB, gs + ((size_t)z * nch + c) * BB, nc * BB);
            }
            // every copy this thread issued has landed before the CTA can exit
            for (int c = q - S < 0 ? 0 : q - S; c < q; c++) mbar_wait(smem_addr(&full[c % S]), (uint32_t)((c / S) & 1));
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {  // MMAs
            int q = 0, k = 0;
            long u = lo;
            bool ok = true;
            while (ok && u < hi) {
                const long seg = u / nchu, e = (seg + 1) * nchu < hi ? (seg + 1) * nchu : hi;
                const int buf = k & 1;
                // the epilogue has read this accumulator's previous piece
                if (k >= 2 && !mbar_wait(smem_addr(&tempty[buf]), (uint32_t)((k / 2 - 1) & 1), &s_abort)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(buf * ACC);
                for (long u0 = u; u < e; u++, q++) {
                    const int st = q % S;
                    if (!mbar_wait(smem_addr(&full[st]), (uint32_t)((q / S) & 1), &s_abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const long c = (u - seg * nchu) * U;
                    const int nc = (int)(nch - c < U ? nch - c : U);
                    for (int j = 0; j < nc; j++) {
                        const uint32_t a = sbase + st * SB + j * AB, b = sbase + st * SB + U * AB + j * BB;
                        if constexpr (kFp8)
                            tc_mma_chunk_fp8(acc, a, b, idesc, u == u0 && j == 0);
                        else
                            tc_mma_chunk(acc, a, b, N * kTcK * 2, idesc, u == u0 && j == 0);
                    }
                    tc_commit(smem_addr(&empty[st]));
                }
                if (!ok) break;
                tc_commit(smem_addr(&tfull[buf]));
                k++;
            }
            if (!ok) s_abort = 1;
            s_mmas = q;
            tc_commit(smem_addr(&done));  // tracks every MMA this thread issued
        }
        __syncwarp();
    } else {  // epilogue warps 2-5: warp w reads TMEM lanes 32(w%4).. = rows
        tc_wait_prior();  // the split kernel's exponents and zeroed counters
        const int qd = warp & 3, rl = qd * 32 + lane;
        const uint32_t tl = tmem + ((uint32_t)(qd * 32) << 16);
        int k = 0;
        long u = lo;
        while (u < hi) {
            const long seg = u / nchu, e = (seg + 1) * nchu < hi ? (seg + 1) * nchu : hi;
            const long z = seg / nrb, rb = seg - z * nrb;
            const int buf = k & 1;
            // one thread polls; the four warps wait for it on a named barrier,
            // which also makes the decision uniform
            const int okw = threadIdx.x == 64 ? (mbar_wait_sleep(smem_addr(&tfull[buf]), (uint32_t)((k / 2) & 1),
                                                                 &s_abort) ? 1 : 0) : 1;
            __syncwarp();
            int all_ok;
            asm volatile(
                "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\t"
                "bar.red.and.pred q, 1, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                : "=r"(all_ok) : "r"(okw) : "memory");
            if (!all_ok) {
                s_abort = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float y[N];
#pragma unroll
            for (int cc = 0; cc < N; cc += 16) {
                int ke[16];
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int b = (int)z * N + cc + j;
                    ke[j] = (kFp8 && b < nbatch) ? kexp[b] : 0;
                    y[cc + j] = 0.f;
                }
#pragma unroll
                for (int t = 0; t < (kFp8 ? kTcTermsFp8 : 1); t++) {
                    uint32_t r[16];
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                        "%15}, [%16];"
                        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                          "=r"(r[14]), "=r"(r[15])
                        : "r"(tl + (uint32_t)(buf * ACC + t * N + cc)));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        y[cc + j] += (kFp8 ? tc_pow2(ke[j] - 4 * t) : 1.f) * __uint_as_float(r[j]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_addr(&tempty[buf])) : "memory");
            // this piece's place in its segment
            const long i0 = tc_unit_cta(seg * nchu, W, P), i1 = tc_unit_cta((seg + 1) * nchu - 1, W, P);
            const int np = (int)(i1 - i0 + 1), j = (int)(ci - i0);
            const int row = (int)rb * kTcRows + rl;
            const float rs = (kFp8 && row < nact) ? rscale[row] : 1.f;
            if (np == 1) {
                if (row < nact)
#pragma unroll
                    for (int n = 0; n < N; n++) {
                        const int b = (int)z * N + n;
                        if (b < nbatch) out[(size_t)b * nact + row] = rs * y[n];
                    }
            } else {
                float *pp = part + ((size_t)seg * maxp + j) * N * kTcRows;
#pragma unroll
                for (int n = 0; n < N; n++) pp[n * kTcRows + rl] = y[n];
                __threadfence();
                asm volatile("bar.sync 1, 128;" ::: "memory");  // the epilogue warps' pieces are stored
                if (threadIdx.x == 64) s_last[buf] = atomicAdd(cnt + seg, 1) == np - 1;
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (s_last[buf]) {  // this CTA completes the segment: add the pieces in index order
                    __threadfence();
                    float sum[N];
#pragma unroll
                    for (int n = 0; n < N; n++) sum[n] = 0.f;
                    for (int jj = 0; jj < np; jj++) {
                        const float *qp = part + ((size_t)seg * maxp + jj) * N * kTcRows;
#pragma unroll
                        for (int n = 0; n < N; n++) sum[n] += __ldcg(qp + n * kTcRows + rl);
                    }
                    if (row < nact)
#pragma unroll
                        for (int n = 0; n < N; n++) {
                            const int b = (int)z * N + n;
                            if (b < nbatch) out[(size_t)b * nact + row] = rs * sum[n];
                        }
                    if (threadIdx.x == 64) cnt[seg] = 0;
                }
            }
            u = e;
            k++;
        }
        if (threadIdx.x == 64) s_units = (int)(u - lo);
    }
    // one thread waits for the MMAs (bounded, twice before the accumulators
    // are freed); the rest of the CTA waits at the barrier
    bool bad = false;
    if (threadIdx.x == 0) {
        bad = !mbar_wait_sleep(smem_addr(&done), 0, nullptr);
        if (bad) mbar_wait_sleep(smem_addr(&done), 0, nullptr);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    const bool skip = __syncthreads_or(bad) || s_abort || s_mmas < nunit || s_units < nunit;
    if (skip && threadIdx.x == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(NCOL) : "memory");
}

}  // namespace mb
