// Batched control-matrix MVM on the 5th-generation tensor cores (tcgen05).
//
// For nbatch instances sharing one BF16 or FP8 control matrix the MVM is a
// GEMM: part[ks][b][row] = sum_{k in slab ks} M[row][k] g[b][k], with M the
// A operand (UMMA M = 128 rows) and the gradients the B operand (UMMA N = the
// batch tile), accumulated in FP32 in tensor memory.
//
// Layout in HBM.  M is stored pre-tiled: tile (row block rb, chunk c) holds
// rows 128rb.. and columns 64c.. contiguously, already in the order the
// tensor core reads from shared memory (K-major, no swizzle: 8x16-byte core
// matrices, core matrix (r/8, k/8) at ((r/8)*8 + k/8)*128 bytes, row r%8 at
// 16*(r%8)).  A BF16 tile is 16 KB; an FP8 tile is 8 KB in an order whose
// 16-byte rows widen to two BF16 core-matrix rows (tc_fp8_off).  The
// gradients are split once per call by k_gsplit into two BF16 terms
// g = hi + lo (lo the BF16 rounding of g - hi), 16 significant bits: each
// product carries a relative error of at most 2^-17 from g, 500 times below
// the BF16 storage rounding of M (2^-8) and further below FP8's; they are
// stored per (batch tile, chunk) as two [N x 64] tiles in the same
// core-matrix order.  Every pipeline stage is therefore two contiguous bulk
// copies (cp.async.bulk, completing on an mbarrier by byte count): no tensor
// map, no per-element address arithmetic, no shared-memory bank conflicts.
//
// CTA (rb, ks, z): 160 threads (5 warps), 128 rows x one K slab x one batch
// tile, with warp roles that meet only on mbarriers:
//   warp 0, lane 0: copies.  Keeps all S stages in flight; a stage is
//     refilled as soon as the MMAs that read it completed ("empty").
//   warp 1, lane 0: MMAs.  Per 64-column chunk, 4 K-steps x 2 terms of
//     tcgen05.mma (M=128, N = batch tile, K=16) into TMEM, committed to the
//     stage's "empty" barrier (and, FP8, to the widened tile's "free").
//   warps 2-4 (FP8 only): widen the stage's FP8 tile to BF16 (exact) into one
//     of two shared-memory tiles and arrive on its "ready" barrier.
// The epilogue reads the accumulators with tcgen05.ld (warps 1-4; warp w
// reaches TMEM lanes 32(w%4).. = rows) and writes the split-K partials.
//
// Every mbarrier wait is bounded.  On a timeout a thread raises the CTA's
// abort flag, every role stops issuing, the copy thread waits (bounded) for
// the copies it issued, all threads wait (bounded) for the MMAs issued, and
// the tensor memory is still freed; the error flag tells the host.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mb {

constexpr int kTcRows = 128;     // UMMA M
constexpr int kTcK = 64;         // columns per chunk (4 MMAs of K=16)
constexpr int kTcThreads = 160;  // copy warp, MMA warp, 3 widening warps (4 epilogue warps)
constexpr int kTcWiden = 96;     // threads of the widening warps
constexpr int kTcTerms = 2;      // BF16 terms of the gradients
constexpr int kTcTileBf16 = kTcRows * kTcK * 2;  // bytes of a BF16 M tile
constexpr int kTcTileFp8 = kTcRows * kTcK;       // bytes of an FP8 M tile

__host__ __device__ constexpr int tc_a_bytes(int dt) { return dt == MB_MVM_BF16 ? kTcTileBf16 : kTcTileFp8; }
__host__ __device__ constexpr int tc_b_bytes(int n) { return kTcTerms * n * kTcK * 2; }
// Pipeline depth: batch tiles of 16 and 32 keep two CTAs per SM (about
// 110 KB each); the 64 tile runs one CTA per SM with a deeper ring.
__host__ __device__ constexpr int tc_stages(int dt, int n) {
    return n <= 16 ? 5 : n <= 32 ? 4 : (dt == MB_MVM_BF16 ? 5 : 6);
}
__host__ __device__ constexpr int tc_smem_bytes(int dt, int n) {
    return tc_stages(dt, n) * (tc_a_bytes(dt) + tc_b_bytes(n)) + (dt == MB_MVM_BF16 ? 0 : 2 * kTcTileBf16);
}

// Byte offset of the 16-byte row holding columns 8*kgrp.. of row r in a
// BF16 [rows x 64] K-major core-matrix tile.
__host__ __device__ __forceinline__ uint32_t tile_off(int r, int kgrp) {
    return (uint32_t)(((r >> 3) * 8 + kgrp) * 128 + (r & 7) * 16);
}
// Byte offset of element (r, k) in an FP8 [128 x 64] tile: 16-byte row
// ((r/8)*4 + k/16)*8 + r%8 holds columns 16(k/16).. of row r, which widen
// to BF16 core-matrix rows (r, 2(k/16)) and (r, 2(k/16)+1).
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

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major,
// M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
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

// Widen one FP8 tile (shared) to a BF16 core-matrix tile (shared): item i is
// the 16-byte FP8 row i, which lands in two BF16 rows of the same row r.
// Eight consecutive threads write eight different 16-byte rows of one
// 128-byte core matrix, so the stores are conflict-free.
__device__ __forceinline__ void tc_widen_fp8(const char *raw, char *tile, int tid) {
    for (int i = tid; i < kTcTileFp8 / 16; i += kTcWiden) {
        const int r = (i >> 5) * 8 + (i & 7), j = (i >> 3) & 3;
        const uint4 q = *reinterpret_cast<const uint4 *>(raw + i * 16);
        const __nv_fp8x2_e4m3 *h = reinterpret_cast<const __nv_fp8x2_e4m3 *>(&q);
        uint32_t w[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const float2 f = static_cast<float2>(h[e]);
            const __nv_bfloat162 b = __floats2bfloat162_rn(f.x, f.y);  // exact: E4M3 fits BF16
            w[e] = *reinterpret_cast<const uint32_t *>(&b);
        }
        *reinterpret_cast<uint4 *>(tile + tile_off(r, 2 * j)) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4 *>(tile + tile_off(r, 2 * j + 1)) = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// grid: (row blocks, K slabs, batch tiles); block kTcThreads; dynamic shared
// memory tc_smem_bytes(DT, N).  Mt: pre-tiled M ([row blocks][nch] tiles of
// tc_a_bytes(DT)); gs: k_gsplit's output; each slab is `cps` chunks.
template <int DT, int N>
__global__ void __launch_bounds__(kTcThreads)
k_mvm_tc(const char *__restrict__ Mt, const char *__restrict__ gs, long nch, int cps, float *__restrict__ part,
         int nact, int nbatch, int *__restrict__ err) {
    static_assert(N == 16 || N == 32 || N == 64, "batch tile");
    constexpr int NCOL = N < 32 ? 32 : N;  // TMEM columns (power of 2, >= 32)
    constexpr int S = tc_stages(DT, N);
    constexpr int AB = tc_a_bytes(DT), BB = tc_b_bytes(N), SB = AB + BB;
    constexpr bool kWiden = DT != MB_MVM_BF16;
    constexpr uint32_t idesc = umma_idesc_bf16(N);
    extern __shared__ __align__(128) char tcsm[];
    __shared__ __align__(8) uint64_t full[S], empty[S], ready[2], tfree[2], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_mmas;
    __shared__ volatile int s_abort;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rb = blockIdx.x, ks = blockIdx.y, z = blockIdx.z;
    const long c0 = (long)ks * cps;
    const int nchunk = (int)((nch - c0) < cps ? (nch - c0) : cps);
    const char *ga = Mt + ((size_t)rb * nch + c0) * AB;
    const char *gb = gs + ((size_t)z * nch + c0) * BB;
    char *widen = tcsm + S * SB;  // FP8 only: two BF16 tiles
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
            mbar_init(smem_addr(&ready[i]), kTcWiden);
            mbar_init(smem_addr(&tfree[i]), 1);
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
                if (kWiden && !mbar_wait(smem_addr(&ready[ch & 1]), (uint32_t)((ch >> 1) & 1), &s_abort)) {
                    s_abort = 1;
                    break;
                }
                if (!mbar_wait(smem_addr(&full[st]), (uint32_t)((ch / S) & 1), &s_abort)) {
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t abase = kWiden ? smem_addr(widen + (ch & 1) * kTcTileBf16) : sbase + st * SB;
                tc_mma_chunk(tmem, abase, sbase + st * SB + AB, N * kTcK * 2, idesc, ch == 0);
                tc_commit(smem_addr(&empty[st]));
                if (kWiden) tc_commit(smem_addr(&tfree[ch & 1]));
                mmas = ch + 1;
            }
            s_mmas = mmas;
            tc_commit(smem_addr(&done));  // tracks every MMA this thread issued
        }
        __syncwarp();
    } else if (kWiden) {  // widening warps
        const int tid = threadIdx.x - 64;
        for (int ch = 0; ch < nchunk; ch++) {
            // one lane per warp polls the barriers; the others wait at the
            // shuffle instead of spinning on the mbarrier unit
            int ok = 1;
            if (lane == 0) {
                ok = mbar_wait(smem_addr(&full[ch % S]), (uint32_t)((ch / S) & 1), &s_abort);
                // the MMAs of chunk ch-2 (the last reader of this BF16 tile) completed
                if (ok && ch >= 2) ok = mbar_wait(smem_addr(&tfree[ch & 1]), (uint32_t)(((ch - 2) >> 1) & 1), &s_abort);
                if (!ok) s_abort = 1;
            }
            if (!__shfl_sync(0xffffffffu, ok, 0)) break;
            tc_widen_fp8(tcsm + (ch % S) * SB, widen + (ch & 1) * kTcTileBf16, tid);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_addr(&ready[ch & 1])) : "memory");
        }
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
    // epilogue: warps 1-4; warp w reads TMEM lanes 32(w%4).. (rows), N columns (instances)
    if (!skip && nchunk > 0 && warp >= 1) {
        const int q = warp & 3;
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16);
        const int row = rb * kTcRows + q * 32 + lane;
#pragma unroll
        for (int cc = 0; cc < N; cc += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr + (uint32_t)cc));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < nact)
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int b = z * N + cc + j;
                    if (b < nbatch) part[((size_t)ks * nbatch + b) * nact + row] = __uint_as_float(r[j]);
                }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(NCOL) : "memory");
}

}  // namespace mb
