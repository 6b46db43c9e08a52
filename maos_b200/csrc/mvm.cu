// Control-matrix MVM: a = M g for a batch of instances sharing M
// (gpu_recon_mvm, cuda/gpu.h:57; curecon_t::mvm cuda/recon.cu:345, which is a
// cuBLAS sgemv in the reference, cuda/solve.h:131).
//
// M is stored row-major [nact][ldm] (ldm = ngrad rounded up to the K tile) in
// FP32, BF16, or FP8-E4M3 with one FP32 scale per row; accumulation is FP32.
// A BF16 or FP8 matrix installed for batches of 4 or more is stored instead
// in the tensor-core tile order of mvm_tc.cuh and multiplied there.
// The kernel is split-K: CTA (rt, ks) multiplies a tile of kRows rows by a
// kK-column slab, with that slab of every instance's gradients staged in
// shared memory, and writes per-split partial sums; a second kernel adds the
// splits in fixed order and applies the row scale (deterministic, no atomics).
// Each warp streams rows with 16-byte vector loads, so M is read exactly once.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "mvm_tc.cuh"

namespace mb {

constexpr int kK = 2048;       // columns per split
constexpr int kRows = 32;      // rows per CTA (4 per warp)
constexpr int kMvmThreads = 256;
constexpr int kMaxBatch = 16;  // instances per launch pass

template <int DT>
struct Elem;
template <>
struct Elem<MB_MVM_F32> {
    using T = float;
    static constexpr int kVec = 4;  // elements per 16 bytes
    __device__ static void from_raw(const uint4 &r, float *v) {
        v[0] = __uint_as_float(r.x); v[1] = __uint_as_float(r.y);
        v[2] = __uint_as_float(r.z); v[3] = __uint_as_float(r.w);
    }
    __device__ static void load(const T *p, float *v) {
        const float4 q = *reinterpret_cast<const float4 *>(p);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    }
};
template <>
struct Elem<MB_MVM_BF16> {
    using T = __nv_bfloat16;
    static constexpr int kVec = 8;
    __device__ static void from_raw(const uint4 &q, float *v) {
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 f = __bfloat1622float2(h[i]);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    }
    __device__ static void load(const T *p, float *v) {
        const uint4 q = *reinterpret_cast<const uint4 *>(p);
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 f = __bfloat1622float2(h[i]);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    }
};
template <>
struct Elem<MB_MVM_FP8> {
    using T = __nv_fp8_e4m3;
    static constexpr int kVec = 16;
    __device__ static void from_raw(const uint4 &q, float *v) {
        const __nv_fp8x2_e4m3 *h = reinterpret_cast<const __nv_fp8x2_e4m3 *>(&q);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const float2 f = static_cast<float2>(h[i]);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    }
    __device__ static void load(const T *p, float *v) {
        const uint4 q = *reinterpret_cast<const uint4 *>(p);
        const __nv_fp8x2_e4m3 *h = reinterpret_cast<const __nv_fp8x2_e4m3 *>(&q);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const float2 f = static_cast<float2>(h[i]);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    }
};

// part[(ks*nbatch + b)*nact + row] = sum over this K slab of M[row][k] g[b][k]
template <int DT, int NB>
__global__ void __launch_bounds__(kMvmThreads)
k_mvm_split(const typename Elem<DT>::T *__restrict__ M, long ldm, const float *__restrict__ g,
            long ngrad, float *__restrict__ part, int nact, int nbatch, int b0) {
    using E = Elem<DT>;
    constexpr int V = E::kVec;
    extern __shared__ float sg[];  // [NB][kK]
    const int ks = blockIdx.y;
    const long k0 = (long)ks * kK;
    const int kn = (int)((ngrad - k0) < kK ? (ngrad - k0) : kK);
    for (int i = threadIdx.x; i < NB * kK; i += blockDim.x) {
        const int b = i / kK, k = i - b * kK;
        sg[i] = (b0 + b < nbatch && k < kn) ? g[(size_t)(b0 + b) * ngrad + k0 + k] : 0.f;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kRowsPerWarp = kRows / (kMvmThreads / 32);
    // small batches: a warp carries RW rows at once, so every lane keeps RW
    // independent 16-byte loads in flight and each staged gradient value
    // serves RW rows
    constexpr int RW = NB <= 2 ? kRowsPerWarp : 1;
    for (int rr = 0; rr < kRowsPerWarp; rr += RW) {
        const int row0 = blockIdx.x * kRows + warp * kRowsPerWarp + rr;
        if (row0 >= nact) break;
        const typename E::T *mrow[RW];
        bool live[RW];
#pragma unroll
        for (int q = 0; q < RW; q++) {
            live[q] = row0 + q < nact;
            mrow[q] = M + (size_t)(live[q] ? row0 + q : row0) * ldm + k0;
        }
        float acc[RW][NB];
#pragma unroll
        for (int q = 0; q < RW; q++)
#pragma unroll
            for (int b = 0; b < NB; b++) acc[q][b] = 0.f;
        // lanes stride by V elements; the slab is a multiple of 32*V elements
        for (int c = lane * V; c < kK; c += 32 * V) {
            float v[RW][V];
#pragma unroll
            for (int q = 0; q < RW; q++) E::load(mrow[q] + c, v[q]);
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const float4 *gb = reinterpret_cast<const float4 *>(sg + b * kK + c);
#pragma unroll
                for (int e4 = 0; e4 < V / 4; e4++) {
                    const float4 g4 = gb[e4];
#pragma unroll
                    for (int q = 0; q < RW; q++)
                        acc[q][b] += v[q][4 * e4] * g4.x + v[q][4 * e4 + 1] * g4.y + v[q][4 * e4 + 2] * g4.z +
                                     v[q][4 * e4 + 3] * g4.w;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < RW; q++)
#pragma unroll
            for (int b = 0; b < NB; b++) {
                float t = acc[q][b];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                if (lane == 0 && live[q] && b0 + b < nbatch)
                    part[((size_t)ks * nbatch + b0 + b) * nact + row0 + q] = t;
            }
    }
}

// Batched form (NB >= 4): a thread owns kRT rows and all NB instances
// (kRT x NB accumulators in registers).  Each step reads 16 bytes of each of
// its rows (all kRT loads issued together) and, per element, one gradient
// vector of NB values from shared memory as a broadcast (every lane reads the
// same address) that feeds kRT x NB FMAs.
// part[(ks*nbatch + b)*nact + row]; grid: (ceil(nact/(kRowThreads*kRT)), nks)
constexpr int kRT = 4;
constexpr int kRowThreads = 128;

template <int DT, int NB>
__global__ void __launch_bounds__(kRowThreads)
k_mvm_rows(const typename Elem<DT>::T *__restrict__ M, long ldm, const float *__restrict__ g, long ngrad,
           float *__restrict__ part, int nact, int nbatch, int b0) {
    static_assert(NB % 4 == 0, "batched form takes multiples of 4 instances");
    using E = Elem<DT>;
    constexpr int V = E::kVec;
    extern __shared__ float sg[];  // [kK][NB]: the NB values of one column are adjacent
    const int ks = blockIdx.y;
    const long k0 = (long)ks * kK;
    const int kn = (int)((ngrad - k0) < kK ? (ngrad - k0) : kK);
    for (int i = threadIdx.x; i < NB * kK; i += blockDim.x) {
        const int b = i / kK, k = i - b * kK;
        sg[k * NB + b] = (b0 + b < nbatch && k < kn) ? g[(size_t)(b0 + b) * ngrad + k0 + k] : 0.f;
    }
    __syncthreads();
    // rows r0 + q*kRowThreads: the lanes of a warp own consecutive rows
    const int r0 = blockIdx.x * kRowThreads * kRT + threadIdx.x;
    const typename E::T *mrow[kRT];
    bool live[kRT];
#pragma unroll
    for (int q = 0; q < kRT; q++) {
        const int row = r0 + q * kRowThreads;
        live[q] = row < nact;
        mrow[q] = M + (size_t)(live[q] ? row : 0) * ldm + k0;
    }
    float acc[kRT][NB];
#pragma unroll
    for (int q = 0; q < kRT; q++)
#pragma unroll
        for (int b = 0; b < NB; b++) acc[q][b] = 0.f;
    for (int c = 0; c < kK; c += V) {
        uint4 raw[kRT];
#pragma unroll
        for (int q = 0; q < kRT; q++) raw[q] = *reinterpret_cast<const uint4 *>(mrow[q] + c);
        float v[kRT][V];
#pragma unroll
        for (int q = 0; q < kRT; q++) E::from_raw(raw[q], v[q]);
#pragma unroll
        for (int e = 0; e < V; e++) {
            const float4 *gc = reinterpret_cast<const float4 *>(sg + (c + e) * NB);
#pragma unroll
            for (int u = 0; u < NB / 4; u++) {
                const float4 g4 = gc[u];
#pragma unroll
                for (int q = 0; q < kRT; q++) {
                    acc[q][4 * u] += v[q][e] * g4.x;
                    acc[q][4 * u + 1] += v[q][e] * g4.y;
                    acc[q][4 * u + 2] += v[q][e] * g4.z;
                    acc[q][4 * u + 3] += v[q][e] * g4.w;
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kRT; q++)
        if (live[q])
#pragma unroll
            for (int b = 0; b < NB; b++)
                if (b0 + b < nbatch) part[((size_t)ks * nbatch + b0 + b) * nact + r0 + q * kRowThreads] = acc[q][b];
}

// out[b][row] = scale[row] * sum_ks part[ks][b][row]
__global__ void k_mvm_reduce(const float *__restrict__ part, const float *__restrict__ scale,
                             float *__restrict__ out, int nact, int nbatch, int nks) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nact * nbatch) return;
    const int b = (int)(t / nact), row = (int)(t - (long)b * nact);
    float s = 0.f;
    for (int k = 0; k < nks; k++) s += part[((size_t)k * nbatch + b) * nact + row];
    out[(size_t)b * nact + row] = scale ? s * scale[row] : s;
}

struct Mvm {
    int dtype = MB_MVM_F32;
    int nact = 0, nbatch = 1, nks = 0;
    long ngrad = 0, ldm = 0;
    bool tiled = false;  // m holds the tensor-core tiles (mvm_tc.cuh) instead of rows
    long nch = 0;        // 64-column chunks per row when tiled (ldm / 64)
    DevBuf<unsigned char> m;  // raw storage
    DevBuf<unsigned char> gs;  // tiled: the gradients' BF16 or E4M3 terms (k_gsplit, k_gsplit8)
    DevBuf<int> kexp;          // tiled FP8: each instance's scale exponent (k_gsplit8)
    DevBuf<int> cnt;           // tiled: stream-K arrival counter per (batch tile, row block)
    DevBuf<float> scale, part, g, out;
    DevBuf<int> err;  // set when a tensor-core MMA wait timed out
    cudaStream_t stream = nullptr;
    ~Mvm() {
        if (stream) cudaStreamDestroy(stream);
    }

    template <int DT, int NB>
    void launch_t(const float *dg, float *dout, cudaStream_t s) {
        const size_t smem = (size_t)NB * kK * sizeof(float);
        static bool attr = false;
        auto kern = [] {
            if constexpr (NB >= 4) return k_mvm_rows<DT, NB>;
            else return k_mvm_split<DT, NB>;
        }();
        if (!attr) {
            MB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr = true;
        }
        const dim3 grid(NB >= 4 ? (nact + kRowThreads * kRT - 1) / (kRowThreads * kRT) : (nact + kRows - 1) / kRows,
                        nks);
        const int threads = NB >= 4 ? kRowThreads : kMvmThreads;
        for (int b0 = 0; b0 < nbatch; b0 += NB) {
            kern<<<grid, threads, smem, s>>>(reinterpret_cast<const typename Elem<DT>::T *>(m.p), ldm, dg, ngrad,
                                            part.p, nact, nbatch, b0);
            MB_CHECK_LAUNCH();
        }
        const long n = (long)nact * nbatch;
        k_mvm_reduce<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(part.p, dtype == MB_MVM_FP8 ? scale.p : nullptr,
                                                                dout, nact, nbatch, nks);
        MB_CHECK_LAUNCH();
    }
    // Batches of 4 or more with BF16 or FP8 storage: the GEMM on the tensor
    // cores (mvm_tc.cuh); MAOS_B200_MVM_TC=0 (read once) keeps the FMA kernels.
    static bool tc_enabled() {
        static const bool on = [] {
            const char *e = std::getenv("MAOS_B200_MVM_TC");
            return !(e && e[0] == '0');
        }();
        return on;
    }
    // Stream-K layout of the tensor-core path, fixed at creation.
    int tc_nrb = 0, tc_P = 0, tc_maxp = 0;
    long tc_W = 0;
    template <int DT, int N>
    static int tc_resident() {  // CTAs of k_mvm_tc<DT, N> resident on the device
        static int n = 0;
        if (!n) {
            constexpr int smem = tc_smem_bytes(DT, N);
            MB_CUDA_TRY(cudaFuncSetAttribute(k_mvm_tc<DT, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            // all of the unified L1 as shared memory, so that two rings fit an SM
            // (the occupancy query and the launch both follow this preference)
            MB_CUDA_TRY(cudaFuncSetAttribute(k_mvm_tc<DT, N>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                             (int)cudaSharedmemCarveoutMaxShared));
            // CTAs per SM from the kernel's own limits (shared memory, registers,
            // threads); a persistent CTA never waits for another, so a count
            // above what is resident only costs a second wave
            int dev = 0, nsm = 0, smsm = 0, rsv = 0, thr = 0;
            MB_CUDA_TRY(cudaGetDevice(&dev));
            MB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            MB_CUDA_TRY(cudaDeviceGetAttribute(&smsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
            MB_CUDA_TRY(cudaDeviceGetAttribute(&rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
            MB_CUDA_TRY(cudaDeviceGetAttribute(&thr, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
            cudaFuncAttributes fa{};
            MB_CUDA_TRY(cudaFuncGetAttributes(&fa, k_mvm_tc<DT, N>));
            const long regs = (long)((fa.numRegs * 32 + 255) / 256 * 256) * (kTcThreads / 32);
            const long by_smem = smsm / ((long)smem + (long)fa.sharedSizeBytes + rsv);
            const long by_regs = 65536 / std::max<long>(regs, 1);
            const long occ = std::max<long>(1, std::min({by_smem, by_regs, (long)(thr / kTcThreads), 2L}));
            n = (int)(nsm * occ);
        }
        return n;
    }
    template <int DT, int N>
    void plan_tc() {
        const int nz = (nbatch + N - 1) / N;
        tc_nrb = (nact + kTcRows - 1) / kTcRows;
        const long nchu = (nch + tc_unit_chunks(DT) - 1) / tc_unit_chunks(DT);
        tc_W = (long)nz * tc_nrb * nchu;
        tc_P = (int)std::min<long>(tc_resident<DT, N>(), tc_W);
        tc_maxp = tc_max_pieces(nchu, tc_W, tc_P);
        gs.alloc((size_t)nz * nch * tc_b_bytes(N));
        gs.zero_async(stream);
        if (DT == MB_MVM_FP8) kexp.alloc((size_t)nz * N);
        part.alloc((size_t)nz * tc_nrb * tc_maxp * N * kTcRows);
        cnt.alloc((size_t)nz * tc_nrb);
        cnt.zero_async(stream);
    }
    template <int DT>
    void plan_tc_dt() {
        if (nbatch <= 16) plan_tc<DT, 16>();
        else if (nbatch <= 32) plan_tc<DT, 32>();
        else plan_tc<DT, 64>();
    }
    template <int DT, int N>
    void launch_tc(const float *dg, float *dout, cudaStream_t s) {
        constexpr int smem = tc_smem_bytes(DT, N);
        const int nz = (nbatch + N - 1) / N, ncnt = nz * tc_nrb;
        if constexpr (DT == MB_MVM_BF16) {
            const long items = (long)nz * nch * N * 8;
            k_gsplit<N><<<(unsigned)((items + 255) / 256), 256, 0, s>>>(dg, ngrad, nbatch, nch, nz,
                                                                        reinterpret_cast<char *>(gs.p), cnt.p, ncnt);
        } else {
            const long share = (nch * 4 + kSplitCta - 1) / kSplitCta * 64;  // bytes of the largest share
            const bool stage = share <= 96 * 1024;
            static bool attr = false;
            if (!attr) {
                MB_CUDA_TRY(cudaFuncSetAttribute(k_gsplit8<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
                attr = true;
            }
            k_gsplit8<N><<<dim3(kSplitCta, nbatch), 256, stage ? (size_t)share : 0, s>>>(
                dg, ngrad, nch, kexp.p, reinterpret_cast<char *>(gs.p), cnt.p, ncnt, stage);
        }
        MB_CHECK_LAUNCH();
        // programmatic dependent launch: the GEMM's CTAs start (TMEM, barriers,
        // the first stages' M tiles) while the split kernel still runs, and
        // wait for its output where they read it (griddepcontrol.wait)
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(tc_P);
        cfg.blockDim = dim3(kTcThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        MB_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_mvm_tc<DT, N>, reinterpret_cast<const char *>(m.p),
                                       reinterpret_cast<const char *>(gs.p), (const int *)kexp.p,
                                       (const float *)(DT == MB_MVM_FP8 ? scale.p : nullptr), tc_nrb, nch, tc_W,
                                       tc_P, tc_maxp, part.p, cnt.p, dout, nact, nbatch, err.p));
    }
    template <int DT>
    void launch_dt(const float *dg, float *dout, cudaStream_t s) {
        if constexpr (DT != MB_MVM_F32) {
            if (tiled) {
                if (nbatch <= 16) launch_tc<DT, 16>(dg, dout, s);
                else if (nbatch <= 32) launch_tc<DT, 32>(dg, dout, s);
                else launch_tc<DT, 64>(dg, dout, s);
                return;
            }
        }
        if (nbatch == 1) launch_t<DT, 1>(dg, dout, s);
        else if (nbatch == 2) launch_t<DT, 2>(dg, dout, s);
        else if (nbatch <= 4) launch_t<DT, 4>(dg, dout, s);
        else if (nbatch <= 8) launch_t<DT, 8>(dg, dout, s);
        else launch_t<DT, kMaxBatch>(dg, dout, s);
    }
    void apply(const float *dg, float *dout, cudaStream_t s) {
        switch (dtype) {
            case MB_MVM_F32: launch_dt<MB_MVM_F32>(dg, dout, s); break;
            case MB_MVM_BF16: launch_dt<MB_MVM_BF16>(dg, dout, s); break;
            default: launch_dt<MB_MVM_FP8>(dg, dout, s); break;
        }
    }
};

}  // namespace mb

struct mb_mvm {
    mb::Mvm M;
};

// ---------------------------------------------------------------------------
// Allocation-free MVM for callers that must not allocate device memory.
//
// The split-K partial sums live in one file-scope device array of
// MB_NOALLOC_MAX_PARTIALS floats (4 MiB), which every GPU that loads this
// library holds until the process exits.  Host code cannot pass the array's
// name to a kernel (on the host it is only a stand-in symbol), so the first
// call on each device looks up its device address with cudaGetSymbolAddress,
// with that device current, and keeps it.  Every partial that the reduction
// reads is written by the same call first, so nothing needs clearing between
// calls; calls that overlap on the GPU share the array and race.
// ---------------------------------------------------------------------------
static __device__ __align__(256) float g_noalloc_partials[MB_NOALLOC_MAX_PARTIALS];

namespace mb {

// Same split-K product as k_mvm_split for an FP32 row-major M with any
// ngrad: full 16-byte vectors up to the last multiple of 4 in the slab, then
// a scalar tail.  ldm must be a multiple of 4 and M 16-byte aligned.
template <int NB>
__global__ void __launch_bounds__(kMvmThreads)
k_mvm_split_f32_ragged(const float *__restrict__ M, long ldm, const float *__restrict__ g,
                       long ngrad, float *__restrict__ part, int nact, int nbatch, int b0) {
    extern __shared__ float sg[];  // [NB][kK]
    const int ks = blockIdx.y;
    const long k0 = (long)ks * kK;
    const int kn = (int)((ngrad - k0) < kK ? (ngrad - k0) : kK);
    const int kn4 = kn & ~3;
    for (int i = threadIdx.x; i < NB * kK; i += blockDim.x) {
        const int b = i / kK, k = i - b * kK;
        sg[i] = (b0 + b < nbatch && k < kn) ? g[(size_t)(b0 + b) * ngrad + k0 + k] : 0.f;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kRowsPerWarp = kRows / (kMvmThreads / 32);
    for (int rr = 0; rr < kRowsPerWarp; rr++) {
        const int row = blockIdx.x * kRows + warp * kRowsPerWarp + rr;
        if (row >= nact) break;
        const float *mrow = M + (size_t)row * ldm + k0;
        float acc[NB];
#pragma unroll
        for (int b = 0; b < NB; b++) acc[b] = 0.f;
        for (int c = lane * 4; c < kn4; c += 128) {
            const float4 v = *reinterpret_cast<const float4 *>(mrow + c);
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const float4 q = *reinterpret_cast<const float4 *>(sg + b * kK + c);
                acc[b] += v.x * q.x + v.y * q.y + v.z * q.z + v.w * q.w;
            }
        }
        for (int c = kn4 + lane; c < kn; c += 32) {
            const float v = mrow[c];
#pragma unroll
            for (int b = 0; b < NB; b++) acc[b] += v * sg[b * kK + c];
        }
#pragma unroll
        for (int b = 0; b < NB; b++) {
            float t = acc[b];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0 && b0 + b < nbatch) part[((size_t)ks * nbatch + b0 + b) * nact + row] = t;
        }
    }
}

static std::mutex g_noalloc_mu;
static float *g_noalloc_ptr[256] = {};

// Once per device, with that device current: the scratch array's device
// address and the shared-memory opt-in of the kernel variants.
static float *noalloc_scratch(int dev) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        float *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_partials);
        if (e != cudaSuccess || !ptr) {
            set_error("cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
            throw CudaError{MB_ECUDA};
        }
        MB_CUDA_TRY(cudaFuncSetAttribute(k_mvm_split_f32_ragged<1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 1 * kK * 4));
        MB_CUDA_TRY(cudaFuncSetAttribute(k_mvm_split_f32_ragged<4>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * kK * 4));
        MB_CUDA_TRY(cudaFuncSetAttribute(k_mvm_split_f32_ragged<8>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * kK * 4));
        g_noalloc_ptr[dev] = ptr;
    }
    return g_noalloc_ptr[dev];
}

template <int NB>
static void noalloc_launch(const float *M, long ldm, const float *g, long ngrad, float *part, int nact,
                           int nbatch, int nks, cudaStream_t s) {
    const dim3 grid((nact + kRows - 1) / kRows, nks);
    for (int b0 = 0; b0 < nbatch; b0 += NB) {
        k_mvm_split_f32_ragged<NB><<<grid, kMvmThreads, (size_t)NB * kK * 4, s>>>(M, ldm, g, ngrad, part, nact,
                                                                                  nbatch, b0);
        MB_CHECK_LAUNCH();
    }
}

}  // namespace mb

extern "C" {

int mb_mvm_create(const double *Mcol, long nact, long ngrad, int dtype, int nbatch, mb_mvm **out) {
    if (!out || !Mcol || nact <= 0 || ngrad <= 0 || nbatch < 1 || nact > (1L << 30)) {
        mb::set_error("mb_mvm_create: invalid arguments");
        return MB_EINVAL;
    }
    if (dtype != MB_MVM_F32 && dtype != MB_MVM_BF16 && dtype != MB_MVM_FP8) {
        mb::set_error("mb_mvm_create: unknown dtype %d", dtype);
        return MB_EINVAL;
    }
    *out = nullptr;
    mb_mvm *h = new (std::nothrow) mb_mvm();
    if (!h) return MB_ENOMEM;
    try {
        mb::Mvm &V = h->M;
        V.dtype = dtype;
        V.nact = (int)nact;
        V.ngrad = ngrad;
        V.nbatch = nbatch;
        V.nks = (int)((ngrad + mb::kK - 1) / mb::kK);
        V.ldm = (long)V.nks * mb::kK;
        MB_CUDA_TRY(cudaStreamCreateWithFlags(&V.stream, cudaStreamNonBlocking));
        // Batches of 4 or more with BF16 or FP8 storage run on the tensor
        // cores and keep M in their tile order; MAOS_B200_MVM_TC=0 keeps rows.
        V.tiled = dtype != MB_MVM_F32 && nbatch >= 4 && mb::Mvm::tc_enabled();
        V.nch = V.ldm / mb::kTcK;
        const long nrow = V.tiled ? (nact + mb::kTcRows - 1) / mb::kTcRows * mb::kTcRows : nact;
        const size_t nel = (size_t)nrow * V.ldm;
        // byte offset of element (r, c) for an element size of el bytes
        auto at = [&](long r, long c, int el) -> size_t {
            if (!V.tiled) return ((size_t)r * V.ldm + c) * el;
            const size_t tile = (size_t)(r / mb::kTcRows) * V.nch + c / mb::kTcK;
            const int rr = (int)(r % mb::kTcRows), cc = (int)(c % mb::kTcK);
            return el == 2 ? tile * mb::kTcTileBf16 + mb::tile_off(rr, cc >> 3) + (cc & 7) * 2
                           : tile * mb::kTcTileFp8 + mb::tc_fp8_off(rr, cc);
        };
        std::vector<float> sc(nact, 1.f);
        if (dtype == MB_MVM_F32) {
            std::vector<float> h32(nel, 0.f);
            for (long r = 0; r < nact; r++)
                for (long c = 0; c < ngrad; c++) h32[(size_t)r * V.ldm + c] = (float)Mcol[(size_t)c * nact + r];
            V.m.alloc(nel * 4);
            MB_CUDA_TRY(cudaMemcpy(V.m.p, h32.data(), nel * 4, cudaMemcpyHostToDevice));
        } else if (dtype == MB_MVM_BF16) {
            std::vector<__nv_bfloat16> h16(nel, __float2bfloat16(0.f));
            for (long r = 0; r < nact; r++)
                for (long c = 0; c < ngrad; c++)
                    h16[at(r, c, 2) / 2] = __float2bfloat16((float)Mcol[(size_t)c * nact + r]);
            V.m.alloc(nel * 2);
            MB_CUDA_TRY(cudaMemcpy(V.m.p, h16.data(), nel * 2, cudaMemcpyHostToDevice));
        } else {
            // per-row scale maps the row's largest magnitude to the e4m3 maximum (448)
            std::vector<__nv_fp8_e4m3> h8(nel, __nv_fp8_e4m3(0.f));
            for (long r = 0; r < nact; r++) {
                double mx = 0;
                for (long c = 0; c < ngrad; c++) mx = std::max(mx, std::fabs(Mcol[(size_t)c * nact + r]));
                const double s = mx > 0 ? mx / 448.0 : 1.0;
                sc[r] = (float)s;
                for (long c = 0; c < ngrad; c++)
                    h8[at(r, c, 1)] = __nv_fp8_e4m3((float)(Mcol[(size_t)c * nact + r] / s));
            }
            V.m.alloc(nel);
            MB_CUDA_TRY(cudaMemcpy(V.m.p, h8.data(), nel, cudaMemcpyHostToDevice));
        }
        if (V.tiled) {
            if (dtype == MB_MVM_BF16) V.plan_tc_dt<MB_MVM_BF16>();
            else V.plan_tc_dt<MB_MVM_FP8>();
        } else {
            V.part.alloc((size_t)V.nks * nbatch * nact);
        }
        V.scale.upload(sc);
        V.err.alloc(1);
        V.err.zero_async(V.stream);
        V.g.alloc((size_t)nbatch * ngrad);
        V.out.alloc((size_t)nbatch * nact);
        // the zeroed buffers are ready before a caller's stream uses them
        MB_CUDA_TRY(cudaStreamSynchronize(V.stream));
    } catch (const mb::CudaError &e) {
        delete h;
        return e.code;
    } catch (...) {
        delete h;
        mb::set_error("mb_mvm_create: unexpected exception");
        return MB_ECUDA;
    }
    *out = h;
    return MB_OK;
}

void mb_mvm_free(mb_mvm *h) { delete h; }

long mb_mvm_bytes(const mb_mvm *h) {
    if (!h) return -1;
    const mb::Mvm &V = h->M;
    const long el = V.dtype == MB_MVM_F32 ? 4 : V.dtype == MB_MVM_BF16 ? 2 : 1;
    return (long)V.nact * V.ngrad * el + (V.dtype == MB_MVM_FP8 ? 4L * V.nact : 0);
}

int mb_mvm_apply_device(mb_mvm *h, const float *d_grad, float *d_out, void *stream) {
    if (!h || !d_grad || !d_out) {
        mb::set_error("mb_mvm_apply_device: invalid arguments");
        return MB_EINVAL;
    }
    try {
        h->M.apply(d_grad, d_out, (cudaStream_t)stream);
    } catch (const mb::CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

int mb_mvm_apply_noalloc(const float *d_M, long nact, long ngrad, long ldm, const float *d_grad,
                         float *d_out, int nbatch, void *stream) {
    if (!d_M || !d_grad || !d_out || nact <= 0 || ngrad <= 0 || nbatch < 1 || ldm < ngrad ||
        (ldm & 3) || ((uintptr_t)d_M & 15)) {
        mb::set_error("mb_mvm_apply_noalloc: invalid arguments (ldm >= ngrad, ldm %% 4 == 0, "
                      "M 16-byte aligned)");
        return MB_EINVAL;
    }
    // bound each factor before multiplying, so the product cannot overflow
    const long nks = (ngrad + mb::kK - 1) / mb::kK;
    const bool too_big = nact > MB_NOALLOC_MAX_PARTIALS || nks > MB_NOALLOC_MAX_PARTIALS ||
                         nbatch > MB_NOALLOC_MAX_PARTIALS ||
                         nks * (long)nbatch > MB_NOALLOC_MAX_PARTIALS / nact;
    const long need = too_big ? -1 : nks * (long)nbatch * nact;
    if (too_big || need > MB_NOALLOC_MAX_PARTIALS) {
        mb::set_error("mb_mvm_apply_noalloc: needs %ld K slabs x %d instances x %ld rows of partial "
                      "sums; the static scratch holds %d",
                      nks, nbatch, nact, (int)MB_NOALLOC_MAX_PARTIALS);
        return MB_EINVAL;
    }
    try {
        int dev = 0;
        MB_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 256) {
            mb::set_error("mb_mvm_apply_noalloc: device index %d", dev);
            return MB_EINVAL;
        }
        float *part = mb::noalloc_scratch(dev);
        cudaStream_t s = (cudaStream_t)stream;
        if (nbatch == 1) mb::noalloc_launch<1>(d_M, ldm, d_grad, ngrad, part, (int)nact, nbatch, (int)nks, s);
        else if (nbatch <= 4) mb::noalloc_launch<4>(d_M, ldm, d_grad, ngrad, part, (int)nact, nbatch, (int)nks, s);
        else mb::noalloc_launch<8>(d_M, ldm, d_grad, ngrad, part, (int)nact, nbatch, (int)nks, s);
        const long n = nact * (long)nbatch;
        mb::k_mvm_reduce<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(part, nullptr, d_out, (int)nact, nbatch,
                                                                    (int)nks);
        MB_CHECK_LAUNCH();
    } catch (const mb::CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

int mb_recon_mvm(mb_mvm *h, const double *grad, double *dmout) {
    if (!h || !grad || !dmout) {
        mb::set_error("mb_recon_mvm: invalid arguments");
        return MB_EINVAL;
    }
    try {
        mb::Mvm &V = h->M;
        const size_t ng = (size_t)V.nbatch * V.ngrad, na = (size_t)V.nbatch * V.nact;
        std::vector<float> tmp(std::max(ng, na));
        for (size_t i = 0; i < ng; i++) tmp[i] = (float)grad[i];
        MB_CUDA_TRY(cudaMemcpyAsync(V.g.p, tmp.data(), ng * 4, cudaMemcpyHostToDevice, V.stream));
        V.apply(V.g.p, V.out.p, V.stream);
        MB_CUDA_TRY(cudaMemcpyAsync(tmp.data(), V.out.p, na * 4, cudaMemcpyDeviceToHost, V.stream));
        int flag = 0;
        MB_CUDA_TRY(cudaMemcpyAsync(&flag, V.err.p, sizeof(int), cudaMemcpyDeviceToHost, V.stream));
        MB_CUDA_TRY(cudaStreamSynchronize(V.stream));
        if (flag) {
            MB_CUDA_TRY(cudaMemsetAsync(V.err.p, 0, sizeof(int), V.stream));
            mb::set_error("mb_recon_mvm: a tensor-core MMA did not complete in time");
            return MB_ECUDA;
        }
        for (size_t i = 0; i < na; i++) dmout[i] = tmp[i];
    } catch (const mb::CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

}  // extern "C"
