// Tomography kernels for B200 (sm_100a).
//
// Every kernel is batched: blockIdx.z (or .y) selects one of `nb` independent
// instances that share the operator tables.  Instance vectors are stored
// instance-major (x[b*nxtot + ...]).  Reductions are deterministic: each block
// writes one FP64 partial, and consumers add the partials in a fixed order.
//
// Reference counterparts (cuda/tomo.cu, cuda/prop_wrap.cu, cuda/pcg.cu):
//   k_hx          gpu_map2map_do forward (prop_wrap.cu:35)    -- bilinear gather
//   k_gp          gpu_gp_do (tomo.cu:362)                     -- GP stencil + TT sums
//   k_pupil_rows  gpu_map2map_do + gpu_gp_do + gpu_gpt_do (tomo.cu:485) + the x half
//                 of gpu_map2map_do 't', fused per block of pupil rows
//   k_hxt_rows    y half of gpu_map2map_do 't' + gpu_laplacian_do (tomo.cu:317)
//   k_fit_hxt     gpu_map2map_do 't' in gather form (DM fit)  -- no atomics
//   k_fd_*        cufdpcg_t::P (fdpcg.cu:168)                 -- own FFTs, half spectrum
//   k_cg_*        gpu_pcg scalar kernels (pcg.cu:27-57)       -- FP64 scalars
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mb {

constexpr int kThreads = 256;
using cplx = float2;  // single-precision complex (re, im)

// One axis entry of the forward bilinear table: source index k (-1: the
// pupil point misses the layer) and the two weights for k and k+1.
struct AxisW {
    int k;
    float w0, w1;
};
// One entry of the transposed (gather) table: pupil index and weight.
struct GatherW {
    int i;
    float w;
};

struct WfsDev {
    int nsa;
    int pos;        // stencil is (pos+1)^2 points
    int goff;       // offset of this WFS's gradients inside one instance
    int has_ptt;
    const int2 *saptr;     // [nsa] lower-left corner on the pupil grid
    const float2 *gp;      // [nsa][(pos+1)^2] (x coefficient, y coefficient)
    const int *samap;      // [np] subaperture whose corner is at this pupil point, -1 if none
    const float *neai;     // [nsa][3] cx, cy, cxy
    const float *ptt;      // [2][2*nsa] column-major (k + 2*i)
};

struct LayerDev {
    int nx, ny;
    long off;       // offset inside one instance
    float l2c;      // biharmonic weight
    int tcol;       // first column of this layer in the row buffer of the separable Hx^T
};

constexpr int kMaxLayers = 16;  // most reconstructed layers (the Hx gather unrolls 8 or 16)

// The layer geometry passed by value (kernel parameter space), for kernels
// whose first dependent step is finding a point's layer.
struct LayerTab {
    LayerDev l[kMaxLayers];
};
// The WFS descriptors by value, for the same reason.
constexpr int kMaxWfs = 16;
struct WfsTab {
    WfsDev w[kMaxWfs];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of one double; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0;
    if (wid == 0) {
        t = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
        t = warp_sum(t);
    }
    __syncthreads();
    return t;
}

// Sum `n` partials in fixed order with one warp; result broadcast to the warp.
__device__ __forceinline__ double warp_sum_partials(const double *part, int n) {
    double v = 0;
    for (int i = threadIdx.x & 31; i < n; i += 32) v += part[i];
    v = warp_sum(v);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Per-CG scalar state, per instance.  sc holds r.z of every iteration
// (0..iters), b.b at iters+1 and the final residual at iters+2; ab the alpha
// and beta of the current iteration; cnt the arrival counters of the
// last-block reductions (zero between kernels).
struct CgScal {
    double *sc;
    int nsc;
    float *ab;       // [nb][2]
    unsigned *cnt;   // [nb]
    float *res;      // [nb]
};

// Every block calls this after writing its partial; it returns true in the
// block that arrived last.  That block alone then adds the partials in a
// fixed order (deterministic) and resets the counter.
__device__ __forceinline__ bool last_block(unsigned *cnt, unsigned nblocks) {
    __shared__ bool s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(cnt, 1u) == nblocks - 1);
    __syncthreads();
    return s_last;
}

// Sum n partials (written by other blocks of this kernel) with one warp,
// bypassing L1; the result is valid in every lane.
__device__ __forceinline__ double warp_sum_fresh(const double *part, int n) {
    double v = 0;
    for (int i = threadIdx.x & 31; i < n; i += 32) v += __ldcg(part + i);
    v = warp_sum(v);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Programmatic dependent launch: the first statement of every kernel here.
// A kernel launched with programmatic stream serialisation may be scheduled
// while its predecessor is still running; griddepcontrol.wait blocks until
// the predecessor has completed and its writes are visible, and
// launch_dependents lets the successor's CTAs be scheduled early.  Both are
// no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Serving: `act` (null: every instance) marks the instances that take part in
// this launch.  Blocks of an inactive instance return before touching memory,
// so its warm-start state stays as it was and no other instance's result
// depends on which instances are active.  Block-uniform (b is a block index).
__device__ __forceinline__ bool inactive(const int *act, int b) { return act && __ldg(act + b) == 0; }

// ---------------------------------------------------------------------------
// Hx: opd[b][w][p] = sum_l bilinear(x_l) at the ray of pupil point p.  The
// layer loop is unrolled to ML (>= nps) so every layer's taps are in flight
// together; the layer geometry comes by value.
// grid: (ceil(np/256), nwfs, nb)
// ---------------------------------------------------------------------------
template <int ML>
__global__ void k_hx(const float *__restrict__ x, float *__restrict__ opd,
                     const AxisW *__restrict__ tab, const __grid_constant__ LayerTab lt, int nps,
                     int nwfs, int nxp, int nyp, long nxtot, const float *__restrict__ w1,
                     double *__restrict__ w1_part, const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.z)) return;
    __shared__ double sh[32];
    const int np = nxp * nyp;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = blockIdx.y, b = blockIdx.z;
    float acc = 0.f;
    if (p < np) {
        const int ix = p % nxp, iy = p / nxp;
        const float *xb = x + (size_t)b * nxtot;
#pragma unroll
        for (int l = 0; l < ML; l++) {
            if (l < nps) {
                const AxisW *t = tab + (size_t)(w * nps + l) * (nxp + nyp);
                const AxisW tx = t[ix], ty = t[nxp + iy];
                const bool ok = tx.k >= 0 && ty.k >= 0;
                const int nx = lt.l[l].nx;
                const float *X = xb + lt.l[l].off + (ok ? (size_t)ty.k * nx + tx.k : 0);
                const float a = tx.w0 * X[0] + tx.w1 * X[1];
                const float c = tx.w0 * X[nx] + tx.w1 * X[nx + 1];
                if (ok) acc += ty.w0 * a + ty.w1 * c;
            }
        }
        opd[((size_t)b * nwfs + w) * np + p] = acc;
    }
    if (w1_part) {  // W1' opd partials for the piston-removed fit weighting
        double v = (p < np) ? (double)w1[p] * acc : 0.0;
        v = block_sum(v, sh);
        if (threadIdx.x == 0) w1_part[((size_t)b * nwfs + w) * gridDim.x + blockIdx.x] = v;
    }
}

// ---------------------------------------------------------------------------
// GP: grad = GP * opd (or the input gradients for the right-hand side), and
// per-block partial sums of PTT * grad for the tip/tilt removal.
// grid: (nblk, nwfs, nb); tt_part[((b*nwfs+w)*nblk + blk)*2 + k]
// ---------------------------------------------------------------------------
__global__ void k_gp(const float *__restrict__ opd, const float *__restrict__ gin,
                     float *__restrict__ grad, double *__restrict__ tt_part,
                     const WfsDev *__restrict__ wfs, int nwfs, int nxp, int np, long ngrad,
                     int do_tt, float *__restrict__ tt_out, unsigned *__restrict__ cnt,
                     const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.z)) return;
    __shared__ double sh[32];
    const int w = blockIdx.y, b = blockIdx.z;
    const WfsDev W = wfs[w];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    float gx = 0.f, gy = 0.f;
    if (s < W.nsa) {
        float *g = grad + (size_t)b * ngrad + W.goff;
        if (gin) {
            const float *gi = gin + (size_t)b * ngrad + W.goff;
            gx = gi[s];
            gy = gi[s + W.nsa];
        } else {
            const int2 c = W.saptr[s];
            const int n1 = W.pos + 1;
            const float2 *cf = W.gp + (size_t)s * n1 * n1;
            const float *o = opd + ((size_t)b * nwfs + w) * np + (size_t)c.y * nxp + c.x;
            for (int ty = 0; ty < n1; ty++)
                for (int tx = 0; tx < n1; tx++) {
                    const float v = o[ty * nxp + tx];
                    const float2 k = cf[ty * n1 + tx];
                    gx += k.x * v;
                    gy += k.y * v;
                }
        }
        g[s] = gx;
        g[s + W.nsa] = gy;
    }
    if (do_tt && W.has_ptt) {
        double tx = 0, ty = 0;
        if (s < W.nsa) {
            const float *P = W.ptt;
            tx = (double)P[2 * s] * gx + (double)P[2 * (s + W.nsa)] * gy;
            ty = (double)P[2 * s + 1] * gx + (double)P[2 * (s + W.nsa) + 1] * gy;
        }
        tx = block_sum(tx, sh);
        ty = block_sum(ty, sh);
        double *base = tt_part + ((size_t)b * nwfs + w) * gridDim.x * 2;
        if (threadIdx.x == 0) {
            base[blockIdx.x * 2] = tx;
            base[blockIdx.x * 2 + 1] = ty;
        }
        if (last_block(cnt + (size_t)b * nwfs + w, gridDim.x) && threadIdx.x < 32) {
            double t0 = 0, t1 = 0;
            for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) {
                t0 += __ldcg(base + 2 * i);
                t1 += __ldcg(base + 2 * i + 1);
            }
            t0 = warp_sum(t0);
            t1 = warp_sum(t1);
            if (threadIdx.x == 0) {
                tt_out[((size_t)b * nwfs + w) * 2] = (float)(-t0);
                tt_out[((size_t)b * nwfs + w) * 2 + 1] = (float)(-t1);
                cnt[(size_t)b * nwfs + w] = 0;
            }
        }
    }
}

// alpha_k = (r.z)_k / (p.Ap), reduced by the last block of the p.Ap producer.
__device__ __forceinline__ void cg_alpha_last(const double *part_b, const CgScal &S, int b, int k) {
    if (last_block(S.cnt + b, gridDim.x) && threadIdx.x < 32) {
        const double pap = warp_sum_fresh(part_b, gridDim.x);
        if (threadIdx.x == 0) {
            double a = S.sc[(size_t)b * S.nsc + k] / pap;
            if (!isfinite(a)) a = 0;  // pcg.c:80-83, pcg.cu:27-30
            S.ab[2 * b] = (float)a;
            S.cnt[b] = 0;
        }
    }
}

struct LowRank {
    const float *nw;        // [n][nnw] column-major (nw[k*n + j]); null: no term
    const double *part;     // NW' x partials [b][k][nblk]
    int nnw, nblk;
};

// Fit transpose HA^T in gather form over padded per-axis lists: for DM
// point (jx, jy) of DM l and fit direction w, the fit-grid points whose
// bilinear footprint covers it are the products of the x list
// fx[((w*ndm + l)*maxn + jx)*kx + e] and the y list (padding: weight 0).
// Every load of a direction depends only on (w, jx, jy), so the loads of
// several directions are in flight together.  Plus the low-rank NW term, an
// optional vector added as is (the slaving term), and the p.Ap partials (last
// block: alpha) for FitL.  grid: (ceil(nact/256), nb).
constexpr int kFitPad = 4;  // widest padded fit list
struct FitPad {
    const GatherW *x, *y;
    int kx, ky, maxn;
};

__global__ void __launch_bounds__(kThreads)
k_fit_hxt(const float *__restrict__ opd2, const float *__restrict__ xin, float *__restrict__ out,
          double *__restrict__ dot_part, FitPad fpd, const __grid_constant__ LayerTab dl, int ndm, int nfit,
          int nfx, int nfy, long nact, LowRank lr, CgScal S, int k, const float *__restrict__ addv,
          const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    __shared__ double sh[32];
    __shared__ float s_t[8];
    const int b = blockIdx.y;
    if (lr.nw) {  // t_k = NW_k' x, summed from partials in fixed order
        const int wid = threadIdx.x >> 5;
        if (wid < lr.nnw) {
            const double t = warp_sum_partials(lr.part + ((size_t)b * lr.nnw + wid) * lr.nblk, lr.nblk);
            if ((threadIdx.x & 31) == 0) s_t[wid] = (float)t;
        }
        __syncthreads();
    }
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double dotv = 0;
    if (j < nact) {
        int l = 0;
        while (l + 1 < ndm && j >= dl.l[l + 1].off) l++;
        const LayerDev L = dl.l[l];
        const int jj = (int)(j - L.off);
        const int jx = jj % L.nx, jy = jj / L.nx;
        const int np = nfx * nfy;
        const size_t wsx = (size_t)ndm * fpd.maxn * fpd.kx, wsy = (size_t)ndm * fpd.maxn * fpd.ky;
        const GatherW *ex0 = fpd.x + ((size_t)l * fpd.maxn + jx) * fpd.kx;
        const GatherW *ey0 = fpd.y + ((size_t)l * fpd.maxn + jy) * fpd.ky;
        const float *ob = opd2 + (size_t)b * nfit * np;
        float acc = 0.f;
#pragma unroll 3
        for (int w = 0; w < nfit; w++) {
            GatherW ex[kFitPad], ey[kFitPad];
#pragma unroll
            for (int e = 0; e < kFitPad; e++) {
                ex[e] = e < fpd.kx ? ex0[w * wsx + e] : GatherW{0, 0.f};
                ey[e] = e < fpd.ky ? ey0[w * wsy + e] : GatherW{0, 0.f};
            }
            const float *o = ob + (size_t)w * np;
#pragma unroll
            for (int ay = 0; ay < kFitPad; ay++) {
                if (ay >= fpd.ky) break;
                float rs = 0.f;
#pragma unroll
                for (int ax = 0; ax < kFitPad; ax++)
                    if (ax < fpd.kx) rs += ex[ax].w * o[ey[ay].i * nfx + ex[ax].i];
                acc += ey[ay].w * rs;
            }
        }
        const float *X = xin ? xin + (size_t)b * nact + L.off : nullptr;
        if (lr.nw) {
            float lt = 0.f;
            for (int q = 0; q < lr.nnw; q++) lt += lr.nw[(size_t)q * nact + j] * s_t[q];
            acc += lt;
        }
        if (addv) acc += addv[(size_t)b * nact + j];  // the slaving term, applied before
        out[(size_t)b * nact + j] = acc;
        if (dot_part && X) dotv = (double)acc * (double)X[jj];
    }
    if (dot_part) {
        dotv = block_sum(dotv, sh);
        if (threadIdx.x == 0) dot_part[(size_t)b * gridDim.x + blockIdx.x] = dotv;
        cg_alpha_last(dot_part + (size_t)b * gridDim.x, S, b, k);
    }
}

// ---------------------------------------------------------------------------
// Tomography normal-equation operator in two kernels.
//
// The bilinear transpose Hx^T is separable: for WFS w and layer l,
//   (Hx^T o)[jy][jx] = sum_{iy in Y(jy)} wy * sum_{ix in X(jx)} wx * o[iy][ix].
// k_pupil_rows works on a block of pupil rows of one (instance, WFS): it
// forms the pupil OPD (Hx, with a halo of `pos` rows), the NEA-weighted
// gradients (GP, NEA) and GP^T of them entirely in shared memory, then
// applies the x half of every layer's transpose and writes the partial
// sums t[w][l][iy][jx] (coalesced).  k_hxt_rows then finishes each layer
// point with the y half over all WFS, adds L2^T L2 x and the p.Ap partial.
// The transposed lists are stored with a fixed width (padding: weight 0 on
// pupil index 0), in the same order as the CSR lists, so the sums are the
// exact adjoint of Hx and independent of the tiling.  Only the footprint of
// each WFS on each layer (the columns and rows whose lists are not empty) is
// computed and read; outside it every term is an exact zero.
// ---------------------------------------------------------------------------
// Asynchronous 4-byte global -> shared copies (cp.async): a CTA issues all of
// a table's words at once and waits once, instead of one round trip per
// loop iteration.
__device__ __forceinline__ void cp_async_word(void *sdst, const void *gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;"
                 :: "r"((unsigned)__cvta_generic_to_shared(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// words [0, n) of src -> dst, spread over the CTA
__device__ __forceinline__ void cp_async_words(void *dst, const void *src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        cp_async_word(static_cast<float *>(dst) + i, static_cast<const float *>(src) + i);
}

struct PadIndex {
    const GatherW *x;   // [(w*kx + e)*ncols + tcol_l + jx]   (per WFS, entry-major over all layers' columns)
    const GatherW *y;   // [((w*nps + l)*maxny + jy)*ky + e]
    const int4 *fp;     // [w*nps + l]: footprint of the WFS on the layer: columns [x, y), rows [z, w)
    int kx, ky, maxnx, maxny;
};

constexpr int kMaxPadX = 8;     // widest x list
constexpr int kMaxPadY = 8;     // widest y list (k_hxt_rows is instantiated up to this)
constexpr int kHxtWfs = 6;      // WFS whose gathers k_hxt_rows issues together for one instance

// Dynamic shared memory of k_pupil_rows, in floats, for `rows` output rows.
__host__ __device__ constexpr int pupil_rows_smem_floats(int rows, int nxp, int nps, int ncols, int kx) {
    return nxp * (3 * (rows + 2) + rows + (rows + 4))      // wg, sid, opd2, opd
           + 3 * nps * (nxp + rows + 4)                     // staged Hx axis tables
           + 2 * ncols * kx;                                // staged x lists of the WFS
}

// grid: (ceil(nyp/rows), nw, nb), WFS w = wbase + blockIdx.y, all with
// subaperture/pupil ratio POS; ML >= nps bounds the unrolled layer loop.  FROM_X: the operator input is the layer
// vector x (Hx, GP in shared memory; no tip/tilt term).  Otherwise the input
// is a gradient vector already in `grad` (right-hand side, or the LHS with
// the tip/tilt projection), with -PTT g per WFS in `tt` when do_tt.
// Thread layout: each thread owns one pupil column (and a phase of the rows)
// for the pupil-grid stages and whole layer columns for the x half of Hx^T,
// so per-item index arithmetic is a few adds; index tables are staged in
// shared memory and a pupil point's layer taps are issued together.
// Grouped launches: one grid over the blocks of several reconstructors of
// different geometries (uneven instances advanced by one launch of an
// operator).  Entry e covers flat blocks [start[e], start[e+1]) with its own
// grid shape and its own arguments (tables, vectors, sizes); a block finds
// its entry and runs the operator's body with the entry's block index.
constexpr int kMaxGroup = 8;
template <class A>
struct GroupTab {
    int n;
    unsigned start[kMaxGroup + 1];
    uint3 grid[kMaxGroup];
    A a[kMaxGroup];
};
template <class A>
__device__ __forceinline__ int group_entry(const GroupTab<A> &g, uint3 &bid) {
    int e = 0;
    while (e + 1 < g.n && blockIdx.x >= g.start[e + 1]) e++;
    const unsigned l = blockIdx.x - g.start[e];
    const uint3 d = g.grid[e];
    bid = make_uint3(l % d.x, (l / d.x) % d.y, l / (d.x * d.y));
    return e;
}

// Arguments of one k_pupil_rows launch.
struct PupilArgs {
    const float *x, *grad, *tt;
    float *t;
    const AxisW *tab;
    LayerTab lt;
    WfsTab wt;
    PadIndex pi;
    int wbase, nps, nwfs, nxp, nyp;
    long nxtot, ngrad, tw;
    int ncols, rows, do_tt;
    const int *act;
};

// The body takes its block index as `bid` (blockIdx, or a block of one
// member of a grouped launch, k_pupil_rows_group).
template <bool FROM_X, int POS, int ML>
__device__ __forceinline__ void
pupil_rows_body(const uint3 bid, const float *__restrict__ x, const float *__restrict__ grad,
                const float *__restrict__ tt, float *__restrict__ t, const AxisW *__restrict__ tab,
                const LayerTab &lt, const WfsTab &wt, const PadIndex &pi, int wbase, int nps, int nwfs, int nxp,
                int nyp, long nxtot, long ngrad, long tw, int ncols, int rows, int do_tt,
                const int *__restrict__ act) {
    pdl_enter();
    constexpr int N1 = POS + 1;
    const int w = wbase + bid.y, b = bid.z;
    if (inactive(act, b)) return;
    extern __shared__ float sm[];
    __shared__ int s_lnx[kMaxLayers], s_tcol[kMaxLayers + 1];
    __shared__ long s_loff[kMaxLayers];
    __shared__ int4 s_fp[kMaxLayers];
    const WfsDev &W = wt.w[w];
    const int r0 = bid.x * rows;
    const int r1 = min(nyp, r0 + rows);      // output pupil rows [r0, r1)
    const int ca = max(0, r0 - POS);         // subaperture corner rows [ca, cb)
    const int cb = min(nyp - POS, r1);
    const int nh = cb + POS - ca;            // pupil rows of the Hx halo block
    const int cr = rows + 2;
    const int ts = nxp + rows + 4;           // staged axis entries per layer
    float2 *s_wg = reinterpret_cast<float2 *>(sm);                  // [cr][nxp]
    int *s_sid = reinterpret_cast<int *>(sm + 2 * cr * nxp);         // [cr][nxp]
    float *s_opd2 = sm + 3 * cr * nxp;                               // [rows][nxp]
    float *s_opd = s_opd2 + rows * nxp;                              // [rows+4][nxp]
    AxisW *s_tab = reinterpret_cast<AxisW *>(s_opd + (rows + 4) * nxp);  // [nps][ts]
    GatherW *s_xp = reinterpret_cast<GatherW *>(reinterpret_cast<float *>(s_tab) + 3 * nps * ts);
    const int nph = blockDim.x / nxp;        // row phases (nxp <= blockDim)
    const int ph = threadIdx.x / nxp, ix = threadIdx.x - ph * nxp;
    const bool colthr = ph < nph;

    // stage the layer geometry and footprints, the x lists of this WFS, the
    // subaperture map of rows [ca, cb) and, for Hx, the axis tables: all
    // copies in flight together
    if (threadIdx.x < nps) {
        const LayerDev &L = lt.l[threadIdx.x];
        s_lnx[threadIdx.x] = L.nx;
        s_loff[threadIdx.x] = L.off;
        s_tcol[threadIdx.x] = L.tcol;
        s_fp[threadIdx.x] = pi.fp[w * nps + threadIdx.x];
    }
    if (threadIdx.x == 0) s_tcol[nps] = ncols;
    {
        constexpr int GW = (int)(sizeof(GatherW) / 4), AW = (int)(sizeof(AxisW) / 4);
        cp_async_words(s_xp, pi.x + (size_t)w * ncols * pi.kx, ncols * pi.kx * GW);
        if (cb > ca) cp_async_words(s_sid, W.samap + (size_t)ca * nxp, (cb - ca) * nxp);
        if (FROM_X) {
            const AxisW *tw0 = tab + (size_t)w * nps * (nxp + nyp);
            for (int l = 0; l < nps; l++) {
                const AxisW *tl = tw0 + (size_t)l * (nxp + nyp);
                cp_async_words(s_tab + l * ts, tl, nxp * AW);                   // x axis
                cp_async_words(s_tab + l * ts + nxp, tl + nxp + ca, nh * AW);   // y axis, rows [ca, ca+nh)
            }
        }
        cp_async_wait_all();
        __syncthreads();
    }
    if (FROM_X) {  // Hx for pupil rows [ca, cb + POS): a point's layer taps are issued together
        const float *xb = x + (size_t)b * nxtot;
        if (colthr)
            for (int r = ph; r < nh; r += nph) {
                float acc = 0.f;
#pragma unroll
                for (int l = 0; l < ML; l++) {
                    if (l < nps) {
                        const AxisW tx = s_tab[l * ts + ix], ty = s_tab[l * ts + nxp + r];
                        const bool ok = tx.k >= 0 && ty.k >= 0;
                        const int nx = s_lnx[l];
                        const float *X = xb + s_loff[l] + (ok ? ty.k * nx + tx.k : 0);
                        const float a = tx.w0 * X[0] + tx.w1 * X[1];
                        const float c = tx.w0 * X[nx] + tx.w1 * X[nx + 1];
                        if (ok) acc += ty.w0 * a + ty.w1 * c;
                    }
                }
                s_opd[r * nxp + ix] = acc;
            }
        __syncthreads();
    }
    {  // NEA-weighted gradients of the subapertures with corners in rows [ca, cb)
        const float *g = FROM_X ? nullptr : grad + (size_t)b * ngrad + W.goff;
        const bool use_tt = !FROM_X && do_tt && W.has_ptt;
        const float ttx = use_tt ? tt[((size_t)b * nwfs + w) * 2] : 0.f;
        const float tty = use_tt ? tt[((size_t)b * nwfs + w) * 2 + 1] : 0.f;
        if (colthr)
            for (int rr = ph; rr < cb - ca; rr += nph) {
                const int i = rr * nxp + ix;
                const int s = s_sid[i];  // staged subaperture map
                if (s < 0) continue;
                const float *ne = W.neai + 3 * s;
                const float n0 = ne[0], n1_ = ne[1], n2 = ne[2];
                float gx = 0.f, gy = 0.f;
                if (FROM_X) {
                    const float2 *cf = W.gp + (size_t)s * N1 * N1;
                    float2 k[N1 * N1];
#pragma unroll
                    for (int q = 0; q < N1 * N1; q++) k[q] = cf[q];
                    const float *o = s_opd + i;
#pragma unroll
                    for (int ty = 0; ty < N1; ty++)
#pragma unroll
                        for (int tx = 0; tx < N1; tx++) {
                            const float v = o[ty * nxp + tx];
                            gx += k[ty * N1 + tx].x * v;
                            gy += k[ty * N1 + tx].y * v;
                        }
                } else {
                    gx = g[s] + ttx;
                    gy = g[s + W.nsa] + tty;
                }
                s_wg[i] = make_float2(n0 * gx + n2 * gy, n2 * gx + n1_ * gy);
            }
        __syncthreads();
    }
    if (colthr) {  // GP^T for the output rows (gather over the covering subapertures)
        for (int pr = ph; pr < r1 - r0; pr += nph) {
            const int py = r0 + pr;
            float2 k[N1 * N1], v[N1 * N1];
#pragma unroll
            for (int dy = 0; dy < N1; dy++)
#pragma unroll
                for (int dx = 0; dx < N1; dx++) {
                    const int cy = py - dy, cx = ix - dx;
                    const int q = dy * N1 + dx;
                    const bool in = cy >= ca && cy < cb && cx >= 0;
                    const int j = in ? (cy - ca) * nxp + cx : 0;
                    const int s = in ? s_sid[j] : -1;
                    k[q] = s >= 0 ? W.gp[(size_t)s * N1 * N1 + q] : make_float2(0.f, 0.f);
                    v[q] = s >= 0 ? s_wg[j] : make_float2(0.f, 0.f);
                }
            float acc = 0.f;
#pragma unroll
            for (int q = 0; q < N1 * N1; q++) acc += k[q].x * v[q].x + k[q].y * v[q].y;
            s_opd2[pr * nxp + ix] = acc;
        }
    }
    __syncthreads();
    {  // x half of Hx^T for every layer: t[w][l][iy][jx]; a thread owns whole layer columns
        float *tb = t + (size_t)(b * nwfs + w) * tw;
        const int kx = pi.kx, nr = r1 - r0;
        for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
            int l = 0;
            while (l + 1 < nps && c >= s_tcol[l + 1]) l++;
            const int tc = s_tcol[l], lnx = s_lnx[l];
            const int4 f = s_fp[l];
            if (c - tc < f.x || c - tc >= f.y) continue;  // no pupil column reaches it: never read
            GatherW e[kMaxPadX];
#pragma unroll
            for (int k = 0; k < kMaxPadX; k++) e[k] = k < kx ? s_xp[k * ncols + c] : GatherW{0, 0.f};  // no bank conflicts
            float *dst = tb + (size_t)nyp * tc + (size_t)r0 * lnx + (c - tc);
            for (int r = 0; r < nr; r++) {
                const float *o = s_opd2 + r * nxp;
                float sx = 0.f;
#pragma unroll
                for (int k = 0; k < kMaxPadX; k++)
                    if (k < kx) sx += e[k].w * o[e[k].i];
                dst[r * lnx] = sx;
            }
        }
    }
}

template <bool FROM_X, int POS, int ML>
__global__ void __launch_bounds__(kThreads, 4)
k_pupil_rows(const float *__restrict__ x, const float *__restrict__ grad, const float *__restrict__ tt,
             float *__restrict__ t, const AxisW *__restrict__ tab, const __grid_constant__ LayerTab lt,
             const __grid_constant__ WfsTab wt, PadIndex pi, int wbase, int nps, int nwfs, int nxp, int nyp,
             long nxtot, long ngrad, long tw, int ncols, int rows, int do_tt,
             const int *__restrict__ act) {
    pupil_rows_body<FROM_X, POS, ML>(blockIdx, x, grad, tt, t, tab, lt, wt, pi, wbase, nps, nwfs, nxp, nyp, nxtot,
                                     ngrad, tw, ncols, rows, do_tt, act);
}
// grid: (sum of the entries' blocks); dynamic shared memory: the largest entry's.
template <bool FROM_X, int POS, int ML>
__global__ void __launch_bounds__(kThreads, 4)
k_pupil_rows_group(const __grid_constant__ GroupTab<PupilArgs> g) {
    uint3 bid;
    const PupilArgs &a = g.a[group_entry(g, bid)];
    pupil_rows_body<FROM_X, POS, ML>(bid, a.x, a.grad, a.tt, a.t, a.tab, a.lt, a.wt, a.pi, a.wbase, a.nps, a.nwfs,
                                     a.nxp, a.nyp, a.nxtot, a.ngrad, a.tw, a.ncols, a.rows, a.do_tt, a.act);
}

// y half of Hx^T over all WFS, + L2^T L2 x and p.Ap partials (last block:
// alpha).  One thread per layer point and NI instances (the index work, the
// footprint tests and the list entries are shared by the instances, and each
// dependent step issues NI times the independent loads; the NI block sums
// and last-block arrivals are taken together);
// grid: (ceil(nxtot/256), ceil(nb/NI)).  KY is the padded y-list width.
// The body takes its block index `bid` and the x extent of its grid `gx`.
template <int KY, int NI>
__device__ __forceinline__ void
hxt_rows_body(const uint3 bid, const unsigned gx, const float *__restrict__ t, const float *__restrict__ xin,
              float *__restrict__ out, double *__restrict__ dot_part, const PadIndex &pi, const LayerTab &lt,
              int nps, int nwfs, int nyp, long nxtot, long tw, int do_l2, const CgScal &S, int kit, int nb,
              const int *__restrict__ act) {
    pdl_enter();
    const int b0 = bid.y * NI;
    bool on[NI];
    bool any = false;
#pragma unroll
    for (int q = 0; q < NI; q++) {
        on[q] = b0 + q < nb && !inactive(act, b0 + q);
        any = any || on[q];
    }
    if (!any) return;
    __shared__ double shq[NI][32];
    __shared__ bool s_last[NI];
    const long j = (long)bid.x * blockDim.x + threadIdx.x;
    double dotv[NI];
#pragma unroll
    for (int q = 0; q < NI; q++) dotv[q] = 0;
    if (j < nxtot) {
        int l = 0;
        while (l + 1 < nps && j >= lt.l[l + 1].off) l++;
        const LayerDev L = lt.l[l];
        const int nx = L.nx, ny = L.ny;
        const int jj = (int)(j - L.off);
        const int jy = jj / nx, jx = jj - jy * nx;
        const float *tl = t + (size_t)b0 * nwfs * tw + (size_t)nyp * L.tcol + jx;
        const size_t tinst = (size_t)nwfs * tw;  // row-buffer stride between instances
        const GatherW *e = pi.y + ((size_t)l * pi.maxny + jy) * KY;
        const int estep = nps * pi.maxny * KY;
        float acc[NI];
#pragma unroll
        for (int q = 0; q < NI; q++) acc[q] = 0.f;
        if constexpr (NI == 1) {
            // one instance: the lists of kHxtWfs WFS are loaded together, then
            // all their row-buffer values, so the WFS cost two round trips
            // instead of two each (same sums, same order)
            for (int w0 = 0; w0 < nwfs; w0 += kHxtWfs) {
                GatherW ge[kHxtWfs][KY];
                bool in[kHxtWfs];
#pragma unroll
                for (int u = 0; u < kHxtWfs; u++) {
                    const int w = w0 + u;
                    in[u] = false;
                    if (w < nwfs) {
                        const int4 f = pi.fp[w * nps + l];
                        in[u] = !(jx < f.x || jx >= f.y || jy < f.z || jy >= f.w);
                    }
#pragma unroll
                    for (int k = 0; k < KY; k++) ge[u][k] = in[u] ? e[(size_t)w * estep + k] : GatherW{0, 0.f};
                }
                float tv[kHxtWfs][KY];
#pragma unroll
                for (int u = 0; u < kHxtWfs; u++)
#pragma unroll
                    for (int k = 0; k < KY; k++)
                        tv[u][k] = (in[u] && on[0]) ? tl[(size_t)(w0 + u) * tw + ge[u][k].i * nx] : 0.f;
#pragma unroll
                for (int u = 0; u < kHxtWfs; u++) {
                    if (!in[u]) continue;
                    float sy = 0.f;
#pragma unroll
                    for (int k = 0; k < KY; k++) sy += ge[u][k].w * tv[u][k];
                    acc[0] += sy;
                }
            }
        } else {
#pragma unroll 2
            for (int w = 0; w < nwfs; w++, e += estep, tl += tw) {
                const int4 f = pi.fp[w * nps + l];
                if (jx < f.x || jx >= f.y || jy < f.z || jy >= f.w) continue;  // outside this WFS's footprint
                GatherW ge[KY];
                float tv[NI][KY];
#pragma unroll
                for (int k = 0; k < KY; k++) ge[k] = e[k];
#pragma unroll
                for (int q = 0; q < NI; q++)
#pragma unroll
                    for (int k = 0; k < KY; k++) tv[q][k] = on[q] ? tl[q * tinst + ge[k].i * nx] : 0.f;
#pragma unroll
                for (int q = 0; q < NI; q++) {
                    float sy = 0.f;
#pragma unroll
                    for (int k = 0; k < KY; k++) sy += ge[k].w * tv[q][k];
                    acc[q] += sy;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NI; q++) {
            if (!on[q]) continue;
            const int b = b0 + q;
            const float *X = xin ? xin + (size_t)b * nxtot + L.off : nullptr;
            float v = acc[q];
            if (do_l2) {  // periodic 13-point biharmonic stencil (tomo.cu gpu_laplacian_do)
                auto wy = [&](int d) { int y = jy + d; y += (y < 0) ? ny : 0; y -= (y >= ny) ? ny : 0; return X + y * nx; };
                auto wx = [&](int d) { int u = jx + d; u += (u < 0) ? nx : 0; u -= (u >= nx) ? nx : 0; return u; };
                const float *Rm2 = wy(-2), *Rm1 = wy(-1), *R0 = X + jy * nx, *Rp1 = wy(1), *Rp2 = wy(2);
                const int xm2 = wx(-2), xm1 = wx(-1), xp1 = wx(1), xp2 = wx(2);
                const float st = 20.f * R0[jx] - 8.f * (R0[xm1] + R0[xp1] + Rm1[jx] + Rp1[jx]) +
                                 2.f * (Rm1[xm1] + Rm1[xp1] + Rp1[xm1] + Rp1[xp1]) +
                                 (Rm2[jx] + R0[xm2] + R0[xp2] + Rp2[jx]);
                v += L.l2c * st;
            }
            out[(size_t)b * nxtot + j] = v;
            if (dot_part && X) dotv[q] = (double)v * (double)X[jj];
        }
    }
    if (dot_part) {
        // block sums of the NI partials (the block_sum tree, NI at a time)
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int q = 0; q < NI; q++) {
            const double v = warp_sum(dotv[q]);
            if (lane == 0) shq[q][wid] = v;
        }
        __syncthreads();
        if (wid == 0)
#pragma unroll
            for (int q = 0; q < NI; q++) {
                double v = lane < (int)(blockDim.x >> 5) ? shq[q][lane] : 0.0;
                v = warp_sum(v);
                if (lane == 0 && on[q]) dot_part[(size_t)(b0 + q) * gx + bid.x] = v;
            }
        // last block per instance: alpha_k = (r.z)_k / (p.Ap) (cg_alpha_last, NI counters at once)
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0)
#pragma unroll
            for (int q = 0; q < NI; q++) s_last[q] = on[q] && atomicAdd(S.cnt + b0 + q, 1u) == gx - 1;
        __syncthreads();
#pragma unroll
        for (int q = 0; q < NI; q++) {
            if (!s_last[q] || threadIdx.x >= 32) continue;
            const int b = b0 + q;
            const double pap = warp_sum_fresh(dot_part + (size_t)b * gx, gx);
            if (threadIdx.x == 0) {
                double a = S.sc[(size_t)b * S.nsc + kit] / pap;
                if (!isfinite(a)) a = 0;  // pcg.c:80-83, pcg.cu:27-30
                S.ab[2 * b] = (float)a;
                S.cnt[b] = 0;
            }
        }
    }
}

template <int KY, int NI>
__global__ void __launch_bounds__(kThreads)
k_hxt_rows(const float *__restrict__ t, const float *__restrict__ xin, float *__restrict__ out,
           double *__restrict__ dot_part, PadIndex pi, const __grid_constant__ LayerTab lt, int nps,
           int nwfs, int nyp, long nxtot, long tw, int do_l2, CgScal S, int kit, int nb,
           const int *__restrict__ act) {
    hxt_rows_body<KY, NI>(blockIdx, gridDim.x, t, xin, out, dot_part, pi, lt, nps, nwfs, nyp, nxtot, tw, do_l2, S,
                          kit, nb, act);
}
// Arguments of one k_hxt_rows launch.
struct HxtArgs {
    const float *t, *xin;
    float *out;
    double *dot_part;
    PadIndex pi;
    LayerTab lt;
    int nps, nwfs, nyp;
    long nxtot, tw;
    int do_l2;
    CgScal S;
    int kit, nb;
    const int *act;
};
template <int KY, int NI>
__global__ void __launch_bounds__(kThreads)
k_hxt_rows_group(const __grid_constant__ GroupTab<HxtArgs> g) {
    uint3 bid;
    const int e = group_entry(g, bid);
    const HxtArgs &a = g.a[e];
    hxt_rows_body<KY, NI>(bid, g.grid[e].x, a.t, a.xin, a.out, a.dot_part, a.pi, a.lt, a.nps, a.nwfs, a.nyp, a.nxtot,
                          a.tw, a.do_l2, a.S, a.kit, a.nb, a.act);
}

// ---------------------------------------------------------------------------
// Fit weighting: y = wt_f (W0 v - W1 (W1' v)) on the fit grid, W0 in CSR.
// grid: (ceil(nf/256), nfit, nb); W1' v from the partials written by k_hx.
// ---------------------------------------------------------------------------
__global__ void k_fit_w(const float *__restrict__ v, float *__restrict__ y,
                        const int *__restrict__ rp, const int *__restrict__ ci,
                        const float *__restrict__ cv, const float *__restrict__ w1,
                        const float *__restrict__ wt, const double *__restrict__ w1_part,
                        int nblk_w1, int nf, int nfit, const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.z)) return;
    __shared__ float s_dot;
    const int f = blockIdx.y, b = blockIdx.z;
    if (threadIdx.x < 32) {
        const double d = warp_sum_partials(w1_part + ((size_t)b * nfit + f) * nblk_w1, nblk_w1);
        if (threadIdx.x == 0) s_dot = (float)d;
    }
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nf) return;
    const float *vb = v + ((size_t)b * nfit + f) * nf;
    float acc = 0.f;
    for (int k = rp[p]; k < rp[p + 1]; k++) acc += cv[k] * vb[ci[k]];
    y[((size_t)b * nfit + f) * nf + p] = wt[f] * (acc - w1[p] * s_dot);
}

// NW' x partials: part[(b*nnw + k)*nblk + blk].  grid: (nblk, nb)
__global__ void k_lowrank_dot(const float *__restrict__ x, const float *__restrict__ nw,
                              double *__restrict__ part, int nnw, long n, const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    __shared__ double sh[32];
    const int b = blockIdx.y;
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const float xv = (j < n) ? x[(size_t)b * n + j] : 0.f;
    for (int k = 0; k < nnw; k++) {
        double v = (j < n) ? (double)nw[(size_t)k * n + j] * xv : 0.0;
        v = block_sum(v, sh);
        if (threadIdx.x == 0) part[((size_t)b * nnw + k) * gridDim.x + blockIdx.x] = v;
    }
}

// ---------------------------------------------------------------------------
// CG vector kernels.  Scalars per instance: sc[b*nsc + k].
// layout: [0..maxit] r.z per iteration, [maxit+1] b.b, [maxit+2] residual
// ---------------------------------------------------------------------------

// r = b - Ax; b.b is reduced by the last block into sc[iters+1].  grid: (nblk, nb)
__global__ void k_cg_init_r(const float *__restrict__ bvec, const float *__restrict__ Ax,
                            float *__restrict__ r, double *__restrict__ bb_part, long n, CgScal S,
                            int iters, const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    __shared__ double sh[32];
    const int b = blockIdx.y;
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0;
    if (j < n) {
        const size_t o = (size_t)b * n + j;
        const float bv = bvec[o];
        r[o] = bv - Ax[o];
        v = (double)bv * bv;
    }
    v = block_sum(v, sh);
    double *pb = bb_part + (size_t)b * gridDim.x;
    if (threadIdx.x == 0) pb[blockIdx.x] = v;
    if (last_block(S.cnt + b, gridDim.x) && threadIdx.x < 32) {
        const double bb = warp_sum_fresh(pb, gridDim.x);
        if (threadIdx.x == 0) {
            S.sc[(size_t)b * S.nsc + iters + 1] = bb;
            S.cnt[b] = 0;
        }
    }
}

// (r.z) reduction shared by the kernels that produce z: the last block
// stores (r.z)_0 when init, otherwise beta = (r.z)_{k+1} / (r.z)_k.
__device__ __forceinline__ void cg_rz_last(const double *part_b, const CgScal &S, int b, int k,
                                           int init) {
    if (last_block(S.cnt + b, gridDim.x) && threadIdx.x < 32) {
        const double rz = warp_sum_fresh(part_b, gridDim.x);
        if (threadIdx.x == 0) {
            if (init) {  // start (or restart, lib/pcg.c:61) at iteration k
                S.sc[(size_t)b * S.nsc + k] = rz;
            } else {
                double be = rz / S.sc[(size_t)b * S.nsc + k];
                if (!isfinite(be)) be = 0;
                S.ab[2 * b + 1] = (float)be;
                S.sc[(size_t)b * S.nsc + k + 1] = rz;
            }
            S.cnt[b] = 0;
        }
    }
}

// v.v partials and (when z aliases r) the r.z of a CG start or restart at
// iteration k.  grid: (nblk, nb)
__global__ void k_dot_self(const float *__restrict__ v, double *__restrict__ part, long n, CgScal S, int k,
                           const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    __shared__ double sh[32];
    const int b = blockIdx.y;
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double t = 0;
    if (j < n) {
        const float a = v[(size_t)b * n + j];
        t = (double)a * a;
    }
    t = block_sum(t, sh);
    if (threadIdx.x == 0) part[(size_t)b * gridDim.x + blockIdx.x] = t;
    cg_rz_last(part + (size_t)b * gridDim.x, S, b, k, 1);
}

// x += alpha p; r -= alpha Ap; r.r partials.  The last block either finishes
// the solve (residual sqrt(r.r/b.b) at the final iteration) or, when z aliases
// r (no preconditioner), produces beta.
__global__ void k_cg_update_xr(float *__restrict__ x, float *__restrict__ r,
                               const float *__restrict__ p, const float *__restrict__ Ap,
                               double *__restrict__ rr_part, long n, CgScal S, int k, int iters,
                               int z_is_r, const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    __shared__ double sh[32];
    const int b = blockIdx.y;
    const float a = S.ab[2 * b];
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0;
    if (j < n) {
        const size_t o = (size_t)b * n + j;
        x[o] += a * p[o];
        const float rv = r[o] - a * Ap[o];
        r[o] = rv;
        v = (double)rv * rv;
    }
    v = block_sum(v, sh);
    double *pb = rr_part + (size_t)b * gridDim.x;
    if (threadIdx.x == 0) pb[blockIdx.x] = v;
    if (k + 1 == iters) {
        if (last_block(S.cnt + b, gridDim.x) && threadIdx.x < 32) {
            const double rr = warp_sum_fresh(pb, gridDim.x);
            if (threadIdx.x == 0) {
                const double res = sqrt(rr / S.sc[(size_t)b * S.nsc + iters + 1]);
                S.sc[(size_t)b * S.nsc + iters + 2] = res;
                S.res[b] = (float)res;
                S.cnt[b] = 0;
            }
        }
    } else if (z_is_r) {
        cg_rz_last(pb, S, b, k, 0);
    }
}

// p = z + beta p (init: p = z).  kUpdP elements per thread (16-byte
// accesses when n is a multiple of 4); every load is issued before the
// participation flag and beta are known, so the thread waits one round trip.
// grid: (ceil(n / (kUpdP * 256)), nb)
constexpr int kUpdP = 4;

__global__ void k_cg_update_p(float *__restrict__ p, const float *__restrict__ z, long n, CgScal S,
                              int init, const int *__restrict__ act) {
    pdl_enter();
    const int b = blockIdx.y;
    const long j = ((long)blockIdx.x * blockDim.x + threadIdx.x) * kUpdP;
    const size_t o = (size_t)b * n + j;
    float zv[kUpdP] = {}, pv[kUpdP] = {};
    const bool vec = (n & 3) == 0 && j + kUpdP <= n;
    if (vec) {
        const float4 a = *reinterpret_cast<const float4 *>(z + o);
        zv[0] = a.x, zv[1] = a.y, zv[2] = a.z, zv[3] = a.w;
        if (!init) {
            const float4 c = *reinterpret_cast<const float4 *>(p + o);
            pv[0] = c.x, pv[1] = c.y, pv[2] = c.z, pv[3] = c.w;
        }
    } else {
#pragma unroll
        for (int u = 0; u < kUpdP; u++)
            if (j + u < n) {
                zv[u] = z[o + u];
                if (!init) pv[u] = p[o + u];
            }
    }
    if (inactive(act, b)) return;
    const float be = init ? 0.f : S.ab[2 * b + 1];
    float r[kUpdP];
#pragma unroll
    for (int u = 0; u < kUpdP; u++) r[u] = init ? zv[u] : zv[u] + be * pv[u];
    if (vec) {
        *reinterpret_cast<float4 *>(p + o) = make_float4(r[0], r[1], r[2], r[3]);
    } else {
#pragma unroll
        for (int u = 0; u < kUpdP; u++)
            if (j + u < n) p[o + u] = r[u];
    }
}

// ---------------------------------------------------------------------------
// FDPCG on the half spectrum.  Each layer's forward transform reads the
// residual straight from the instance-major vector and writes
// H[hoff_l + b*hs_l + ky*(nx/2+1) + kx], hs_l = ny*(nx/2+1); the inverse
// writes z back the same way.
// ---------------------------------------------------------------------------
enum { kFdConj = 1, kFdStore = 2 };
struct FdIndex {
    int base;    // hoff_l + position of the member in the layer's half spectrum
    int stride;  // hs_l (instance stride)
    int flags;   // kFdConj: the member is the conjugate of the stored value;
                 // kFdStore: this member writes the stored value
    int pad;
};

// Batched 2-D real FFTs of the layer grids, one CTA per (layer, instance),
// entirely in shared memory.  Length-n complex transforms are mixed-radix
// Stockham stages (radix 2, 3, 4, 5; no reordering pass), twiddles
// exp(-2 pi i k/n) come from a table computed on the host in FP64.  Two real
// rows travel as one complex row.  Forward: rows, then columns of the half
// spectrum; output layout [ky][kx], kx <= nx/2.  Inverse: columns, then
// rows, with the imaginary parts of the kx = 0 and kx = nx/2 bins dropped
// (the real part of the inverse of the Hermitian extension).  Neither
// direction is normalised.
struct FdLayer {
    int nx, ny;          // grid (x fastest); both even
    long off;            // offset of the layer in an instance vector
    int hoff, hs;        // half-spectrum offset of instance 0 and the instance stride
    int twx, twy;        // offsets of the twiddle tables for n = nx and n = ny
    int nrx, nry;        // radix stages along x and y
    signed char rx[8], ry[8];
    int px, py;          // two-pass factor pair (index into kFftPairs) along x and y, -1: stages
};
struct FdTab {  // per layer, by value (kernel parameter space)
    FdLayer l[kMaxLayers];
};

// Lengths the two-pass FFT handles, as n = N1 * N2 (both passes' DFTs held
// in registers).  The host picks the first pair whose product is n.
constexpr int kFftPairs[][2] = {{4, 4}, {8, 4}, {6, 6}, {8, 5}, {8, 6}, {10, 6}, {8, 8}, {12, 6}, {10, 8},
                                {12, 8}, {10, 10}, {12, 10}, {12, 12}, {16, 10}, {16, 12}, {16, 16}, {16, 8}};
constexpr int kNumFftPairs = (int)(sizeof(kFftPairs) / sizeof(kFftPairs[0]));

__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cplx cconj(cplx a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ cplx mul_mi(cplx a) { return make_float2(a.y, -a.x); }  // -i a

// One Stockham stage of radix R over `count` transforms of length n
// (element stride es, transform stride ts), a -> b.  Ns = product of the
// radices of the previous stages.  A thread keeps one butterfly position j
// (and its twiddles) for the whole stage and steps over the transforms.
// Requires n / R <= blockDim.x.
template <int R>
__device__ __forceinline__ void fft_stage(const cplx *__restrict__ a, cplx *__restrict__ b, int n, int count,
                                          int es, int ts, int Ns, const cplx *__restrict__ tw, bool inv) {
    const int nbf = n / R;
    const int cstep = blockDim.x / nbf;
    const int c0 = threadIdx.x / nbf, j = threadIdx.x - c0 * nbf;
    if (c0 >= cstep) return;
    const int jm = j % Ns;
    const int tmul = n / (Ns * R);
    cplx w[R], d[R];  // stage twiddles, radix-R roots of unity
#pragma unroll
    for (int r = 0; r < R; r++) {
        w[r] = tw[r * jm * tmul];
        d[r] = tw[r * nbf];
        if (inv) {
            w[r].y = -w[r].y;
            d[r].y = -d[r].y;
        }
    }
    const int o = (j / Ns) * Ns * R + jm;
    for (int c = c0; c < count; c += cstep) {
        const cplx *src = a + (size_t)c * ts;
        cplx *dst = b + (size_t)c * ts;
        cplx v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const cplx x = src[(j + r * nbf) * es];
            v[r] = r == 0 ? x : cmul(x, w[r]);
        }
        if (R == 2) {
            dst[o * es] = cadd(v[0], v[1]);
            dst[(o + Ns) * es] = csub(v[0], v[1]);
        } else if (R == 4) {
            const cplx s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
            const cplx s13 = cadd(v[1], v[3]);
            cplx d13 = mul_mi(csub(v[1], v[3]));  // -i (v1 - v3)
            if (inv) d13 = make_float2(-d13.x, -d13.y);
            dst[o * es] = cadd(s02, s13);
            dst[(o + Ns) * es] = cadd(d02, d13);
            dst[(o + 2 * Ns) * es] = csub(s02, s13);
            dst[(o + 3 * Ns) * es] = csub(d02, d13);
        } else {
#pragma unroll
            for (int q = 0; q < R; q++) {
                cplx acc = v[0];
#pragma unroll
                for (int r = 1; r < R; r++) acc = cadd(acc, cmul(v[r], d[(r * q) % R]));
                dst[(o + q * Ns) * es] = acc;
            }
        }
    }
}

// All stages of `count` length-n transforms, ping-ponging between a and b;
// returns the buffer that holds the result.  Ends with a barrier.
__device__ cplx *fft_many(cplx *a, cplx *b, int n, int count, int es, int ts, const signed char *rad, int nr,
                          const cplx *__restrict__ tw, bool inv) {
    int Ns = 1;
    for (int s = 0; s < nr; s++) {
        const int R = rad[s];
        switch (R) {
            case 2: fft_stage<2>(a, b, n, count, es, ts, Ns, tw, inv); break;
            case 3: fft_stage<3>(a, b, n, count, es, ts, Ns, tw, inv); break;
            case 4: fft_stage<4>(a, b, n, count, es, ts, Ns, tw, inv); break;
            default: fft_stage<5>(a, b, n, count, es, ts, Ns, tw, inv); break;
        }
        __syncthreads();
        cplx *t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// ---------------------------------------------------------------------------
// Two-pass (four-step) FFT of length n = N1 * N2.  With input index
// i = k2 + N2 m and output index k = k1 + N1 j2:
//   X[k1 + N1 j2] = sum_k2 W_N2^(k2 j2) W_n^(k2 k1) sum_m x[k2 + N2 m] W_N1^(m k1).
// Pass 1 (one item per (transform, k2)) does the N1-point DFT over m in
// registers and the twiddle W_n^(k2 k1); pass 2 (one item per (transform,
// k1)) does the N2-point DFT over k2.  Between the passes the values go
// through a scratch buffer laid out so that both passes read and write
// shared memory without bank conflicts: rows of a row transform are padded
// to an odd stride, column transforms keep the column index fastest.  Two
// barriers per transform instead of one per radix stage.  All twiddles come
// from the n-entry table tw (W_n^e = tw[e], conjugated for the inverse).
// ---------------------------------------------------------------------------
__device__ __forceinline__ cplx tw_at(const cplx *tw, int e, bool inv) {
    cplx w = tw[e];
    if (inv) w.y = -w.y;
    return w;
}

// In-register DFT of N points; W_N^m = tw[m * ts].
template <int N>
__device__ __forceinline__ void rdft(cplx *v, const cplx *tw, int ts, bool inv) {
    if constexpr (N == 1) {
        return;
    } else if constexpr (N == 2) {
        const cplx a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (N == 4) {
        const cplx s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const cplx s13 = cadd(v[1], v[3]);
        cplx d13 = mul_mi(csub(v[1], v[3]));  // -i (v1 - v3)
        if (inv) d13 = make_float2(-d13.x, -d13.y);
        v[0] = cadd(s02, s13);
        v[1] = cadd(d02, d13);
        v[2] = csub(s02, s13);
        v[3] = csub(d02, d13);
    } else if constexpr (N == 3 || N == 5) {
        cplx o[N];
#pragma unroll
        for (int q = 0; q < N; q++) {
            cplx acc = v[0];
#pragma unroll
            for (int r = 1; r < N; r++) acc = cadd(acc, cmul(v[r], tw_at(tw, ((r * q) % N) * ts, inv)));
            o[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < N; q++) v[q] = o[q];
    } else {
        constexpr int A = (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : (N % 3 == 0) ? 3 : 5;
        constexpr int B = N / A;
        static_assert(A * B == N, "radix");
        cplx t[N];
#pragma unroll
        for (int b = 0; b < B; b++) {
            cplx u[A];
#pragma unroll
            for (int a = 0; a < A; a++) u[a] = v[b + B * a];
            rdft<A>(u, tw, ts * B, inv);
#pragma unroll
            for (int ka = 0; ka < A; ka++)
                t[b + B * ka] = (b * ka == 0) ? u[ka] : cmul(u[ka], tw_at(tw, b * ka * ts, inv));
        }
#pragma unroll
        for (int ka = 0; ka < A; ka++) {
            cplx w[B];
#pragma unroll
            for (int b = 0; b < B; b++) w[b] = t[b + B * ka];
            rdft<B>(w, tw, ts * A, inv);
#pragma unroll
            for (int kb = 0; kb < B; kb++) v[ka + A * kb] = w[kb];
        }
    }
}

// `count` transforms of length N1*N2 over x -> x, scratch s.  ROWS: transform
// c is x[c*ld + i] (contiguous); otherwise x[i*ld + c] (columns).  Ends with
// a barrier.
template <bool ROWS, int N1, int N2>
__device__ void fft2(cplx *x, cplx *s, int count, int ld, const cplx *tw, bool inv) {
    constexpr int P = N2 | 1;  // padded scratch row (odd stride) for row transforms
    for (int it = threadIdx.x; it < count * N2; it += blockDim.x) {
        int c, k2;
        if (ROWS) {
            c = it / N2;
            k2 = it - c * N2;
        } else {
            k2 = it / count;
            c = it - k2 * count;
        }
        cplx v[N1];
#pragma unroll
        for (int m = 0; m < N1; m++) v[m] = ROWS ? x[c * ld + k2 + N2 * m] : x[(k2 + N2 * m) * ld + c];
        rdft<N1>(v, tw, N2, inv);
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) {
            const cplx y = k1 == 0 ? v[0] : cmul(v[k1], tw_at(tw, k1 * k2, inv));
            if (ROWS) s[(c * N1 + k1) * P + k2] = y;
            else s[(k1 * N2 + k2) * count + c] = y;
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < count * N1; it += blockDim.x) {
        int c, k1;
        if (ROWS) {
            c = it / N1;
            k1 = it - c * N1;
        } else {
            k1 = it / count;
            c = it - k1 * count;
        }
        cplx w[N2];
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) w[k2] = ROWS ? s[(c * N1 + k1) * P + k2] : s[(k1 * N2 + k2) * count + c];
        rdft<N2>(w, tw, N1, inv);
#pragma unroll
        for (int j2 = 0; j2 < N2; j2++) {
            if (ROWS) x[c * ld + k1 + N1 * j2] = w[j2];
            else x[(k1 + N1 * j2) * ld + c] = w[j2];
        }
    }
    __syncthreads();
}

// Scratch (complex values) fft2 needs for `count` transforms of pair `pair`.
inline int fft2_scratch(int pair, bool rows, int count) {
    const int n1 = kFftPairs[pair][0], n2 = kFftPairs[pair][1];
    return rows ? count * n1 * (n2 | 1) : count * n1 * n2;
}

// Transforms of one direction of a layer: the two-pass form when the
// length has a factor pair (pair >= 0; result in place in a), else the
// radix stages (result in a or b).  Returns the buffer with the result.
template <bool ROWS>
__device__ cplx *fft_dir(int pair, cplx *a, cplx *b, int n, int count, int ld, const signed char *rad, int nr,
                         const cplx *tw, bool inv) {
    switch (pair) {
#define MB_FFT_CASE(i)                                                          \
    case i:                                                                     \
        fft2<ROWS, kFftPairs[i][0], kFftPairs[i][1]>(a, b, count, ld, tw, inv); \
        return a;
        MB_FFT_CASE(0) MB_FFT_CASE(1) MB_FFT_CASE(2) MB_FFT_CASE(3) MB_FFT_CASE(4) MB_FFT_CASE(5)
        MB_FFT_CASE(6) MB_FFT_CASE(7) MB_FFT_CASE(8) MB_FFT_CASE(9) MB_FFT_CASE(10) MB_FFT_CASE(11)
        MB_FFT_CASE(12) MB_FFT_CASE(13) MB_FFT_CASE(14) MB_FFT_CASE(15) MB_FFT_CASE(16)
#undef MB_FFT_CASE
        default:
            return ROWS ? fft_many(a, b, n, count, 1, ld, rad, nr, tw, inv)
                        : fft_many(a, b, n, count, ld, 1, rad, nr, tw, inv);
    }
}
static_assert(kNumFftPairs == 17, "fft_dir lists one case per factor pair");

constexpr int kFftThreads = 512;  // threads of a layer-FFT CTA
// threads of a k_fd_fused CTA (one 30 m instance's step: 1.09-1.12 ms with
// 512, 1.16-1.17 with 256, 1.37 with 1024, which spills)
constexpr int kFusedThreads = 512;

// Forward: r (instance-major) -> half spectra H.  grid: (nps, nb), block:
// kFftThreads; dynamic shared memory: two buffers of `bufn` complex values,
// then the layer's twiddle tables for n = nx and n = ny.  With `ab`, the CG
// update of this iteration comes first on the layer's points:
// x += alpha p, r -= alpha Ap (alpha = ab[2b]), and the updated r is
// transformed (the k_cg_update_xr of a non-final iteration, fused).  A thread
// issues the loads of kFdLoads row pairs before using any of them, so the
// global round trips overlap instead of following one another.
constexpr int kFdLoads = 5;

__global__ void __launch_bounds__(kFftThreads, 2)
k_fd_fwd(float *__restrict__ r, cplx *__restrict__ H, const __grid_constant__ FdTab ft, const cplx *__restrict__ tw,
         long nxtot, int bufn, float *__restrict__ xw, const float *__restrict__ pv,
         const float *__restrict__ Apv, const float *__restrict__ ab, const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    extern __shared__ cplx fsm[];
    const FdLayer &L = ft.l[blockIdx.x];
    const int b = blockIdx.y;
    const int nx = L.nx, ny = L.ny, h = nx / 2 + 1, np2 = ny / 2;
    cplx *A = fsm, *B = fsm + bufn, *twx = fsm + 2 * bufn, *twy = twx + nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) twx[i] = tw[L.twx + i];
    for (int i = threadIdx.x; i < ny; i += blockDim.x) twy[i] = tw[L.twy + i];
    const size_t base = (size_t)b * nxtot + L.off;
    float *rb = r + base;
    const int xs = blockDim.x / nx, x0 = threadIdx.x / nx, xc = threadIdx.x - x0 * nx;  // nx <= blockDim
    if (x0 < xs) {
        if (ab) {
            const float a = ab[2 * b];
            float *xb = xw + base;
            const float *pb = pv + base, *qb = Apv + base;
            for (int p0 = x0; p0 < np2; p0 += kFdLoads * xs) {
                float xv[kFdLoads][2], pp[kFdLoads][2], rv[kFdLoads][2], qq[kFdLoads][2];
#pragma unroll
                for (int u = 0; u < kFdLoads; u++) {
                    const int p = p0 + u * xs;
                    if (p < np2) {
                        const int o0 = (2 * p) * nx + xc, o1 = o0 + nx;
                        xv[u][0] = xb[o0];
                        xv[u][1] = xb[o1];
                        pp[u][0] = pb[o0];
                        pp[u][1] = pb[o1];
                        rv[u][0] = rb[o0];
                        rv[u][1] = rb[o1];
                        qq[u][0] = qb[o0];
                        qq[u][1] = qb[o1];
                    }
                }
#pragma unroll
                for (int u = 0; u < kFdLoads; u++) {
                    const int p = p0 + u * xs;
                    if (p < np2) {
                        const int o0 = (2 * p) * nx + xc, o1 = o0 + nx;
                        xb[o0] = xv[u][0] + a * pp[u][0];
                        xb[o1] = xv[u][1] + a * pp[u][1];
                        const float r0 = rv[u][0] - a * qq[u][0], r1 = rv[u][1] - a * qq[u][1];
                        rb[o0] = r0;
                        rb[o1] = r1;
                        A[p * nx + xc] = make_float2(r0, r1);
                    }
                }
            }
        } else {
            for (int p0 = x0; p0 < np2; p0 += kFdLoads * xs) {
                float rv[kFdLoads][2];
#pragma unroll
                for (int u = 0; u < kFdLoads; u++) {
                    const int p = p0 + u * xs;
                    if (p < np2) {
                        rv[u][0] = rb[(2 * p) * nx + xc];
                        rv[u][1] = rb[(2 * p + 1) * nx + xc];
                    }
                }
#pragma unroll
                for (int u = 0; u < kFdLoads; u++) {
                    const int p = p0 + u * xs;
                    if (p < np2) A[p * nx + xc] = make_float2(rv[u][0], rv[u][1]);
                }
            }
        }
    }
    __syncthreads();
    cplx *Z = fft_dir<true>(L.px, A, B, nx, np2, nx, L.rx, L.nrx, twx, false);
    cplx *S = (Z == A) ? B : A;
    const int hs_ = blockDim.x / h, h0 = threadIdx.x / h, k = threadIdx.x - h0 * h;
    for (int p = h0; h0 < hs_ && p < np2; p += hs_) {
        const cplx zk = Z[p * nx + k], zm = cconj(Z[p * nx + (k == 0 ? 0 : nx - k)]);
        S[(2 * p) * h + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
        const cplx d = csub(zk, zm);
        S[(2 * p + 1) * h + k] = make_float2(0.5f * d.y, -0.5f * d.x);  // -i/2 (zk - conj(z_-k))
    }
    __syncthreads();
    const cplx *C = fft_dir<false>(L.py, S, Z, ny, h, h, L.ry, L.nry, twy, false);
    cplx *out = H + L.hoff + (size_t)b * L.hs;
    for (int i = threadIdx.x; i < ny * h; i += blockDim.x) out[i] = C[i];
}

// Per-frequency block solve on the blocks of the non-positive x frequencies
// (the leading blocks of the reference's ordering, which reach every stored
// bin): Y_i = sum_j M[blk][j*bs+i] X_j.  A CTA takes floor(256/bs) whole
// blocks and up to NI instances: a thread keeps its row of M in
// registers for all of them, gathers its own member X_i of every instance
// at once (one round trip, not one per instance), stages them in shared
// memory, then forms its row of each instance from the block's members.
// NI (2, 4, 8 or 16) is the batch shape mb_autotune picks: more instances
// per CTA read M fewer times, fewer give more CTAs.
// grid: (ceil(nblk / floor(256/bs)), ceil(nbatch / NI))
constexpr int kFdInst = 8;  // default instances per CTA
constexpr int kMaxBs = 16;

template <int kFdInst>
__global__ void __launch_bounds__(kThreads)
k_fd_mul(const cplx *__restrict__ X, cplx *__restrict__ Y, const cplx *__restrict__ M,
         const FdIndex *__restrict__ idx, int nblk, int bs, int nbatch, const int *__restrict__ act) {
    pdl_enter();
    __shared__ cplx xs[kFdInst][kThreads];
    const int per = kThreads / bs;
    const int lb = threadIdx.x / bs, i = threadIdx.x - lb * bs;
    const int blk = blockIdx.x * per + lb;
    const bool live = lb < per && blk < nblk;
    const int b0 = blockIdx.y * kFdInst, nq = min(kFdInst, nbatch - b0);
    bool on[kFdInst];
#pragma unroll
    for (int q = 0; q < kFdInst; q++) on[q] = q < nq && !inactive(act, b0 + q);
    FdIndex o{};
    cplx m[kMaxBs];
    if (live) {
        o = idx[(size_t)blk * bs + i];
        const cplx *Mb = M + (size_t)blk * bs * bs + i;
#pragma unroll
        for (int jj = 0; jj < kMaxBs; jj++) m[jj] = jj < bs ? Mb[jj * bs] : make_float2(0.f, 0.f);
        cplx xv[kFdInst];
#pragma unroll
        for (int q = 0; q < kFdInst; q++)
            xv[q] = on[q] ? X[o.base + (size_t)(b0 + q) * o.stride] : make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < kFdInst; q++) {
            if (o.flags & kFdConj) xv[q].y = -xv[q].y;
            xs[q][threadIdx.x] = xv[q];
        }
    }
    __syncthreads();
    if (!live || !(o.flags & kFdStore)) return;
#pragma unroll
    for (int q = 0; q < kFdInst; q++) {
        if (!on[q]) continue;
        const cplx *xb = xs[q] + lb * bs;
        float re = 0.f, im = 0.f;
#pragma unroll
        for (int jj = 0; jj < kMaxBs; jj++) {
            if (jj < bs) {
                const cplx xv = xb[jj];
                re += m[jj].x * xv.x - m[jj].y * xv.y;
                im += m[jj].x * xv.y + m[jj].y * xv.x;
            }
        }
        Y[o.base + (size_t)(b0 + q) * o.stride] = make_float2(re, (o.flags & kFdConj) ? -im : im);
    }
}

// ---------------------------------------------------------------------------
// FDPCG blocks rebuilt on the device after a Cn2 update (maos/fdpcg.c:331-580
// fdpcg_prepare, its inversion step).  Per block b, in FP64:
//   M = Hermitian part of (data term + diag(invpsd * l2c_new / l2c_setup)),
//   entries below 1e-15 in magnitude dropped (cspdroptol), then
//   Minv = pseudo-inverse of M with eigenvalues at or below 1e-7 of the
//   largest dropped (the reference's SVD rule: for a Hermitian M the singular
//   values are the eigenvalue magnitudes).  The eigensystem comes from cyclic
//   complex Jacobi rotations, one warp per block: a rotation of columns
//   p, q by c and s e^{i th} (e^{i th} = M_pq / |M_pq|), then of rows p, q,
//   lanes owning rows (column step) or columns (row step).  At most
//   kPrepSweeps sweeps; a sweep is skipped once the off-diagonal norm is
//   below 1e-15 of the diagonal norm.  Blocks are column-major, (i, j) at
//   (b*bs + j)*bs + i, as mb_fdpcg_desc.mbinv.
// ---------------------------------------------------------------------------
constexpr int kPrepWarps = 4;
constexpr int kPrepSweeps = 20;

__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 zaxpy(double a, double2 x, double2 y) { return make_double2(a * x.x + y.x, a * x.y + y.y); }
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// grid: ceil(nb / kPrepWarps) x (32 * kPrepWarps)
__global__ void __launch_bounds__(32 * kPrepWarps)
k_fd_prepare(const double2 *__restrict__ mdata, const double *__restrict__ mdiag, const int *__restrict__ mlayer,
             const double *__restrict__ lscale, double2 *__restrict__ minv, int nb, int bs) {
    __shared__ double2 sA[kPrepWarps][kMaxBs][kMaxBs + 1];
    __shared__ double2 sV[kPrepWarps][kMaxBs][kMaxBs + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * kPrepWarps + warp;
    if (b >= nb) return;  // whole warps only: no CTA-wide barrier below
    double2(*A)[kMaxBs + 1] = sA[warp];
    double2(*V)[kMaxBs + 1] = sV[warp];
    const double2 *Mb = mdata + (size_t)b * bs * bs;
    constexpr int kPer = (kMaxBs * kMaxBs + 31) / 32;
    double2 h[kPer];
#pragma unroll
    for (int u = 0; u < kPer; u++) {  // Hermitian part plus the scaled diagonal
        const int e = lane + 32 * u;
        if (e < bs * bs) {
            const int j = e / bs, i = e - j * bs;
            const double2 a = Mb[e], at = zconj(Mb[(size_t)i * bs + j]);
            double2 v = make_double2(0.5 * (a.x + at.x), 0.5 * (a.y + at.y));
            if (i == j) v.x += mdiag[(size_t)b * bs + i] * lscale[mlayer[(size_t)b * bs + i]];
            if (sqrt(v.x * v.x + v.y * v.y) < 1e-15) v = make_double2(0.0, 0.0);  // cspdroptol
            h[u] = v;
        }
    }
#pragma unroll
    for (int u = 0; u < kPer; u++) {
        const int e = lane + 32 * u;
        if (e < bs * bs) {
            const int j = e / bs, i = e - j * bs;
            A[i][j] = h[u];
            V[i][j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
        }
    }
    __syncwarp();
    for (int sweep = 0; sweep < kPrepSweeps; sweep++) {
        double off = 0, dia = 0;
        for (int e = lane; e < bs * bs; e += 32) {
            const int j = e / bs, i = e - j * bs;
            const double m2 = A[i][j].x * A[i][j].x + A[i][j].y * A[i][j].y;
            if (i == j) dia += m2;
            else off += m2;
        }
        off = warp_allsum(off);
        dia = warp_allsum(dia);
        if (off <= 1e-30 * dia) break;
        for (int p = 0; p < bs - 1; p++)
            for (int q = p + 1; q < bs; q++) {
                const double2 apq = A[p][q];
                const double r = sqrt(apq.x * apq.x + apq.y * apq.y);
                if (r == 0.0) continue;  // uniform over the warp
                const double2 e = make_double2(apq.x / r, apq.y / r);
                const double tau = (A[q][q].x - A[p][p].x) / (2.0 * r);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double c = 1.0 / sqrt(1.0 + t * t), sn = t * c;
                const double2 se = make_double2(sn * e.x, sn * e.y), sec = zconj(se);
                __syncwarp();
                if (lane < bs) {  // columns p, q of A and V
                    const double2 cp = A[lane][p], cq = A[lane][q];
                    A[lane][p] = zaxpy(c, cp, make_double2(-(sec.x * cq.x - sec.y * cq.y), -(sec.x * cq.y + sec.y * cq.x)));
                    A[lane][q] = zaxpy(c, cq, zmul(se, cp));
                    const double2 vp = V[lane][p], vq = V[lane][q];
                    V[lane][p] = zaxpy(c, vp, make_double2(-(sec.x * vq.x - sec.y * vq.y), -(sec.x * vq.y + sec.y * vq.x)));
                    V[lane][q] = zaxpy(c, vq, zmul(se, vp));
                }
                __syncwarp();
                if (lane < bs) {  // rows p, q of A
                    const double2 rp = A[p][lane], rq = A[q][lane];
                    A[p][lane] = zaxpy(c, rp, make_double2(-(se.x * rq.x - se.y * rq.y), -(se.x * rq.y + se.y * rq.x)));
                    A[q][lane] = zaxpy(c, rq, zmul(sec, rp));
                }
                __syncwarp();
            }
    }
    __syncwarp();
    // pseudo-inverse from the eigensystem
    double lmax = 0;
    for (int k = lane; k < bs; k += 32) lmax = fmax(lmax, fabs(A[k][k].x));
    lmax = warp_max(lmax);
    const double thr = 1e-7 * lmax;
    double2 *out = minv + (size_t)b * bs * bs;
    for (int e = lane; e < bs * bs; e += 32) {
        const int j = e / bs, i = e - j * bs;
        double2 acc = make_double2(0.0, 0.0);
        for (int k = 0; k < bs; k++) {
            const double lam = A[k][k].x;
            if (fabs(lam) <= thr) continue;
            const double2 t2 = zmul(V[i][k], zconj(V[j][k]));
            acc.x += t2.x / lam;
            acc.y += t2.y / lam;
        }
        out[e] = acc;
    }
}

// The blocks the half-spectrum solve uses: Hermitian average with the block
// of the negated frequencies (partner bp[b], member map sig) and the FFT
// scaling folded in, as the host does at setup; FP32 out.
// grid: ceil(nbh*bs*bs / 256) x 256
__global__ void k_fd_fold(const double2 *__restrict__ minv, const int *__restrict__ bp, const int *__restrict__ sig,
                          const double *__restrict__ sc, cplx *__restrict__ M, int nbh, int bs) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long)nbh * bs * bs) return;
    const int b = (int)(k / (bs * bs)), r = (int)(k - (long)b * bs * bs);
    const int j = r / bs, i = r - j * bs;
    const long kp = ((long)bp[b] * bs + sig[b * bs + j]) * bs + sig[b * bs + i];
    const double2 a = minv[k], p = minv[kp];
    const double s = sc[b * bs + i] * sc[b * bs + j];
    M[k] = make_float2((float)(0.5 * (a.x + p.x) * s), (float)(0.5 * (a.y - p.y) * s));
}

// ---------------------------------------------------------------------------
// The FDPCG blocks' data term formed on the device (maos/fdpcg.c:427-480), in
// FP64, one CTA per frequency block b:
//   D_b = sum_w sum_{f1,f2} P_w(f1)^H Mmid(f1, f2) P_w(f2) / neam_w^2,
//   Mmid(f1, f2) = (conj(gx_f1) gx_f2 + conj(gy_f1) gy_f2) R(f2 - f1),
// f over the pupil frequencies aliasing to the block (pos x pos of them),
// P_w(f)[a] the propagation of pupil frequency f to member a (layer l at
// shifted frequency (jx, jy)) along WFS w: exp(2 pi i (fx dx_w + fy dy_w))
// with dx_w = ht_l theta_w, times the bilinear alias factor when the layer
// is sampled at half the pupil rate (fdpcg.c:253 fdpcg_prop); zero when f
// does not map to the member.  The v table and the Mmid table are formed once
// per block in shared memory.  out: [nb][bs][bs] column-major, as
// mb_fdpcg_desc.mdata.
// ---------------------------------------------------------------------------
struct FdGeomDev {
    int nxp, nyp, pos, adimx, adimy, nsel, needscale, nwfs, bs;
    double dxp, scale0;  // pupil sampling; nx0*ny0
};
constexpr int kFdDataThreads = 256;

__global__ void __launch_bounds__(kFdDataThreads)
k_fd_data(FdGeomDev G, const int4 *__restrict__ mem, const int2 *__restrict__ blk,
          const double2 *__restrict__ gx, const double2 *__restrict__ gy, const int2 *__restrict__ seld,
          const double2 *__restrict__ selr, const double *__restrict__ neam, const double *__restrict__ thx,
          const double *__restrict__ thy, const double *__restrict__ lht, const int *__restrict__ lnx,
          const int *__restrict__ lny, double2 *__restrict__ out) {
    extern __shared__ double2 fdsm[];
    __shared__ int s_kx[16], s_ky[16];
    const int b = blockIdx.x, bs = G.bs, nw = G.nwfs;
    const int npf = G.pos * G.pos;
    double2 *v = fdsm, *mm = fdsm + (size_t)npf * nw * bs;
    const double dkx = 1.0 / (G.nxp * G.dxp), dky = 1.0 / (G.nyp * G.dxp);
    if (threadIdx.x < npf) {  // pupil frequencies of this block, centred
        const int mxp = threadIdx.x / G.pos, myp = threadIdx.x - mxp * G.pos;
        const int2 bk = blk[b];
        const int kx = bk.x + G.adimx * mxp, ky = bk.y + G.adimy * myp;
        s_kx[threadIdx.x] = ((kx + G.nxp / 2) % G.nxp + G.nxp) % G.nxp - G.nxp / 2;
        s_ky[threadIdx.x] = ((ky + G.nyp / 2) % G.nyp + G.nyp) % G.nyp - G.nyp / 2;
    }
    __syncthreads();
    for (int it = threadIdx.x; it < npf * nw * bs; it += blockDim.x) {
        const int f = it / (nw * bs), w = (it / bs) % nw, a = it % bs;
        const int4 m = mem[(size_t)b * bs + a];  // layer, shifted jx, shifted jy
        const int nx = lnx[m.x], ny = lny[m.x];
        const int kx = s_kx[f], ky = s_ky[f];
        double2 val = make_double2(0.0, 0.0);
        if ((kx + nx / 2 + nx) % nx == m.y && (ky + ny / 2 + ny) % ny == m.z) {
            const double fx = (m.y - nx / 2) * dkx, fy = (m.z - ny / 2) * dky;
            const double ph = 2.0 * M_PI * (fx * (lht[m.x] * thx[w]) + fy * (lht[m.x] * thy[w]));
            double sn, cs;
            sincos(ph, &sn, &cs);
            double amp = 1.0;
            if (G.nxp / nx == 2)
                amp = (1.0 + cos(2.0 * M_PI * (kx * dkx) * G.dxp)) * (1.0 + cos(2.0 * M_PI * (ky * dky) * G.dxp)) * 0.5;
            val = make_double2(cs * amp / neam[w], sn * amp / neam[w]);
        }
        v[((size_t)f * nw + w) * bs + a] = val;
    }
    for (int it = threadIdx.x; it < npf * npf; it += blockDim.x) {
        const int f1 = it / npf, f2 = it - f1 * npf;
        const int p1x = s_kx[f1] + G.nxp / 2, p1y = s_ky[f1] + G.nyp / 2;
        const int p2x = s_kx[f2] + G.nxp / 2, p2y = s_ky[f2] + G.nyp / 2;
        const int dx = ((p2x - p1x) % G.nxp + G.nxp) % G.nxp, dy = ((p2y - p1y) % G.nyp + G.nyp) % G.nyp;
        double2 r = make_double2(0.0, 0.0);
        for (int k = 0; k < G.nsel; k++)
            if (seld[k].x == dx && seld[k].y == dy) r = selr[k];
        const double2 a1 = gx[(size_t)p1y * G.nxp + p1x], a2 = gx[(size_t)p2y * G.nxp + p2x];
        const double2 c1 = gy[(size_t)p1y * G.nxp + p1x], c2 = gy[(size_t)p2y * G.nxp + p2x];
        const double2 g = make_double2(a1.x * a2.x + a1.y * a2.y + c1.x * c2.x + c1.y * c2.y,
                                       a1.x * a2.y - a1.y * a2.x + c1.x * c2.y - c1.y * c2.x);  // conj(g1) g2
        mm[it] = make_double2(g.x * r.x - g.y * r.y, g.x * r.y + g.y * r.x);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < bs * bs; e += blockDim.x) {
        const int i = e % bs, j = e / bs;  // row (member i), column (member j)
        double re = 0.0, im = 0.0;
        for (int f1 = 0; f1 < npf; f1++)
            for (int f2 = 0; f2 < npf; f2++) {
                const double2 q = mm[f1 * npf + f2];
                if (q.x == 0.0 && q.y == 0.0) continue;
                for (int w = 0; w < nw; w++) {
                    const double2 a = v[((size_t)f1 * nw + w) * bs + i], c = v[((size_t)f2 * nw + w) * bs + j];
                    const double ur = a.x * c.x + a.y * c.y, ui = a.x * c.y - a.y * c.x;  // conj(a) c
                    re += ur * q.x - ui * q.y;
                    im += ur * q.y + ui * q.x;
                }
            }
        if (!G.needscale) {
            re *= G.scale0;
            im *= G.scale0;
        }
        out[((size_t)b * bs + j) * bs + i] = make_double2(re, im);
    }
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Inverse: half spectra H -> z (instance-major), plus the r.z partial of this
// (layer, instance); the last CTA of an instance leaves (r.z)_0 or beta.
// grid: (nps, nb); shared memory as k_fd_fwd.
// PU (CG step, launched as clusters of the nps layer CTAs of one instance):
// the CTAs exchange their r.z partials through distributed shared memory
// behind a cluster barrier, each forms r.z (same order, same value) and
// beta, and updates its own layer of p = z + beta p (init: p = z), which
// replaces the separate p update launch; z is not written.  Rank 0 records
// the CG scalars as cg_rz_last does.
template <bool PU>
__global__ void __launch_bounds__(kFftThreads, 2)
k_fd_inv(const cplx *__restrict__ H, const float *__restrict__ r, float *__restrict__ z,
         double *__restrict__ rz_part, const __grid_constant__ FdTab ft, const cplx *__restrict__ tw, long nxtot,
         int bufn, CgScal SC, int kit, int init, const int *__restrict__ act, float *__restrict__ pv) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    extern __shared__ cplx fsm[];
    __shared__ double sh[32];
    const FdLayer &L = ft.l[blockIdx.x];
    const int b = blockIdx.y;
    const int nx = L.nx, ny = L.ny, h = nx / 2 + 1, np2 = ny / 2;
    cplx *A = fsm, *B = fsm + bufn, *twx = fsm + 2 * bufn, *twy = twx + nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) twx[i] = tw[L.twx + i];
    for (int i = threadIdx.x; i < ny; i += blockDim.x) twy[i] = tw[L.twy + i];
    const cplx *in = H + L.hoff + (size_t)b * L.hs;
    constexpr int kLd = 2 * kFdLoads;  // spectrum values a thread loads before storing any
    for (int i0 = threadIdx.x; i0 < ny * h; i0 += kLd * blockDim.x) {
        cplx v[kLd];
#pragma unroll
        for (int u = 0; u < kLd; u++) {
            const int i = i0 + u * blockDim.x;
            if (i < ny * h) v[u] = in[i];
        }
#pragma unroll
        for (int u = 0; u < kLd; u++) {
            const int i = i0 + u * blockDim.x;
            if (i < ny * h) A[i] = v[u];
        }
    }
    __syncthreads();
    cplx *C = fft_dir<false>(L.py, A, B, ny, h, h, L.ry, L.nry, twy, true);
    cplx *Zb = (C == A) ? B : A;
    const int xs = blockDim.x / nx, x0 = threadIdx.x / nx, k = threadIdx.x - x0 * nx;
    for (int p = x0; x0 < xs && p < np2; p += xs) {
        const int i = p * nx + k;
        const bool hi = k > nx / 2;
        const int kk = hi ? nx - k : k;
        cplx a = C[(2 * p) * h + kk], c = C[(2 * p + 1) * h + kk];
        if (kk == 0 || kk == nx / 2) {
            a.y = 0.f;
            c.y = 0.f;
        }
        if (hi) {
            a = cconj(a);
            c = cconj(c);
        }
        Zb[i] = make_float2(a.x - c.y, a.y + c.x);  // a + i c
    }
    __syncthreads();
    const cplx *Zo = fft_dir<true>(L.px, Zb, C, nx, np2, nx, L.rx, L.nrx, twx, true);
    const size_t base = (size_t)b * nxtot + L.off;
    double v = 0;
    for (int p0 = x0; x0 < xs && p0 < np2; p0 += kFdLoads * xs) {
        float rv[kFdLoads][2];
#pragma unroll
        for (int u = 0; u < kFdLoads; u++) {
            const int p = p0 + u * xs;
            if (p < np2) {
                const size_t o0 = base + (size_t)(2 * p) * nx + k;
                rv[u][0] = r[o0];
                rv[u][1] = r[o0 + nx];
            }
        }
#pragma unroll
        for (int u = 0; u < kFdLoads; u++) {
            const int p = p0 + u * xs;
            if (p < np2) {
                const cplx q = Zo[p * nx + k];
                const size_t o0 = base + (size_t)(2 * p) * nx + k, o1 = o0 + nx;
                if (!PU) {
                    z[o0] = q.x;
                    z[o1] = q.y;
                }
                v += (double)q.x * rv[u][0] + (double)q.y * rv[u][1];
            }
        }
    }
    v = block_sum(v, sh);
    if constexpr (!PU) {
        if (threadIdx.x == 0) rz_part[(size_t)b * gridDim.x + blockIdx.x] = v;
        if (SC.sc) cg_rz_last(rz_part + (size_t)b * gridDim.x, SC, b, kit, init);
    } else {
        __shared__ double s_part, s_be;
        if (threadIdx.x == 0) s_part = v;
        cluster_sync_all();  // every rank's partial is in its shared memory
        if (threadIdx.x < 32) {
            // lane i reads rank i (the layer order), summed as warp_sum_fresh sums rz_part
            double t = 0;
            if (threadIdx.x < (int)gridDim.x) {
                const unsigned la = (unsigned)__cvta_generic_to_shared(&s_part);
                unsigned ra;
                asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(la), "r"((unsigned)threadIdx.x));
                asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(t) : "r"(ra) : "memory");
            }
            t = warp_sum(t);
            if (threadIdx.x == 0) {
                const double rz = t;
                double be = 0;
                if (!init) {
                    be = rz / SC.sc[(size_t)b * SC.nsc + kit];
                    if (!isfinite(be)) be = 0;
                }
                s_be = be;
                if (blockIdx.x == 0) {  // rank 0 keeps the CG scalars
                    if (init) {  // start (or restart) at iteration kit
                        SC.sc[(size_t)b * SC.nsc + kit] = rz;
                    } else {
                        SC.ab[2 * b + 1] = (float)be;
                        SC.sc[(size_t)b * SC.nsc + kit + 1] = rz;
                    }
                }
            }
        }
        __syncthreads();
        asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");  // done reading the others
        const float be = (float)s_be;
        for (int p0 = x0; x0 < xs && p0 < np2; p0 += kFdLoads * xs) {
            float pp[kFdLoads][2];
#pragma unroll
            for (int u = 0; u < kFdLoads; u++) {
                const int p = p0 + u * xs;
                if (p < np2 && !init) {
                    const size_t o0 = base + (size_t)(2 * p) * nx + k;
                    pp[u][0] = pv[o0];
                    pp[u][1] = pv[o0 + nx];
                }
            }
#pragma unroll
            for (int u = 0; u < kFdLoads; u++) {
                const int p = p0 + u * xs;
                if (p < np2) {
                    const cplx q = Zo[p * nx + k];
                    const size_t o0 = base + (size_t)(2 * p) * nx + k;
                    pv[o0] = init ? q.x : q.x + be * pp[u][0];
                    pv[o0 + nx] = init ? q.y : q.y + be * pp[u][1];
                }
            }
        }
        asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");  // no rank leaves while read
    }
}

// ---------------------------------------------------------------------------
// The whole preconditioner of one CG step in one launch, for small batches.
//
// An instance's layers are split over the CTAs of one thread-block cluster
// (at most 16): layer l gets K_l CTAs, K_l proportional to its size, so a
// 96 x 96 ground layer is transformed by 4 CTAs and a 48 x 48 one by 1.  A
// CTA owns a range of row pairs and a range of half-spectrum columns of its
// layer.  Phases, separated by cluster barriers, with the data exchanged
// through distributed shared memory (ld/st.shared::cluster):
//   F1  x += a p, r -= a Ap on its row pairs (the CG update, when ab is set),
//       row FFTs of r, unpacking into half-spectrum rows stored straight into
//       the column owners' SC (stores into the receiver's shared memory before
//       the barrier: no remote load waits on a round trip);
//   F2  column FFTs (SC);
//   M   its share of the frequency blocks: members gathered from the column
//       owners' SC, Y = Mbinv X, each stored bin written into its owner's SY;
//   I1  inverse column FFTs of SY, row pairs stored straight into the row
//       owners' R (Hermitian mirror);
//   I2  inverse row FFTs, then r.z over the cluster, beta and p = z + beta p.
// Every shared-memory region sits at the same offset in every CTA of the
// kernel, so a peer's copy is the local address mapped to the peer's rank.
// ---------------------------------------------------------------------------
constexpr int kMaxFdParts = 16;  // CTAs in an instance's cluster
struct FdPart {
    short l, q, K, rbase;  // layer, split index, splits of the layer, cluster rank of its split 0
    short p0, p1;          // row pairs [p0, p1)
    short c0, c1;          // half-spectrum columns [c0, c1)
    int b0, b1;            // frequency blocks solved [b0, b1)
};
struct FdFusedTab {
    FdPart c[kMaxFdParts];
    int C;                 // CTAs per instance (cluster size)
    int oTY, oR, oS, oSC, oSY;  // shared-memory offsets (complex elements); twiddles x at 0
};
// One member of a solved block: the cluster rank that owns its bin, the bin's
// offset in that CTA's SC / SY, and the conjugate / store flags of FdIndex.
struct FdMem {
    int off;
    short rank;
    short flags;
};

__device__ __forceinline__ unsigned dsm_base(const void *local, unsigned rank) {
    const unsigned la = (unsigned)__cvta_generic_to_shared(local);
    unsigned ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(la), "r"(rank));
    return ra;
}
__device__ __forceinline__ cplx dsm_ld(unsigned a) {
    float x, y;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "r"(a) : "memory");
    return make_float2(x, y);
}
__device__ __forceinline__ double dsm_ld_f64(unsigned a) {
    double t;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(t) : "r"(a) : "memory");
    return t;
}
__device__ __forceinline__ void dsm_st(unsigned a, cplx v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}

// The transform of fft_dir with its result moved back into a (the shared
// layout peers read needs the result at a fixed place).  Ends with a barrier.
template <bool ROWS>
__device__ void fft_dir_inplace(int pair, cplx *a, cplx *b, int n, int count, int ld, const signed char *rad,
                                int nr, const cplx *tw, bool inv) {
    const cplx *res = fft_dir<ROWS>(pair, a, b, n, count, ld, rad, nr, tw, inv);
    if (res != a) {
        const int tot = ROWS ? count * ld : n * ld;
        for (int i = threadIdx.x; i < tot; i += blockDim.x) a[i] = res[i];
        __syncthreads();
    }
}

// grid: (C, nb), clusters of C CTAs along x; block: kFusedThreads (one CTA
// per SM: the registers carry r, p and a block row between phases).
__global__ void __launch_bounds__(kFusedThreads, 1)
k_fd_fused(float *__restrict__ r, const __grid_constant__ FdTab ft, const __grid_constant__ FdFusedTab fu,
           const cplx *__restrict__ tw, const cplx *__restrict__ M, const FdMem *__restrict__ mem, int bs,
           long nxtot, float *__restrict__ xw, const float *__restrict__ Apv, CgScal SC, int kit, int init,
           const int *__restrict__ act, float *__restrict__ pv) {
    pdl_enter();
    // an instance's CTAs are one cluster: all return or none does
    if (inactive(act, blockIdx.y)) return;
    extern __shared__ cplx fsm[];
    __shared__ double sh[32];
    const FdPart P = fu.c[blockIdx.x];
    const FdLayer &L = ft.l[P.l];
    const int b = blockIdx.y;
    const int nx = L.nx, ny = L.ny, h = nx / 2 + 1;
    const int npr = P.p1 - P.p0, ncl = P.c1 - P.c0;
    cplx *twx = fsm, *twy = fsm + fu.oTY, *R = fsm + fu.oR, *S = fsm + fu.oS;
    cplx *SCb = fsm + fu.oSC, *SY = fsm + fu.oSY;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) twx[i] = tw[L.twx + i];
    for (int i = threadIdx.x; i < ny; i += blockDim.x) twy[i] = tw[L.twy + i];
    const size_t base = (size_t)b * nxtot + L.off;
    float *rb = r + base;
    const int xs = blockDim.x / nx, x0 = threadIdx.x / nx, xc = threadIdx.x - x0 * nx;  // nx <= blockDim
    // ---- F1: CG update and row FFTs of this CTA's row pairs.  When a thread's
    // rows fit one pass (one = true), the updated r and the old p stay in its
    // registers for the r.z and the p update at the end.
    const bool one = npr <= kFdLoads * xs;
    float rv[kFdLoads][2], pp[kFdLoads][2];
    if (x0 < xs) {
        const float a = SC.ab ? SC.ab[2 * b] : 0.f;
        for (int p0 = P.p0 + x0; p0 < P.p1; p0 += kFdLoads * xs) {
            float xv[kFdLoads][2], qq[kFdLoads][2];
#pragma unroll
            for (int u = 0; u < kFdLoads; u++) {
                const int p = p0 + u * xs;
                if (p < P.p1) {
                    const int o0 = (2 * p) * nx + xc, o1 = o0 + nx;
                    rv[u][0] = rb[o0];
                    rv[u][1] = rb[o1];
                    if (xw) {
                        xv[u][0] = xw[base + o0];
                        xv[u][1] = xw[base + o1];
                        pp[u][0] = pv[base + o0];
                        pp[u][1] = pv[base + o1];
                        qq[u][0] = Apv[base + o0];
                        qq[u][1] = Apv[base + o1];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kFdLoads; u++) {
                const int p = p0 + u * xs;
                if (p < P.p1) {
                    const int o0 = (2 * p) * nx + xc, o1 = o0 + nx;
                    float r0 = rv[u][0], r1 = rv[u][1];
                    if (xw) {
                        xw[base + o0] = xv[u][0] + a * pp[u][0];
                        xw[base + o1] = xv[u][1] + a * pp[u][1];
                        r0 -= a * qq[u][0];
                        r1 -= a * qq[u][1];
                        rb[o0] = r0;
                        rb[o1] = r1;
                        rv[u][0] = r0;
                        rv[u][1] = r1;
                    }
                    R[(p - P.p0) * nx + xc] = make_float2(r0, r1);
                }
            }
        }
    }
    __syncthreads();
    fft_dir_inplace<true>(L.px, R, S, nx, npr, nx, L.rx, L.nrx, twx, false);
    {  // unpack into half-spectrum rows, each bin stored straight into its
       // column owner's SC (distributed shared memory: stores, no round trip)
        const int hs_ = blockDim.x / h, h0 = threadIdx.x / h, k = threadIdx.x - h0 * h;
        int q = P.K - 1;  // the column owner of bin k
        while (fu.c[P.rbase + q].c0 > k) q--;
        const FdPart O = fu.c[P.rbase + q];
        const int on = O.c1 - O.c0;
        const unsigned oa = dsm_base(SCb, (unsigned)(P.rbase + q)) + 8u * (unsigned)(k - O.c0);
        for (int p = h0; h0 < hs_ && p < npr; p += hs_) {
            const cplx zk = R[p * nx + k], zm = cconj(R[p * nx + (k == 0 ? 0 : nx - k)]);
            const cplx d = csub(zk, zm);
            const int i = 2 * (P.p0 + p);  // the layer row of the first of the pair
            dsm_st(oa + 8u * (unsigned)(i * on), make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y)));
            dsm_st(oa + 8u * (unsigned)((i + 1) * on), make_float2(0.5f * d.y, -0.5f * d.x));  // -i/2 (zk - conj(z_-k))
        }
    }
    cluster_sync_all();  // B1: every CTA's columns are complete in its SC
    // ---- F2: column FFTs of this CTA's columns
    fft_dir_inplace<false>(L.py, SCb, S, ny, ncl, ncl, L.ry, L.nry, twy, false);
    cluster_sync_all();  // B2: spectra final in every SC; no SR is read any more
    // ---- M: this CTA's frequency blocks: a thread gathers one member of a
    // block into shared memory, then forms its row of Y = Mbinv X
    {
        const int per = blockDim.x / bs;
        const int lb = threadIdx.x / bs, i = threadIdx.x - lb * bs;
        cplx *xsb = R;  // staging of the gathered members (R is free now)
        for (int blk0 = P.b0; blk0 < P.b1; blk0 += per) {
            const int blk = blk0 + lb;
            const bool live = lb < per && blk < P.b1;
            FdMem e{};
            cplx m[kMaxBs];
            if (live) {
                e = mem[(size_t)blk * bs + i];
                const cplx *Mb = M + (size_t)blk * bs * bs + i;
#pragma unroll
                for (int jj = 0; jj < kMaxBs; jj++) m[jj] = jj < bs ? Mb[jj * bs] : make_float2(0.f, 0.f);
                cplx xv = dsm_ld(dsm_base(SCb, (unsigned)e.rank) + 8u * (unsigned)e.off);
                if (e.flags & kFdConj) xv.y = -xv.y;
                xsb[threadIdx.x] = xv;
            }
            __syncthreads();
            if (live && (e.flags & kFdStore)) {
                const cplx *xb = xsb + lb * bs;
                float re = 0.f, im = 0.f;
#pragma unroll
                for (int jj = 0; jj < kMaxBs; jj++) {
                    if (jj < bs) {
                        const cplx xv = xb[jj];
                        re += m[jj].x * xv.x - m[jj].y * xv.y;
                        im += m[jj].x * xv.y + m[jj].y * xv.x;
                    }
                }
                dsm_st(dsm_base(SY, (unsigned)e.rank) + 8u * (unsigned)e.off,
                       make_float2(re, (e.flags & kFdConj) ? -im : im));
            }
            __syncthreads();
        }
    }
    cluster_sync_all();  // B3: every stored bin of every SY written; no SC is read any more
    // ---- I1: inverse column FFTs, then each column's row pairs stored straight
    // into the row owners' R as a + i c (and, mirrored, at nx - k)
    fft_dir_inplace<false>(L.py, SY, S, ny, ncl, ncl, L.ry, L.nry, twy, true);
    for (int it = threadIdx.x; it < (ny / 2) * ncl; it += blockDim.x) {
        const int p = it / ncl, cl = it - p * ncl;  // layer row pair p, local column cl
        const int kk = P.c0 + cl;
        cplx a = SY[(2 * p) * ncl + cl], c = SY[(2 * p + 1) * ncl + cl];
        if (kk == 0 || kk == nx / 2) {
            a.y = 0.f;
            c.y = 0.f;
        }
        int q = P.K - 1;  // the row owner of pair p
        while (fu.c[P.rbase + q].p0 > p) q--;
        const unsigned ra = dsm_base(R, (unsigned)(P.rbase + q)) +
                            8u * (unsigned)((p - fu.c[P.rbase + q].p0) * nx);
        dsm_st(ra + 8u * (unsigned)kk, make_float2(a.x - c.y, a.y + c.x));  // a + i c
        if (kk > 0 && kk < nx / 2) {
            a = cconj(a);
            c = cconj(c);
            dsm_st(ra + 8u * (unsigned)(nx - kk), make_float2(a.x - c.y, a.y + c.x));
        }
    }
    cluster_sync_all();  // B4: every CTA's row pairs are complete in its R
    // ---- I2: inverse row FFTs
    fft_dir_inplace<true>(L.px, R, S, nx, npr, nx, L.rx, L.nrx, twx, true);
    double v = 0;
    if (x0 < xs)
        for (int p0 = P.p0 + x0; p0 < P.p1; p0 += kFdLoads * xs) {
            if (!one) {
#pragma unroll
                for (int u = 0; u < kFdLoads; u++) {
                    const int p = p0 + u * xs;
                    if (p < P.p1) {
                        const size_t o0 = (size_t)(2 * p) * nx + xc;
                        rv[u][0] = rb[o0];
                        rv[u][1] = rb[o0 + nx];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kFdLoads; u++) {
                const int p = p0 + u * xs;
                if (p < P.p1) {
                    const cplx q = R[(p - P.p0) * nx + xc];
                    v += (double)q.x * rv[u][0] + (double)q.y * rv[u][1];
                }
            }
        }
    v = block_sum(v, sh);
    __shared__ double s_part, s_be;
    if (threadIdx.x == 0) s_part = v;
    cluster_sync_all();  // B5: every rank's r.z partial is in its shared memory; no SY is read any more
    if (threadIdx.x < 32) {
        // lane i reads rank i, in rank order
        double t = 0;
        if (threadIdx.x < fu.C) t = dsm_ld_f64(dsm_base(&s_part, (unsigned)threadIdx.x));
        t = warp_sum(t);
        if (threadIdx.x == 0) {
            double be = 0;
            if (!init) {
                be = t / SC.sc[(size_t)b * SC.nsc + kit];
                if (!isfinite(be)) be = 0;
            }
            s_be = be;
            if (blockIdx.x == 0) {  // rank 0 keeps the CG scalars
                if (init) {  // start (or restart) at iteration kit
                    SC.sc[(size_t)b * SC.nsc + kit] = t;
                } else {
                    SC.ab[2 * b + 1] = (float)be;
                    SC.sc[(size_t)b * SC.nsc + kit + 1] = t;
                }
            }
        }
    }
    __syncthreads();
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");  // done reading the others
    const float be = (float)s_be;
    if (x0 < xs)
        for (int p0 = P.p0 + x0; p0 < P.p1; p0 += kFdLoads * xs) {
            if (!one || !xw) {  // the old p is in registers only after a CG update pass
#pragma unroll
                for (int u = 0; u < kFdLoads; u++) {
                    const int p = p0 + u * xs;
                    if (p < P.p1 && !init) {
                        const size_t o0 = base + (size_t)(2 * p) * nx + xc;
                        pp[u][0] = pv[o0];
                        pp[u][1] = pv[o0 + nx];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kFdLoads; u++) {
                const int p = p0 + u * xs;
                if (p < P.p1) {
                    const cplx q = R[(p - P.p0) * nx + xc];
                    const size_t o0 = base + (size_t)(2 * p) * nx + xc;
                    pv[o0] = init ? q.x : q.x + be * pp[u][0];
                    pv[o0 + nx] = init ? q.y : q.y + be * pp[u][1];
                }
            }
        }
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");  // no rank leaves while read
}

// float <-> double staging helpers for the host-facing API
__global__ void k_scale_copy(const float *__restrict__ a, float *__restrict__ o, float s, long n) {
    pdl_enter();
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) o[j] = s * a[j];
}

}  // namespace mb
