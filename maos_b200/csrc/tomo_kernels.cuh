// Tomography kernels for B200 (sm_100a).
//
// Every kernel is batched: blockIdx.z (or .y) selects one of `nb` independent
// instances that share the operator tables.  Instance vectors are stored
// instance-major (x[b*nxtot + ...]).  Reductions are deterministic: each block
// writes one FP64 partial, and consumers add the partials in a fixed order.
//
// Reference counterparts (cuda/tomo.cu, cuda/prop_wrap.cu, cuda/pcg.cu):
//   k_hx        gpu_map2map_do forward (prop_wrap.cu:35)      -- bilinear gather
//   k_gp        gpu_gp_do (tomo.cu:362)                       -- GP stencil + TT sums
//   k_gpt       gpu_gpt_do (tomo.cu:485)                      -- gather form, no atomics
//   k_hxt       gpu_map2map_do 't' + gpu_laplacian_do         -- gather form, no atomics
//   k_cg_*      gpu_pcg scalar kernels (pcg.cu:27-57)         -- FP64 scalars
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

// Serving: `act` (null: every instance) marks the instances that take part in
// this launch.  Blocks of an inactive instance return before touching memory,
// so its warm-start state stays as it was and no other instance's result
// depends on which instances are active.  Block-uniform (b is a block index).
__device__ __forceinline__ bool inactive(const int *act, int b) { return act && __ldg(act + b) == 0; }

// ---------------------------------------------------------------------------
// Hx: opd[b][w][p] = sum_l bilinear(x_l) at the ray of pupil point p.
// grid: (ceil(np/256), nwfs, nb)
// ---------------------------------------------------------------------------
__global__ void k_hx(const float *__restrict__ x, float *__restrict__ opd,
                     const AxisW *__restrict__ tab, const LayerDev *__restrict__ lay, int nps,
                     int nwfs, int nxp, int nyp, long nxtot, const float *__restrict__ w1,
                     double *__restrict__ w1_part, const int *__restrict__ act) {
    if (inactive(act, blockIdx.z)) return;
    __shared__ double sh[32];
    const int np = nxp * nyp;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = blockIdx.y, b = blockIdx.z;
    float acc = 0.f;
    if (p < np) {
        const int ix = p % nxp, iy = p / nxp;
        const float *xb = x + (size_t)b * nxtot;
        for (int l = 0; l < nps; l++) {
            const AxisW *t = tab + (size_t)(w * nps + l) * (nxp + nyp);
            const AxisW tx = t[ix], ty = t[nxp + iy];
            if (tx.k < 0 || ty.k < 0) continue;
            const int nx = lay[l].nx;
            const float *X = xb + lay[l].off + (size_t)ty.k * nx + tx.k;
            const float a = tx.w0 * X[0] + tx.w1 * X[1];
            const float c = tx.w0 * X[nx] + tx.w1 * X[nx + 1];
            acc += ty.w0 * a + ty.w1 * c;
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

// ---------------------------------------------------------------------------
// GP^T NEA^-1 (I - TT PTT) in gather form: each pupil point collects from the
// (pos+1)^2 subapertures whose stencil covers it.
// grid: (ceil(np/256), nwfs, nb)
// ---------------------------------------------------------------------------
__global__ void k_gpt(const float *__restrict__ grad, const float *__restrict__ tt,
                      float *__restrict__ opd2, const WfsDev *__restrict__ wfs, int nwfs,
                      int nxp, int nyp, long ngrad, int do_tt, float alpha,
                      const int *__restrict__ act) {
    if (inactive(act, blockIdx.z)) return;
    const int w = blockIdx.y, b = blockIdx.z;
    const WfsDev W = wfs[w];
    const bool use_tt = do_tt && W.has_ptt;
    const int np = nxp * nyp;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int px = p % nxp, py = p / nxp;
    const int n1 = W.pos + 1;
    const float *g = grad + (size_t)b * ngrad + W.goff;
    const float ttx = use_tt ? tt[((size_t)b * nwfs + w) * 2] : 0.f;
    const float tty = use_tt ? tt[((size_t)b * nwfs + w) * 2 + 1] : 0.f;
    float acc = 0.f;
    for (int dy = 0; dy < n1; dy++) {
        const int cy = py - dy;
        if (cy < 0) break;
        for (int dx = 0; dx < n1; dx++) {
            const int cx = px - dx;
            if (cx < 0) break;
            const int s = W.samap[cy * nxp + cx];
            if (s < 0) continue;
            const float gx = g[s] + ttx;
            const float gy = g[s + W.nsa] + tty;
            const float *ne = W.neai + 3 * s;
            const float nx_ = ne[0] * gx + ne[2] * gy;
            const float ny_ = ne[2] * gx + ne[1] * gy;
            const float2 k = W.gp[(size_t)s * n1 * n1 + dy * n1 + dx];
            acc += k.x * nx_ + k.y * ny_;
        }
    }
    opd2[((size_t)b * nwfs + w) * np + p] = alpha * acc;
}

// ---------------------------------------------------------------------------
// Hx^T in gather form (+ L2^T L2 regularisation and p.Ap partial for the LHS).
// Layer points are flattened over all layers; grid: (nblk_x, nb).
// The transposed table for (w, l, axis) is a CSR list per layer column/row.
// ---------------------------------------------------------------------------
struct GatherIndex {
    const int *ptr;        // [ntab] offsets of each (w,l,axis) CSR in `idx_ptr`
    const int *idx_ptr;    // concatenated CSR row pointers
    const GatherW *ent;    // concatenated entries
};

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

__global__ void k_hxt(const float *__restrict__ opd2, const float *__restrict__ xin,
                      float *__restrict__ out, double *__restrict__ dot_part, GatherIndex gi,
                      const LayerDev *__restrict__ lay, int nps, int nwfs, int nxp, int nyp,
                      long nxtot, int do_l2, float alpha, LowRank lr, CgScal S, int k,
                      const int *__restrict__ act) {
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
    if (j < nxtot) {
        int l = 0;
        while (l + 1 < nps && j >= lay[l + 1].off) l++;
        const LayerDev L = lay[l];
        const int jj = (int)(j - L.off);
        const int jx = jj % L.nx, jy = jj / L.nx;
        const int np = nxp * nyp;
        float acc = 0.f;
        for (int w = 0; w < nwfs; w++) {
            const int tx = gi.ptr[(w * nps + l) * 2 + 0];
            const int ty = gi.ptr[(w * nps + l) * 2 + 1];
            const int ax0 = gi.idx_ptr[tx + jx], ax1 = gi.idx_ptr[tx + jx + 1];
            const int ay0 = gi.idx_ptr[ty + jy], ay1 = gi.idx_ptr[ty + jy + 1];
            if (ax0 == ax1 || ay0 == ay1) continue;
            const float *o = opd2 + ((size_t)b * nwfs + w) * np;
            for (int ay = ay0; ay < ay1; ay++) {
                const GatherW ey = gi.ent[ay];
                float rs = 0.f;
                for (int ax = ax0; ax < ax1; ax++) {
                    const GatherW ex = gi.ent[ax];
                    rs += ex.w * o[ey.i * nxp + ex.i];
                }
                acc += ey.w * rs;
            }
        }
        const float *X = xin ? xin + (size_t)b * nxtot + L.off : nullptr;
        if (do_l2) {
            const int nx = L.nx, ny = L.ny;
            auto at = [&](int dx, int dy) {
                int xx = jx + dx, yy = jy + dy;
                xx += (xx < 0) ? nx : 0;
                xx -= (xx >= nx) ? nx : 0;
                yy += (yy < 0) ? ny : 0;
                yy -= (yy >= ny) ? ny : 0;
                return X[yy * nx + xx];
            };
            const float st = 20.f * at(0, 0) -
                             8.f * (at(-1, 0) + at(1, 0) + at(0, -1) + at(0, 1)) +
                             2.f * (at(-1, -1) + at(1, -1) + at(-1, 1) + at(1, 1)) +
                             (at(0, -2) + at(-2, 0) + at(2, 0) + at(0, 2));
            acc = alpha * acc + alpha * L.l2c * st;
        } else {
            acc = alpha * acc;
        }
        if (lr.nw) {
            float lt = 0.f;
            for (int k = 0; k < lr.nnw; k++) lt += lr.nw[(size_t)k * nxtot + j] * s_t[k];
            acc += alpha * lt;
        }
        out[(size_t)b * nxtot + j] = acc;
        if (dot_part && X) dotv = (double)acc * (double)X[jj];
    }
    if (dot_part) {
        dotv = block_sum(dotv, sh);
        if (threadIdx.x == 0) dot_part[(size_t)b * gridDim.x + blockIdx.x] = dotv;
        cg_alpha_last(dot_part + (size_t)b * gridDim.x, S, b, k);
    }
}

// ---------------------------------------------------------------------------
// Tiled Hx^T (+ L2^T L2 and p.Ap partials) for the tomography.
// One CTA = one instance x one tile of `ny` consecutive rows of one layer.
// The bilinear transpose is separable, so per WFS the CTA
//   1. stages that WFS's x-gather lists for the layer in shared memory,
//   2. x pass: t[iy][jx] = sum_x w * opd2[iy][ix] for the pupil rows that
//      reach the tile (coalesced reads along each pupil row),
//   3. y pass: acc[jy][jx] += sum_y w * t[iy][jx] into registers.
// grid: (ntiles, nb); dynamic smem: maxrows*maxnx floats + lists.
// ---------------------------------------------------------------------------
struct TileDesc {
    int l;     // layer
    int jy0;   // first layer row
    int ny;    // rows in this tile
};
constexpr int kMaxOwn = 8;  // layer points per thread (tile rows * nx <= 256 * kMaxOwn)

__global__ void __launch_bounds__(kThreads)
k_hxt_tiled(const float *__restrict__ opd2, const float *__restrict__ xin, float *__restrict__ out,
            double *__restrict__ dot_part, GatherIndex gi, const LayerDev *__restrict__ lay,
            const TileDesc *__restrict__ tiles, const int2 *__restrict__ rowrange, int nps, int nwfs,
            int nxp, int nyp, long nxtot, int do_l2, float alpha, int maxrows, int maxnx,
            int maxent, CgScal S, int kit, const int *__restrict__ act) {
    if (inactive(act, blockIdx.y)) return;
    extern __shared__ float smem[];
    __shared__ double sh[32];
    const int tid = blockIdx.x, b = blockIdx.y;
    const TileDesc T = tiles[tid];
    const LayerDev L = lay[T.l];
    const int nx = L.nx;
    const int nown = T.ny * nx;
    float *t = smem;
    int *xptr = reinterpret_cast<int *>(t + (size_t)maxrows * maxnx);
    GatherW *xent = reinterpret_cast<GatherW *>(xptr + ((maxnx + 2) & ~1));
    const int np = nxp * nyp;
    float acc[kMaxOwn];
#pragma unroll
    for (int k = 0; k < kMaxOwn; k++) acc[k] = 0.f;
    for (int w = 0; w < nwfs; w++) {
        const int2 rr = rowrange[(size_t)tid * nwfs + w];
        if (rr.y < rr.x) continue;  // uniform over the CTA
        const int tx = gi.ptr[(w * nps + T.l) * 2 + 0];
        const int ty = gi.ptr[(w * nps + T.l) * 2 + 1];
        const int e0 = gi.idx_ptr[tx];
        const int ne = gi.idx_ptr[tx + nx] - e0;
        for (int i = threadIdx.x; i <= nx; i += blockDim.x) xptr[i] = gi.idx_ptr[tx + i] - e0;
        for (int i = threadIdx.x; i < ne && i < maxent; i += blockDim.x) xent[i] = gi.ent[e0 + i];
        __syncthreads();
        const int nr = rr.y - rr.x + 1;
        const float *o = opd2 + ((size_t)b * nwfs + w) * np + (size_t)rr.x * nxp;
        for (int idx = threadIdx.x; idx < nr * nx; idx += blockDim.x) {
            const int r = idx / nx, jx = idx - r * nx;
            float sx = 0.f;
            for (int e = xptr[jx]; e < xptr[jx + 1]; e++) {
                const GatherW ge = xent[e];
                sx += ge.w * o[(size_t)r * nxp + ge.i];
            }
            t[r * maxnx + jx] = sx;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kMaxOwn; k++) {
            const int oi = threadIdx.x + k * kThreads;
            if (oi < nown) {
                const int jy = T.jy0 + oi / nx, jx = oi % nx;
                const int a0 = gi.idx_ptr[ty + jy], a1 = gi.idx_ptr[ty + jy + 1];
                float sy = 0.f;
                for (int a = a0; a < a1; a++) {
                    const GatherW ge = gi.ent[a];
                    sy += ge.w * t[(ge.i - rr.x) * maxnx + jx];
                }
                acc[k] += sy;
            }
        }
        __syncthreads();
    }
    const float *X = xin ? xin + (size_t)b * nxtot + L.off : nullptr;
    double dotv = 0;
#pragma unroll
    for (int k = 0; k < kMaxOwn; k++) {
        const int oi = threadIdx.x + k * kThreads;
        if (oi < nown) {
            const int jy = T.jy0 + oi / nx, jx = oi % nx;
            float v = alpha * acc[k];
            if (do_l2) {
                const int ny_ = L.ny;
                auto at = [&](int dx, int dy) {
                    int xx = jx + dx, yy = jy + dy;
                    xx += (xx < 0) ? nx : 0;
                    xx -= (xx >= nx) ? nx : 0;
                    yy += (yy < 0) ? ny_ : 0;
                    yy -= (yy >= ny_) ? ny_ : 0;
                    return X[yy * nx + xx];
                };
                const float st = 20.f * at(0, 0) - 8.f * (at(-1, 0) + at(1, 0) + at(0, -1) + at(0, 1)) +
                                 2.f * (at(-1, -1) + at(1, -1) + at(-1, 1) + at(1, 1)) +
                                 (at(0, -2) + at(-2, 0) + at(2, 0) + at(0, 2));
                v += alpha * L.l2c * st;
            }
            const long j = L.off + (long)jy * nx + jx;
            out[(size_t)b * nxtot + j] = v;
            if (dot_part && X) dotv += (double)v * (double)X[jy * nx + jx];
        }
    }
    if (dot_part) {
        dotv = block_sum(dotv, sh);
        if (threadIdx.x == 0) dot_part[(size_t)b * gridDim.x + blockIdx.x] = dotv;
        cg_alpha_last(dot_part + (size_t)b * gridDim.x, S, b, kit);
    }
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
            if (init) {
                S.sc[(size_t)b * S.nsc] = rz;
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

// v.v partials and (when z aliases r) the start-of-CG r.z.  grid: (nblk, nb)
__global__ void k_dot_self(const float *__restrict__ v, double *__restrict__ part, long n, CgScal S,
                           const int *__restrict__ act) {
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
    cg_rz_last(part + (size_t)b * gridDim.x, S, b, 0, 1);
}

// x += alpha p; r -= alpha Ap; r.r partials.  The last block either finishes
// the solve (residual sqrt(r.r/b.b) at the final iteration) or, when z aliases
// r (no preconditioner), produces beta.
__global__ void k_cg_update_xr(float *__restrict__ x, float *__restrict__ r,
                               const float *__restrict__ p, const float *__restrict__ Ap,
                               double *__restrict__ rr_part, long n, CgScal S, int k, int iters,
                               int z_is_r, const int *__restrict__ act) {
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

// p = z + beta p (init: p = z).  grid: (nblk, nb)
__global__ void k_cg_update_p(float *__restrict__ p, const float *__restrict__ z, long n, CgScal S,
                              int init, const int *__restrict__ act) {
    if (inactive(act, blockIdx.y)) return;
    const int b = blockIdx.y;
    const float be = init ? 0.f : S.ab[2 * b + 1];
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) {
        const size_t o = (size_t)b * n + j;
        p[o] = init ? z[o] : z[o] + be * p[o];
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
};

__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cplx cconj(cplx a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ cplx mul_mi(cplx a) { return make_float2(a.y, -a.x); }  // -i a

// One Stockham stage of radix R over `count` transforms of length n
// (element stride es, transform stride ts), a -> b.  Ns = product of the
// radices of the previous stages.
template <int R>
__device__ __forceinline__ void fft_stage(const cplx *__restrict__ a, cplx *__restrict__ b, int n, int count,
                                          int es, int ts, int Ns, const cplx *__restrict__ tw, bool inv) {
    const int nbf = n / R;
    const int tmul = n / (Ns * R);
    const int tot = nbf * count;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int c = t / nbf, j = t - c * nbf;
        const cplx *src = a + (size_t)c * ts;
        cplx *dst = b + (size_t)c * ts;
        const int jm = j % Ns;
        cplx v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            cplx x = src[(j + r * nbf) * es];
            if (r > 0 && jm > 0) {
                cplx w = tw[r * jm * tmul];
                if (inv) w.y = -w.y;
                x = cmul(x, w);
            }
            v[r] = x;
        }
        const int o = (j / Ns) * Ns * R + jm;
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
                for (int r = 1; r < R; r++) {
                    cplx w = tw[((r * q) % R) * nbf];
                    if (inv) w.y = -w.y;
                    acc = cadd(acc, cmul(v[r], w));
                }
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

// Forward: r (instance-major) -> half spectra H.  grid: (nps, nb); dynamic
// shared memory: two buffers of `bufn` complex values.
__global__ void __launch_bounds__(kThreads)
k_fd_fwd(const float *__restrict__ r, cplx *__restrict__ H, const FdLayer *__restrict__ fl,
         const cplx *__restrict__ tw, long nxtot, int bufn, const int *__restrict__ act) {
    if (inactive(act, blockIdx.y)) return;
    extern __shared__ cplx fsm[];
    const FdLayer L = fl[blockIdx.x];
    const int b = blockIdx.y;
    const int nx = L.nx, ny = L.ny, h = nx / 2 + 1, np2 = ny / 2;
    cplx *A = fsm, *B = fsm + bufn;
    const float *rb = r + (size_t)b * nxtot + L.off;
    for (int i = threadIdx.x; i < np2 * nx; i += blockDim.x) {
        const int p = i / nx, x = i - p * nx;
        A[i] = make_float2(rb[(2 * p) * nx + x], rb[(2 * p + 1) * nx + x]);
    }
    __syncthreads();
    cplx *Z = fft_many(A, B, nx, np2, 1, nx, L.rx, L.nrx, tw + L.twx, false);
    cplx *S = (Z == A) ? B : A;
    for (int i = threadIdx.x; i < np2 * h; i += blockDim.x) {
        const int p = i / h, k = i - p * h;
        const cplx zk = Z[p * nx + k], zm = cconj(Z[p * nx + (nx - k) % nx]);
        S[(2 * p) * h + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
        const cplx d = csub(zk, zm);
        S[(2 * p + 1) * h + k] = make_float2(0.5f * d.y, -0.5f * d.x);  // -i/2 (zk - conj(z_-k))
    }
    __syncthreads();
    const cplx *C = fft_many(S, Z, ny, h, h, 1, L.ry, L.nry, tw + L.twy, false);
    cplx *out = H + L.hoff + (size_t)b * L.hs;
    for (int i = threadIdx.x; i < ny * h; i += blockDim.x) out[i] = C[i];
}

// Per-frequency block solve on the blocks of the non-positive x frequencies
// (the leading blocks of the reference's ordering, which reach every stored
// bin): Y_i = sum_j M[blk][j*bs+i] X_j.  A CTA takes floor(256/bs) whole
// blocks: every thread first stages its own member X_i in shared memory,
// then forms its row from the block's staged members.
// grid: (ceil(nblk / floor(256/bs)), nbatch)
__global__ void __launch_bounds__(kThreads)
k_fd_mul(const cplx *__restrict__ X, cplx *__restrict__ Y, const cplx *__restrict__ M,
         const FdIndex *__restrict__ idx, int nblk, int bs, const int *__restrict__ act) {
    if (inactive(act, blockIdx.y)) return;
    __shared__ cplx xs[kThreads];
    const int b = blockIdx.y;
    const int per = kThreads / bs;
    const int lb = threadIdx.x / bs, i = threadIdx.x - lb * bs;
    const int blk = blockIdx.x * per + lb;
    const bool live = lb < per && blk < nblk;
    FdIndex o{};
    if (live) {
        o = idx[(size_t)blk * bs + i];
        cplx xv = X[o.base + (size_t)b * o.stride];
        if (o.flags & kFdConj) xv.y = -xv.y;
        xs[threadIdx.x] = xv;
    }
    __syncthreads();
    if (!live) return;
    const cplx *Mb = M + (size_t)blk * bs * bs + i;
    const cplx *xb = xs + lb * bs;
    float re = 0.f, im = 0.f;
#pragma unroll 4
    for (int jj = 0; jj < bs; jj++) {
        const cplx m = Mb[jj * bs];
        const cplx xv = xb[jj];
        re += m.x * xv.x - m.y * xv.y;
        im += m.x * xv.y + m.y * xv.x;
    }
    if (o.flags & kFdStore)
        Y[o.base + (size_t)b * o.stride] = make_float2(re, (o.flags & kFdConj) ? -im : im);
}

// Inverse: half spectra H -> z (instance-major), plus the r.z partial of this
// (layer, instance); the last CTA of an instance leaves (r.z)_0 or beta.
// grid: (nps, nb)
__global__ void __launch_bounds__(kThreads)
k_fd_inv(const cplx *__restrict__ H, const float *__restrict__ r, float *__restrict__ z,
         double *__restrict__ rz_part, const FdLayer *__restrict__ fl, const cplx *__restrict__ tw, long nxtot,
         int bufn, CgScal SC, int kit, int init, const int *__restrict__ act) {
    if (inactive(act, blockIdx.y)) return;
    extern __shared__ cplx fsm[];
    __shared__ double sh[32];
    const FdLayer L = fl[blockIdx.x];
    const int b = blockIdx.y;
    const int nx = L.nx, ny = L.ny, h = nx / 2 + 1, np2 = ny / 2;
    cplx *A = fsm, *B = fsm + bufn;
    const cplx *in = H + L.hoff + (size_t)b * L.hs;
    for (int i = threadIdx.x; i < ny * h; i += blockDim.x) A[i] = in[i];
    __syncthreads();
    cplx *C = fft_many(A, B, ny, h, h, 1, L.ry, L.nry, tw + L.twy, true);
    cplx *Zb = (C == A) ? B : A;
    for (int i = threadIdx.x; i < np2 * nx; i += blockDim.x) {
        const int p = i / nx, k = i - p * nx;
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
    const cplx *Zo = fft_many(Zb, C, nx, np2, 1, nx, L.rx, L.nrx, tw + L.twx, true);
    const size_t base = (size_t)b * nxtot + L.off;
    double v = 0;
    for (int i = threadIdx.x; i < np2 * nx; i += blockDim.x) {
        const int p = i / nx, x = i - p * nx;
        const cplx q = Zo[i];
        const size_t o0 = base + (size_t)(2 * p) * nx + x, o1 = o0 + nx;
        z[o0] = q.x;
        z[o1] = q.y;
        v += (double)q.x * r[o0] + (double)q.y * r[o1];
    }
    v = block_sum(v, sh);
    if (threadIdx.x == 0) rz_part[(size_t)b * gridDim.x + blockIdx.x] = v;
    if (SC.sc) cg_rz_last(rz_part + (size_t)b * gridDim.x, SC, b, kit, init);
}

// float <-> double staging helpers for the host-facing API
__global__ void k_scale_copy(const float *__restrict__ a, float *__restrict__ o, float s, long n) {
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) o[j] = s * a[j];
}

}  // namespace mb
