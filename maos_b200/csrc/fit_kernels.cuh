// Kernels of the assembled DM fit (sparse plus low rank) for B200 (sm_100a).
//
// The reference's default GPU fit (cuda/solve.cu cusolve_sparse, cumuv_t)
// applies FR and FL as cuSPARSE csrmv plus two cuBLAS gemv per operator,
// one instance at a time.  Here every operator is two launches for all
// instances sharing the matrices:
//   k_lr_dot   t[b][q] = V_q' x_b (FP64 block partials, the last block to
//              arrive adds them in a fixed order)
//   k_spmv_lr  y_b = M x_b - U t_b, M in CSR as (column, value) pairs read
//              once per group of NI instances, optionally + p.Ap partials and
//              alpha for CG.
// Every instance's sums are formed independently of the others (a warp per
// row, each lane holding NI instance sums, a butterfly over the warp), so
// results do not depend on which instances run together.
#pragma once
#include "tomo_kernels.cuh"

namespace mb {

constexpr int kMaxLr = 16;  // low-rank columns (FR: fit directions; FL: + NW)

// grid: (ceil(n/256), nb); part [nb][nq][gridDim.x]; t [nb][kMaxLr]
__global__ void __launch_bounds__(kThreads)
k_lr_dot(const float *__restrict__ x, const float *__restrict__ V, int nq, long n, double *__restrict__ part,
         float *__restrict__ t, unsigned *__restrict__ cnt, const int *__restrict__ act) {
    pdl_enter();
    if (inactive(act, blockIdx.y)) return;
    __shared__ double sh[kThreads / 32][kMaxLr];
    const int b = blockIdx.y;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const float xv = (j < n) ? x[(size_t)b * n + j] : 0.f;
    for (int q = 0; q < nq; q++) {
        double v = (j < n) ? (double)V[(size_t)q * n + j] * (double)xv : 0.0;
        v = warp_sum(v);
        if (lane == 0) sh[wid][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < nq) {
        double s = 0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; w++) s += sh[w][threadIdx.x];
        part[((size_t)b * nq + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
    if (last_block(cnt + b, gridDim.x)) {
        for (int q = wid; q < nq; q += kThreads / 32) {
            const double s = warp_sum_fresh(part + ((size_t)b * nq + q) * gridDim.x, gridDim.x);
            if (lane == 0) t[(size_t)b * kMaxLr + q] = (float)s;
        }
        if (threadIdx.x == 0) cnt[b] = 0;
    }
}

// y[b][i] = sum_e M[i][e] x[b][col_e] - sum_q U[q*nrow + i] t[b][q] (+ add[b][i]).
// One warp per row (8 rows per CTA); grid: (ceil(nb/NI), ceil(nrow/8)).
// With dot_part: the p.Ap partials (dot_x = p) per CTA, [nb][gridDim.y], and
// the last CTA of each instance group leaves alpha_k = (r.z)_k / p.Ap.
template <int NI>
__global__ void __launch_bounds__(kThreads)
k_spmv_lr(const int *__restrict__ rp, const GatherW *__restrict__ ent, int nrow, long ncol,
          const float *__restrict__ x, float *__restrict__ y, const float *__restrict__ U,
          const float *__restrict__ t, int nq, const float *__restrict__ add, const float *__restrict__ dot_x,
          double *__restrict__ dot_part, CgScal S, int k, int nbatch, const int *__restrict__ act) {
    pdl_enter();
    const int b0 = blockIdx.x * NI;
    const int ni = min(NI, nbatch - b0);
    bool on[NI];
    bool any = false;
#pragma unroll
    for (int q = 0; q < NI; q++) {
        on[q] = q < ni && !inactive(act, b0 + q);
        any |= on[q];
    }
    if (!any) return;  // uniform over the instance group
    __shared__ double sh[kThreads / 32][NI];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int row = blockIdx.y * (kThreads / 32) + wid;
    float acc[NI];
#pragma unroll
    for (int q = 0; q < NI; q++) acc[q] = 0.f;
    if (row < nrow) {
        const int e1 = rp[row + 1];
        for (int e = rp[row] + lane; e < e1; e += 32) {
            const GatherW g = ent[e];
#pragma unroll
            for (int q = 0; q < NI; q++)
                if (on[q]) acc[q] += g.w * x[(size_t)(b0 + q) * ncol + g.i];
        }
    }
#pragma unroll
    for (int q = 0; q < NI; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    // lane q finishes instance b0 + q
    float mine = 0.f;
    bool mon = false;
#pragma unroll
    for (int q = 0; q < NI; q++)
        if (lane == q) {
            mine = acc[q];
            mon = on[q];
        }
    double dv = 0.0;
    if (row < nrow && lane < NI && mon) {
        const int b = b0 + lane;
        float lr = 0.f;
        for (int q = 0; q < nq; q++) lr += U[(size_t)q * nrow + row] * t[(size_t)b * kMaxLr + q];
        float v = mine - lr;
        if (add) v += add[(size_t)b * nrow + row];
        y[(size_t)b * nrow + row] = v;
        if (dot_part) dv = (double)v * (double)dot_x[(size_t)b * nrow + row];
    }
    if (!dot_part) return;  // uniform
    if (lane < NI) sh[wid][lane] = dv;
    __syncthreads();
    if (threadIdx.x < ni) {  // instances past nbatch have no row in dot_part
        double s = 0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; w++) s += sh[w][threadIdx.x];
        dot_part[(size_t)(b0 + threadIdx.x) * gridDim.y + blockIdx.y] = s;
    }
    if (last_block(S.cnt + b0, gridDim.y)) {
        if (wid < ni && !inactive(act, b0 + wid)) {
            const int b = b0 + wid;
            const double pap = warp_sum_fresh(dot_part + (size_t)b * gridDim.y, gridDim.y);
            if (lane == 0) {
                double a = S.sc[(size_t)b * S.nsc + k] / pap;
                if (!isfinite(a)) a = 0;  // pcg.c:80-83, pcg.cu:27-30
                S.ab[2 * b] = (float)a;
            }
        }
        if (threadIdx.x == 0) S.cnt[b0] = 0;
    }
}

}  // namespace mb
