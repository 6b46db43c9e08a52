// Host side of the tomography reconstructor: table preparation, buffers,
// the CG/FDPCG schedule captured in one CUDA graph, and the C ABI
// (include/maos_b200.h).
//
// Table preparation mirrors what the reference does when it copies RECON_T to
// the GPU (cuda/tomo.cu:30-139 prep_GP/prep_saptr/convert_neai,
// cuda/prop_wrap.cu:357 gpu_map2map_prep), with two differences chosen for
// parity with the reference CPU path: GP is kept exactly (FP32 stencil
// coefficients, not short2-quantised) and every transpose is the exact
// transpose of the forward table, evaluated in gather form.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <atomic>
#include <climits>
#include <cstdint>
#include <functional>
#include <vector>

#include "common.cuh"
#include "tomo_kernels.cuh"
#include "fit_kernels.cuh"

namespace mb {

static thread_local char g_err[1024] = "";
void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char *last_error() { return g_err; }
static std::atomic<long> g_launches{0};
void count_launches(long n) { g_launches += n; }

static inline unsigned nblocks(long n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }
constexpr int kCgRestart = 100;  // lib/pcg.c:61

// Every kernel of the reconstructor is launched through here.  While a
// reconstructor captures its graphs (PdlScope) with the mode the autotuner
// chose, or with MAOS_B200_PDL=1, the launches carry programmatic stream
// serialisation (the kernels open with pdl_enter), so a kernel's launch and
// CTA ramp overlap the tail of its predecessor.  Mode 0: none; 1: the plain
// launches; 2: the cluster launches too.  Measured on the 30 m system: one
// instance 1.02 ms with mode 1, 1.06 with 2, 1.09 with 0; four instances
// best with 0; 32 instances 3.49 ms with 2 against 3.56.
static thread_local int g_pdl_mode = 0;
struct PdlScope {
    int old;
    explicit PdlScope(int mode) : old(g_pdl_mode) { g_pdl_mode = mode; }
    ~PdlScope() { g_pdl_mode = old; }
};
static bool pdl_enabled() {
    static const bool env = std::getenv("MAOS_B200_PDL") != nullptr;
    return g_pdl_mode >= 1 || env;
}
static bool pdl_cluster_enabled() { return g_pdl_mode >= 2; }

template <typename... KArgs, typename... Args>
static void launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
    if (e != cudaSuccess) {
        set_error("kernel launch: %s", cudaGetErrorString(e));
        throw CudaError{MB_ECUDA};
    }
    count_launches(1);
}

// A launch in thread-block clusters of `cx` CTAs along x.
template <typename... KArgs, typename... Args>
static void launch_cluster(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, int cx,
                           Args &&...args) {
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cx;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = pdl_cluster_enabled() ? 1 : 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
    if (e != cudaSuccess) {
        set_error("cluster launch: %s", cudaGetErrorString(e));
        throw CudaError{MB_ECUDA};
    }
    count_launches(1);
}

// Forward tables for (direction d, source grid t) on the device, and their
// exact transposes as per-axis CSR lists over the source grid (gather form)
// on the host, from which the padded gather lists of the kernels are built.
struct RayTables {
    DevBuf<AxisW> fwd;
    std::vector<int> h_ptr, h_idxptr;
    std::vector<GatherW> h_ent;
};

struct Recon {
    int device = 0;
    cudaStream_t stream = nullptr;
    int nb = 1;  // batch
    int nwfs = 0, nps = 0, nxp = 0, nyp = 0, np = 0;
    long nxtot = 0, ngrad = 0;
    int maxit = 0, precond = 0, split = 1;
    int nsc = 0;            // scalars per instance
    int nblk_x = 0;         // blocks over nxtot
    int hxt_threads = kThreads, nblk_hxt = 0;  // k_hxt_rows's CTA size (autotuned) and CTAs per instance
    int nblk_tt = 0;        // blocks over the largest nsa
    std::vector<long> xoff, goff;
    std::vector<int> nsa;

    // tables
    RayTables hx;
    // separable Hx^T: fixed-width transposed lists and the pupil-row buffer
    DevBuf<GatherW> xpad, ypad;
    DevBuf<int4> footprint;
    int kx = 0, ky = 0, maxnx = 0, maxny = 0;
    int prows = 0, ptiles = 0, ncols = 0;  // pupil rows per CTA, CTAs per WFS, sum of layer widths
    long tw = 0;                           // row-buffer floats per (instance, WFS)
    size_t pupil_smem = 0;
    DevBuf<float> tbuf;
    PadIndex pad() const { return PadIndex{xpad.p, ypad.p, footprint.p, kx, ky, maxnx, maxny}; }
    DevBuf<LayerDev> lay;
    std::vector<LayerDev> lay_h;
    LayerTab laytab{};  // lay_h by value, for kernel parameters
    std::vector<mb_grid> xgrid;   // host copy of the layer grids
    DevBuf<WfsDev> wfs;
    std::vector<std::unique_ptr<DevBuf<int2>>> saptr;
    std::vector<std::unique_ptr<DevBuf<float2>>> gp;
    std::vector<std::unique_ptr<DevBuf<int>>> samap;
    std::vector<std::unique_ptr<DevBuf<float>>> neai, ptt;
    std::vector<WfsDev> wfs_h;
    // FDPCG
    int fd_nb = 0, fd_bs = 0, fd_nbh = 0;  // blocks, block size, blocks solved (half spectrum)
    DevBuf<cplx> fd_M;
    DevBuf<FdIndex> fd_idx;
    // device rebuild of the blocks after a Cn2 update (k_fd_prepare, k_fd_fold)
    bool fd_dev = false;                    // the data term below is present
    DevBuf<double2> fd_mdata, fd_minv;      // [nb][bs][bs] column-major
    DevBuf<double> fd_mdiag, fd_sc, fd_lscale;
    DevBuf<int> fd_mlayer, fd_bp, fd_sig;
    std::vector<double> fd_l2c_ref;         // l2c at which fd_mdiag holds invpsd
    std::vector<double> l2c_now;            // l2c last installed
    DevBuf<FdLayer> fd_lay;                 // per layer: FFT geometry and radices
    FdTab fdtab{};                          // the same, by value for kernel parameters
    WfsTab wfstab{};                        // wfs_h by value for kernel parameters
    DevBuf<cplx> fd_tw;                     // twiddle tables exp(-2 pi i k/n)
    int fd_bufn = 0;                        // complex elements per FFT shared buffer
    size_t fd_smem = 0;

    DevBuf<cplx> spec, spec2;               // half spectra

    // state and work buffers
    DevBuf<float> x, r, p, z, Ap, rhs, opd, grad, gin;
    DevBuf<double> tt_part, pap_part, rr_part, rz_part, bb_part, sc;
    DevBuf<float> res, ab, tt;
    DevBuf<unsigned> cnt, cnt_tt;
    CgScal scal() const { return CgScal{sc.p, nsc, ab.p, cnt.p, res.p}; }

    // Serving: per-instance participation flags read by every kernel of the
    // step (1: run, 0: leave the instance untouched).  All ones except while a
    // masked step is queued; the host copy is pinned so the upload is
    // asynchronous, and `mask_ev` guards its reuse.
    DevBuf<int> active;
    int *mask_host = nullptr;
    cudaEvent_t mask_ev = nullptr;
    bool mask_all = true;
    const int *act() const { return active.p; }
    void set_mask(const int *m, cudaStream_t s);

    // DM fit
    int has_fit = 0, nfit = 0, ndm = 0, nfx = 0, nfy = 0, nf = 0, nnw = 0, fit_maxit = 0;
    int nblk_a = 0, nblk_f = 0, fnsc = 0;
    long nact = 0;
    RayTables hxp, ha;
    DevBuf<GatherW> fxpad, fypad;  // HA^T as padded per-axis lists (k_fit_hxt)
    int fkx = 0, fky = 0, fmaxn = 0;
    LayerTab dmtab{};
    FitPad fitpad() const { return FitPad{fxpad.p, fypad.p, fkx, fky, fmaxn}; }
    DevBuf<LayerDev> dmlay;
    std::vector<LayerDev> dmlay_h;
    DevBuf<int> w0_rp, w0_ci;
    DevBuf<float> w0_v, w1v, fwt, nwv;
    DevBuf<float> fa, fr, fp, fAp, frhs, opdf, opdw;
    DevBuf<double> w1_part, nw_part, f_pap, f_rr, f_rz, f_bb, fsc;
    DevBuf<float> fres, fab;
    DevBuf<unsigned> fcnt;
    CgScal fscal() const { return CgScal{fsc.p, fnsc, fab.p, fcnt.p, fres.p}; }
    // grid fit: slaving term of FitL (CSR), applied into fslv and added by k_fit_hxt
    bool has_slave = false;
    DevBuf<int> as_rp;
    DevBuf<GatherW> as_e;
    DevBuf<float> fslv;
    // assembled fit (fit_sparse): FR, FL as CSR (column, value) plus low rank
    bool fit_sparse = false;
    int nfr = 0, nfl = 0, nrb_a = 0;       // low-rank columns; 8-row blocks over the actuators
    DevBuf<int> frm_rp, flm_rp;
    DevBuf<GatherW> frm_e, flm_e;
    DevBuf<float> fru, frv, flu, flv;
    DevBuf<double> lr_part;
    DevBuf<float> lr_t;
    DevBuf<unsigned> lr_cnt;
    void spmv(const DevBuf<int> &rp, const DevBuf<GatherW> &e, int nrow, long ncol, const float *xin, float *out,
              const float *U, int nq, const float *add, double *dot, int k, cudaStream_t s);
    void lr_dot(const float *xin, const float *V, int nq, long n, cudaStream_t s);
    void build_fit_sparse(const mb_fit_sparse_desc *f);
    void alloc_fit_state();

    // pinned host staging for the FP64 <-> FP32 conversions of the host-buffer calls
    float *hstage = nullptr;
    size_t hstage_n = 0;
    float *stage(size_t n) {
        if (n > hstage_n) {
            if (hstage) cudaFreeHost(hstage);
            hstage = nullptr;
            hstage_n = 0;
            MB_CUDA_TRY(cudaHostAlloc(&hstage, n * sizeof(float), cudaHostAllocDefault));
            hstage_n = n;
        }
        return hstage;
    }

    cudaGraphExec_t graph = nullptr;       // tomography step
    cudaGraphExec_t graph_fit = nullptr;   // fit step
    cudaGraphExec_t graph_step = nullptr;  // tomography + fit
    long graph_kernels = 0, graph_fit_kernels = 0, graph_step_kernels = 0;
    long graph_version = 0;  // counts recaptures (a ReconGroup recaptures after a member did)
    int pdl = 0;             // programmatic dependent launch in the step graphs (PdlScope mode, autotuned)

    ~Recon() {
        if (hstage) cudaFreeHost(hstage);
        if (mask_ev) cudaEventDestroy(mask_ev);
        if (mask_host) cudaFreeHost(mask_host);
        if (graph) cudaGraphExecDestroy(graph);
        if (graph_fit) cudaGraphExecDestroy(graph_fit);
        if (graph_step) cudaGraphExecDestroy(graph_step);
        if (stream) cudaStreamDestroy(stream);
    }

    // ------------------------------------------------------------------
    void build(const mb_recon_desc *d);
    void build_hx_tables(const mb_recon_desc *d);
    void build_pad(int min_kx = 1, int min_ky = 1);
    void set_pupil_rows(int rows);
    void rebuild_fdpcg_device();
    int autotune(int reps, float *ms_out);
    void pupil_rows(bool from_x, const float *xin, cudaStream_t s);
    void hxt_rows(const float *xin, float *out, double *dot_part, int do_l2, int k, cudaStream_t s);
    // the arguments of those launches (also gathered by a ReconGroup)
    PupilArgs pupil_args(bool from_x, const float *xin, int w0) const;
    HxtArgs hxt_args(const float *xin, float *out, double *dot_part, int do_l2, int k) const;
    int hxt_ni() const { return nb > 1 ? 2 : 1; }
    void build_wfs_tables(const mb_recon_desc *d);
    void build_fdpcg(const mb_fdpcg_desc *fd);
    void build_fit(const mb_fit_desc *f);
    void set_neai(int iwfs, const double *neai, const double *ptt);
    void set_l2c(const double *l2c);

    // operator pieces (enqueue on `s`)
    void op_hx(const float *xin, cudaStream_t s);
    void op_rhs(const float *g, float *out, cudaStream_t s);
    void op_lhs(const float *xin, float *out, double *dot_part, cudaStream_t s, int k = 0);
    bool op_fdpcg(float *rin, float *zout, double *rz_part, cudaStream_t s, int k = 0, int init = 0,
                  bool in_cg = false, float *xupd = nullptr, const float *pupd = nullptr,
                  const float *Apupd = nullptr, float *pnext = nullptr);
    bool fd_cluster = false;  // k_fd_inv<true> fits as clusters of nps CTAs
    // the fused preconditioner (k_fd_fused): an instance's layers split over
    // one cluster of fused_tab.C CTAs; fd_mode 1 = three kernels, 2 = fused
    bool fd_fused_ok = false;
    int fd_mode = 1;
    int fd_mul_ni = kFdInst;  // instances per k_fd_mul CTA (the form-1 batch shape)
    void fd_mul(cudaStream_t s);
    FdFusedTab fused_tab{};
    DevBuf<FdMem> fd_mem;
    size_t fd_fsmem = 0;
    void build_fdpcg_fused(const std::vector<FdIndex> &idx, const std::vector<long> &hoff);
    // the FDPCG data term's geometry (mb_fdpcg_geom), for k_fd_data
    bool fd_geom = false;
    FdGeomDev fdg{};
    DevBuf<int4> fdg_mem;
    DevBuf<int2> fdg_blk, fdg_seld;
    DevBuf<double2> fdg_gx, fdg_gy, fdg_selr;
    DevBuf<double> fdg_neam, fdg_thx, fdg_thy, fdg_lht;
    DevBuf<int> fdg_lnx, fdg_lny;
    std::vector<double> wfs_thx, wfs_thy;
    void build_fdpcg_geom(const mb_fdpcg_desc *fd);
    void form_fdpcg_data(const double *neam);
    void set_fdpcg_mode(int mode);
    void enqueue_solve(cudaStream_t s);
    struct CgBufs {
        float *x, *r, *p, *z, *Ap, *rhs;
        double *pap, *rr, *rz, *bb;
        CgScal S;
    };
    using AmulFn = std::function<void(const float *, float *, double *, int)>;
    // preconditioners return true when they also left p = z + beta p
    using MmulFn = std::function<bool(float *, float *, double *, int, int)>;
    using XrMmulFn = std::function<bool(int)>;
    void enqueue_cg(const CgBufs &B, long n, int nblk, int iters, const AmulFn &Amul,
                    const MmulFn &Mmul, cudaStream_t s, const XrMmulFn &XrMmul = XrMmulFn());
    // One CG solve taken apart at its operator applications, so that a
    // ReconGroup can apply the operator of several reconstructors in one
    // launch: after A x -> cg_init; after A p_k -> cg_post (true: done).
    struct CgRun {
        CgBufs B;
        long n;
        int nblk, iters;
        MmulFn Mmul;
        XrMmulFn XrMmul;
        float *zp;
    };
    void cg_init(CgRun &c, int k, cudaStream_t s);
    bool cg_post(CgRun &c, int k, cudaStream_t s);
    CgRun solve_run(cudaStream_t s);  // the tomography CG (its preconditioner launched on s)
    void op_rhs_gp(const float *g, cudaStream_t s);  // the first launch of op_rhs (gradient weighting)
    void op_fitR(const float *xin, float *out, cudaStream_t s);
    void op_fitL(const float *ain, float *out, double *dot_part, cudaStream_t s, int k = 0);
    void enqueue_fit(cudaStream_t s);
    void time_stages(int reps, float *ms, double *bytes, int *launches);
    void capture_graph();
    void capture(const std::function<void(cudaStream_t)> &body, long &nkernels, cudaGraphExec_t &exec);
    void run_graph(cudaStream_t s);
};

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------

// Bilinear weights of one axis: output coordinate c maps to source index
// u = (c*scale + disp - o)/d.  Same inclusion rule as the reference CPU ray
// tracer (lib/prop_grid.c): 0 <= u <= n-1, a point on the last sample uses
// that sample alone.  With `snap`, coordinates within 1e-9 of a sample are
// moved onto it first (lib/mkh.c keeps a corner whose weight exceeds EPS, so
// a ray a rounding error outside the first or last sample still counts).
static void axis_weights(int n_out, double o_out, double d_out, double scale, double disp,
                         double o_in, double d_in, int n_in, bool snap, std::vector<AxisW> &out) {
    for (int i = 0; i < n_out; i++) {
        const double c = o_out + i * d_out;
        double u = (c * scale + disp - o_in) / d_in;
        if (snap) {
            const double r = std::round(u);
            if (std::fabs(u - r) < 1e-9) u = r;
        }
        long k = (long)std::floor(u);
        double f = u - k;
        if (k == n_in - 1 && f < 1e-12) {
            k = n_in - 2;
            f = 1.0;
        }
        AxisW e;
        if (u >= 0 && k >= 0 && k <= n_in - 2) {
            e.k = (int)k;
            e.w0 = (float)(1.0 - f);
            e.w1 = (float)f;
        } else {
            e.k = -1;
            e.w0 = e.w1 = 0.f;
        }
        out.push_back(e);
    }
}


static void build_ray_tables(const mb_grid &og, int ndir, int nt, const mb_grid *tg,
                             const std::function<void(int, int, double &, double &, double &)> &geom,
                             bool snap, RayTables &rt) {
    const int nxo = og.nx, nyo = og.ny;
    std::vector<AxisW> tab;
    tab.reserve((size_t)ndir * nt * (nxo + nyo));
    for (int d = 0; d < ndir; d++)
        for (int t = 0; t < nt; t++) {
            double scale, dx, dy;
            geom(d, t, scale, dx, dy);
            const mb_grid &g = tg[t];
            axis_weights(nxo, og.ox, og.dx, scale, dx, g.ox, g.dx, g.nx, snap, tab);
            axis_weights(nyo, og.oy, og.dy, scale, dy, g.oy, g.dy, g.ny, snap, tab);
        }
    rt.fwd.upload(tab);
    std::vector<int> ptr, idxptr;
    std::vector<GatherW> ent;
    for (int d = 0; d < ndir; d++)
        for (int t = 0; t < nt; t++) {
            const AxisW *tt = tab.data() + (size_t)(d * nt + t) * (nxo + nyo);
            for (int axis = 0; axis < 2; axis++) {
                const int n_in = axis ? tg[t].ny : tg[t].nx;
                const int n_out = axis ? nyo : nxo;
                const AxisW *ta = tt + (axis ? nxo : 0);
                ptr.push_back((int)idxptr.size());
                std::vector<std::vector<GatherW>> lists(n_in);
                for (int i = 0; i < n_out; i++) {
                    if (ta[i].k < 0) continue;
                    lists[ta[i].k].push_back(GatherW{i, ta[i].w0});
                    lists[ta[i].k + 1].push_back(GatherW{i, ta[i].w1});
                }
                for (int j = 0; j < n_in; j++) {
                    idxptr.push_back((int)ent.size());
                    for (auto &e : lists[j]) ent.push_back(e);
                }
                idxptr.push_back((int)ent.size());
            }
        }
    rt.h_ptr = std::move(ptr);
    rt.h_idxptr = std::move(idxptr);
    rt.h_ent = std::move(ent);
}

void Recon::build_hx_tables(const mb_recon_desc *d) {
    build_ray_tables(d->pmap, nwfs, nps, d->xmap,
                     [&](int w, int l, double &scale, double &dx, double &dy) {
                         const mb_wfs_desc &W = d->wfs[w];
                         const double ht = d->xmap[l].ht;
                         scale = std::isinf(W.hs) ? 1.0 : 1.0 - ht / W.hs;
                         dx = W.thetax * ht;
                         dy = W.thetay * ht;
                     },
                     false, hx);
}

// Fixed-width copies of the transposed x and y lists of every (WFS, layer),
// padded with (index 0, weight 0) after the real entries (at least min_kx /
// min_ky wide: a ReconGroup gives its members one width, and the padding
// adds exact zeros), and the pupil-row blocking of k_pupil_rows.
void Recon::build_pad(int min_kx, int min_ky) {
    maxnx = maxny = 0;
    for (int l = 0; l < nps; l++) {
        maxnx = std::max(maxnx, lay_h[l].nx);
        maxny = std::max(maxny, lay_h[l].ny);
    }
    kx = std::max(1, min_kx);
    ky = std::max(1, min_ky);
    for (int w = 0; w < nwfs; w++)
        for (int l = 0; l < nps; l++)
            for (int axis = 0; axis < 2; axis++) {
                const int tb = hx.h_ptr[(w * nps + l) * 2 + axis];
                const int n = axis ? lay_h[l].ny : lay_h[l].nx;
                int &K = axis ? ky : kx;
                for (int j = 0; j < n; j++) K = std::max(K, hx.h_idxptr[tb + j + 1] - hx.h_idxptr[tb + j]);
            }
    MB_REQUIRE(nps <= kMaxLayers, "at most %d reconstructed layers (%d)", kMaxLayers, nps);
    MB_REQUIRE(kx <= kMaxPadX, "transposed x lists wider than %d (%d)", kMaxPadX, kx);
    MB_REQUIRE(ky <= kMaxPadY, "transposed y lists wider than %d (%d)", kMaxPadY, ky);
    MB_REQUIRE(nxp <= kThreads, "pupil grid wider than %d (%d)", kThreads, nxp);
    std::vector<GatherW> xp((size_t)nwfs * ncols * kx, GatherW{0, 0.f});
    std::vector<GatherW> yp((size_t)nwfs * nps * maxny * ky, GatherW{0, 0.f});
    for (int w = 0; w < nwfs; w++)
        for (int l = 0; l < nps; l++)
            for (int axis = 0; axis < 2; axis++) {
                const int tb = hx.h_ptr[(w * nps + l) * 2 + axis];
                const int n = axis ? lay_h[l].ny : lay_h[l].nx;
                for (int j = 0; j < n; j++)
                    for (int a = hx.h_idxptr[tb + j], k = 0; a < hx.h_idxptr[tb + j + 1]; a++, k++) {
                        if (axis) yp[((size_t)(w * nps + l) * maxny + j) * ky + k] = hx.h_ent[a];
                        else xp[((size_t)w * kx + k) * ncols + lay_h[l].tcol + j] = hx.h_ent[a];  // entry-major
                    }
            }
    xpad.upload(xp);
    ypad.upload(yp);
    // footprint of every WFS on every layer: first and last+1 column and row
    // with a non-empty transposed list
    std::vector<int4> fp((size_t)nwfs * nps);
    for (int w = 0; w < nwfs; w++)
        for (int l = 0; l < nps; l++) {
            int lo[2] = {INT32_MAX, INT32_MAX}, hi[2] = {-1, -1};
            for (int axis = 0; axis < 2; axis++) {
                const int tb = hx.h_ptr[(w * nps + l) * 2 + axis];
                const int n = axis ? lay_h[l].ny : lay_h[l].nx;
                for (int j = 0; j < n; j++)
                    if (hx.h_idxptr[tb + j + 1] > hx.h_idxptr[tb + j]) {
                        lo[axis] = std::min(lo[axis], j);
                        hi[axis] = j;
                    }
            }
            fp[(size_t)w * nps + l] = hi[0] < 0 || hi[1] < 0 ? make_int4(0, 0, 0, 0)
                                                             : make_int4(lo[0], hi[0] + 1, lo[1], hi[1] + 1);
        }
    footprint.upload(fp);
    // pupil rows per CTA: as many row blocks per WFS as one wave of 4 CTAs on
    // each of 148 SMs holds, at least 3 and with at least 4 rows per block
    // (the measured optimum of the 30 m system at 1, 32 and 64 instances);
    // Recon::autotune replaces the guess by measurement.
    const long nmax = (nyp + 3) / 4;
    const long tiles = std::max(3L, std::min(nmax, (long)(4 * 148) / std::max(1L, (long)nwfs * nb)));
    int rows = (int)((nyp + tiles - 1) / tiles);
    if (const char *e = std::getenv("MAOS_B200_PUPIL_ROWS")) {  // tuning override
        const int v = std::atoi(e);
        if (v >= 1 && v <= 64) rows = v;
    }
    tw = (long)nyp * ncols;
    set_pupil_rows(rows);
}

void Recon::set_pupil_rows(int rows) {
    const size_t sm = (size_t)pupil_rows_smem_floats(rows, nxp, nps, ncols, kx) * sizeof(float);
    MB_REQUIRE(sm <= 200 * 1024, "pupil row block needs %zu bytes of shared memory", sm);
    prows = rows;
    ptiles = (nyp + prows - 1) / prows;
    pupil_smem = sm;
    for (auto k : {k_pupil_rows<true, 1, 8>, k_pupil_rows<true, 2, 8>, k_pupil_rows<false, 1, 8>,
                   k_pupil_rows<false, 2, 8>, k_pupil_rows<true, 1, 16>, k_pupil_rows<true, 2, 16>,
                   k_pupil_rows<false, 1, 16>, k_pupil_rows<false, 2, 16>})
        MB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pupil_smem));
}

PupilArgs Recon::pupil_args(bool from_x, const float *xin, int w0) const {
    return PupilArgs{xin,    grad.p, tt.p,   tbuf.p, hx.fwd.p, laytab, wfstab, pad(), w0,    nps, nwfs, nxp,
                     nyp,    nxtot,  ngrad,  tw,     ncols,    prows,  from_x ? 0 : 1, act()};
}

// The k_pupil_rows instantiation for a subaperture/pupil ratio and layer count.
using PupilKern = void (*)(const float *, const float *, const float *, float *, const AxisW *, LayerTab, WfsTab,
                           PadIndex, int, int, int, int, int, long, long, long, int, int, int, const int *);
static PupilKern pupil_kern(bool from_x, bool p2, bool few) {
    return from_x ? (p2 ? (few ? k_pupil_rows<true, 2, 8> : k_pupil_rows<true, 2, 16>)
                        : (few ? k_pupil_rows<true, 1, 8> : k_pupil_rows<true, 1, 16>))
                  : (p2 ? (few ? k_pupil_rows<false, 2, 8> : k_pupil_rows<false, 2, 16>)
                        : (few ? k_pupil_rows<false, 1, 8> : k_pupil_rows<false, 1, 16>));
}
using PupilGroupKern = void (*)(GroupTab<PupilArgs>);
static PupilGroupKern pupil_group_kern(bool from_x, bool p2, bool few) {
    return from_x ? (p2 ? (few ? k_pupil_rows_group<true, 2, 8> : k_pupil_rows_group<true, 2, 16>)
                        : (few ? k_pupil_rows_group<true, 1, 8> : k_pupil_rows_group<true, 1, 16>))
                  : (p2 ? (few ? k_pupil_rows_group<false, 2, 8> : k_pupil_rows_group<false, 2, 16>)
                        : (few ? k_pupil_rows_group<false, 1, 8> : k_pupil_rows_group<false, 1, 16>));
}

// Launch k_pupil_rows over every WFS: one launch per run of consecutive WFS
// with the same subaperture/pupil ratio.
void Recon::pupil_rows(bool from_x, const float *xin, cudaStream_t s) {
    for (int w0 = 0; w0 < nwfs;) {
        int w1 = w0 + 1;
        while (w1 < nwfs && wfs_h[w1].pos == wfs_h[w0].pos) w1++;
        const PupilArgs a = pupil_args(from_x, xin, w0);
        launch(pupil_kern(from_x, wfs_h[w0].pos == 2, nps <= 8), dim3(ptiles, w1 - w0, nb), dim3(kThreads),
               pupil_smem, s, a.x, a.grad, a.tt, a.t, a.tab, a.lt, a.wt, a.pi, a.wbase, a.nps, a.nwfs, a.nxp, a.nyp,
               a.nxtot, a.ngrad, a.tw, a.ncols, a.rows, a.do_tt, a.act);
        w0 = w1;
    }
}

HxtArgs Recon::hxt_args(const float *xin, float *out, double *dot_part, int do_l2, int k) const {
    return HxtArgs{tbuf.p, xin, out, dot_part, pad(), laytab, nps, nwfs, nyp, nxtot, tw, do_l2, scal(), k, nb, act()};
}

using HxtKern = void (*)(const float *, const float *, float *, double *, PadIndex, LayerTab, int, int, int, long,
                         long, int, CgScal, int, int, const int *);
static HxtKern hxt_kern(int ky, int ni) {
    static const HxtKern tab1[kMaxPadY] = {k_hxt_rows<1, 1>, k_hxt_rows<2, 1>, k_hxt_rows<3, 1>, k_hxt_rows<4, 1>,
                                           k_hxt_rows<5, 1>, k_hxt_rows<6, 1>, k_hxt_rows<7, 1>, k_hxt_rows<8, 1>};
    static const HxtKern tab2[kMaxPadY] = {k_hxt_rows<1, 2>, k_hxt_rows<2, 2>, k_hxt_rows<3, 2>, k_hxt_rows<4, 2>,
                                           k_hxt_rows<5, 2>, k_hxt_rows<6, 2>, k_hxt_rows<7, 2>, k_hxt_rows<8, 2>};
    return ni == 2 ? tab2[ky - 1] : tab1[ky - 1];
}
using HxtGroupKern = void (*)(GroupTab<HxtArgs>);
static HxtGroupKern hxt_group_kern(int ky, int ni) {
    static const HxtGroupKern tab1[kMaxPadY] = {k_hxt_rows_group<1, 1>, k_hxt_rows_group<2, 1>, k_hxt_rows_group<3, 1>,
                                                k_hxt_rows_group<4, 1>, k_hxt_rows_group<5, 1>, k_hxt_rows_group<6, 1>,
                                                k_hxt_rows_group<7, 1>, k_hxt_rows_group<8, 1>};
    static const HxtGroupKern tab2[kMaxPadY] = {k_hxt_rows_group<1, 2>, k_hxt_rows_group<2, 2>, k_hxt_rows_group<3, 2>,
                                                k_hxt_rows_group<4, 2>, k_hxt_rows_group<5, 2>, k_hxt_rows_group<6, 2>,
                                                k_hxt_rows_group<7, 2>, k_hxt_rows_group<8, 2>};
    return ni == 2 ? tab2[ky - 1] : tab1[ky - 1];
}

// k_hxt_rows at the padded y-list width, two instances per thread when the
// batch has more than one.
void Recon::hxt_rows(const float *xin, float *out, double *dot_part, int do_l2, int k, cudaStream_t s) {
    const int ni = hxt_ni();
    const HxtArgs a = hxt_args(xin, out, dot_part, do_l2, k);
    launch(hxt_kern(ky, ni), dim3(nblk_hxt, (nb + ni - 1) / ni), dim3(hxt_threads), 0, s, a.t, a.xin, a.out,
           a.dot_part, a.pi, a.lt, a.nps, a.nwfs, a.nyp, a.nxtot, a.tw, a.do_l2, a.S, a.kit, a.nb, a.act);
}

void Recon::build_wfs_tables(const mb_recon_desc *d) {
    const mb_grid &pm = d->pmap;
    wfs_h.resize(nwfs);
    for (int w = 0; w < nwfs; w++) {
        const mb_wfs_desc &W = d->wfs[w];
        const int ns = W.nsa;
        MB_REQUIRE(ns > 0 && W.salocx && W.salocy && W.gp_p && W.gp_i && W.gp_x && W.neai,
                   "wfs %d: missing arrays", w);
        const double posd = W.dsa / pm.dx;
        const int pos = (int)std::lround(posd);
        if (!(pos == 1 || pos == 2) || std::fabs(posd - pos) > 1e-9) {
            set_error("wfs %d: subaperture/pupil sampling ratio %g is not 1 or 2", w, posd);
            throw InvalidArg{MB_EUNSUP};
        }
        const int n1 = pos + 1;
        // share tables between WFS that pass identical arrays (like tomo.cu:259-276)
        int share = -1;
        for (int v = 0; v < w; v++) {
            const mb_wfs_desc &V = d->wfs[v];
            if (V.gp_x == W.gp_x && V.gp_p == W.gp_p && V.salocx == W.salocx && V.nsa == ns &&
                V.dsa == W.dsa)
                share = v;
        }
        std::vector<int2> sp(ns);
        std::vector<float2> coef((size_t)ns * n1 * n1, make_float2(0.f, 0.f));
        if (share < 0) {
            std::vector<int> sm(np, -1);
            for (int s = 0; s < ns; s++) {
                const long ix = std::lround((W.salocx[s] - pm.ox) / pm.dx);
                const long iy = std::lround((W.salocy[s] - pm.oy) / pm.dy);
                MB_REQUIRE(ix >= 0 && iy >= 0 && ix + pos < nxp && iy + pos < nyp,
                           "wfs %d subaperture %d lies outside the pupil grid", w, s);
                sp[s] = make_int2((int)ix, (int)iy);
                MB_REQUIRE(sm[iy * nxp + ix] < 0, "wfs %d: two subapertures share a corner", w);
                sm[iy * nxp + ix] = s;
            }
            // GP in CSC: columns are pupil points, rows gradients.  Entries
            // outside a subaperture's stencil are accepted only as rounding
            // noise of the GP construction (below 1e-9 of the largest
            // coefficient, e.g. 1e-14 when dsa is not exact in binary) and
            // dropped.
            double gmax = 0;
            for (long k = 0; k < W.gp_p[np]; k++) gmax = std::max(gmax, std::fabs(W.gp_x[k]));
            for (int col = 0; col < np; col++) {
                const int px = col % nxp, py = col / nxp;
                for (int k = W.gp_p[col]; k < W.gp_p[col + 1]; k++) {
                    const int row = W.gp_i[k];
                    MB_REQUIRE(row >= 0 && row < 2 * ns, "wfs %d: GP row %d out of range", w, row);
                    const int s = row < ns ? row : row - ns;
                    const int tx = px - sp[s].x, ty = py - sp[s].y;
                    if (tx < 0 || tx > pos || ty < 0 || ty > pos) {
                        if (std::fabs(W.gp_x[k]) > 1e-9 * gmax) {
                            set_error("wfs %d: GP couples subaperture %d to a pupil point outside "
                                      "its %dx%d stencil", w, s, n1, n1);
                            throw InvalidArg{MB_EUNSUP};
                        }
                        continue;
                    }
                    float2 &c = coef[(size_t)s * n1 * n1 + ty * n1 + tx];
                    if (row < ns) c.x += (float)W.gp_x[k];
                    else c.y += (float)W.gp_x[k];
                }
            }
            saptr.emplace_back(new DevBuf<int2>());
            saptr.back()->upload(sp);
            gp.emplace_back(new DevBuf<float2>());
            gp.back()->upload(coef);
            samap.emplace_back(new DevBuf<int>());
            samap.back()->upload(sm);
            wfs_h[w].saptr = saptr.back()->p;
            wfs_h[w].gp = gp.back()->p;
            wfs_h[w].samap = samap.back()->p;
        } else {
            wfs_h[w].saptr = wfs_h[share].saptr;
            wfs_h[w].gp = wfs_h[share].gp;
            wfs_h[w].samap = wfs_h[share].samap;
        }
        wfs_h[w].nsa = ns;
        wfs_h[w].pos = pos;
        wfs_h[w].goff = (int)goff[w];
        neai.emplace_back(new DevBuf<float>());
        ptt.emplace_back(new DevBuf<float>());
        set_neai(w, W.neai, W.ptt);
    }
    wfs.upload(wfs_h);
    MB_REQUIRE(nwfs <= kMaxWfs, "at most %d WFS", kMaxWfs);
    for (int w = 0; w < nwfs; w++) wfstab.w[w] = wfs_h[w];
}

void Recon::set_neai(int w, const double *ne, const double *pt) {
    const int ns = nsa[w];
    std::vector<float> h(3 * (size_t)ns);
    for (size_t i = 0; i < h.size(); i++) {
        MB_REQUIRE(std::isfinite(ne[i]), "wfs %d: non-finite NEA", w);
        h[i] = (float)ne[i];
    }
    neai[w]->upload(h);
    wfs_h[w].neai = neai[w]->p;
    if (pt) {
        std::vector<float> q(4 * (size_t)ns);
        for (size_t i = 0; i < q.size(); i++) q[i] = (float)pt[i];
        ptt[w]->upload(q);
        wfs_h[w].ptt = ptt[w]->p;
        wfs_h[w].has_ptt = 1;
    } else {
        wfs_h[w].ptt = nullptr;
        wfs_h[w].has_ptt = 0;
    }
}

void Recon::set_l2c(const double *l2c) {
    for (int l = 0; l < nps; l++) {
        MB_REQUIRE(std::isfinite(l2c[l]) && l2c[l] >= 0, "layer %d: invalid l2c", l);
        lay_h[l].l2c = (float)l2c[l];
    }
    lay.upload(lay_h);
    MB_REQUIRE(nps <= kMaxLayers, "at most %d layers", kMaxLayers);
    for (int l = 0; l < nps; l++) laytab.l[l] = lay_h[l];  // captured graphs are re-captured by the caller
    l2c_now.assign(l2c, l2c + nps);
}

// FDPCG tables for the half spectrum.  The reference orders the frequency
// blocks with the non-positive x frequencies first (maos/fdpcg.c:119-197,
// fdpcg_perm); those leading blocks reach every stored bin of each layer's
// real-to-complex spectrum, some bins twice (once directly, once as a
// conjugate).  Each stored bin gets exactly one writer, preferring the
// direct member, so the result does not depend on write order.
void Recon::build_fdpcg(const mb_fdpcg_desc *fd) {
    MB_REQUIRE(fd && fd->perm && fd->mbinv && fd->nb > 0 && fd->bs > 0, "fdpcg tables missing");
    MB_REQUIRE((long)fd->nb * fd->bs == nxtot, "fdpcg: nb*bs=%ld differs from nxtot=%ld",
               (long)fd->nb * fd->bs, nxtot);
    MB_REQUIRE(fd->bs <= kMaxBs, "fdpcg: block size %d above %d", fd->bs, kMaxBs);
    fd_nb = fd->nb;
    fd_bs = fd->bs;
    std::vector<long> hoff(nps), hsz(nps);
    long acc = 0;
    for (int l = 0; l < nps; l++) {
        MB_REQUIRE(lay_h[l].nx % 2 == 0 && lay_h[l].ny % 2 == 0, "fdpcg: layer %d grid %dx%d is not even", l,
                   lay_h[l].nx, lay_h[l].ny);
        hsz[l] = (long)lay_h[l].ny * (lay_h[l].nx / 2 + 1);
        hoff[l] = acc;
        acc += (long)nb * hsz[l];
    }
    MB_REQUIRE(acc < (1L << 31), "fdpcg: batch too large for 32-bit spectrum index");
    struct Mem { int l; long pos; bool conj; };
    auto member = [&](long q) {
        if (q < 0) q = -q;
        MB_REQUIRE(q < nxtot, "fdpcg: perm out of range");
        int l = 0;
        while (l + 1 < nps && q >= xoff[l + 1]) l++;
        const long local = q - xoff[l];
        const int nx = lay_h[l].nx, ny = lay_h[l].ny;
        long jx = local % nx, jy = local / nx;
        bool cj = false;
        if (jx > nx / 2) {  // bin of a positive-x frequency: the conjugate of a stored bin
            cj = true;
            jx = nx - jx;
            jy = (ny - jy) % ny;
        }
        return Mem{l, jy * (nx / 2 + 1) + jx, cj};
    };
    // solve the leading blocks until every stored bin has a writer
    std::vector<std::vector<long>> writer(nps);
    long ntot = 0, nreach = 0;
    for (int l = 0; l < nps; l++) {
        writer[l].assign(hsz[l], -1);
        ntot += hsz[l];
    }
    int nbh = 0;
    for (int blk = 0; blk < fd_nb && nreach < ntot; blk++, nbh++)
        for (int m = 0; m < fd_bs; m++) {
            const long i = (long)blk * fd_bs + m;
            const Mem e = member(fd->perm[i]);
            long &wr = writer[e.l][e.pos];
            if (wr < 0) {
                wr = i;
                nreach++;
            } else if (!e.conj && member(fd->perm[wr]).conj) {
                wr = i;  // prefer the direct member
            }
        }
    if (nreach < ntot) {
        set_error("fdpcg: the block ordering does not reach the half spectrum (%ld of %ld bins)", nreach, ntot);
        throw InvalidArg{MB_EUNSUP};
    }
    fd_nbh = nbh;
    std::vector<FdIndex> idx((size_t)nbh * fd_bs);
    std::vector<double> sc((size_t)nbh * fd_bs);
    for (long i = 0; i < (long)nbh * fd_bs; i++) {
        const Mem e = member(fd->perm[i]);
        idx[i].base = (int)(hoff[e.l] + e.pos);
        idx[i].stride = (int)hsz[e.l];
        idx[i].flags = (e.conj ? kFdConj : 0) | (writer[e.l][e.pos] == i ? kFdStore : 0);
        idx[i].pad = 0;
        sc[i] = fd->scale ? 1.0 / std::sqrt((double)lay_h[e.l].nx * lay_h[e.l].ny) : 1.0;
    }
    // The reference's CPU preconditioner keeps the real part of the inverse
    // FFT of M X over the full spectrum (maos/fdpcg.c:612-644).  Its blocks
    // are Hermitian-consistent (M at -k equal to conj(M) at k) only to about
    // 1e-6, so solving half of them and mirroring would be a different
    // operator, and 30 PCG iterations turn that 1e-6 into 1e-4 of the result.
    // The real part equals the mirrored half with the Hermitian average of
    // each block and the block of its negated frequencies:
    //   Ms[b](i,j) = (M[b](i,j) + conj(M[b'](s(i), s(j)))) / 2,
    // b' the block holding the negated frequencies, s the member map.
    std::vector<long> inv(nxtot, -1);
    for (long i = 0; i < nxtot; i++) {
        const long q = fd->perm[i];
        MB_REQUIRE(q >= 0 && q < nxtot && inv[q] < 0, "fdpcg: perm is not a permutation of the spectra");
        inv[q] = i;
    }
    auto negated = [&](long q) {
        int l = 0;
        while (l + 1 < nps && q >= xoff[l + 1]) l++;
        const long local = q - xoff[l];
        const int nx = lay_h[l].nx, ny = lay_h[l].ny;
        const long jx = local % nx, jy = local / nx;
        return xoff[l] + ((ny - jy) % ny) * nx + (nx - jx) % nx;
    };
    std::vector<double> ms((size_t)nbh * fd_bs * fd_bs * 2);
    std::vector<int> bpv(nbh), sigv((size_t)nbh * fd_bs);
    for (long b = 0; b < nbh; b++) {
        long bp = -1;
        int *sig = sigv.data() + b * fd_bs;
        for (int i = 0; i < fd_bs; i++) {
            const long P = inv[negated(fd->perm[b * fd_bs + i])];
            if (i == 0) bp = P / fd_bs;
            MB_REQUIRE(P / fd_bs == bp, "fdpcg: block %ld: its negated frequencies span several blocks", b);
            sig[i] = (int)(P % fd_bs);
        }
        bpv[b] = (int)bp;
        for (int j = 0; j < fd_bs; j++)
            for (int i = 0; i < fd_bs; i++) {
                const size_t k = ((size_t)b * fd_bs + j) * fd_bs + i;
                const size_t kp = ((size_t)bp * fd_bs + sig[j]) * fd_bs + sig[i];
                ms[2 * k] = 0.5 * (fd->mbinv[2 * k] + fd->mbinv[2 * kp]);
                ms[2 * k + 1] = 0.5 * (fd->mbinv[2 * k + 1] - fd->mbinv[2 * kp + 1]);
            }
    }
    // fold the 1/sqrt(n) of the forward and inverse FFTs into the blocks
    std::vector<cplx> M((size_t)nbh * fd_bs * fd_bs);
    for (long b = 0; b < nbh; b++)
        for (int j = 0; j < fd_bs; j++)
            for (int i = 0; i < fd_bs; i++) {
                const size_t k = (size_t)b * fd_bs * fd_bs + (size_t)j * fd_bs + i;
                const double s = sc[b * fd_bs + i] * sc[b * fd_bs + j];
                M[k] = make_float2((float)(ms[2 * k] * s), (float)(ms[2 * k + 1] * s));
            }
    fd_M.upload(M);
    fd_idx.upload(idx);
    // the data term for device rebuilds (k_fd_prepare, k_fd_fold)
    fd_dev = fd->mdiag && (fd->mdata || fd->geom);
    fd_geom = false;
    if (fd_dev) {
        const size_t nel = (size_t)fd_nb * fd_bs * fd_bs;
        if (fd->geom) {  // the data term formed on the device from its geometry
            build_fdpcg_geom(fd);
        } else {
            std::vector<double2> md(nel);
            for (size_t k = 0; k < nel; k++) md[k] = make_double2(fd->mdata[2 * k], fd->mdata[2 * k + 1]);
            fd_mdata.upload(md);
        }
        fd_mdiag.upload(std::vector<double>(fd->mdiag, fd->mdiag + (size_t)fd_nb * fd_bs));
        std::vector<int> ml((size_t)fd_nb * fd_bs);
        for (long i = 0; i < (long)fd_nb * fd_bs; i++) ml[i] = member(fd->perm[i]).l;
        fd_mlayer.upload(ml);
        fd_bp.upload(bpv);
        fd_sig.upload(sigv);
        fd_sc.upload(sc);
        fd_minv.alloc(nel);
        fd_lscale.alloc(nps);
        fd_l2c_ref = l2c_now;
    }
    spec.alloc(acc);
    spec2.alloc(acc);
    spec.zero_async(stream);  // spectra of instances that never ran stay finite
    spec2.zero_async(stream);
    // FFT geometry per layer: radix stages (4 first, then 2, 3, 5) and one
    // twiddle table per distinct length, computed in FP64
    std::vector<FdLayer> fl(nps);
    std::vector<cplx> tw;
    std::vector<std::pair<int, int>> twof;  // (n, offset)
    auto table = [&](int n) {
        for (auto &e : twof)
            if (e.first == n) return e.second;
        const int o = (int)tw.size();
        for (int k = 0; k < n; k++) {
            const double a = -2.0 * M_PI * k / n;
            tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
        twof.push_back({n, o});
        return o;
    };
    auto radices = [&](int n, signed char *rad, int &nr) {
        nr = 0;
        for (int R : {4, 2, 3, 5})
            while (n % R == 0 && nr < 8) {
                rad[nr++] = (signed char)R;
                n /= R;
            }
        return n == 1;
    };
    fd_bufn = 0;
    int twn = 0;  // twiddle entries a layer CTA stages (nx + ny)
    for (int l = 0; l < nps; l++) {
        FdLayer &F = fl[l];
        F.nx = lay_h[l].nx;
        F.ny = lay_h[l].ny;
        if (!radices(F.nx, F.rx, F.nrx) || !radices(F.ny, F.ry, F.nry)) {
            set_error("fdpcg: layer %d grid %dx%d is not a product of 2, 3 and 5 in 8 stages", l, F.nx, F.ny);
            throw InvalidArg{MB_EUNSUP};
        }
        MB_REQUIRE(F.nx <= kFftThreads && F.ny <= 2 * kFftThreads, "fdpcg: layer %d grid %dx%d too large", l,
                   F.nx, F.ny);
        F.off = lay_h[l].off;
        F.hoff = (int)hoff[l];
        F.hs = (int)hsz[l];
        F.twx = table(F.nx);
        F.twy = table(F.ny);
        F.px = F.py = -1;  // two-pass FFT where a factor pair is listed
        for (int i = 0; i < kNumFftPairs; i++) {
            if (F.px < 0 && kFftPairs[i][0] * kFftPairs[i][1] == F.nx) F.px = i;
            if (F.py < 0 && kFftPairs[i][0] * kFftPairs[i][1] == F.ny) F.py = i;
        }
        fd_bufn = std::max(fd_bufn, std::max(F.ny / 2 * F.nx, F.ny * (F.nx / 2 + 1)));
        if (F.px >= 0) fd_bufn = std::max(fd_bufn, fft2_scratch(F.px, true, F.ny / 2));
        if (F.py >= 0) fd_bufn = std::max(fd_bufn, fft2_scratch(F.py, false, F.nx / 2 + 1));
        twn = std::max(twn, F.nx + F.ny);
    }
    fd_lay.upload(fl);
    for (int l = 0; l < nps; l++) fdtab.l[l] = fl[l];
    fd_tw.upload(tw);
    fd_smem = (2 * (size_t)fd_bufn + twn) * sizeof(cplx);
    MB_REQUIRE(fd_smem <= 200 * 1024, "fdpcg: layer FFT needs %zu bytes of shared memory", fd_smem);
    MB_CUDA_TRY(cudaFuncSetAttribute(k_fd_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fd_smem));
    MB_CUDA_TRY(cudaFuncSetAttribute(k_fd_inv<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fd_smem));
    MB_CUDA_TRY(cudaFuncSetAttribute(k_fd_inv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fd_smem));
    // the CG step's inverse runs as clusters of the nps layer CTAs of an instance when such a cluster fits
    fd_cluster = false;
    if (nps <= 16) {
        if (nps > 8)
            MB_CUDA_TRY(cudaFuncSetAttribute(k_fd_inv<true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)nps;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nps, nb);
        cfg.blockDim = dim3(kFftThreads);
        cfg.dynamicSmemBytes = fd_smem;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int ncl = 0;
        fd_cluster = cudaOccupancyMaxActiveClusters(&ncl, k_fd_inv<true>, &cfg) == cudaSuccess && ncl > 0;
        cudaGetLastError();  // a size the device refuses only means the unclustered path
        if (const char *e = std::getenv("MAOS_B200_FD_CLUSTER")) fd_cluster = fd_cluster && e[0] != '0';
    }
    build_fdpcg_fused(idx, hoff);
}

// Split each layer over K_l CTAs of an instance's cluster (K_l proportional
// to its size, at most 16 CTAs in all), the CTAs' row-pair, column and block
// ranges, the common shared-memory layout, and each block member's owner.
void Recon::build_fdpcg_fused(const std::vector<FdIndex> &idx, const std::vector<long> &hoff) {
    fd_fused_ok = false;
    fd_mode = 1;
    long nmin = LONG_MAX;
    for (int l = 0; l < nps; l++) nmin = std::min(nmin, (long)lay_h[l].nx * lay_h[l].ny);
    // CTAs per layer proportional to its size, scaled up to as many as the
    // cluster holds (kMaxFdParts, or MAOS_B200_FD_CTAS, a tuning override)
    int cmax = kMaxFdParts;
    if (const char *e = std::getenv("MAOS_B200_FD_CTAS")) {
        const int v = std::atoi(e);
        if (v >= 1 && v <= kMaxFdParts) cmax = v;
    }
    std::vector<int> K(nps);
    int C = 0;
    auto split = [&](double scale) {
        int c = 0;
        for (int l = 0; l < nps; l++) {
            const FdLayer &F = fdtab.l[l];
            K[l] = (int)std::max(1L, std::lround(scale * F.nx * F.ny / (double)nmin));
            K[l] = std::min(K[l], std::min(F.ny / 2, F.nx / 2 + 1));
            c += K[l];
        }
        return c;
    };
    double sbest = 1.0;
    int cbest = split(1.0);
    for (double sc = 1.05; sc <= 8.0; sc += 0.05) {
        const int c = split(sc);
        if (c <= cmax && c > cbest) {
            cbest = c;
            sbest = sc;
        }
    }
    C = split(sbest);
    while (C > cmax) {  // take CTAs from the most split layer
        int lm = 0;
        for (int l = 1; l < nps; l++)
            if (K[l] > K[lm]) lm = l;
        if (K[lm] <= 1) return;  // more layers than cluster CTAs: the three-kernel form only
        K[lm]--;
        C--;
    }
    for (int l = 0; l < nps; l++)
        if (fdtab.l[l].nx > kFusedThreads) return;  // a row per thread: the three-kernel form only
    FdFusedTab T{};
    T.C = C;
    int maxnx = 0, maxny = 0;
    long nR = kFusedThreads, nS = 0, nSC = 0;
    int rank = 0;
    std::vector<int> rbase(nps);
    for (int l = 0; l < nps; l++) {
        const FdLayer &F = fdtab.l[l];
        const int np2 = F.ny / 2, h = F.nx / 2 + 1;
        maxnx = std::max(maxnx, F.nx);
        maxny = std::max(maxny, F.ny);
        rbase[l] = rank;
        for (int q = 0; q < K[l]; q++, rank++) {
            FdPart &P = T.c[rank];
            P.l = (short)l;
            P.q = (short)q;
            P.K = (short)K[l];
            P.rbase = (short)rbase[l];
            P.p0 = (short)(q * np2 / K[l]);
            P.p1 = (short)((q + 1) * np2 / K[l]);
            P.c0 = (short)(q * h / K[l]);
            P.c1 = (short)((q + 1) * h / K[l]);
            P.b0 = (int)((long)rank * fd_nbh / C);
            P.b1 = (int)((long)(rank + 1) * fd_nbh / C);
            const int npr = P.p1 - P.p0, ncl = P.c1 - P.c0;
            MB_REQUIRE(npr >= 1 && ncl >= 1, "fdpcg: layer %d split %d is empty", l, q);
            nR = std::max(nR, (long)npr * F.nx);
            nS = std::max(nS, (long)(F.px >= 0 ? fft2_scratch(F.px, true, npr) : npr * F.nx));
            nS = std::max(nS, (long)(F.py >= 0 ? fft2_scratch(F.py, false, ncl) : (long)F.ny * ncl));
            nSC = std::max(nSC, (long)F.ny * ncl);
        }
    }
    for (int c = 0; c < C; c++)  // the rank's blocks are uniform over the whole cluster
        MB_REQUIRE(T.c[c].b1 > T.c[c].b0, "fdpcg: fewer frequency blocks than cluster CTAs");
    T.oTY = maxnx;
    T.oR = maxnx + maxny;
    T.oS = (int)(T.oR + nR);
    T.oSC = (int)(T.oS + nS);
    T.oSY = (int)(T.oSC + nSC);
    fd_fsmem = (size_t)(T.oSY + nSC) * sizeof(cplx);
    if (fd_fsmem > 200 * 1024) return;  // else the three-kernel form
    // member owners: the CTA whose columns hold the member's bin
    std::vector<FdMem> mem(idx.size());
    for (size_t i = 0; i < idx.size(); i++) {
        int l = 0;
        while (l + 1 < nps && idx[i].base >= hoff[l + 1]) l++;
        const FdLayer &F = fdtab.l[l];
        const int h = F.nx / 2 + 1;
        const long pos = idx[i].base - hoff[l];  // instance 0's half spectrum of layer l
        MB_REQUIRE(pos >= 0 && pos < (long)F.ny * h, "fdpcg: member %zu outside its layer", i);
        const int ky = (int)(pos / h), kx = (int)(pos % h);
        int q = K[l] - 1;
        while (T.c[rbase[l] + q].c0 > kx) q--;
        const FdPart &O = T.c[rbase[l] + q];
        mem[i].rank = (short)(rbase[l] + q);
        mem[i].off = ky * (O.c1 - O.c0) + (kx - O.c0);
        mem[i].flags = (short)idx[i].flags;
    }
    // the cluster must be schedulable
    if (C > 8) {
        if (cudaFuncSetAttribute(k_fd_fused, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
    }
    MB_CUDA_TRY(cudaFuncSetAttribute(k_fd_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fd_fsmem));
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, nb);
    cfg.blockDim = dim3(kFusedThreads);
    cfg.dynamicSmemBytes = fd_fsmem;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    const bool fits = cudaOccupancyMaxActiveClusters(&ncl, k_fd_fused, &cfg) == cudaSuccess && ncl > 0;
    cudaGetLastError();
    if (!fits) return;
    fd_mem.upload(mem);
    fused_tab = T;
    fd_fused_ok = true;
}

// The data term's geometry on the device: per block its base pupil
// frequency, per member its layer and shifted frequency (from fd->perm, the
// natural-order FFT index), the transfer functions, the selection
// autocorrelation, the layer heights and WFS directions; then the data term
// at the setup's mean NEA.
void Recon::build_fdpcg_geom(const mb_fdpcg_desc *fd) {
    const mb_fdpcg_geom *g = fd->geom;
    MB_REQUIRE(g->nxp > 0 && g->nyp > 0 && g->dxp > 0 && g->pos >= 1 && g->pos <= 4 && g->adimx > 0 &&
                   g->adimy > 0 && g->gx && g->gy && g->neam && g->nsel >= 0 && g->nsel <= 64 &&
                   (g->nsel == 0 || (g->sel_dx && g->sel_dy && g->sel_r)),
               "fdpcg geometry: invalid sizes or missing arrays");
    MB_REQUIRE(nwfs <= kMaxWfs, "fdpcg geometry: at most %d WFS", kMaxWfs);
    fdg.nxp = g->nxp;
    fdg.nyp = g->nyp;
    fdg.pos = g->pos;
    fdg.adimx = g->adimx;
    fdg.adimy = g->adimy;
    fdg.nsel = g->nsel;
    fdg.needscale = g->needscale;
    fdg.nwfs = nwfs;
    fdg.bs = fd_bs;
    fdg.dxp = g->dxp;
    fdg.scale0 = (double)lay_h[0].nx * lay_h[0].ny;
    std::vector<int> lnx(nps), lny(nps);
    std::vector<double> lht(nps);
    for (int l = 0; l < nps; l++) {
        lnx[l] = lay_h[l].nx;
        lny[l] = lay_h[l].ny;
        lht[l] = xgrid[l].ht;
        const int ratio = g->nxp / lnx[l];
        MB_REQUIRE(ratio <= 2 && g->nyp / lny[l] == ratio, "fdpcg geometry: layer %d sampled at 1/%d of the pupil",
                   l, ratio);
    }
    std::vector<int4> mem((size_t)fd_nb * fd_bs);
    std::vector<int2> blk(fd_nb);
    for (long i = 0; i < (long)fd_nb * fd_bs; i++) {
        const long q = fd->perm[i];
        int l = 0;
        while (l + 1 < nps && q >= xoff[l + 1]) l++;
        const long local = q - xoff[l];
        const int nx = lay_h[l].nx, ny = lay_h[l].ny;
        const int jx = (int)(local % nx), jy = (int)(local / nx);
        mem[i] = make_int4(l, (jx + nx / 2) % nx, (jy + ny / 2) % ny, 0);
        if (i % fd_bs == 0) {  // member 0 of a block: layer 0, the block's own frequency
            MB_REQUIRE(l == 0, "fdpcg geometry: block %ld does not start on layer 0", i / fd_bs);
            blk[i / fd_bs] = make_int2(jx >= nx / 2 ? jx - nx : jx, jy >= ny / 2 ? jy - ny : jy);
        }
    }
    std::vector<double2> gx((size_t)g->nxp * g->nyp), gy(gx.size()), sr(std::max(g->nsel, 1));
    for (size_t k = 0; k < gx.size(); k++) {
        gx[k] = make_double2(g->gx[2 * k], g->gx[2 * k + 1]);
        gy[k] = make_double2(g->gy[2 * k], g->gy[2 * k + 1]);
    }
    std::vector<int2> sd(std::max(g->nsel, 1), make_int2(-1, -1));
    for (int k = 0; k < g->nsel; k++) {
        sd[k] = make_int2(((g->sel_dx[k] % g->nxp) + g->nxp) % g->nxp, ((g->sel_dy[k] % g->nyp) + g->nyp) % g->nyp);
        sr[k] = make_double2(g->sel_r[2 * k], g->sel_r[2 * k + 1]);
    }
    fdg_mem.upload(mem);
    fdg_blk.upload(blk);
    fdg_gx.upload(gx);
    fdg_gy.upload(gy);
    fdg_seld.upload(sd);
    fdg_selr.upload(sr);
    fdg_thx.upload(wfs_thx);
    fdg_thy.upload(wfs_thy);
    fdg_lht.upload(lht);
    fdg_lnx.upload(lnx);
    fdg_lny.upload(lny);
    fdg_neam.alloc(nwfs);
    fd_mdata.alloc((size_t)fd_nb * fd_bs * fd_bs);
    fd_geom = true;
    form_fdpcg_data(g->neam);
}

// The data term at mean NEA neam [nwfs] (host), into fd_mdata.  Synchronous.
void Recon::form_fdpcg_data(const double *neam) {
    for (int w = 0; w < nwfs; w++)
        MB_REQUIRE(neam[w] > 0 && std::isfinite(neam[w]), "fdpcg: neam of WFS %d is %g", w, neam[w]);
    MB_CUDA_TRY(cudaMemcpyAsync(fdg_neam.p, neam, nwfs * sizeof(double), cudaMemcpyHostToDevice, stream));
    const int npf = fdg.pos * fdg.pos;
    const size_t smem = ((size_t)npf * nwfs * fd_bs + (size_t)npf * npf) * sizeof(double2);
    MB_REQUIRE(smem <= 48 * 1024, "fdpcg geometry: %zu bytes of shared memory per block", smem);
    k_fd_data<<<fd_nb, kFdDataThreads, smem, stream>>>(fdg, fdg_mem.p, fdg_blk.p, fdg_gx.p, fdg_gy.p, fdg_seld.p,
                                                       fdg_selr.p, fdg_neam.p, fdg_thx.p, fdg_thy.p, fdg_lht.p,
                                                       fdg_lnx.p, fdg_lny.p, fd_mdata.p);
    MB_CHECK_LAUNCH();
    MB_CUDA_TRY(cudaStreamSynchronize(stream));
}

// 1: three kernels per preconditioner (k_fd_fwd, k_fd_mul, k_fd_inv);
// 2: the fused cluster kernel (when it fits); 0: the fused one when it fits.
// The step graphs are captured again.
void Recon::set_fdpcg_mode(int mode) {
    fd_mode = (mode == 2 || mode == 0) && fd_fused_ok ? 2 : 1;
    if (graph) capture_graph();
}

// FDPCG blocks from the stored data term at the current l2c: the invpsd
// diagonal scales with each layer's l2c (fdpcg.c:375-403: invpsd is the
// spectrum of L2^T L2).  Synchronous.
void Recon::rebuild_fdpcg_device() {
    MB_REQUIRE(fd_dev, "fdpcg: no data term on the device (mb_fdpcg_desc.mdata/mdiag at setup)");
    std::vector<double> ls(nps);
    for (int l = 0; l < nps; l++) {
        MB_REQUIRE(fd_l2c_ref[l] > 0, "fdpcg: layer %d has no regularisation to scale", l);
        ls[l] = l2c_now[l] / fd_l2c_ref[l];
    }
    MB_CUDA_TRY(cudaMemcpyAsync(fd_lscale.p, ls.data(), nps * sizeof(double), cudaMemcpyHostToDevice, stream));
    k_fd_prepare<<<(fd_nb + kPrepWarps - 1) / kPrepWarps, 32 * kPrepWarps, 0, stream>>>(
        fd_mdata.p, fd_mdiag.p, fd_mlayer.p, fd_lscale.p, fd_minv.p, fd_nb, fd_bs);
    MB_CHECK_LAUNCH();
    const long n = (long)fd_nbh * fd_bs * fd_bs;
    k_fd_fold<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(fd_minv.p, fd_bp.p, fd_sig.p, fd_sc.p, fd_M.p,
                                                             fd_nbh, fd_bs);
    MB_CHECK_LAUNCH();
    MB_CUDA_TRY(cudaStreamSynchronize(stream));
}

void Recon::build(const mb_recon_desc *d) {
    MB_REQUIRE(d, "null descriptor");
    MB_REQUIRE(d->nps > 0 && d->nwfs > 0 && d->xmap && d->wfs && d->l2c, "empty descriptor");
    MB_REQUIRE(d->nbatch >= 1, "nbatch must be >= 1");
    MB_REQUIRE(d->maxit >= 1, "maxit must be >= 1");
    MB_REQUIRE(d->precond == 0 || d->precond == 1, "precond must be 0 or 1");
    MB_CUDA_TRY(cudaGetDevice(&device));
    MB_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    nb = d->nbatch;
    nwfs = d->nwfs;
    nps = d->nps;
    nxp = d->pmap.nx;
    nyp = d->pmap.ny;
    np = nxp * nyp;
    maxit = d->maxit;
    precond = d->precond;
    split = d->split;
    MB_REQUIRE(nxp > 1 && nyp > 1 && d->pmap.dx > 0, "invalid pupil grid");
    xoff.assign(nps + 1, 0);
    lay_h.resize(nps);
    for (int l = 0; l < nps; l++) {
        const mb_grid &g = d->xmap[l];
        MB_REQUIRE(g.nx >= 5 && g.ny >= 5 && g.dx > 0 && g.dy > 0, "layer %d: invalid grid", l);
        lay_h[l].nx = g.nx;
        lay_h[l].ny = g.ny;
        lay_h[l].off = xoff[l];
        lay_h[l].tcol = ncols;
        ncols += g.nx;
        xoff[l + 1] = xoff[l] + (long)g.nx * g.ny;
    }
    nxtot = xoff[nps];
    xgrid.assign(d->xmap, d->xmap + nps);
    goff.assign(nwfs + 1, 0);
    nsa.resize(nwfs);
    int nsamax = 0;
    wfs_thx.resize(nwfs);
    wfs_thy.resize(nwfs);
    for (int w = 0; w < nwfs; w++) {
        nsa[w] = d->wfs[w].nsa;
        nsamax = std::max(nsamax, nsa[w]);
        goff[w + 1] = goff[w] + 2L * nsa[w];
        wfs_thx[w] = d->wfs[w].thetax;
        wfs_thy[w] = d->wfs[w].thetay;
    }
    ngrad = goff[nwfs];
    set_l2c(d->l2c);
    build_hx_tables(d);
    build_pad();
    build_wfs_tables(d);
    nblk_x = (int)nblocks(nxtot);
    nblk_hxt = nblk_x;
    nblk_tt = (int)nblocks(nsamax);
    nsc = maxit + 3;
    const size_t NX = (size_t)nb * nxtot;
    x.alloc(NX); r.alloc(NX); p.alloc(NX); z.alloc(NX); Ap.alloc(NX); rhs.alloc(NX);
    opd.alloc((size_t)nb * nwfs * np);
    tbuf.alloc((size_t)nb * nwfs * tw);
    grad.alloc((size_t)nb * ngrad);
    gin.alloc((size_t)nb * ngrad);
    tt_part.alloc((size_t)nb * nwfs * nblk_tt * 2);
    pap_part.alloc((size_t)nb * nblocks(nxtot, 64));  // room for k_hxt_rows CTAs down to 64 threads
    rr_part.alloc((size_t)nb * nblk_x);
    rz_part.alloc((size_t)nb * nblk_x);
    bb_part.alloc((size_t)nb * nblk_x);
    sc.alloc((size_t)nb * nsc);
    res.alloc(nb);
    ab.alloc((size_t)nb * 2);
    tt.alloc((size_t)nb * nwfs * 2);
    cnt.alloc(nb);
    cnt_tt.alloc((size_t)nb * nwfs);
    active.alloc(nb);
    MB_CUDA_TRY(cudaHostAlloc(&mask_host, (size_t)nb * sizeof(int), cudaHostAllocDefault));
    MB_CUDA_TRY(cudaEventCreateWithFlags(&mask_ev, cudaEventDisableTiming));
    for (int b = 0; b < nb; b++) mask_host[b] = 1;
    MB_CUDA_TRY(cudaMemcpyAsync(active.p, mask_host, (size_t)nb * sizeof(int), cudaMemcpyHostToDevice, stream));
    MB_CUDA_TRY(cudaEventRecord(mask_ev, stream));
    if (precond) build_fdpcg(d->fdpcg);
    MB_REQUIRE(!(d->fit && d->fit_sparse), "give either the grid-form fit or the assembled fit, not both");
    if (d->fit) build_fit(d->fit);
    if (d->fit_sparse) build_fit_sparse(d->fit_sparse);
    x.zero_async(stream);
    gin.zero_async(stream);
    sc.zero_async(stream);
    res.zero_async(stream);
    ab.zero_async(stream);
    tt.zero_async(stream);
    cnt.zero_async(stream);
    cnt_tt.zero_async(stream);
    MB_CUDA_TRY(cudaStreamSynchronize(stream));
    capture_graph();
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
void Recon::op_hx(const float *xin, cudaStream_t s) {
    launch(nps <= 8 ? k_hx<8> : k_hx<16>, dim3(nblocks(np), nwfs, nb), dim3(kThreads), 0, s, xin, opd.p, hx.fwd.p, laytab, nps, nwfs,
                                                         nxp, nyp, nxtot, nullptr, nullptr, act());
}

void Recon::op_rhs_gp(const float *g, cudaStream_t s) {
    launch(k_gp, dim3(nblk_tt, nwfs, nb), dim3(kThreads), 0, s, nullptr, g, grad.p, tt_part.p, wfs.p, nwfs,
                                                      nxp, np, ngrad, 1, tt.p, cnt_tt.p, act());
}

void Recon::op_rhs(const float *g, float *out, cudaStream_t s) {
    // TomoR: x = Hx^T GP^T NEA^-1 (I - TT PTT) g   (recon_utils.c:397, tomo.cu:607)
    op_rhs_gp(g, s);
    pupil_rows(false, nullptr, s);
    hxt_rows(nullptr, out, nullptr, 0, 0, s);
}

void Recon::op_lhs(const float *xin, float *out, double *dot_part, cudaStream_t s, int k) {
    // TomoL: Hx^T GP^T NEA^-1 (I - TT PTT) GP Hx x + L2^T L2 x   (recon_utils.c:447, tomo.cu:639)
    if (split) {  // no tip/tilt term: Hx, GP, NEA, GP^T fused per pupil-row block
        pupil_rows(true, xin, s);
    } else {      // the tip/tilt projection needs every gradient of a WFS first
        op_hx(xin, s);
        launch(k_gp, dim3(nblk_tt, nwfs, nb), dim3(kThreads), 0, s, opd.p, nullptr, grad.p, tt_part.p, wfs.p,
                                                          nwfs, nxp, np, ngrad, 1, tt.p, cnt_tt.p, act());
        pupil_rows(false, nullptr, s);
    }
    hxt_rows(xin, out, dot_part, 1, k, s);
}

// The block solve of every (half-spectrum block, instance), fd_mul_ni
// instances per CTA.
void Recon::fd_mul(cudaStream_t s) {
    using K = void (*)(const cplx *, cplx *, const cplx *, const FdIndex *, int, int, int, const int *);
    const K k = fd_mul_ni == 2 ? k_fd_mul<2> : fd_mul_ni == 4 ? k_fd_mul<4> : fd_mul_ni == 16 ? k_fd_mul<16>
                                                                                            : k_fd_mul<8>;
    const int per = kThreads / fd_bs;
    launch(k, dim3((fd_nbh + per - 1) / per, (nb + fd_mul_ni - 1) / fd_mul_ni), dim3(kThreads), 0, s, spec.p, spec2.p,
           fd_M.p, fd_idx.p, fd_nbh, fd_bs, nb, act());
}

bool Recon::op_fdpcg(float *rin, float *zout, double *rzp, cudaStream_t s, int k, int init, bool in_cg,
                     float *xupd, const float *pupd, const float *Apupd, float *pnext) {
    // fdpcg_precond (maos/fdpcg.c:661): FFT -> permute -> block solve -> permute back -> IFFT,
    // on the half spectrum as in cuda/fdpcg.cu (fdpcg_mul_block_sync_half)
    if (in_cg && pnext && fd_mode == 2) {  // one launch: layers split over an instance's cluster
        launch_cluster(k_fd_fused, dim3(fused_tab.C, nb), dim3(kFusedThreads), fd_fsmem, s, fused_tab.C, rin, fdtab,
                       fused_tab, fd_tw.p, fd_M.p, fd_mem.p, fd_bs, nxtot, xupd, Apupd, scal(), k, init, act(),
                       pnext);
        return true;
    }
    launch(k_fd_fwd, dim3(nps, nb), dim3(kFftThreads), fd_smem, s, rin, spec.p, fdtab, fd_tw.p, nxtot, fd_bufn, xupd,
                                                        pupd, Apupd, xupd ? ab.p : nullptr, act());
    fd_mul(s);
    CgScal S = in_cg ? scal() : CgScal{};
    if (in_cg && pnext && fd_cluster) {  // the p update inside, clusters of the layer CTAs
        launch_cluster(k_fd_inv<true>, dim3(nps, nb), dim3(kFftThreads), fd_smem, s, nps, spec2.p, rin, zout, rzp,
                       fdtab, fd_tw.p, nxtot, fd_bufn, S, k, init, act(), pnext);
        return true;
    }
    launch(k_fd_inv<false>, dim3(nps, nb), dim3(kFftThreads), fd_smem, s, spec2.p, rin, zout, rzp, fdtab, fd_tw.p,
           nxtot, fd_bufn, S, k, init, act(), (float *)nullptr);
    return false;
}

void Recon::cg_init(CgRun &c, int k, cudaStream_t s) {
    // after Ap = A x: r = b - A x, b.b, z = M r, (r.z)_k, p = z
    const CgBufs &B = c.B;
    launch(k_cg_init_r, dim3(c.nblk, nb), dim3(kThreads), 0, s, B.rhs, B.Ap, B.r, B.bb, c.n, B.S, c.iters, act());
    bool pdone = false;
    if (c.Mmul) {
        pdone = c.Mmul(B.r, B.z, B.rz, k, 1);
    } else {
        launch(k_dot_self, dim3(c.nblk, nb), dim3(kThreads), 0, s, B.r, B.rz, c.n, B.S, k, act());  // z aliases r
    }
    if (!pdone)
        launch(k_cg_update_p, dim3(nblocks((c.n + kUpdP - 1) / kUpdP), nb), dim3(kThreads), 0, s, B.p, c.zp, c.n, B.S,
               1, act());
}

bool Recon::cg_post(CgRun &c, int k, cudaStream_t s) {
    // after Ap = A p_k (whose last block left alpha_k)
    const CgBufs &B = c.B;
    bool pdone;
    if (c.XrMmul && k + 1 < c.iters) {
        pdone = c.XrMmul(k);  // x, r update and preconditioner; beta_k (and p, when it says so)
    } else {
        launch(k_cg_update_xr, dim3(c.nblk, nb), dim3(kThreads), 0, s, B.x, B.r, B.p, B.Ap, B.rr, c.n, B.S, k,
               c.iters, c.Mmul ? 0 : 1, act());
        if (k + 1 == c.iters) return true;
        pdone = c.Mmul ? c.Mmul(B.r, B.z, B.rz, k, 0) : false;  // beta_k (and p, when it says so)
    }
    if (!pdone)
        launch(k_cg_update_p, dim3(nblocks((c.n + kUpdP - 1) / kUpdP), nb), dim3(kThreads), 0, s, B.p, c.zp, c.n, B.S,
               0, act());
    return false;
}

// (Preconditioned) CG with FP64 scalars, the schedule of lib/pcg.c:28: the
// residual is recomputed from x every kCgRestart = 100 iterations as the
// reference's CPU solver does (its GPU solver, cuda/pcg.cu:87, every 500),
// which matters to the long solves of the control-matrix build.  x holds the
// warm start.
// XrMmul, when given, performs the x/r update of a non-final iteration
// together with the preconditioner.
void Recon::enqueue_cg(const CgBufs &B, long n, int nblk, int iters, const AmulFn &Amul,
                       const MmulFn &Mmul, cudaStream_t s, const XrMmulFn &XrMmul) {
    CgRun c{B, n, nblk, iters, Mmul, XrMmul, Mmul ? B.z : B.r};
    Amul(B.x, B.Ap, nullptr, 0);
    cg_init(c, 0, s);
    for (int k = 0; k < iters; k++) {
        if (k > 0 && k % kCgRestart == 0) {
            // restart as lib/pcg.c:61 does every 100 iterations: r = b - A x,
            // z = M r, p = z, (r.z)_k afresh (the p of the previous step is dropped)
            Amul(B.x, B.Ap, nullptr, 0);
            cg_init(c, k, s);
        }
        Amul(B.p, B.Ap, B.pap, k);  // its last block leaves alpha_k
        if (cg_post(c, k, s)) break;
    }
}

Recon::CgRun Recon::solve_run(cudaStream_t s) {
    CgRun c{CgBufs{x.p, r.p, p.p, z.p, Ap.p, rhs.p, pap_part.p, rr_part.p, rz_part.p, bb_part.p, scal()},
            nxtot, nblk_x, maxit, MmulFn(), XrMmulFn(), r.p};
    if (precond) {
        c.Mmul = [this, s](float *in, float *out, double *dot, int k, int init) {
            return op_fdpcg(in, out, dot, s, k, init, true, nullptr, nullptr, nullptr, p.p);
        };
        c.XrMmul = [this, s](int k) { return op_fdpcg(r.p, z.p, rz_part.p, s, k, 0, true, x.p, p.p, Ap.p, p.p); };
        c.zp = z.p;
    }
    return c;
}

// The whole per-step tomography: RHS, then (FD)PCG from the warm start in x.
void Recon::enqueue_solve(cudaStream_t s) {
    op_rhs(gin.p, rhs.p, s);
    CgRun c = solve_run(s);
    AmulFn A = [&](const float *in, float *out, double *dot, int k) { op_lhs(in, out, dot, s, k); };
    enqueue_cg(c.B, c.n, c.nblk, c.iters, A, c.Mmul, s, c.XrMmul);
}

// y = M x - U (V'x) for all instances: one warp per row, NI instances per CTA.
void Recon::spmv(const DevBuf<int> &rp, const DevBuf<GatherW> &e, int nrow, long ncol, const float *xin, float *out,
                 const float *U, int nq, const float *add, double *dot, int k, cudaStream_t s) {
    const unsigned ry = (unsigned)((nrow + kThreads / 32 - 1) / (kThreads / 32));
    const CgScal S = dot ? fscal() : CgScal{};
    const float *dx = dot ? xin : nullptr;
#define MB_SPMV(NI)                                                                                            \
    launch(k_spmv_lr<NI>, dim3((unsigned)((nb + NI - 1) / NI), ry), dim3(kThreads), 0, s, rp.p, e.p, nrow, ncol, \
           xin, out, U, lr_t.p, nq, add, dx, dot, S, k, nb, act())
    if (nb == 1) MB_SPMV(1);
    else if (nb == 2) MB_SPMV(2);
    else if (nb <= 4) MB_SPMV(4);
    else MB_SPMV(8);
#undef MB_SPMV
}

// t[b][q] = V_q' x_b (FP64 partials, fixed-order total)
void Recon::lr_dot(const float *xin, const float *V, int nq, long n, cudaStream_t s) {
    launch(k_lr_dot, dim3(nblocks(n), nb), dim3(kThreads), 0, s, xin, V, nq, n, lr_part.p, lr_t.p, lr_cnt.p, act());
}

// FitR: sum_f wt_f HA_f^T (W0 - W1 W1^T) Hxp_f x   (recon_utils.c:483, fit.cu:190)
// assembled: FR.M x - FR.U (FR.V' x)                 (lib/muv.c:37, solve.cu:36)
void Recon::op_fitR(const float *xin, float *out, cudaStream_t s) {
    if (fit_sparse) {
        if (nfr) lr_dot(xin, frv.p, nfr, nxtot, s);
        spmv(frm_rp, frm_e, (int)nact, nxtot, xin, out, nfr ? fru.p : nullptr, nfr, nullptr, nullptr, 0, s);
        return;
    }
    launch(nps <= 8 ? k_hx<8> : k_hx<16>, dim3(nblk_f, nfit, nb), dim3(kThreads), 0, s, xin, opdf.p, hxp.fwd.p, laytab, nps, nfit, nfx, nfy,
                                                    nxtot, w1v.p, w1_part.p, act());
    launch(k_fit_w, dim3(nblk_f, nfit, nb), dim3(kThreads), 0, s, opdf.p, opdw.p, w0_rp.p, w0_ci.p, w0_v.p, w1v.p,
                                                       fwt.p, w1_part.p, nblk_f, nf, nfit, act());
    launch(k_fit_hxt, dim3(nblk_a, nb), dim3(kThreads), 0, s, opdw.p, nullptr, out, nullptr, fitpad(), dmtab, ndm,
           nfit, nfx, nfy, nact, LowRank{}, fscal(), 0, (const float *)nullptr, act());
}

// FitL: sum_f wt_f HA_f^T (W0 - W1 W1^T) HA_f a + NW NW^T a + actslave a
//       (recon_utils.c:536, fit.cu:213-235)
// assembled: FL.M a - FL.U (FL.V' a)                 (lib/muv.c:37, solve.cu:36)
void Recon::op_fitL(const float *ain, float *out, double *dot_part, cudaStream_t s, int k) {
    if (fit_sparse) {
        if (nfl) lr_dot(ain, flv.p, nfl, nact, s);
        spmv(flm_rp, flm_e, (int)nact, nact, ain, out, nfl ? flu.p : nullptr, nfl, nullptr, dot_part, k, s);
        return;
    }
    LowRank lr{};
    if (nnw) {
        launch(k_lowrank_dot, dim3(nblk_a, nb), dim3(kThreads), 0, s, ain, nwv.p, nw_part.p, nnw, nact, act());
        lr = LowRank{nwv.p, nw_part.p, nnw, nblk_a};
    }
    if (has_slave)
        spmv(as_rp, as_e, (int)nact, nact, ain, fslv.p, nullptr, 0, nullptr, nullptr, 0, s);
    launch(ndm <= 8 ? k_hx<8> : k_hx<16>, dim3(nblk_f, nfit, nb), dim3(kThreads), 0, s, ain, opdf.p, ha.fwd.p, dmtab, ndm, nfit, nfx, nfy,
                                                    nact, w1v.p, w1_part.p, act());
    launch(k_fit_w, dim3(nblk_f, nfit, nb), dim3(kThreads), 0, s, opdf.p, opdw.p, w0_rp.p, w0_ci.p, w0_v.p, w1v.p,
                                                       fwt.p, w1_part.p, nblk_f, nf, nfit, act());
    launch(k_fit_hxt, dim3(nblk_a, nb), dim3(kThreads), 0, s, opdw.p, ain, out, dot_part, fitpad(), dmtab, ndm,
           nfit, nfx, nfy, nact, lr, fscal(), k, has_slave ? (const float *)fslv.p : nullptr, act());
}

// The DM fit of one step: RHS from the tomography solution, then CG warm-
// started from the previous commands (curecon_t::fit, cuda/recon.cu:277).
void Recon::enqueue_fit(cudaStream_t s) {
    op_fitR(x.p, frhs.p, s);
    CgBufs B{fa.p, fr.p, fp.p, fr.p, fAp.p, frhs.p, f_pap.p, f_rr.p, f_rz.p, f_bb.p, fscal()};
    AmulFn A = [&](const float *in, float *out, double *dot, int k) { op_fitL(in, out, dot, s, k); };
    enqueue_cg(B, nact, nblk_a, fit_maxit, A, MmulFn(), s);
}

// CSC (the reference's dsp) -> CSR rows of (column, value) pairs.
static void csc_to_csr(const mb_csc &m, const char *what, std::vector<int> &rp, std::vector<GatherW> &ent) {
    MB_REQUIRE(m.p && m.nrow > 0 && m.ncol > 0, "%s: empty matrix", what);
    const long nnz = m.p[m.ncol];
    MB_REQUIRE(nnz >= 0 && (nnz == 0 || (m.i && m.x)), "%s: missing arrays", what);
    rp.assign((size_t)m.nrow + 1, 0);
    for (int c = 0; c < m.ncol; c++)
        MB_REQUIRE(m.p[c] <= m.p[c + 1], "%s: column pointers decrease at %d", what, c);
    for (long k = 0; k < nnz; k++) {
        MB_REQUIRE(m.i[k] >= 0 && m.i[k] < m.nrow, "%s: row index %d out of range", what, m.i[k]);
        rp[m.i[k] + 1]++;
    }
    for (int r = 0; r < m.nrow; r++) rp[r + 1] += rp[r];
    ent.assign((size_t)nnz, GatherW{0, 0.f});
    std::vector<int> fill(rp.begin(), rp.end() - 1);
    for (int c = 0; c < m.ncol; c++)
        for (int k = m.p[c]; k < m.p[c + 1]; k++) ent[fill[m.i[k]]++] = GatherW{c, (float)m.x[k]};
}

static void upload_f32(DevBuf<float> &d, const double *h, size_t n) {
    std::vector<float> t(n);
    for (size_t i = 0; i < n; i++) t[i] = (float)h[i];
    d.upload(t);
}

// CG state and scratch of the fit (both forms), sized by nact.
void Recon::alloc_fit_state() {
    nblk_a = (int)nblocks(nact);
    nrb_a = (int)((nact + kThreads / 32 - 1) / (kThreads / 32));
    MB_REQUIRE(nrb_a < 65535, "fit: too many actuators (%ld)", nact);
    fnsc = fit_maxit + 3;
    const size_t NA = (size_t)nb * nact;
    fa.alloc(NA); fr.alloc(NA); fp.alloc(NA); fAp.alloc(NA); frhs.alloc(NA);
    // the p.Ap partials of the sparse operator are per 8-row block, of the grid one per 256 actuators
    f_pap.alloc((size_t)nb * std::max(nblk_a, nrb_a)); f_rr.alloc((size_t)nb * nblk_a);
    f_rz.alloc((size_t)nb * nblk_a); f_bb.alloc((size_t)nb * nblk_a);
    fsc.alloc((size_t)nb * fnsc);
    fres.alloc(nb);
    fab.alloc((size_t)nb * 2);
    fcnt.alloc(nb);
    fa.zero_async(stream);
    fsc.zero_async(stream);
    fres.zero_async(stream);
    fab.zero_async(stream);
    fcnt.zero_async(stream);
}

void Recon::build_fit_sparse(const mb_fit_sparse_desc *f) {
    MB_REQUIRE(f->maxit >= 1, "fit_sparse: maxit must be >= 1");
    MB_REQUIRE(f->frm.p && f->flm.p, "fit_sparse: FR.M and FL.M are required");
    MB_REQUIRE(f->frm.ncol == nxtot, "fit_sparse: FR.M has %d columns, the layers %ld points", f->frm.ncol, nxtot);
    MB_REQUIRE(f->flm.nrow == f->frm.nrow && f->flm.ncol == f->frm.nrow,
               "fit_sparse: FL.M must be nact x nact with nact = FR.M rows (%d)", f->frm.nrow);
    MB_REQUIRE(f->nfr >= 0 && f->nfr <= kMaxLr && f->nfl >= 0 && f->nfl <= kMaxLr,
               "fit_sparse: at most %d low-rank columns", kMaxLr);
    MB_REQUIRE((f->nfr == 0 || (f->fru && f->frv)) && (f->nfl == 0 || (f->flu && f->flv)),
               "fit_sparse: low-rank arrays missing");
    has_fit = 1;
    fit_sparse = true;
    nact = f->frm.nrow;
    fit_maxit = f->maxit;
    nfr = f->nfr;
    nfl = f->nfl;
    std::vector<int> rp;
    std::vector<GatherW> ent;
    csc_to_csr(f->frm, "FR.M", rp, ent);
    frm_rp.upload(rp);
    frm_e.upload(ent);
    csc_to_csr(f->flm, "FL.M", rp, ent);
    flm_rp.upload(rp);
    flm_e.upload(ent);
    if (nfr) {
        upload_f32(fru, f->fru, (size_t)nact * nfr);
        upload_f32(frv, f->frv, (size_t)nxtot * nfr);
    }
    if (nfl) {
        upload_f32(flu, f->flu, (size_t)nact * nfl);
        upload_f32(flv, f->flv, (size_t)nact * nfl);
    }
    lr_part.alloc((size_t)nb * kMaxLr * std::max(nblocks(nxtot), nblocks(nact)));
    lr_t.alloc((size_t)nb * kMaxLr);
    lr_cnt.alloc(nb);
    lr_t.zero_async(stream);
    lr_cnt.zero_async(stream);
    alloc_fit_state();
}

void Recon::build_fit(const mb_fit_desc *f) {
    MB_REQUIRE(f->nfit >= 1 && f->ndm >= 1 && f->thetax && f->thetay && f->wt && f->hs && f->amap,
               "fit: missing arrays");
    MB_REQUIRE(f->w0_p && f->w0_i && f->w0_x && f->w1, "fit: W0/W1 missing");
    MB_REQUIRE(f->nnw >= 0 && f->nnw <= 8 && (f->nnw == 0 || f->nw), "fit: 0..8 low-rank columns");
    MB_REQUIRE(f->maxit >= 1, "fit: maxit must be >= 1");
    has_fit = 1;
    nfit = f->nfit;
    ndm = f->ndm;
    nfx = f->floc.nx;
    nfy = f->floc.ny;
    nf = nfx * nfy;
    nnw = f->nnw;
    fit_maxit = f->maxit;
    dmlay_h.resize(ndm);
    long off = 0;
    for (int d = 0; d < ndm; d++) {
        MB_REQUIRE(f->amap[d].nx >= 2 && f->amap[d].ny >= 2 && f->amap[d].dx > 0, "fit: DM %d grid", d);
        dmlay_h[d].nx = f->amap[d].nx;
        dmlay_h[d].ny = f->amap[d].ny;
        dmlay_h[d].off = off;
        dmlay_h[d].l2c = 0.f;
        off += (long)f->amap[d].nx * f->amap[d].ny;
    }
    nact = off;
    dmlay.upload(dmlay_h);
    // the layer grids are needed for Hxp: keep a host copy of the layer grids
    build_ray_tables(f->floc, nfit, nps, xgrid.data(),
                     [&](int d, int t, double &scale, double &dx, double &dy) {
                         const double ht = xgrid[t].ht - f->floc.ht;
                         scale = std::isinf(f->hs[d]) ? 1.0 : 1.0 - ht / f->hs[d];
                         dx = f->thetax[d] * ht;
                         dy = f->thetay[d] * ht;
                     },
                     true, hxp);
    build_ray_tables(f->floc, nfit, ndm, f->amap,
                     [&](int d, int t, double &scale, double &dx, double &dy) {
                         const double ht = f->amap[t].ht - f->floc.ht;
                         scale = std::isinf(f->hs[d]) ? 1.0 : 1.0 - ht / f->hs[d];
                         dx = f->thetax[d] * ht;
                         dy = f->thetay[d] * ht;
                     },
                     true, ha);
    // HA^T as padded per-axis lists over the DM grids
    MB_REQUIRE(ndm <= kMaxLayers, "fit: at most %d DMs", kMaxLayers);
    for (int d = 0; d < ndm; d++) dmtab.l[d] = dmlay_h[d];
    fkx = fky = 1;
    fmaxn = 0;
    for (int d = 0; d < ndm; d++) fmaxn = std::max(fmaxn, std::max(dmlay_h[d].nx, dmlay_h[d].ny));
    for (int w = 0; w < nfit; w++)
        for (int d = 0; d < ndm; d++)
            for (int axis = 0; axis < 2; axis++) {
                const int tb = ha.h_ptr[(w * ndm + d) * 2 + axis];
                const int n = axis ? dmlay_h[d].ny : dmlay_h[d].nx;
                int &K = axis ? fky : fkx;
                for (int j = 0; j < n; j++) K = std::max(K, ha.h_idxptr[tb + j + 1] - ha.h_idxptr[tb + j]);
            }
    MB_REQUIRE(fkx <= kFitPad && fky <= kFitPad, "fit: transposed lists wider than %d (%d, %d)", kFitPad, fkx,
               fky);
    {
        std::vector<GatherW> xq((size_t)nfit * ndm * fmaxn * fkx, GatherW{0, 0.f});
        std::vector<GatherW> yq((size_t)nfit * ndm * fmaxn * fky, GatherW{0, 0.f});
        for (int w = 0; w < nfit; w++)
            for (int d = 0; d < ndm; d++)
                for (int axis = 0; axis < 2; axis++) {
                    const int tb = ha.h_ptr[(w * ndm + d) * 2 + axis];
                    const int n = axis ? dmlay_h[d].ny : dmlay_h[d].nx, K = axis ? fky : fkx;
                    for (int j = 0; j < n; j++) {
                        GatherW *dst = (axis ? yq.data() : xq.data()) + ((size_t)(w * ndm + d) * fmaxn + j) * K;
                        for (int a = ha.h_idxptr[tb + j], e = 0; a < ha.h_idxptr[tb + j + 1]; a++, e++)
                            dst[e] = ha.h_ent[a];
                    }
                }
        fxpad.upload(xq);
        fypad.upload(yq);
    }
    // W0: CSC -> CSR
    std::vector<int> rp(nf + 1, 0), ci;
    std::vector<float> cv;
    const long nnz = f->w0_p[nf];
    for (long k = 0; k < nnz; k++) {
        MB_REQUIRE(f->w0_i[k] >= 0 && f->w0_i[k] < nf, "fit: W0 row out of range");
        rp[f->w0_i[k] + 1]++;
    }
    for (int i = 0; i < nf; i++) rp[i + 1] += rp[i];
    ci.resize(nnz);
    cv.resize(nnz);
    std::vector<int> fill(rp.begin(), rp.end() - 1);
    for (int c = 0; c < nf; c++)
        for (int k = f->w0_p[c]; k < f->w0_p[c + 1]; k++) {
            const int r = f->w0_i[k];
            ci[fill[r]] = c;
            cv[fill[r]++] = (float)f->w0_x[k];
        }
    w0_rp.upload(rp);
    w0_ci.upload(ci);
    w0_v.upload(cv);
    std::vector<float> h1(nf), hw(nfit), hn((size_t)nact * nnw);
    for (int i = 0; i < nf; i++) h1[i] = (float)f->w1[i];
    for (int i = 0; i < nfit; i++) hw[i] = (float)f->wt[i];
    for (size_t i = 0; i < hn.size(); i++) hn[i] = (float)f->nw[i];
    w1v.upload(h1);
    fwt.upload(hw);
    if (nnw) nwv.upload(hn);
    nblk_f = (int)nblocks(nf);
    if (f->actslave.p) {  // cufit_grid::L's slaving term (cuda/fit.cu:232-234)
        MB_REQUIRE(f->actslave.nrow == nact && f->actslave.ncol == nact,
                   "fit: actslave must be %ld x %ld (the DM grids)", nact, nact);
        std::vector<int> rp;
        std::vector<GatherW> ent;
        csc_to_csr(f->actslave, "actslave", rp, ent);
        as_rp.upload(rp);
        as_e.upload(ent);
        has_slave = true;
        fslv.alloc((size_t)nb * nact);
    }
    alloc_fit_state();
    opdf.alloc((size_t)nb * nfit * nf);
    opdw.alloc((size_t)nb * nfit * nf);
    w1_part.alloc((size_t)nb * nfit * nblk_f);
    nw_part.alloc((size_t)nb * std::max(nnw, 1) * nblk_a);
}

// Time each kernel of a CG iteration alone and report its algorithmic
// traffic per launch: every per-instance operand once per instance, and every
// table the instances share (ray-tracing lists, WFS stencils and NEA, the
// FDPCG blocks and their member index) once per launch, since one launch
// reads it for all nb instances.
void Recon::time_stages(int reps, float *ms, double *bytes, int *launches) {
    const int ns = mb_num_stages();
    set_mask(nullptr, stream);
    cudaEvent_t e0, e1;
    MB_CUDA_TRY(cudaEventCreate(&e0));
    MB_CUDA_TRY(cudaEventCreate(&e1));
    const double B = nb, F = 4.0;
    double tab_wfs = 0;  // stencil coefficients, NEA, corner map
    for (int w = 0; w < nwfs; w++) {
        const int n1 = wfs_h[w].pos + 1;
        tab_wfs += nsa[w] * (8.0 * n1 * n1 + 12.0) + 4.0 * np;
    }
    const double nx = (double)nxtot;
    const double trow = (double)nwfs * tw;  // row-buffer floats per instance
    const double nbk = (double)fd_nbh * fd_bs;  // block members (spectrum bins read by k_fd_mul)
    double nh = 0;                              // half-spectrum bins per instance
    for (int l = 0; l < nps; l++) nh += (double)lay_h[l].ny * (lay_h[l].nx / 2 + 1);
    const double by[8] = {
        B * (F * nx + F * trow) + (double)hx.fwd.n * sizeof(AxisW) + tab_wfs + (double)xpad.n * sizeof(GatherW),
        B * (F * trow + 2 * F * nx) + (double)ypad.n * sizeof(GatherW),       // t, p -> Ap
        B * (6 * F * nx),                                                    // x,r,p,Ap read; x,r written
        B * (3 * F * nx),                                                    // p,z read; p written
        B * (6 * F * nx + 8.0 * nh),                          // x,r,p,Ap read; x,r written; spectrum written
        B * (2 * 8.0 * nbk) + 8.0 * fd_bs * fd_bs * fd_nbh + (double)sizeof(FdIndex) * nbk,  // X, Y; M, idx once
        B * (8.0 * nh + (fd_cluster ? 3 : 2) * F * nx),       // spectrum, r read; p read+written (or z written)
        // fused: x, r, p, Ap read, x, r written, r read again, p written; M and the member table once
        B * (9 * F * nx) + 8.0 * fd_bs * fd_bs * fd_nbh + (double)sizeof(FdMem) * nbk};
    // launches per step: with the preconditioner the x/r update of all but
    // the last iteration runs inside k_fd_fwd (timed with it), and with the
    // clustered inverse the p update runs inside k_fd_inv (timed with it)
    const bool pin = precond && fd_cluster;
    const bool fused = precond && fd_mode == 2;
    const int nsep = precond && !fused ? maxit : 0;
    const int lps[8] = {maxit + 2, maxit + 2, precond ? 1 : maxit, (pin || fused) ? 0 : maxit, nsep, nsep, nsep,
                        fused ? maxit : 0};
    const int per = kThreads / std::max(fd_bs, 1);
    for (int st = 0; st < ns; st++) {
        bytes[st] = by[st];
        launches[st] = lps[st];
        ms[st] = 0.f;
        if (st >= 4 && !precond) continue;
        if (st == 7 && !fd_fused_ok) continue;
        // the vectors written here are scratch (z, rhs, spectra): the warm
        // start in x, r and p is left as it was
        auto run_stage = [&]() {
            switch (st) {
                case 0: pupil_rows(true, p.p, stream); break;
                case 1: hxt_rows(p.p, Ap.p, pap_part.p, 1, 0, stream); break;
                case 2:
                    launch(k_cg_update_xr, dim3(nblk_x, nb), dim3(kThreads), 0, stream, z.p, rhs.p, p.p, Ap.p,
                           rr_part.p, nxtot, scal(), 0, maxit, 0, act());
                    break;
                case 3:
                    launch(k_cg_update_p, dim3(nblocks((nxtot + kUpdP - 1) / kUpdP), nb), dim3(kThreads), 0,
                           stream, rhs.p, z.p, nxtot, scal(), 0, act());
                    break;
                case 4:
                    launch(k_fd_fwd, dim3(nps, nb), dim3(kFftThreads), fd_smem, stream, rhs.p, spec.p, fdtab,
                           fd_tw.p, nxtot, fd_bufn, z.p, p.p, Ap.p, ab.p, act());
                    break;
                case 5: fd_mul(stream); break;
                case 7:  // fused: scratch vectors (rhs as r, z as x, Ap, rhs as p)
                    launch_cluster(k_fd_fused, dim3(fused_tab.C, nb), dim3(kFusedThreads), fd_fsmem, stream,
                                   fused_tab.C, rhs.p, fdtab, fused_tab, fd_tw.p, fd_M.p, fd_mem.p, fd_bs, nxtot,
                                   z.p, Ap.p, scal(), 0, 0, act(), z.p);
                    break;
                case 6:
                    if (pin)
                        launch_cluster(k_fd_inv<true>, dim3(nps, nb), dim3(kFftThreads), fd_smem, stream, nps,
                                       spec2.p, r.p, z.p, rz_part.p, fdtab, fd_tw.p, nxtot, fd_bufn, scal(), 0, 0,
                                       act(), rhs.p);
                    else
                        launch(k_fd_inv<false>, dim3(nps, nb), dim3(kFftThreads), fd_smem, stream, spec2.p, r.p,
                               z.p, rz_part.p, fdtab, fd_tw.p, nxtot, fd_bufn, CgScal{}, 0, 0, act(),
                               (float *)nullptr);
                    break;
            }
        };
        run_stage();  // warm
        MB_CUDA_TRY(cudaEventRecord(e0, stream));
        for (int i = 0; i < reps; i++) run_stage();
        MB_CUDA_TRY(cudaEventRecord(e1, stream));
        MB_CUDA_TRY(cudaEventSynchronize(e1));
        float t = 0;
        MB_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
        ms[st] = t / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// Time the tomography operator with each admissible pupil-row blocking and
// keep the fastest (results do not depend on the blocking); the graphs are
// captured again.  ms_out[i]: ms per operator for 4, 8, 16 rows (-1: not
// admissible).  Returns the rows kept.
int Recon::autotune(int reps, float *ms_out) {
    // 4, 8 and 16 rows (reported in ms_out), then every even split of the
    // pupil rows into k blocks (ceil(nyp/k) rows, 1..32: one 30 m instance
    // runs fastest with 2)
    std::vector<int> cand = {4, 8, 16};
    for (int k = 1; k <= nyp; k++) {
        const int r = (nyp + k - 1) / k;
        if (r >= 1 && r <= 32 && std::find(cand.begin(), cand.end(), r) == cand.end()) cand.push_back(r);
    }
    set_mask(nullptr, stream);
    cudaEvent_t e0, e1;
    MB_CUDA_TRY(cudaEventCreate(&e0));
    MB_CUDA_TRY(cudaEventCreate(&e1));
    int best = prows;
    float tbest = 1e30f;
    for (size_t c = 0; c < cand.size(); c++) {
        if (ms_out && c < 3) ms_out[c] = -1.f;
        if ((size_t)pupil_rows_smem_floats(cand[c], nxp, nps, ncols, kx) * sizeof(float) > 200 * 1024) continue;
        set_pupil_rows(cand[c]);
        op_lhs(p.p, Ap.p, nullptr, stream);  // warm
        MB_CUDA_TRY(cudaEventRecord(e0, stream));
        for (int i = 0; i < reps; i++) op_lhs(p.p, Ap.p, nullptr, stream);
        MB_CUDA_TRY(cudaEventRecord(e1, stream));
        MB_CUDA_TRY(cudaEventSynchronize(e1));
        float t = 0;
        MB_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
        t /= reps;
        if (ms_out && c < 3) ms_out[c] = t;
        if (t < tbest) {
            tbest = t;
            best = cand[c];
        }
    }
    set_pupil_rows(best);
    // k_hxt_rows's CTA size: 256, 128 or 64 threads (smaller CTAs spread a
    // small batch over more SMs)
    {
        int bt = hxt_threads;
        float tb = 1e30f;
        for (int th : {256, 128, 64}) {
            hxt_threads = th;
            nblk_hxt = (int)nblocks(nxtot, th);
            op_lhs(p.p, Ap.p, nullptr, stream);  // warm
            MB_CUDA_TRY(cudaEventRecord(e0, stream));
            for (int i = 0; i < reps; i++) op_lhs(p.p, Ap.p, nullptr, stream);
            MB_CUDA_TRY(cudaEventRecord(e1, stream));
            MB_CUDA_TRY(cudaEventSynchronize(e1));
            float t = 0;
            MB_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
            if (t < tb) {
                tb = t;
                bt = th;
            }
        }
        hxt_threads = bt;
        nblk_hxt = (int)nblocks(nxtot, bt);
    }
    capture_graph();
    // the preconditioner's form: three kernels, or one fused cluster kernel,
    // timed as whole tomography steps (graph launches)
    if (precond) {
        // the three-kernel form with 2, 4, 8 or 16 instances per block-solve
        // CTA (the batch shape; shapes above twice the batch are skipped),
        // and the fused form when its cluster fits
        auto time_graph = [&]() {
            MB_CUDA_TRY(cudaGraphLaunch(graph, stream));  // warm
            MB_CUDA_TRY(cudaEventRecord(e0, stream));
            const int nrep = std::max(2, reps / 4);
            for (int i = 0; i < nrep; i++) MB_CUDA_TRY(cudaGraphLaunch(graph, stream));
            MB_CUDA_TRY(cudaEventRecord(e1, stream));
            MB_CUDA_TRY(cudaEventSynchronize(e1));
            float t = 0;
            MB_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
            return t;
        };
        int best_ni = fd_mul_ni, best_mode = 1;
        float tb = 1e30f;
        for (int ni : {2, 4, 8, 16}) {
            if (ni > 2 * nb && ni != 2) continue;
            fd_mul_ni = ni;
            set_fdpcg_mode(1);  // recaptures
            const float t = time_graph();
            if (t < tb) {
                tb = t;
                best_ni = ni;
            }
        }
        fd_mul_ni = best_ni;
        if (fd_fused_ok) {
            set_fdpcg_mode(2);
            if (time_graph() < tb) best_mode = 2;
        }
        set_fdpcg_mode(best_mode);
    }
    // launches with or without programmatic dependent launch, timed as whole
    // steps (graph launches)
    {
        float tp[3] = {0, 0, 0};
        for (int on = 0; on < 3; on++) {
            pdl = on;
            capture_graph();
            cudaGraphExec_t g = has_fit ? graph_step : graph;
            MB_CUDA_TRY(cudaGraphLaunch(g, stream));  // warm
            MB_CUDA_TRY(cudaEventRecord(e0, stream));
            const int nrep = std::max(2, reps / 4);
            for (int i = 0; i < nrep; i++) MB_CUDA_TRY(cudaGraphLaunch(g, stream));
            MB_CUDA_TRY(cudaEventRecord(e1, stream));
            MB_CUDA_TRY(cudaEventSynchronize(e1));
            MB_CUDA_TRY(cudaEventElapsedTime(&tp[on], e0, e1));
        }
        pdl = tp[1] < tp[0] ? (tp[2] < tp[1] ? 2 : 1) : (tp[2] < tp[0] ? 2 : 0);
        capture_graph();
    }
    {
        // the timing steps moved the warm start: start the instances cold again
        x.zero_async(stream);
        if (has_fit) fa.zero_async(stream);
        MB_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// Capture `body` into `exec`: an existing executable graph of the same shape
// (a table update changes kernel arguments, not the launch sequence) is
// updated in place, which costs a fraction of a new instantiation.
static void capture_into(cudaStream_t stream, const std::function<void(cudaStream_t)> &body, long &nkernels,
                         cudaGraphExec_t &exec) {
    cudaGraph_t g = nullptr;
    const long before = g_launches.load();
    MB_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
        body(stream);
    } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    MB_CUDA_TRY(cudaStreamEndCapture(stream, &g));
    nkernels = g_launches.load() - before;
    g_launches -= nkernels;  // captured, not launched
    if (exec) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(exec, g, &info) == cudaSuccess) {
            cudaGraphDestroy(g);
            return;
        }
        (void)cudaGetLastError();  // not updatable: instantiate anew
        cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        exec = nullptr;
        set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e));
        throw CudaError{MB_ECUDA};
    }
}

void Recon::capture(const std::function<void(cudaStream_t)> &body, long &nkernels, cudaGraphExec_t &exec) {
    capture_into(stream, body, nkernels, exec);
}

void Recon::capture_graph() {
    graph_version++;
    PdlScope ps(pdl);
    capture([&](cudaStream_t s) { enqueue_solve(s); }, graph_kernels, graph);
    if (has_fit) {
        capture([&](cudaStream_t s) { enqueue_fit(s); }, graph_fit_kernels, graph_fit);
        capture(
            [&](cudaStream_t s) {
                enqueue_solve(s);
                enqueue_fit(s);
            },
            graph_step_kernels, graph_step);
    }
}

// Queue the upload of a participation mask (null: all instances) on `s`.
void Recon::set_mask(const int *m, cudaStream_t s) {
    if (!m && mask_all) return;
    MB_CUDA_TRY(cudaEventSynchronize(mask_ev));  // the previous upload has left mask_host
    for (int b = 0; b < nb; b++) mask_host[b] = m ? (m[b] != 0) : 1;
    MB_CUDA_TRY(cudaMemcpyAsync(active.p, mask_host, (size_t)nb * sizeof(int), cudaMemcpyHostToDevice, s));
    MB_CUDA_TRY(cudaEventRecord(mask_ev, s));
    mask_all = (m == nullptr);
}

void Recon::run_graph(cudaStream_t s) {
    set_mask(nullptr, s);
    MB_CUDA_TRY(cudaGraphLaunch(graph, s));
    count_launches(graph_kernels);
}

// ---------------------------------------------------------------------------
// ReconGroup: reconstructors of different geometries (uneven instances)
// stepped together in one graph.  The tomography operators -- the RHS and
// every CG iteration's A p (k_pupil_rows: Hx, GP, NEA, GP^T, x half of Hx^T;
// k_hxt_rows: y half of Hx^T, L2, p.Ap and alpha) -- are one launch for all
// members (GroupTab: per-member arguments and block ranges); each member's
// own CG vector updates, preconditioner and DM fit run between them on the
// member's side stream, so those of different members overlap.  Every
// member's arithmetic is that of its own step, so a member's result is the
// same in the group as alone.  Members share the CG iteration count; their
// padded list widths are made equal (the padding adds exact zeros).
// ---------------------------------------------------------------------------
struct ReconGroup {
    std::vector<Recon *> m;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> side;
    cudaEvent_t fork_ev = nullptr;
    std::vector<cudaEvent_t> join_ev;
    cudaGraphExec_t graph = nullptr;
    long graph_kernels = 0;
    std::vector<long> versions;  // members' graph_version at the group's capture
    int device = 0, maxit = 0;
    size_t pupil_smem = 0;
    std::vector<int> order;  // members by decreasing work per grouped launch

    ~ReconGroup() {
        if (graph) cudaGraphExecDestroy(graph);
        for (auto e : join_ev) cudaEventDestroy(e);
        if (fork_ev) cudaEventDestroy(fork_ev);
        for (auto q : side) cudaStreamDestroy(q);
        if (stream) cudaStreamDestroy(stream);
    }
    void fork(cudaStream_t s) {
        MB_CUDA_TRY(cudaEventRecord(fork_ev, s));
        for (auto q : side) MB_CUDA_TRY(cudaStreamWaitEvent(q, fork_ev, 0));
    }
    void join(cudaStream_t s) {
        for (size_t i = 0; i < m.size(); i++) {
            MB_CUDA_TRY(cudaEventRecord(join_ev[i], side[i]));
            MB_CUDA_TRY(cudaStreamWaitEvent(s, join_ev[i], 0));
        }
    }
    // k_pupil_rows of the listed members in as few launches as their
    // subaperture/pupil ratios and layer counts allow (one for the presets)
    void pupil_rows(bool from_x, const std::vector<int> &who, const std::vector<const float *> &xin,
                    cudaStream_t s) {
        struct E {
            PupilArgs a;
            uint3 grid;
            int key;
            size_t smem;
        };
        std::vector<E> es;
        for (int i : who) {
            const Recon &R = *m[i];
            for (int w0 = 0; w0 < R.nwfs;) {
                int w1 = w0 + 1;
                while (w1 < R.nwfs && R.wfs_h[w1].pos == R.wfs_h[w0].pos) w1++;
                es.push_back(E{R.pupil_args(from_x, xin[i], w0),
                               make_uint3((unsigned)R.ptiles, (unsigned)(w1 - w0), (unsigned)R.nb),
                               (R.wfs_h[w0].pos == 2 ? 2 : 0) + (R.nps <= 8 ? 1 : 0), R.pupil_smem});
                w0 = w1;
            }
        }
        for (int key = 0; key < 4; key++) {
            std::vector<const E *> b;
            for (const E &e : es)
                if (e.key == key) b.push_back(&e);
            for (size_t c0 = 0; c0 < b.size(); c0 += kMaxGroup) {
                GroupTab<PupilArgs> g{};
                g.n = (int)std::min(b.size() - c0, (size_t)kMaxGroup);
                g.start[0] = 0;
                for (int e = 0; e < g.n; e++) {
                    const E &x = *b[c0 + e];
                    MB_REQUIRE(x.smem <= pupil_smem, "group: a member's pupil rows need %zu bytes of shared memory",
                               x.smem);
                    g.a[e] = x.a;
                    g.grid[e] = x.grid;
                    g.start[e + 1] = g.start[e] + x.grid.x * x.grid.y * x.grid.z;
                }
                launch(pupil_group_kern(from_x, key & 2, key & 1), dim3(g.start[g.n]), dim3(kThreads), pupil_smem, s,
                       g);
            }
        }
    }
    void hxt_rows(const std::vector<int> &who, const std::vector<const float *> &xin, const std::vector<float *> &out,
                  const std::vector<double *> &dot, int do_l2, int k, cudaStream_t s) {
        int ni = 1;
        for (int i : who) ni = std::max(ni, m[i]->hxt_ni());
        for (int ky = 1; ky <= kMaxPadY; ky++) {
            std::vector<int> b;
            for (int i : who)
                if (m[i]->ky == ky) b.push_back(i);
            for (size_t c0 = 0; c0 < b.size(); c0 += kMaxGroup) {
                GroupTab<HxtArgs> g{};
                g.n = (int)std::min(b.size() - c0, (size_t)kMaxGroup);
                g.start[0] = 0;
                for (int e = 0; e < g.n; e++) {
                    const int i = b[c0 + e];
                    const Recon &R = *m[i];
                    g.a[e] = R.hxt_args(xin[i], out[i], dot[i], do_l2, k);
                    g.grid[e] = make_uint3((unsigned)R.nblk_x, (unsigned)((R.nb + ni - 1) / ni), 1u);
                    g.start[e + 1] = g.start[e] + g.grid[e].x * g.grid[e].y;
                }
                launch(hxt_group_kern(ky, ni), dim3(g.start[g.n]), dim3(kThreads), 0, s, g);
            }
        }
    }
    // A p for every member (TomoL): grouped where the tip/tilt split allows
    void lhs(const std::vector<const float *> &xin, const std::vector<float *> &out, const std::vector<double *> &dot,
             int k, cudaStream_t s) {
        std::vector<int> who;
        for (int i : order) {
            if (m[i]->split) who.push_back(i);
            else m[i]->op_lhs(xin[i], out[i], dot[i], s, k);
        }
        if (who.empty()) return;
        pupil_rows(true, who, xin, s);
        hxt_rows(who, xin, out, dot, 1, k, s);
    }
    void enqueue(cudaStream_t s) {
        const int n = (int)m.size();
        const std::vector<int> &all = order;
        std::vector<const float *> none(n, nullptr), xs(n), ps(n);
        std::vector<float *> rhs(n), Ap(n);
        std::vector<double *> nod(n, nullptr), pap(n);
        for (int i = 0; i < n; i++) {
            xs[i] = m[i]->x.p;
            ps[i] = m[i]->p.p;
            rhs[i] = m[i]->rhs.p;
            Ap[i] = m[i]->Ap.p;
            pap[i] = m[i]->pap_part.p;
        }
        // RHS: gradient weighting per member, then the two operator halves for all
        fork(s);
        for (int i = 0; i < n; i++) m[i]->op_rhs_gp(m[i]->gin.p, side[i]);
        join(s);
        pupil_rows(false, all, none, s);
        hxt_rows(all, none, rhs, nod, 0, 0, s);
        // CG from the warm start, iteration by iteration
        std::vector<Recon::CgRun> run;
        for (int i = 0; i < n; i++) run.push_back(m[i]->solve_run(side[i]));
        std::vector<bool> done(n, false);
        lhs(xs, Ap, nod, 0, s);
        fork(s);
        for (int i = 0; i < n; i++) m[i]->cg_init(run[i], 0, side[i]);
        join(s);
        for (int k = 0; k < maxit; k++) {
            if (k > 0 && k % kCgRestart == 0) {
                lhs(xs, Ap, nod, 0, s);
                fork(s);
                for (int i = 0; i < n; i++) m[i]->cg_init(run[i], k, side[i]);
                join(s);
            }
            lhs(ps, Ap, pap, k, s);
            fork(s);
            for (int i = 0; i < n; i++)
                if (!done[i]) done[i] = m[i]->cg_post(run[i], k, side[i]);
            join(s);
        }
        // DM fits, overlapping
        fork(s);
        for (int i = 0; i < n; i++)
            if (m[i]->has_fit) m[i]->enqueue_fit(side[i]);
        join(s);
    }
    void capture() {
        // the grouped k_pupil_rows runs with the largest member's shared memory,
        // taken now: a member's pupil-row blocking (autotune) may have changed
        pupil_smem = 0;
        for (Recon *r : m) pupil_smem = std::max(pupil_smem, r->pupil_smem);
        for (bool fx : {false, true})
            for (int key = 0; key < 4; key++)
                MB_CUDA_TRY(cudaFuncSetAttribute(pupil_group_kern(fx, key & 2, key & 1),
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pupil_smem));
        capture_into(stream, [&](cudaStream_t s) { enqueue(s); }, graph_kernels, graph);
        versions.clear();
        for (Recon *r : m) versions.push_back(r->graph_version);
    }
    void build() {
        MB_REQUIRE(!m.empty(), "empty group");
        device = m[0]->device;
        maxit = m[0]->maxit;
        int kx = 1, ky = 1;
        for (Recon *r : m) {
            MB_REQUIRE(r->device == device, "members on different devices (%d, %d)", device, r->device);
            MB_REQUIRE(r->maxit == maxit, "members with different CG iteration counts (%d, %d)", maxit, r->maxit);
            kx = std::max(kx, r->kx);
            ky = std::max(ky, r->ky);
        }
        for (size_t i = 0; i < m.size(); i++)
            for (size_t j = 0; j < i; j++) MB_REQUIRE(m[i] != m[j], "a reconstructor appears twice in the group");
        // grouped launches list the member with the most unknowns first, so
        // its blocks (the longest chains) are scheduled first
        order.resize(m.size());
        for (size_t i = 0; i < m.size(); i++) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return (long)m[a]->nb * m[a]->nxtot > (long)m[b]->nb * m[b]->nxtot;
        });
        MB_CUDA_TRY(cudaSetDevice(device));
        // one list width for all members (their own graphs are recaptured)
        for (Recon *r : m)
            if (r->kx != kx || r->ky != ky) {
                const int rows = r->prows;
                r->build_pad(kx, ky);
                r->set_pupil_rows(rows);
                r->capture_graph();
            }
        MB_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        MB_CUDA_TRY(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
        for (size_t i = 0; i < m.size(); i++) {
            cudaStream_t q;
            MB_CUDA_TRY(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
            side.push_back(q);
            cudaEvent_t e;
            MB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            join_ev.push_back(e);
        }
        capture();
    }
    bool stale() const {
        for (size_t i = 0; i < m.size(); i++)
            if (m[i]->graph_version != versions[i]) return true;
        return false;
    }
};

}  // namespace mb

// ===========================================================================
// C ABI
// ===========================================================================
struct mb_recon {
    mb::Recon R;
};

using mb::CudaError;
using mb::InvalidArg;

#define MB_API_BEGIN try {
#define MB_API_END                                   \
    }                                                \
    catch (const CudaError &e) { return e.code; }    \
    catch (const InvalidArg &e) { return e.code; }   \
    catch (const std::bad_alloc &) {                 \
        mb::set_error("host allocation failed");     \
        return MB_ENOMEM;                            \
    }                                                \
    catch (...) {                                    \
        mb::set_error("unexpected C++ exception");   \
        return MB_ECUDA;                             \
    }                                                \
    return MB_OK;

extern "C" {

int mb_version(void) { return 1; }

const char *mb_error_string(int code) {
    switch (code) {
        case MB_OK: return "ok";
        case MB_EINVAL: return "invalid argument";
        case MB_ECUDA: return "CUDA error";
        case MB_ENOMEM: return "out of device memory";
        case MB_ESTATE: return "invalid state";
        case MB_EUNSUP: return "unsupported geometry";
        case MB_ENUM: return "numerical failure";
        default: return "unknown error";
    }
}
const char *mb_last_error_message(void) { return mb::last_error(); }

long mb_kernel_launches(int reset) {
    long v = mb::g_launches.load();
    if (reset) mb::g_launches = 0;
    return v;
}

int mb_init(int device) {
    MB_API_BEGIN
    int n = 0;
    MB_CUDA_TRY(cudaGetDeviceCount(&n));
    MB_REQUIRE(device >= 0 && device < n, "device %d out of range (%d devices)", device, n);
    MB_CUDA_TRY(cudaSetDevice(device));
    MB_API_END
}

void mb_cleanup(void) {}

int mb_setup_recon(const mb_recon_desc *desc, mb_recon **out) {
    if (!out) {
        mb::set_error("out is NULL");
        return MB_EINVAL;
    }
    *out = nullptr;
    mb_recon *h = new (std::nothrow) mb_recon();
    if (!h) return MB_ENOMEM;
    try {
        h->R.build(desc);
    } catch (const CudaError &e) {
        delete h;
        return e.code;
    } catch (const InvalidArg &e) {
        delete h;
        return e.code;
    } catch (...) {
        delete h;
        mb::set_error("unexpected exception in setup");
        return MB_ECUDA;
    }
    *out = h;
    return MB_OK;
}

void mb_recon_free(mb_recon *r) { delete r; }

long mb_ngrad(const mb_recon *r) { return r ? r->R.ngrad : -1; }
long mb_nxtot(const mb_recon *r) { return r ? r->R.nxtot : -1; }
int mb_nbatch(const mb_recon *r) { return r ? r->R.nb : -1; }

int mb_recon_reset(mb_recon *h) {
    MB_API_BEGIN
    MB_REQUIRE(h, "null handle");
    h->R.x.zero_async(h->R.stream);
    if (h->R.has_fit) h->R.fa.zero_async(h->R.stream);
    MB_CUDA_TRY(cudaStreamSynchronize(h->R.stream));
    MB_API_END
}

int mb_update_recon_nea(mb_recon *h, int iwfs, const double *neai, const double *ptt) {
    MB_API_BEGIN
    MB_REQUIRE(h && neai && iwfs >= 0 && iwfs < h->R.nwfs, "invalid arguments");
    MB_CUDA_TRY(cudaStreamSynchronize(h->R.stream));
    h->R.set_neai(iwfs, neai, ptt);
    h->R.wfs.upload(h->R.wfs_h);
    for (int w = 0; w < h->R.nwfs; w++) h->R.wfstab.w[w] = h->R.wfs_h[w];
    h->R.capture_graph();
    MB_API_END
}

int mb_update_recon_neam(mb_recon *h, const double *neam) {
    MB_API_BEGIN
    MB_REQUIRE(h && neam, "invalid arguments");
    mb::Recon &R = h->R;
    if (!R.precond || !R.fd_geom || !R.fd_dev) {
        mb::set_error("mb_update_recon_neam: no FDPCG data-term geometry (mb_fdpcg_desc.geom, .mdiag) at setup");
        return MB_EINVAL;
    }
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    R.form_fdpcg_data(neam);
    R.rebuild_fdpcg_device();
    MB_API_END
}

int mb_fdpcg_data(mb_recon *h, double *out) {
    MB_API_BEGIN
    MB_REQUIRE(h && out, "invalid arguments");
    mb::Recon &R = h->R;
    if (!R.precond || !R.fd_dev) {
        mb::set_error("mb_fdpcg_data: no FDPCG data term on the device");
        return MB_EINVAL;
    }
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    MB_CUDA_TRY(cudaMemcpy(out, R.fd_mdata.p, R.fd_mdata.n * sizeof(double2), cudaMemcpyDeviceToHost));
    MB_API_END
}

int mb_update_recon_cn2(mb_recon *h, const double *l2c, const mb_fdpcg_desc *fd) {
    MB_API_BEGIN
    MB_REQUIRE(h && l2c, "invalid arguments");
    MB_CUDA_TRY(cudaStreamSynchronize(h->R.stream));
    h->R.set_l2c(l2c);
    if (h->R.precond) {
        if (fd) h->R.build_fdpcg(fd);
        else h->R.rebuild_fdpcg_device();  // new invpsd from the stored data term, on the GPU
    }
    h->R.capture_graph();
    MB_API_END
}

static void to_float_dev(float *d, const double *hsrc, size_t n, cudaStream_t s) {
    std::vector<float> tmp(n);
    for (size_t i = 0; i < n; i++) tmp[i] = (float)hsrc[i];
    MB_CUDA_TRY(cudaMemcpyAsync(d, tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice, s));
    MB_CUDA_TRY(cudaStreamSynchronize(s));
}
static void from_float_dev(double *hdst, const float *d, size_t n, cudaStream_t s) {
    std::vector<float> tmp(n);
    MB_CUDA_TRY(cudaMemcpyAsync(tmp.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    MB_CUDA_TRY(cudaStreamSynchronize(s));
    for (size_t i = 0; i < n; i++) hdst[i] = tmp[i];
}

int mb_tomo(mb_recon *h, const double *grad, double *opdr, float *cgres) {
    MB_API_BEGIN
    MB_REQUIRE(h && grad, "invalid arguments");
    mb::Recon &R = h->R;
    const size_t ng = (size_t)R.nb * R.ngrad;
    for (size_t i = 0; i < ng; i++)
        if (!std::isfinite(grad[i])) {
            mb::set_error("gradient %zu is not finite", i);
            return MB_ENUM;
        }
    to_float_dev(R.gin.p, grad, ng, R.stream);
    R.run_graph(R.stream);
    if (opdr) from_float_dev(opdr, R.x.p, (size_t)R.nb * R.nxtot, R.stream);
    if (cgres) MB_CUDA_TRY(cudaMemcpyAsync(cgres, R.res.p, R.nb * sizeof(float), cudaMemcpyDeviceToHost, R.stream));
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    MB_API_END
}

int mb_tomo_device(mb_recon *h, const float *d_grad, void *stream) {
    MB_API_BEGIN
    MB_REQUIRE(h && d_grad, "invalid arguments");
    mb::Recon &R = h->R;
    cudaStream_t s = (cudaStream_t)stream;
    MB_CUDA_TRY(cudaMemcpyAsync(R.gin.p, d_grad, (size_t)R.nb * R.ngrad * sizeof(float),
                                cudaMemcpyDeviceToDevice, s));
    R.run_graph(s);
    MB_API_END
}

const float *mb_tomo_solution(mb_recon *h) { return h ? h->R.x.p : nullptr; }
const float *mb_fit_solution(mb_recon *h) { return h && h->R.has_fit ? h->R.fa.p : nullptr; }
long mb_nact(const mb_recon *h) { return h && h->R.has_fit ? h->R.nact : 0; }

int mb_fit(mb_recon *h, double *dmout, float *cgres) {
    MB_API_BEGIN
    MB_REQUIRE(h, "null handle");
    mb::Recon &R = h->R;
    if (!R.has_fit) {
        mb::set_error("reconstructor was set up without a DM fit");
        return MB_ESTATE;
    }
    R.set_mask(nullptr, R.stream);
    MB_CUDA_TRY(cudaGraphLaunch(R.graph_fit, R.stream));
    mb::count_launches(R.graph_fit_kernels);
    if (dmout) from_float_dev(dmout, R.fa.p, (size_t)R.nb * R.nact, R.stream);
    if (cgres) MB_CUDA_TRY(cudaMemcpyAsync(cgres, R.fres.p, R.nb * sizeof(float), cudaMemcpyDeviceToHost, R.stream));
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    MB_API_END
}

int mb_tomo_wfs(mb_recon *h, const double *const *grad, double *const *opdr, float *cgres) {
    MB_API_BEGIN
    MB_REQUIRE(h && grad, "invalid arguments");
    mb::Recon &R = h->R;
    MB_REQUIRE(R.nb == 1, "mb_tomo_wfs serves one instance (nbatch %d)", R.nb);
    float *st = R.stage((size_t)std::max(R.ngrad, R.nxtot));
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));  // the staging buffer is free
    for (int w = 0; w < R.nwfs; w++) {
        const long n = R.goff[w + 1] - R.goff[w];
        float *d = st + R.goff[w];
        if (!grad[w]) {
            std::fill(d, d + n, 0.f);
            continue;
        }
        for (long i = 0; i < n; i++) {
            if (!std::isfinite(grad[w][i])) {
                mb::set_error("gradient %ld of WFS %d is not finite", i, w);
                return MB_ENUM;
            }
            d[i] = (float)grad[w][i];
        }
    }
    MB_CUDA_TRY(cudaMemcpyAsync(R.gin.p, st, (size_t)R.ngrad * sizeof(float), cudaMemcpyHostToDevice, R.stream));
    R.run_graph(R.stream);
    if (opdr) MB_CUDA_TRY(cudaMemcpyAsync(st, R.x.p, (size_t)R.nxtot * sizeof(float), cudaMemcpyDeviceToHost, R.stream));
    if (cgres) MB_CUDA_TRY(cudaMemcpyAsync(cgres, R.res.p, sizeof(float), cudaMemcpyDeviceToHost, R.stream));
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    if (opdr)
        for (int l = 0; l < R.nps; l++)
            if (opdr[l])
                for (long i = R.xoff[l]; i < R.xoff[l + 1]; i++) opdr[l][i - R.xoff[l]] = st[i];
    MB_API_END
}

int mb_fit_opdr(mb_recon *h, const double *const *opdr, double *dmout, float *cgres) {
    MB_API_BEGIN
    MB_REQUIRE(h && opdr, "invalid arguments");
    mb::Recon &R = h->R;
    if (!R.has_fit) {
        mb::set_error("reconstructor was set up without a DM fit");
        return MB_ESTATE;
    }
    MB_REQUIRE(R.nb == 1, "mb_fit_opdr serves one instance (nbatch %d)", R.nb);
    float *st = R.stage((size_t)std::max<long>(R.nxtot, R.nact));
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    for (int l = 0; l < R.nps; l++)
        for (long i = R.xoff[l]; i < R.xoff[l + 1]; i++) st[i] = opdr[l] ? (float)opdr[l][i - R.xoff[l]] : 0.f;
    MB_CUDA_TRY(cudaMemcpyAsync(R.x.p, st, (size_t)R.nxtot * sizeof(float), cudaMemcpyHostToDevice, R.stream));
    R.set_mask(nullptr, R.stream);
    MB_CUDA_TRY(cudaGraphLaunch(R.graph_fit, R.stream));
    mb::count_launches(R.graph_fit_kernels);
    if (dmout) MB_CUDA_TRY(cudaMemcpyAsync(st, R.fa.p, (size_t)R.nact * sizeof(float), cudaMemcpyDeviceToHost, R.stream));
    if (cgres) MB_CUDA_TRY(cudaMemcpyAsync(cgres, R.fres.p, sizeof(float), cudaMemcpyDeviceToHost, R.stream));
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    if (dmout)
        for (long i = 0; i < R.nact; i++) dmout[i] = st[i];
    MB_API_END
}

int mb_recon_step_device(mb_recon *h, const float *d_grad, void *stream) {
    MB_API_BEGIN
    MB_REQUIRE(h && d_grad, "invalid arguments");
    mb::Recon &R = h->R;
    if (!R.has_fit) {
        mb::set_error("reconstructor was set up without a DM fit");
        return MB_ESTATE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MB_CUDA_TRY(cudaMemcpyAsync(R.gin.p, d_grad, (size_t)R.nb * R.ngrad * sizeof(float),
                                cudaMemcpyDeviceToDevice, s));
    R.set_mask(nullptr, s);
    MB_CUDA_TRY(cudaGraphLaunch(R.graph_step, s));
    mb::count_launches(R.graph_step_kernels);
    MB_API_END
}

struct mb_group {
    mb::ReconGroup G;
};

int mb_group_create(mb_recon *const *members, int n, mb_group **out) {
    if (!out) {
        mb::set_error("out is NULL");
        return MB_EINVAL;
    }
    *out = nullptr;
    MB_API_BEGIN
    MB_REQUIRE(members && n >= 1, "no members");
    auto *g = new mb_group();
    try {
        for (int i = 0; i < n; i++) {
            MB_REQUIRE(members[i], "member %d is NULL", i);
            g->G.m.push_back(&members[i]->R);
        }
        g->G.build();
    } catch (...) {
        delete g;
        throw;
    }
    *out = g;
    MB_API_END
}

int mb_group_step_device(mb_group *g, const float *const *d_grad, void *stream) {
    MB_API_BEGIN
    MB_REQUIRE(g && d_grad, "invalid arguments");
    mb::ReconGroup &G = g->G;
    for (size_t i = 0; i < G.m.size(); i++) {
        MB_REQUIRE(d_grad[i], "gradients of member %zu are NULL", i);
        MB_REQUIRE(G.m[i]->has_fit, "member %zu was set up without a DM fit", i);
    }
    if (G.stale()) G.capture();  // a member's tables changed (update, autotune)
    cudaStream_t s = (cudaStream_t)stream;
    for (size_t i = 0; i < G.m.size(); i++) {
        mb::Recon &R = *G.m[i];
        MB_CUDA_TRY(cudaMemcpyAsync(R.gin.p, d_grad[i], (size_t)R.nb * R.ngrad * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s));
        R.set_mask(nullptr, s);
    }
    MB_CUDA_TRY(cudaGraphLaunch(G.graph, s));
    mb::count_launches(G.graph_kernels);
    MB_API_END
}

long mb_group_graph_kernels(const mb_group *g) { return g ? g->G.graph_kernels : -1; }

void mb_group_free(mb_group *g) { delete g; }

int mb_apply_fit_R(mb_recon *h, const double *xin, double *aout) {
    MB_API_BEGIN
    MB_REQUIRE(h && xin && aout && h->R.has_fit, "invalid arguments or no fit");
    mb::Recon &R = h->R;
    R.set_mask(nullptr, R.stream);
    to_float_dev(R.z.p, xin, (size_t)R.nb * R.nxtot, R.stream);
    R.op_fitR(R.z.p, R.frhs.p, R.stream);
    from_float_dev(aout, R.frhs.p, (size_t)R.nb * R.nact, R.stream);
    MB_API_END
}

int mb_apply_fit_L(mb_recon *h, const double *ain, double *aout) {
    MB_API_BEGIN
    MB_REQUIRE(h && ain && aout && h->R.has_fit, "invalid arguments or no fit");
    mb::Recon &R = h->R;
    R.set_mask(nullptr, R.stream);
    to_float_dev(R.fp.p, ain, (size_t)R.nb * R.nact, R.stream);
    R.op_fitL(R.fp.p, R.fAp.p, nullptr, R.stream);
    from_float_dev(aout, R.fAp.p, (size_t)R.nb * R.nact, R.stream);
    MB_API_END
}

void *mb_recon_stream(mb_recon *h) { return h ? (void *)h->R.stream : nullptr; }

static const char *kStageNames[] = {"lhs_pupil", "lhs_layer", "cg_update_xr", "cg_update_p",
                                    "fd_fwd",    "fd_mul",    "fd_inv",       "fd_fused"};
int mb_num_stages(void) { return (int)(sizeof(kStageNames) / sizeof(kStageNames[0])); }
const char *mb_stage_name(int i) { return (i >= 0 && i < mb_num_stages()) ? kStageNames[i] : ""; }

int mb_time_stages(mb_recon *h, int reps, float *ms, double *bytes, int *launches) {
    MB_API_BEGIN
    MB_REQUIRE(h && ms && bytes && launches && reps > 0, "invalid arguments");
    h->R.time_stages(reps, ms, bytes, launches);
    MB_API_END
}

int mb_fdpcg_mode(mb_recon *h, int mode) {
    MB_API_BEGIN
    MB_REQUIRE(h && mode >= -1 && mode <= 2, "invalid arguments");
    mb::Recon &R = h->R;
    MB_REQUIRE(R.precond, "reconstructor has no FDPCG preconditioner");
    if (mode < 0) return R.fd_mode;
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    R.set_fdpcg_mode(mode);
    return R.fd_mode;
    MB_API_END
}

int mb_fdpcg_shape(mb_recon *h, int ni) {
    MB_API_BEGIN
    MB_REQUIRE(h && (ni == -1 || ni == 2 || ni == 4 || ni == 8 || ni == 16), "invalid arguments");
    mb::Recon &R = h->R;
    MB_REQUIRE(R.precond, "reconstructor has no FDPCG preconditioner");
    if (ni < 0) return R.fd_mul_ni;
    MB_CUDA_TRY(cudaStreamSynchronize(R.stream));
    R.fd_mul_ni = ni;
    if (R.graph) R.capture_graph();
    return R.fd_mul_ni;
    MB_API_END
}

int mb_autotune(mb_recon *h, int reps, int *rows, float *ms) {
    MB_API_BEGIN
    MB_REQUIRE(h && reps > 0, "invalid arguments");
    MB_CUDA_TRY(cudaStreamSynchronize(h->R.stream));
    const int r = h->R.autotune(reps, ms);
    if (rows) *rows = r;
    MB_API_END
}

int mb_tomo_residual(mb_recon *h, float *cgres) {
    MB_API_BEGIN
    MB_REQUIRE(h && cgres, "invalid arguments");
    MB_CUDA_TRY(cudaMemcpyAsync(cgres, h->R.res.p, h->R.nb * sizeof(float), cudaMemcpyDeviceToHost,
                                h->R.stream));
    MB_CUDA_TRY(cudaStreamSynchronize(h->R.stream));
    MB_API_END
}

int mb_apply_tomo_R(mb_recon *h, const double *grad, double *xout) {
    MB_API_BEGIN
    MB_REQUIRE(h && grad && xout, "invalid arguments");
    mb::Recon &R = h->R;
    R.set_mask(nullptr, R.stream);
    to_float_dev(R.gin.p, grad, (size_t)R.nb * R.ngrad, R.stream);
    R.op_rhs(R.gin.p, R.rhs.p, R.stream);
    from_float_dev(xout, R.rhs.p, (size_t)R.nb * R.nxtot, R.stream);
    MB_API_END
}

int mb_apply_tomo_L(mb_recon *h, const double *xin, double *xout) {
    MB_API_BEGIN
    MB_REQUIRE(h && xin && xout, "invalid arguments");
    mb::Recon &R = h->R;
    R.set_mask(nullptr, R.stream);
    to_float_dev(R.z.p, xin, (size_t)R.nb * R.nxtot, R.stream);
    R.op_lhs(R.z.p, R.Ap.p, nullptr, R.stream);
    from_float_dev(xout, R.Ap.p, (size_t)R.nb * R.nxtot, R.stream);
    MB_API_END
}

int mb_apply_fdpcg(mb_recon *h, const double *xin, double *xout) {
    MB_API_BEGIN
    MB_REQUIRE(h && xin && xout, "invalid arguments");
    mb::Recon &R = h->R;
    R.set_mask(nullptr, R.stream);
    if (!R.precond) {
        mb::set_error("reconstructor has no FDPCG preconditioner");
        return MB_ESTATE;
    }
    to_float_dev(R.Ap.p, xin, (size_t)R.nb * R.nxtot, R.stream);
    R.op_fdpcg(R.Ap.p, R.z.p, R.rz_part.p, R.stream);
    from_float_dev(xout, R.z.p, (size_t)R.nb * R.nxtot, R.stream);
    MB_API_END
}

// ---------------------------------------------------------------------------
// Serving: per-slot state and masked steps
// ---------------------------------------------------------------------------
static void check_slot(const mb_recon *h, int slot) {
    MB_REQUIRE(h, "null handle");
    MB_REQUIRE(slot >= 0 && slot < h->R.nb, "slot %d out of range (%d slots)", slot, h->R.nb);
}

int mb_recon_reset_slot(mb_recon *h, int slot, void *stream) {
    MB_API_BEGIN
    check_slot(h, slot);
    mb::Recon &R = h->R;
    cudaStream_t s = (cudaStream_t)stream;
    MB_CUDA_TRY(cudaMemsetAsync(R.x.p + (size_t)slot * R.nxtot, 0, R.nxtot * sizeof(float), s));
    if (R.has_fit) MB_CUDA_TRY(cudaMemsetAsync(R.fa.p + (size_t)slot * R.nact, 0, R.nact * sizeof(float), s));
    MB_API_END
}

int mb_slot_upload(mb_recon *h, int slot, const float *grad, void *stream) {
    MB_API_BEGIN
    check_slot(h, slot);
    MB_REQUIRE(grad, "null gradients");
    mb::Recon &R = h->R;
    MB_CUDA_TRY(cudaMemcpyAsync(R.gin.p + (size_t)slot * R.ngrad, grad, R.ngrad * sizeof(float),
                                cudaMemcpyDefault, (cudaStream_t)stream));
    MB_API_END
}

int mb_slot_download(mb_recon *h, int slot, float *out, void *stream) {
    MB_API_BEGIN
    check_slot(h, slot);
    MB_REQUIRE(out, "null output");
    mb::Recon &R = h->R;
    const float *src = R.has_fit ? R.fa.p + (size_t)slot * R.nact : R.x.p + (size_t)slot * R.nxtot;
    const size_t n = R.has_fit ? (size_t)R.nact : (size_t)R.nxtot;
    MB_CUDA_TRY(cudaMemcpyAsync(out, src, n * sizeof(float), cudaMemcpyDefault, (cudaStream_t)stream));
    MB_API_END
}

int mb_recon_step_slots(mb_recon *h, const int *active, void *stream) {
    MB_API_BEGIN
    MB_REQUIRE(h && active, "invalid arguments");
    mb::Recon &R = h->R;
    cudaStream_t s = (cudaStream_t)stream;
    R.set_mask(active, s);
    if (R.has_fit) {
        MB_CUDA_TRY(cudaGraphLaunch(R.graph_step, s));
        mb::count_launches(R.graph_step_kernels);
    } else {
        MB_CUDA_TRY(cudaGraphLaunch(R.graph, s));
        mb::count_launches(R.graph_kernels);
    }
    MB_API_END
}

int mb_recon_serve_step(mb_recon *h, const int *active, const float *grad, float *out, void *stream) {
    MB_API_BEGIN
    MB_REQUIRE(h && active && grad && out, "invalid arguments");
    mb::Recon &R = h->R;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nout = R.has_fit ? (size_t)R.nact : (size_t)R.nxtot;
    float *res = R.has_fit ? R.fa.p : R.x.p;
    // one copy per run of consecutive active slots, each way
    auto runs = [&](const std::function<void(int, int)> &f) {
        for (int b = 0; b < R.nb;) {
            if (!active[b]) {
                b++;
                continue;
            }
            int e = b;
            while (e < R.nb && active[e]) e++;
            f(b, e - b);
            b = e;
        }
    };
    runs([&](int b, int n) {
        MB_CUDA_TRY(cudaMemcpyAsync(R.gin.p + (size_t)b * R.ngrad, grad + (size_t)b * R.ngrad,
                                    (size_t)n * R.ngrad * sizeof(float), cudaMemcpyDefault, s));
    });
    R.set_mask(active, s);
    if (R.has_fit) {
        MB_CUDA_TRY(cudaGraphLaunch(R.graph_step, s));
        mb::count_launches(R.graph_step_kernels);
    } else {
        MB_CUDA_TRY(cudaGraphLaunch(R.graph, s));
        mb::count_launches(R.graph_kernels);
    }
    runs([&](int b, int n) {
        MB_CUDA_TRY(cudaMemcpyAsync(out + (size_t)b * nout, res + (size_t)b * nout, (size_t)n * nout * sizeof(float),
                                    cudaMemcpyDefault, s));
    });
    MB_API_END
}

int mb_apply_hx(mb_recon *h, const double *xin, double *opd) {
    MB_API_BEGIN
    MB_REQUIRE(h && xin && opd, "invalid arguments");
    mb::Recon &R = h->R;
    R.set_mask(nullptr, R.stream);
    to_float_dev(R.z.p, xin, (size_t)R.nb * R.nxtot, R.stream);
    R.op_hx(R.z.p, R.stream);
    from_float_dev(opd, R.opd.p, (size_t)R.nb * R.nwfs * R.np, R.stream);
    MB_API_END
}

}  // extern "C"
