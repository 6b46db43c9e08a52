/*
 * maos_gpu_glue.c -- the reconstruction entry points maos calls through
 * cuda/gpu.h, implemented on top of the maos_b200 C ABI (include/maos_b200.h).
 *
 * A maintainer adds this file to maos in place of cuda/recon.cu (and the
 * gpu_init / gpu_cleanup of cuda/cudata.cu) and links libmaosb200.so; maos's
 * own callers (maos/maos.c:127,163, maos/recon.c:79,89,295, maos/sim.c:84,211,
 * maos/setup_recon.c:751, maos/setup_recon_mvm.c:243, maos/sim_utils.c:1409)
 * stay as they are.  The file copies fields out of PARMS_T / RECON_T /
 * POWFS_T / SIM_T, which only maos knows, into the flat descriptors; the
 * library never sees maos types.
 *
 *   gpu_init              cuda/cudata.cu:144     mb_init
 *   gpu_cleanup           cuda/cudata.cu         mb_recon_free, mb_mvm_free
 *   gpu_setup_recon       cuda/recon.cu:477      mb_setup_recon
 *   gpu_setup_recon_mvm   cuda/recon.cu:489      mb_mvm_create (recon->MVM)
 *   gpu_update_recon      cuda/recon.cu:510      mb_update_recon_nea + FDPCG tables
 *   gpu_update_recon_cn2  cuda/recon.cu:522      mb_update_recon_cn2
 *   gpu_recon_reset       cuda/recon.cu:534      mb_recon_reset
 *   gpu_recon_free        cuda/gpu.h:54          mb_recon_free
 *   gpu_tomo              cuda/recon.cu:564      mb_tomo_wfs (+ simu->opdr, gngsmvst)
 *   gpu_fit               cuda/recon.cu:584      mb_fit / mb_fit_opdr
 *   gpu_recon_mvm         cuda/recon.cu:598      mb_recon_mvm
 *
 * DM fit: gpu.fit=1 (the maos default) hands recon->fit->FR and FL (the
 * assembled sparse plus low-rank matrices, any aloc) to the library;
 * gpu.fit=2 hands the grid form (fmap, W0/W1, amap, NW, actslave).
 * Errors: maos aborts on a GPU error (cuda/common.h:103); so does this file,
 * through maos's error(), with the library's message.
 */
#include "maos/common.h"
#include "lib/laplacian.h"
#include "maos_b200.h"

static mb_recon *g_recon = NULL;
static mb_mvm *g_mvm = NULL;
static int g_device = 0;

#define MB_CHECK(call)                                                         \
    do {                                                                       \
        int rc_ = (call);                                                      \
        if (rc_ != MB_OK) error("%s: %s\n", #call, mb_last_error_message()); \
    } while (0)

static mb_grid grid_of(const map_t *m) {
    mb_grid g;
    g.nx = (int)m->nx;
    g.ny = (int)m->ny;
    g.dx = m->dx;
    g.dy = m->dy;
    g.ox = m->ox;
    g.oy = m->oy;
    g.ht = m->h;
    return g;
}

/* Host arrays the descriptors point into, released after the setup call. */
typedef struct {
    void **p;
    int n, cap;
} keep_t;
static void *keep(keep_t *k, void *ptr) {
    if (k->n == k->cap) {
        k->cap = k->cap ? 2 * k->cap : 64;
        k->p = realloc(k->p, sizeof(void *) * k->cap);
    }
    k->p[k->n++] = ptr;
    return ptr;
}
static void keep_free(keep_t *k) {
    for (int i = 0; i < k->n; i++) free(k->p[i]);
    free(k->p);
    k->p = NULL;
    k->n = k->cap = 0;
}

/* A dsp (spint may be 32 or 64 bit) as the ABI's int CSC. */
static mb_csc csc_of(const dsp *A, keep_t *k) {
    mb_csc c = {0};
    if (!A) return c;
    const long nnz = A->p[A->ny];
    int *p = keep(k, malloc(sizeof(int) * (A->ny + 1)));
    int *i = keep(k, malloc(sizeof(int) * (nnz > 0 ? nnz : 1)));
    for (long j = 0; j <= A->ny; j++) p[j] = (int)A->p[j];
    for (long j = 0; j < nnz; j++) i[j] = (int)A->i[j];
    c.nrow = (int)A->nx;
    c.ncol = (int)A->ny;
    c.p = p;
    c.i = i;
    c.x = A->x;
    return c;
}

/* The biharmonic weight of each layer as cuda/tomo.cu:159-163 forms it. */
static void layer_l2c(const PARMS_T *parms, const RECON_T *recon, double *l2c) {
    for (int ips = 0; ips < recon->npsr; ips++) {
        const double c = laplacian_coef(recon->r0, recon->wt->p[ips], recon->xmap->p[ips]->dx) * 0.25;
        l2c[ips] = c * c * parms->tomo.cxxscale * TOMOSCALE;
    }
}

/* The inverse NEA of one WFS as [cx, cy, cxy] per subaperture: the diagonal
 * block of recon->saneai, read as cuda/tomo.cu:111 convert_neai reads it. */
static double *neai_of(const RECON_T *recon, int iwfs, int nwfs, keep_t *k) {
    const dsp *nea = recon->saneai->p[iwfs + iwfs * nwfs];
    const long nsa = nea->ny / 2;
    double *out = keep(k, calloc(3 * nsa, sizeof(double)));
    for (long ic = 0; ic < nea->ny; ic++) {
        const long isa = ic < nsa ? ic : ic - nsa;
        for (long j = nea->p[ic]; j < nea->p[ic + 1]; j++) {
            const long ir = nea->i[j];
            if (ir == ic) out[3 * isa + (ic == isa ? 0 : 1)] = nea->x[j];
            else if (ir == ic - nsa || ir == ic + nsa) out[3 * isa + 2] = nea->x[j];
            else error("saneai of WFS %d has an entry off the 2x2 blocks\n", iwfs);
        }
    }
    return out;
}

/* recon->fdpcg as the ABI's descriptor: the ccell of bs x bs blocks is
 * contiguous complex doubles, i.e. interleaved (re, im) pairs. */
static mb_fdpcg_desc fdpcg_of(const RECON_T *recon, keep_t *k) {
    mb_fdpcg_desc fd = {0};
    const FDPCG_T *f = recon->fdpcg;
    const long nb = f->Mbinv->nx, bs = f->bs;
    double *mb = keep(k, malloc(sizeof(double) * 2 * nb * bs * bs));
    for (long ib = 0; ib < nb; ib++)
        memcpy(mb + 2 * ib * bs * bs, f->Mbinv->p[ib]->p, sizeof(double) * 2 * bs * bs);
    fd.nb = (int)nb;
    fd.bs = (int)bs;
    fd.scale = f->scale;
    fd.perm = f->perm->p;
    fd.mbinv = mb;
    return fd;
}

/* A dcell stacked into one column-major matrix (rows of all cells). */
static double *stack_rows(const dcell *c, long *nrow, long *ncol, keep_t *k) {
    dmat *m = dcell2m((dcell *)c);
    double *out = keep(k, malloc(sizeof(double) * (m->nx * m->ny > 0 ? m->nx * m->ny : 1)));
    memcpy(out, m->p, sizeof(double) * m->nx * m->ny);
    *nrow = m->nx;
    *ncol = m->ny;
    dfree(m);
    return out;
}

int gpu_init(const PARMS_T *parms, int *gpus, int ngpu) {
    (void)parms;
    g_device = 0;
    if (gpus && ngpu > 0) {
        if (gpus[0] < 0) return 0; /* CUDA disabled by the user (cuda/cudata.cu:150-156) */
        g_device = gpus[0];
    }
    return mb_init(g_device) == MB_OK;
}

void gpu_recon_free(void) {
    if (g_recon) mb_recon_free(g_recon);
    g_recon = NULL;
}

void gpu_cleanup(void) {
    gpu_recon_free();
    if (g_mvm) mb_mvm_free(g_mvm);
    g_mvm = NULL;
    mb_cleanup();
}

void gpu_setup_recon(const PARMS_T *parms, POWFS_T *powfs, RECON_T *recon) {
    keep_t k = {0};
    const int nps = recon->npsr, nwfs = parms->nwfsr;
    if (parms->recon.alg != 0) error("maos_b200 serves the minimum-variance reconstructor (recon.alg=0)\n");
    mb_grid *xmap = keep(&k, malloc(sizeof(mb_grid) * nps));
    double *l2c = keep(&k, malloc(sizeof(double) * nps));
    for (int i = 0; i < nps; i++) xmap[i] = grid_of(recon->xmap->p[i]);
    layer_l2c(parms, recon, l2c);
    mb_wfs_desc *wfs = keep(&k, calloc(nwfs, sizeof(mb_wfs_desc)));
    for (int iw = 0; iw < nwfs; iw++) {
        const int ipowfs = parms->wfsr[iw].powfs;
        const loc_t *saloc = powfs[ipowfs].saloc;
        const mb_csc gp = csc_of(recon->GP->p[iw], &k);
        wfs[iw].thetax = parms->wfsr[iw].thetax;
        wfs[iw].thetay = parms->wfsr[iw].thetay;
        wfs[iw].hs = parms->wfsr[iw].hs;
        wfs[iw].nsa = (int)saloc->nloc;
        wfs[iw].dsa = saloc->dx;
        wfs[iw].salocx = saloc->locx;
        wfs[iw].salocy = saloc->locy;
        wfs[iw].gp_p = gp.p;
        wfs[iw].gp_i = gp.i;
        wfs[iw].gp_x = gp.x;
        wfs[iw].neai = neai_of(recon, iw, nwfs, &k);
        wfs[iw].ptt = (recon->PTT && recon->PTT->p[iw + iw * nwfs]) ? recon->PTT->p[iw + iw * nwfs]->p : NULL;
    }
    mb_fdpcg_desc fd = {0};
    if (parms->tomo.precond == 1) fd = fdpcg_of(recon, &k);
    mb_fit_desc fit = {0};
    mb_fit_sparse_desc fsp = {0};
    int use_grid = 0, use_sparse = 0;
    if (parms->gpu.fit == 2) { /* cufit_grid (cuda/fit.cu:46), fit.square=1 */
        const FIT_T *f = recon->fit;
        const int ndm = parms->ndm;
        mb_grid *amap = keep(&k, malloc(sizeof(mb_grid) * ndm));
        for (int d = 0; d < ndm; d++) amap[d] = grid_of(recon->amap->p[d]);
        fit.floc = grid_of(recon->fmap);
        fit.nfit = parms->fit.nfit;
        fit.thetax = parms->fit.thetax->p;
        fit.thetay = parms->fit.thetay->p;
        fit.wt = parms->fit.wt->p;
        fit.hs = parms->fit.hs->p;
        const mb_csc w0 = csc_of(recon->W0, &k);
        fit.w0_p = w0.p;
        fit.w0_i = w0.i;
        fit.w0_x = w0.x;
        fit.w1 = recon->W1->p;
        fit.ndm = ndm;
        fit.amap = amap;
        if (f->NW) {
            long nr, nc;
            fit.nw = stack_rows(f->NW, &nr, &nc, &k);
            fit.nnw = (int)nc;
        }
        fit.maxit = parms->fit.maxit;
        if (f->actslave) {
            dsp *s = dspcell2sp(f->actslave);
            fit.actslave = csc_of(s, &k);
            double *x = keep(&k, malloc(sizeof(double) * (s->p[s->ny] > 0 ? s->p[s->ny] : 1)));
            memcpy(x, s->x, sizeof(double) * s->p[s->ny]);
            fit.actslave.x = x;
            dspfree(s);
        }
        use_grid = 1;
    } else if (parms->gpu.fit == 1) { /* cusolve_sparse over FR and FL (cuda/solve.cu:36-90) */
        const FIT_T *f = recon->fit;
        if (!f->FR.M || !f->FL.M) error("gpu.fit=1 needs the assembled fit matrices (fit.assemble=1)\n");
        dsp *frm = dspcell2sp((dspcell *)f->FR.M);
        dsp *flm = dspcell2sp((dspcell *)f->FL.M);
        fsp.frm = csc_of(frm, &k);
        fsp.flm = csc_of(flm, &k);
        double *frx = keep(&k, malloc(sizeof(double) * (frm->p[frm->ny] + 1)));
        double *flx = keep(&k, malloc(sizeof(double) * (flm->p[flm->ny] + 1)));
        memcpy(frx, frm->x, sizeof(double) * frm->p[frm->ny]);
        memcpy(flx, flm->x, sizeof(double) * flm->p[flm->ny]);
        fsp.frm.x = frx;
        fsp.flm.x = flx;
        dspfree(frm);
        dspfree(flm);
        long nr, nc;
        if (f->FR.U && f->FR.V) {
            fsp.fru = stack_rows(f->FR.U, &nr, &nc, &k);
            fsp.frv = stack_rows(f->FR.V, &nr, &nc, &k);
            fsp.nfr = (int)nc;
        }
        if (f->FL.U && f->FL.V) {
            fsp.flu = stack_rows(f->FL.U, &nr, &nc, &k);
            fsp.flv = stack_rows(f->FL.V, &nr, &nc, &k);
            fsp.nfl = (int)nc;
        }
        fsp.maxit = parms->fit.maxit;
        use_sparse = 1;
    }
    mb_recon_desc d = {0};
    d.pmap = grid_of(recon->pmap);
    d.nps = nps;
    d.xmap = xmap;
    d.l2c = l2c;
    d.nwfs = nwfs;
    d.wfs = wfs;
    d.maxit = parms->tomo.maxit;
    d.precond = parms->tomo.precond;
    d.split = parms->recon.split;
    d.fdpcg = parms->tomo.precond == 1 ? &fd : NULL;
    d.nbatch = 1;
    d.fit = use_grid ? &fit : NULL;
    d.fit_sparse = use_sparse ? &fsp : NULL;
    gpu_recon_free();
    MB_CHECK(mb_init(g_device));
    MB_CHECK(mb_setup_recon(&d, &g_recon));
    keep_free(&k);
}

void gpu_setup_recon_mvm(const PARMS_T *parms, RECON_T *recon, POWFS_T *powfs) {
    (void)parms;
    (void)powfs;
    if (!recon->MVM)
        error("maos_b200: assemble recon->MVM first (the control-matrix build is maos_b200.mvm_build)\n");
    if (g_mvm) mb_mvm_free(g_mvm);
    g_mvm = NULL;
    /* FP32 storage as the reference's cusolve_mvm (cuda/solve.h:123-135) */
    MB_CHECK(mb_mvm_create(recon->MVM->p, recon->MVM->nx, recon->MVM->ny, MB_MVM_F32, 1, &g_mvm));
}

void gpu_update_recon(const PARMS_T *parms, POWFS_T *powfs, RECON_T *recon) {
    (void)powfs;
    if (!parms->gpu.tomo || !g_recon) return;
    keep_t k = {0};
    const int nwfs = parms->nwfsr;
    for (int iw = 0; iw < nwfs; iw++) {
        const double *ptt =
            (recon->PTT && recon->PTT->p[iw + iw * nwfs]) ? recon->PTT->p[iw + iw * nwfs]->p : NULL;
        MB_CHECK(mb_update_recon_nea(g_recon, iw, neai_of(recon, iw, nwfs, &k), ptt));
    }
    if (parms->tomo.precond == 1) { /* maos rebuilt recon->fdpcg for the new noise */
        double *l2c = keep(&k, malloc(sizeof(double) * recon->npsr));
        layer_l2c(parms, recon, l2c);
        mb_fdpcg_desc fd = fdpcg_of(recon, &k);
        MB_CHECK(mb_update_recon_cn2(g_recon, l2c, &fd));
    }
    keep_free(&k);
}

void gpu_update_recon_cn2(const PARMS_T *parms, RECON_T *recon) {
    if (!parms->gpu.tomo || !g_recon) return;
    keep_t k = {0};
    double *l2c = keep(&k, malloc(sizeof(double) * recon->npsr));
    layer_l2c(parms, recon, l2c);
    if (parms->tomo.precond == 1 && recon->fdpcg) {
        mb_fdpcg_desc fd = fdpcg_of(recon, &k);
        MB_CHECK(mb_update_recon_cn2(g_recon, l2c, &fd));
    } else {
        MB_CHECK(mb_update_recon_cn2(g_recon, l2c, NULL));
    }
    keep_free(&k);
}

void gpu_recon_reset(const PARMS_T *parms) {
    (void)parms;
    if (g_recon) MB_CHECK(mb_recon_reset(g_recon));
}

void gpu_tomo(SIM_T *simu, dcell *gradin) {
    const PARMS_T *parms = simu->parms;
    RECON_T *recon = simu->recon;
    const int nwfs = parms->nwfsr, nps = recon->npsr;
    /* copy the layer OPD back when maos reads it on the CPU (cuda/recon.cu:574-578) */
    const int copy2cpu = parms->plot.run > 1 || !parms->gpu.fit || parms->save.opdr ||
                         (recon->moao && !parms->gpu.moao) || parms->evl.tomo || recon->GXL;
    const double *g[nwfs];
    for (int iw = 0; iw < nwfs; iw++) g[iw] = (gradin && gradin->p[iw]) ? gradin->p[iw]->p : NULL;
    double *opd[nps];
    if (copy2cpu) {
        if (!simu->opdr) simu->opdr = dcellnew3(nps, 1, recon->xnloc->p, NULL);
        for (int i = 0; i < nps; i++) opd[i] = simu->opdr->p[i]->p;
    }
    float res = 0;
    MB_CHECK(mb_tomo_wfs(g_recon, g, copy2cpu ? opd : NULL, &res));
    if (simu->cgres) simu->cgres->p[0]->p[simu->reconisim] = res;
    if (recon->GXL) { /* NGS modes of the layer solution (cuda/recon.cu:269-272) */
        dcellmm(&simu->gngsmvst, recon->GXL, simu->opdr, "nn", 1);
    }
}

void gpu_fit(dcell **dmout, SIM_T *simu) {
    const PARMS_T *parms = simu->parms;
    RECON_T *recon = simu->recon;
    const int ndm = parms->ndm;
    long nact = 0;
    for (int d = 0; d < ndm; d++) nact += parms->gpu.fit == 2 ? recon->anx->p[d] * recon->any->p[d] : recon->anloc->p[d];
    if (!*dmout) {
        if (parms->gpu.fit == 2) *dmout = dcellnew3(ndm, 1, recon->anx->p, recon->any->p);
        else *dmout = dcellnew3(ndm, 1, recon->anloc->p, NULL);
    }
    double *a = malloc(sizeof(double) * nact);
    float res = 0;
    if (parms->gpu.tomo) {
        MB_CHECK(mb_fit(g_recon, a, &res));
    } else { /* the tomography ran on the CPU: fit simu->opdr (cuda/recon.cu:603-604) */
        const double *opd[recon->npsr];
        for (int i = 0; i < recon->npsr; i++) opd[i] = simu->opdr ? simu->opdr->p[i]->p : NULL;
        MB_CHECK(mb_fit_opdr(g_recon, opd, a, &res));
    }
    /* overwrite, like add2cpu(_dmfit, 0, dmfit_vec, 1) at cuda/recon.cu:285 */
    long off = 0;
    for (int d = 0; d < ndm; d++) {
        dmat *m = (*dmout)->p[d];
        memcpy(m->p, a + off, sizeof(double) * m->nx * m->ny);
        off += m->nx * m->ny;
    }
    free(a);
    if (simu->cgres) simu->cgres->p[1]->p[simu->reconisim] = res;
}

void gpu_recon_mvm(dcell **dmout, dcell *gradin) {
    if (!g_mvm) error("maos_b200: gpu_setup_recon_mvm was not called\n");
    long ng = 0, na = 0;
    for (int i = 0; i < gradin->nx * gradin->ny; i++) ng += gradin->p[i] ? gradin->p[i]->nx * gradin->p[i]->ny : 0;
    for (int i = 0; i < (*dmout)->nx * (*dmout)->ny; i++) na += (*dmout)->p[i]->nx * (*dmout)->p[i]->ny;
    double *g = malloc(sizeof(double) * ng), *a = malloc(sizeof(double) * na);
    long off = 0;
    for (int i = 0; i < gradin->nx * gradin->ny; i++)
        if (gradin->p[i]) {
            const long n = gradin->p[i]->nx * gradin->p[i]->ny;
            memcpy(g + off, gradin->p[i]->p, sizeof(double) * n);
            off += n;
        }
    MB_CHECK(mb_recon_mvm(g_mvm, g, a));
    off = 0;
    for (int i = 0; i < (*dmout)->nx * (*dmout)->ny; i++) {
        const long n = (*dmout)->p[i]->nx * (*dmout)->p[i]->ny;
        memcpy((*dmout)->p[i]->p, a + off, sizeof(double) * n);
        off += n;
    }
    free(g);
    free(a);
}
