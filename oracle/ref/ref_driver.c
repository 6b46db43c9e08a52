/*
 * Flat C driver around the reference MAOS CPU reconstruction -- TEST
 * INFRASTRUCTURE ONLY.  It is linked into oracle/_ref/libmaosref.so together
 * with the reference's own sys/, math/, lib/ and maos/ objects (see Makefile)
 * and lets the Python tests run the reference's functions on exactly the
 * tables the B200 path consumes:
 *
 *   TomoR, TomoL           maos/recon_utils.c:397,447
 *   fdpcg_prepare          maos/fdpcg.c:331
 *   fdpcg_precond          maos/fdpcg.c:661
 *   pcg                    lib/pcg.c:28
 *   mkg                    lib/mkg.c:470
 *   dcellpinv (PTT)        used by maos/setup_recon.c:255
 *   prop_grid_stat         lib/accphi.c + lib/prop_grid.c
 *   prop_grid (loc out)    lib/accphi.c:426
 *   WFS pts/amp/GS0        maos/setup_powfs.c:328-337,565 (ptsnew, pts2loc,
 *                          mkamp -> locannular, mkg)
 *
 * The driver fills only the PARMS_T / RECON_T / POWFS_T fields those
 * functions read; everything else stays zero.  All arrays crossing this ABI
 * are plain doubles / ints / longs, column-major like dmat.
 */
#include "maos/common.h"
#include "maos/recon_utils.h"
#include "maos/fdpcg.h"
#include "lib/pcg.h"
#include "lib/mkg.h"
#include "lib/accphi.h"
#include "lib/mkh.h"
#include "lib/mkw.h"
#include "lib/servo.h"
#include "lib/slaving.h"

typedef struct {
    int nwfs, nps, nthread;
    PARMS_T *parms;
    RECON_T *recon;
    POWFS_T *powfs;
    SIM_T *simu;
    int *nsa;
    long *goff; /* gradient offsets per wfs */
    long *xoff; /* x offsets per layer */
    int finalized;
} refh_t;

int maosref_driver_version(void) { return 2; }

static map_t *mk_map(int nx, int ny, double dx, double dy, double ox, double oy) {
    map_t *m = mapnew(nx, ny, dx, dy, NULL);
    m->ox = ox;
    m->oy = oy;
    return m;
}

static loc_t *mk_square_loc(int nx, int ny, double dx, double dy, double ox, double oy) {
    map_t *m = mk_map(nx, ny, dx, dy, ox, oy);
    dset((dmat *)m, 1);
    loc_t *loc = map2loc(m, 0);
    mapfree(m);
    return loc;
}

void *ref_new(int nwfs, int nps, int nthread) {
    refh_t *h = calloc(1, sizeof(refh_t));
    h->nwfs = nwfs;
    h->nps = nps;
    h->nthread = nthread > 0 ? nthread : 1;
    h->parms = calloc(1, sizeof(PARMS_T));
    h->recon = calloc(1, sizeof(RECON_T));
    h->powfs = calloc(1, sizeof(POWFS_T));
    h->simu = calloc(1, sizeof(SIM_T));
    h->nsa = calloc(nwfs, sizeof(int));
    h->goff = calloc(nwfs + 1, sizeof(long));
    h->xoff = calloc(nps + 1, sizeof(long));
    PARMS_T *parms = h->parms;
    RECON_T *recon = h->recon;
    parms->nwfs = parms->nwfsr = nwfs;
    parms->npowfs = 1;
    parms->powfs = calloc(1, sizeof(POWFS_CFG_T));
    parms->wfs = calloc(nwfs, sizeof(WFS_CFG_T));
    parms->wfsr = parms->wfs;
    parms->powfs[0].nwfs = parms->powfs[0].nwfsr = nwfs;
    parms->powfs[0].wfs = lnew(nwfs, 1);
    parms->powfs[0].wfsr = lnew(nwfs, 1);
    parms->powfs[0].wfsind = lnew(nwfs, 1);
    for (int i = 0; i < nwfs; i++) {
        parms->powfs[0].wfs->p[i] = i;
        parms->powfs[0].wfsr->p[i] = i;
        parms->powfs[0].wfsind->p[i] = i;
    }
    parms->powfs[0].dtrat = 1;
    parms->tomo.square = 1;
    parms->tomo.cxx = 0;
    parms->tomo.cxxscale = 1;
    parms->atmr.os = lnew(nps, 1);
    parms->atmr.ht = dnew(nps, 1);
    parms->atmr.wt = dnew(nps, 1);
    parms->atmr.nps = nps;
    recon->npsr = nps;
    recon->ht = dnew(nps, 1);
    recon->wt = dnew(nps, 1);
    recon->os = dnew(nps, 1);
    recon->dx = dnew(nps, 1);
    recon->xloc = loccellnew(nps, 1);
    recon->xmap = mapcellnew(nps, 1);
    recon->xnx = lnew(nps, 1);
    recon->xny = lnew(nps, 1);
    recon->xnloc = lnew(nps, 1);
    recon->GP = dspcellnew(nwfs, 1);
    recon->saneai = dspcellnew(nwfs, nwfs);
    recon->sanea = dspcellnew(nwfs, nwfs);
    recon->TT = dcellnew(nwfs, nwfs);
    recon->neam = dnew(nwfs, 1);
    recon->nthread = h->nthread;
    recon->cxx = 0;
    if (!global) global = calloc(1, sizeof(GLOBAL_T));
    return h;
}

void ref_set_system(void *hh, double r0, double cxxscale, double dt, int tomo_pos, int split,
                    int precond, int maxit) {
    refh_t *h = hh;
    h->recon->r0 = r0;
    h->parms->tomo.cxxscale = cxxscale;
    h->parms->sim.dt = dt;
    h->parms->tomo.pos = tomo_pos;
    h->parms->recon.split = split;
    h->parms->tomo.precond = precond;
    h->parms->tomo.maxit = maxit;
}

void ref_set_pmap(void *hh, int nx, int ny, double dx, double ox, double oy) {
    refh_t *h = hh;
    RECON_T *recon = h->recon;
    recon->ploc = mk_square_loc(nx, ny, dx, dx, ox, oy);
    loc_create_map_npad(recon->ploc, 0, 0, 0);
    recon->pmap = recon->ploc->map;
    loc_create_stat(recon->ploc);
}

void ref_set_layer(void *hh, int ips, int nx, int ny, double dx, double ox, double oy, double ht,
                   double wt, int os) {
    refh_t *h = hh;
    RECON_T *recon = h->recon;
    recon->ht->p[ips] = ht;
    recon->wt->p[ips] = wt;
    recon->os->p[ips] = os;
    recon->dx->p[ips] = dx;
    h->parms->atmr.os->p[ips] = os;
    h->parms->atmr.ht->p[ips] = ht;
    h->parms->atmr.wt->p[ips] = wt;
    recon->xloc->p[ips] = mk_square_loc(nx, ny, dx, dx, ox, oy);
    recon->xloc->p[ips]->ht = ht;
    loc_create_stat(recon->xloc->p[ips]);
    recon->xmap->p[ips] = mk_map(nx, ny, dx, dx, ox, oy);
    recon->xmap->p[ips]->h = ht;
    recon->xnx->p[ips] = nx;
    recon->xny->p[ips] = ny;
    recon->xnloc->p[ips] = (long)nx * ny;
}

static dsp *mk_csc(long nrow, long ncol, const int *p, const int *i, const double *x) {
    long nnz = p[ncol];
    dsp *A = dspnew(nrow, ncol, nnz);
    for (long k = 0; k <= ncol; k++) A->p[k] = p[k];
    for (long k = 0; k < nnz; k++) { A->i[k] = i[k]; A->x[k] = x[k]; }
    return A;
}

/* GP is passed in CSC (rows = 2*nsa gradients, cols = pupil points). */
void ref_set_wfs(void *hh, int iwfs, double thetax, double thetay, double hs, int nsa, double dsa,
                 const double *salocx, const double *salocy, const double *saa, const int *gp_p,
                 const int *gp_i, const double *gp_x, const double *saneai, const double *sanea,
                 int trs) {
    refh_t *h = hh;
    PARMS_T *parms = h->parms;
    RECON_T *recon = h->recon;
    parms->wfs[iwfs].thetax = thetax;
    parms->wfs[iwfs].thetay = thetay;
    parms->wfs[iwfs].hs = hs;
    parms->wfs[iwfs].powfs = 0;
    parms->powfs[0].trs = trs;
    parms->powfs[0].hs = hs;
    h->nsa[iwfs] = nsa;
    if (iwfs == 0) {
        loc_t *saloc = locnew(nsa, dsa, dsa);
        memcpy(saloc->locx, salocx, sizeof(double) * nsa);
        memcpy(saloc->locy, salocy, sizeof(double) * nsa);
        h->powfs[0].saloc = saloc;
        h->powfs[0].saa = dnew(nsa, 1);
        memcpy(h->powfs[0].saa->p, saa, sizeof(double) * nsa);
    }
    recon->GP->p[iwfs] = mk_csc(2L * nsa, recon->ploc->nloc, gp_p, gp_i, gp_x);
    recon->saneai->p[iwfs + iwfs * h->nwfs] = dspnewdiag(2L * nsa, (double *)saneai, 1.);
    recon->sanea->p[iwfs + iwfs * h->nwfs] = dspnewdiag(2L * nsa, (double *)sanea, 1.);
    if (trs) {
        dmat *TT = dnew(2L * nsa, 2);
        for (int isa = 0; isa < nsa; isa++) {
            TT->p[isa] = 1;
            TT->p[2L * nsa + nsa + isa] = 1;
        }
        recon->TT->p[iwfs + iwfs * h->nwfs] = TT;
    }
}

void ref_set_neam(void *hh, int iwfs, double neam) { ((refh_t *)hh)->recon->neam->p[iwfs] = neam; }

int ref_finalize(void *hh) {
    refh_t *h = hh;
    PARMS_T *parms = h->parms;
    RECON_T *recon = h->recon;
    int nps = h->nps, nwfs = h->nwfs;
    h->goff[0] = 0;
    for (int i = 0; i < nwfs; i++) h->goff[i + 1] = h->goff[i] + 2L * h->nsa[i];
    h->xoff[0] = 0;
    for (int i = 0; i < nps; i++) h->xoff[i + 1] = h->xoff[i] + recon->xnloc->p[i];
    /* tip/tilt removal operators (setup_recon.c:255) */
    int anytt = 0;
    for (int i = 0; i < nwfs * nwfs; i++) anytt |= recon->TT->p[i] != NULL;
    if (anytt) {
        recon->PTT = dcellpinv(recon->TT, recon->saneai);
        recon->TTF = dcellref(recon->TT);
        recon->PTTF = dcellref(recon->PTT);
    }
    /* biharmonic regularisation (setup_recon.c:291-335), tomo.square=1 */
    recon->L2 = dspcellnew(nps, nps);
    for (int ips = 0; ips < nps; ips++) {
        recon->L2->p[ips + nps * ips] =
            mklaplacian_map(recon->xmap->p[ips]->nx, recon->xmap->p[ips]->nx,
                            recon->xloc->p[ips]->dx, recon->r0, recon->wt->p[ips]);
    }
    dspcellscale(recon->L2, sqrt(parms->tomo.cxxscale * TOMOSCALE));
    global->parms = parms;
    global->recon = recon;
    global->powfs = h->powfs;
    global->simu = h->simu;
    h->finalized = 1;
    return 0;
}

/* PTT for one wfs as computed by the reference: 2 x 2nsa column-major */
int ref_get_ptt(void *hh, int iwfs, double *out) {
    refh_t *h = hh;
    if (!h->recon->PTT) return -1;
    dmat *P = h->recon->PTT->p[iwfs + iwfs * h->nwfs];
    if (!P) return -1;
    memcpy(out, P->p, sizeof(double) * P->nx * P->ny);
    return (int)(P->nx * P->ny);
}

static dcell *vec2cell(const double *v, const long *off, int n) {
    dcell *c = dcellnew(n, 1);
    for (int i = 0; i < n; i++) {
        c->p[i] = dnew(off[i + 1] - off[i], 1);
        if (v) memcpy(c->p[i]->p, v + off[i], sizeof(double) * (off[i + 1] - off[i]));
    }
    return c;
}
static void cell2vec(double *v, const dcell *c, const long *off, int n) {
    for (int i = 0; i < n; i++) {
        long len = off[i + 1] - off[i];
        if (c && c->p[i]) memcpy(v + off[i], c->p[i]->p, sizeof(double) * len);
        else memset(v + off[i], 0, sizeof(double) * len);
    }
}

void ref_tomoR(void *hh, const double *g, double alpha, double *xout) {
    refh_t *h = hh;
    dcell *gin = vec2cell(g, h->goff, h->nwfs);
    dcell *x = vec2cell(NULL, h->xoff, h->nps);
    TomoR(&x, h->recon, gin, alpha);
    cell2vec(xout, x, h->xoff, h->nps);
    dcellfree(gin);
    dcellfree(x);
}

void ref_tomoL(void *hh, const double *xin, double alpha, double *xout) {
    refh_t *h = hh;
    dcell *x = vec2cell(xin, h->xoff, h->nps);
    dcell *y = vec2cell(NULL, h->xoff, h->nps);
    TomoL(&y, h->recon, x, alpha);
    cell2vec(xout, y, h->xoff, h->nps);
    dcellfree(x);
    dcellfree(y);
}

/* Hx for one wfs: sum over layers of prop_grid_stat onto ploc */
void ref_hx(void *hh, int iwfs, const double *xin, double *opd) {
    refh_t *h = hh;
    RECON_T *recon = h->recon;
    PARMS_T *parms = h->parms;
    long np = recon->ploc->nloc;
    memset(opd, 0, sizeof(double) * np);
    for (int ips = 0; ips < h->nps; ips++) {
        double ht = recon->ht->p[ips];
        map_t xmap;
        memcpy(&xmap, recon->xmap->p[ips], sizeof(map_t));
        xmap.p = (double *)xin + h->xoff[ips];
        double scale = 1. - ht / parms->wfs[iwfs].hs;
        prop_grid_stat(&xmap, recon->ploc->stat, opd, 1, parms->wfs[iwfs].thetax * ht,
                       parms->wfs[iwfs].thetay * ht, scale, 0, 0, 0);
    }
}

/* Build the reference FDPCG tables from the system. */
int ref_fdpcg_prepare(void *hh, long *nb, long *bs) {
    refh_t *h = hh;
    h->parms->powfs[0].lo = 0;
    h->parms->powfs[0].skip = 0;
    h->recon->fdpcg = fdpcg_prepare(h->parms, h->recon, h->powfs, NULL);
    if (!h->recon->fdpcg) return -1;
    *nb = h->recon->fdpcg->Mbinv->nx;
    *bs = h->recon->fdpcg->bs;
    return h->recon->fdpcg->scale;
}

/* Export Mbinv (nb blocks of bs x bs complex, column-major, re/im interleaved) and perm. */
void ref_fdpcg_get(void *hh, double *mbinv, long *perm) {
    refh_t *h = hh;
    FDPCG_T *fd = h->recon->fdpcg;
    long bs = fd->bs;
    for (long ib = 0; ib < fd->Mbinv->nx; ib++) {
        cmat *B = fd->Mbinv->p[ib];
        for (long k = 0; k < bs * bs; k++) {
            mbinv[2 * (ib * bs * bs + k)] = creal(B->p[k]);
            mbinv[2 * (ib * bs * bs + k) + 1] = cimag(B->p[k]);
        }
    }
    memcpy(perm, fd->perm->p, sizeof(long) * fd->perm->nx);
}

/* Install externally built FDPCG tables (same layout as ref_fdpcg_get). */
void ref_fdpcg_set(void *hh, long nb, long bs, const double *mbinv, const long *perm, int scale) {
    refh_t *h = hh;
    FDPCG_T *fd = calloc(1, sizeof(FDPCG_T));
    fd->bs = bs;
    fd->scale = scale;
    fd->square = 1;
    fd->xloc = h->recon->xloc;
    fd->nxtot = h->xoff[h->nps];
    fd->perm = lnew(nb * bs, 1);
    memcpy(fd->perm->p, perm, sizeof(long) * nb * bs);
    fd->Mbinv = ccellnew(nb, 1);
    for (long ib = 0; ib < nb; ib++) {
        fd->Mbinv->p[ib] = cnew(bs, bs);
        for (long k = 0; k < bs * bs; k++)
            fd->Mbinv->p[ib]->p[k] = mbinv[2 * (ib * bs * bs + k)] + I * mbinv[2 * (ib * bs * bs + k) + 1];
    }
    h->recon->fdpcg = fd;
}

void ref_fdpcg_precond(void *hh, const double *r, double *z) {
    refh_t *h = hh;
    dcell *rin = vec2cell(r, h->xoff, h->nps);
    dcell *zout = NULL;
    fdpcg_precond(&zout, h->recon, rin);
    cell2vec(z, zout, h->xoff, h->nps);
    dcellfree(rin);
    dcellfree(zout);
}

/* Tomography solve with the reference pcg: x (in/out) warm start. */
double ref_tomo_pcg(void *hh, const double *b, double *x, int warm, int maxit, int precond) {
    refh_t *h = hh;
    dcell *bb = vec2cell(b, h->xoff, h->nps);
    dcell *xx = vec2cell(x, h->xoff, h->nps);
    double res = pcg(&xx, TomoL, h->recon, precond ? fdpcg_precond : NULL, h->recon, bb, warm, maxit);
    cell2vec(x, xx, h->xoff, h->nps);
    dcellfree(bb);
    dcellfree(xx);
    return res;
}

/* mkg on a square pupil grid (OPD grid = pupil grid). Returns nnz; fills CSC if p != NULL. */
static dsp *last_gp = NULL;
long ref_mkg(int nx, int ny, double dx, double ox, double oy, const double *amp, int nsa, double dsa,
             const double *salocx, const double *salocy) {
    loc_t *ploc = mk_square_loc(nx, ny, dx, dx, ox, oy);
    loc_create_map_npad(ploc, 0, 0, 0);
    dmat *a = dnew(ploc->nloc, 1);
    memcpy(a->p, amp, sizeof(double) * ploc->nloc);
    loc_t *saloc = locnew(nsa, dsa, dsa);
    memcpy(saloc->locx, salocx, sizeof(double) * nsa);
    memcpy(saloc->locy, salocy, sizeof(double) * nsa);
    if (last_gp) dspfree(last_gp);
    last_gp = mkg(ploc, ploc, a, saloc, 1, 0, 0, 1);
    dfree(a);
    locfree(saloc);
    locfree(ploc);
    return last_gp->p[last_gp->ny];
}
void ref_mkg_get(int *p, int *i, double *x, long *nrow, long *ncol) {
    *nrow = last_gp->nx;
    *ncol = last_gp->ny;
    long nnz = last_gp->p[last_gp->ny];
    for (long k = 0; k <= last_gp->ny; k++) p[k] = last_gp->p[k];
    for (long k = 0; k < nnz; k++) { i[k] = last_gp->i[k]; x[k] = last_gp->x[k]; }
}

/* loc ordering check: coordinates of a square loc built like ploc/xloc */
void ref_loc_coords(int nx, int ny, double dx, double ox, double oy, double *x, double *y) {
    loc_t *l = mk_square_loc(nx, ny, dx, dx, ox, oy);
    memcpy(x, l->locx, sizeof(double) * l->nloc);
    memcpy(y, l->locy, sizeof(double) * l->nloc);
    locfree(l);
}

/* ------------------------------------------------------------------------
 * DM fit.  FIT_T is filled from the caller's fit grid, W0/W1, DM actuator
 * locations and low-rank NW; HA and HXF are built by the reference's own mkh
 * (lib/mkh.c:47) exactly as setup_fit_HA / setup_fit_HXF do
 * (maos/setup_recon_fit.c:26-70).
 * ---------------------------------------------------------------------- */
static FIT_T *g_fit = NULL;
static long *g_aoff = NULL;
static int g_ndm = 0;

int ref_fit_setup(void *hh, int nfit, const double *thetax, const double *thetay, const double *wt,
                  const double *hs, int nf, const int *w0p, const int *w0i, const double *w0x,
                  const double *w1, int ndm, const double *dmht, const double *dmdx, const int *nact,
                  const double *alocx, const double *alocy, int nnw, const double *nw) {
    refh_t *h = hh;
    FIT_T *fit = calloc(1, sizeof(FIT_T));
    fit->thetax = dnew(nfit, 1);
    fit->thetay = dnew(nfit, 1);
    fit->wt = dnew(nfit, 1);
    fit->hs = dnew(nfit, 1);
    for (int i = 0; i < nfit; i++) {
        fit->thetax->p[i] = thetax[i];
        fit->thetay->p[i] = thetay[i];
        fit->wt->p[i] = wt[i];
        fit->hs->p[i] = hs[i];
    }
    fit->floc = h->recon->ploc; /* fit grid is the pupil grid */
    fit->xloc = h->recon->xloc;
    fit->W0 = mk_csc(nf, nf, w0p, w0i, w0x);
    fit->W1 = dnew(nf, 1);
    memcpy(fit->W1->p, w1, sizeof(double) * nf);
    fit->aloc = loccellnew(ndm, 1);
    free(g_aoff);
    g_aoff = calloc(ndm + 1, sizeof(long));
    g_ndm = ndm;
    for (int d = 0; d < ndm; d++) {
        loc_t *a = locnew(nact[d], dmdx[d], dmdx[d]);
        memcpy(a->locx, alocx + g_aoff[d], sizeof(double) * nact[d]);
        memcpy(a->locy, alocy + g_aoff[d], sizeof(double) * nact[d]);
        a->ht = dmht[d];
        fit->aloc->p[d] = a;
        g_aoff[d + 1] = g_aoff[d] + nact[d];
    }
    const int npsr = h->nps;
    fit->HXF = dspcellnew(nfit, npsr);
    fit->HA = dspcellnew(nfit, ndm);
    for (int f = 0; f < nfit; f++) {
        for (int ips = 0; ips < npsr; ips++) {
            const double ht = fit->xloc->p[ips]->ht - fit->floc->ht;
            const double scale = 1. - ht / hs[f];
            fit->HXF->p[f + ips * nfit] =
                mkh(fit->xloc->p[ips], fit->floc, thetax[f] * ht, thetay[f] * ht, scale);
        }
        for (int d = 0; d < ndm; d++) {
            const double ht = fit->aloc->p[d]->ht - fit->floc->ht;
            const double scale = 1. - ht / hs[f];
            fit->HA->p[f + d * nfit] =
                mkh(fit->aloc->p[d], fit->floc, thetax[f] * ht, thetay[f] * ht, scale);
        }
    }
    if (nnw > 0) {
        fit->NW = dcellnew(ndm, 1);
        long ntot = g_aoff[ndm];
        for (int d = 0; d < ndm; d++) {
            fit->NW->p[d] = dnew(nact[d], nnw);
            for (int k = 0; k < nnw; k++)
                memcpy(fit->NW->p[d]->p + (long)k * nact[d], nw + (long)k * ntot + g_aoff[d],
                       sizeof(double) * nact[d]);
        }
    }
    g_fit = fit;
    return 0;
}

/* HA[f][d] of the reference (CSC, nfloc x nact). Returns nnz; fills when p != NULL. */
long ref_fit_ha(int f, int d, int *p, int *i, double *x) {
    dsp *A = g_fit->HA->p[f + d * g_fit->thetax->nx];
    long nnz = A->p[A->ny];
    if (p) {
        for (long k = 0; k <= A->ny; k++) p[k] = A->p[k];
        for (long k = 0; k < nnz; k++) { i[k] = A->i[k]; x[k] = A->x[k]; }
    }
    return nnz;
}

static dcell *avec2cell(const double *v) {
    dcell *c = dcellnew(g_ndm, 1);
    for (int d = 0; d < g_ndm; d++) {
        c->p[d] = dnew(g_aoff[d + 1] - g_aoff[d], 1);
        if (v) memcpy(c->p[d]->p, v + g_aoff[d], sizeof(double) * (g_aoff[d + 1] - g_aoff[d]));
    }
    return c;
}

void ref_fitR(void *hh, const double *xin, double alpha, double *aout) {
    refh_t *h = hh;
    dcell *x = vec2cell(xin, h->xoff, h->nps);
    dcell *a = avec2cell(NULL);
    FitR(&a, g_fit, x, alpha);
    cell2vec(aout, a, g_aoff, g_ndm);
    dcellfree(x);
    dcellfree(a);
}

void ref_fitL(void *hh, const double *ain, double alpha, double *aout) {
    (void)hh;
    dcell *a = avec2cell(ain);
    dcell *y = avec2cell(NULL);
    FitL(&y, g_fit, a, alpha);
    cell2vec(aout, y, g_aoff, g_ndm);
    dcellfree(a);
    dcellfree(y);
}

double ref_fit_pcg(void *hh, const double *b, double *a, int warm, int maxit) {
    (void)hh;
    dcell *bb = avec2cell(b);
    dcell *aa = avec2cell(a);
    double res = pcg(&aa, FitL, g_fit, NULL, NULL, bb, warm, maxit);
    cell2vec(a, aa, g_aoff, g_ndm);
    dcellfree(bb);
    dcellfree(aa);
    return res;
}

/* mkw_amp (lib/mkw.c:41) on a square grid; returns nnz of W0 (CSC) */
static dsp *last_w0 = NULL;
static dmat *last_w1 = NULL;
long ref_mkw_amp(int nx, int ny, double dx, double ox, double oy, const double *amp) {
    loc_t *loc = mk_square_loc(nx, ny, dx, dx, ox, oy);
    if (last_w0) dspfree(last_w0);
    if (last_w1) dfree(last_w1);
    mkw_amp(loc, (double *)amp, &last_w0, &last_w1);
    locfree(loc);
    return last_w0->p[last_w0->ny];
}
void ref_mkw_amp_get(int *p, int *i, double *x, double *w1) {
    long nnz = last_w0->p[last_w0->ny];
    for (long k = 0; k <= last_w0->ny; k++) p[k] = last_w0->p[k];
    for (long k = 0; k < nnz; k++) { i[k] = last_w0->i[k]; x[k] = last_w0->x[k]; }
    memcpy(w1, last_w1->p, sizeof(double) * last_w1->nx);
}

/* .bin I/O through the reference's own writer and reader (math/cell.c
 * writebin, read_by_id), for checking maos_b200.binio. */
int ref_bin_write_dmat(const char *fn, const double *p, long nx, long ny, const char *header) {
    dmat *d = dnew(nx, ny);
    memcpy(d->p, p, sizeof(double) * nx * ny);
    if (header && header[0]) d->header = strdup(header);
    writebin(d, "%s", fn);
    dfree(d);
    return 0;
}
/* a 3 x 1 cell {a, empty, b} */
int ref_bin_write_dcell3(const char *fn, const double *a, long anx, long any, const double *b, long bnx, long bny) {
    dcell *c = dcellnew(3, 1);
    c->p[0] = dnew(anx, any);
    memcpy(c->p[0]->p, a, sizeof(double) * anx * any);
    c->p[2] = dnew(bnx, bny);
    memcpy(c->p[2]->p, b, sizeof(double) * bnx * bny);
    writebin(c, "%s", fn);
    dcellfree(c);
    return 0;
}
/* reads a dmat; returns the number of elements copied (-1: too large) */
long ref_bin_read_dmat(const char *fn, double *p, long cap, long *nx, long *ny, char *hdr, long hcap) {
    dmat *d = dread("%s", fn);
    *nx = d->nx;
    *ny = d->ny;
    long n = d->nx * d->ny;
    if (n > cap) { dfree(d); return -1; }
    memcpy(p, d->p, sizeof(double) * n);
    if (hdr && hcap > 0) {
        hdr[0] = 0;
        if (d->header) { strncpy(hdr, d->header, hcap - 1); hdr[hcap - 1] = 0; }
    }
    dfree(d);
    return n;
}
/* reads a dcell; element k's size into nx[k], ny[k] (0 for empty), data concatenated */
long ref_bin_read_dcell(const char *fn, double *p, long cap, long *ncell, long *nx, long *ny, long kcap) {
    dcell *c = dcellread("%s", fn);
    long off = 0;
    *ncell = c->nx * c->ny;
    for (long k = 0; k < *ncell && k < kcap; k++) {
        const dmat *e = c->p[k];
        nx[k] = e ? e->nx : 0;
        ny[k] = e ? e->ny : 0;
        if (e) {
            if (off + e->nx * e->ny > cap) { dcellfree(c); return -1; }
            memcpy(p + off, e->p, sizeof(double) * e->nx * e->ny);
            off += e->nx * e->ny;
        }
    }
    dcellfree(c);
    return off;
}

/* servo_new / servo_filter (lib/servo.c) on n command values in one cell;
 * ep column-major ep_nx x ep_ny; the command after each step is mint[0]. */
void *ref_servo_new(long n, const double *ap, int nap, int al, double dt, const double *ep, int ep_nx, int ep_ny) {
    dmat *apm = NULL;
    if (nap > 0) {
        apm = dnew(nap, 1);
        memcpy(apm->p, ap, sizeof(double) * nap);
    }
    dmat *epm = dnew(ep_nx, ep_ny);
    memcpy(epm->p, ep, sizeof(double) * ep_nx * ep_ny);
    SERVO_T *st = servo_new(NULL, apm, al, dt, epm);
    dfree(apm);
    dfree(epm);
    (void)n;
    return st;
}
int ref_servo_filter(void *h, const double *merr, long n, double *cmd) {
    SERVO_T *st = (SERVO_T *)h;
    dcell *m = dcellnew(1, 1);
    m->p[0] = dnew(n, 1);
    memcpy(m->p[0]->p, merr, sizeof(double) * n);
    int up = servo_filter(st, m);
    dcellfree(m);
    const dcell *c = st->mint->p[0];
    if (c && c->p[0]) memcpy(cmd, c->p[0]->p, sizeof(double) * n);
    else memset(cmd, 0, sizeof(double) * n);
    return up;
}
void ref_servo_free(void *h) { servo_free((SERVO_T *)h); }

/* Geometric WFS of one powfs, built as maos/setup_powfs.c:328-337 and :565 do:
 * pts of nx x nx points per subaperture at saloc + dx/2, loc = pts2loc(pts),
 * amp = locannular(loc, D/2, din/2) (maos/utils.c:446 mkamp without a map),
 * GS0 = mkg(loc, loc, amp, saloc, 1, 0, 0, 1).  Returns nnz of GS0. */
static loc_t *last_wloc = NULL;
static dmat *last_wamp = NULL;
static dsp *last_gs0 = NULL;
long ref_wfs_gs0(int nsa, double dsa, int nx, const double *salocx, const double *salocy, double D, double din) {
    const double dx = dsa / nx;
    pts_t *pts = ptsnew(nsa, dsa, dsa, nx, dx, dx);
    for (int isa = 0; isa < nsa; isa++) {
        pts->origx[isa] = salocx[isa] + dx * 0.5;
        pts->origy[isa] = salocy[isa] + dx * 0.5;
    }
    if (last_wloc) locfree(last_wloc);
    if (last_wamp) dfree(last_wamp);
    if (last_gs0) dspfree(last_gs0);
    last_wloc = pts2loc(pts);
    last_wamp = dnew(last_wloc->nloc, 1);
    locannular(last_wamp->p, last_wloc, 0, 0, D * 0.5, din * 0.5, 1);
    loc_t *saloc = locnew(nsa, dsa, dsa);
    memcpy(saloc->locx, salocx, sizeof(double) * nsa);
    memcpy(saloc->locy, salocy, sizeof(double) * nsa);
    last_gs0 = mkg(last_wloc, last_wloc, last_wamp, saloc, 1, 0, 0, 1);
    locfree(saloc);
    ptsfree(pts);
    return last_gs0->p[last_gs0->ny];
}
void ref_wfs_gs0_get(double *locx, double *locy, double *amp, int *p, int *i, double *x, long *nrow,
                     long *ncol) {
    const long nloc = last_wloc->nloc;
    memcpy(locx, last_wloc->locx, sizeof(double) * nloc);
    memcpy(locy, last_wloc->locy, sizeof(double) * nloc);
    memcpy(amp, last_wamp->p, sizeof(double) * nloc);
    *nrow = last_gs0->nx;
    *ncol = last_gs0->ny;
    long nnz = last_gs0->p[last_gs0->ny];
    for (long k = 0; k <= last_gs0->ny; k++) p[k] = last_gs0->p[k];
    for (long k = 0; k < nnz; k++) { i[k] = last_gs0->i[k]; x[k] = last_gs0->x[k]; }
}

/* out += prop_grid(screen on an nx x ny map, points (locx, locy)): lib/accphi.c:426. */
void ref_prop_grid(int nx, int ny, double dx, double ox, double oy, const double *screen, long nloc,
                   const double *locx, const double *locy, double alpha, double displacex, double displacey,
                   double scale, int wrap, double *out) {
    map_t *m = mk_map(nx, ny, dx, dx, ox, oy);
    memcpy(m->p, screen, sizeof(double) * nx * ny);
    loc_t *loc = locnew(nloc, dx, dx);
    memcpy(loc->locx, locx, sizeof(double) * nloc);
    memcpy(loc->locy, locy, sizeof(double) * nloc);
    prop_grid(m, loc, out, alpha, displacex, displacey, scale, wrap, 0, 0);
    locfree(loc);
    mapfree(m);
}

/* Geometric gradients of nwfs WFS of the powfs last built by ref_wfs_gs0, as
 * the reference's CPU simulation forms them: OPD on loc = sum over maps of
 * prop_grid (atmosphere: displacement ht*theta - v*dt*isim, wrap; DMs:
 * ht*theta, alpha -1, no wrap; scale 1 - ht/hs), then GS0 * OPD
 * (maos/wfsgrad.c:241 dspmm).  One WFS per thread of an OpenMP team of
 * nthread threads, as maos/sim.c runs wfsgrad_iwfs as one task per WFS;
 * idle threads take prop_grid's own taskloop chunks.  grad: [nwfs][2 nsa]. */
void ref_wfs_geom_grads(int nwfs, const double *thetax, const double *thetay, const double *hs, int nscr,
                        const int *nx, const int *ny, const double *dx, const double *ox, const double *oy,
                        const double *ht, const double *vx, const double *vy, const double *alpha, const int *wrap,
                        const double *screens, double dt, long isim, int nthread, double *grad) {
    map_t **maps = calloc(nscr, sizeof(map_t *));
    long off = 0;
    for (int s = 0; s < nscr; s++) {
        maps[s] = mk_map(nx[s], ny[s], dx[s], dx[s], ox[s], oy[s]);
        memcpy(maps[s]->p, screens + off, sizeof(double) * nx[s] * ny[s]);
        off += (long)nx[s] * ny[s];
    }
    const long nloc = last_wloc->nloc;
    dmat **opd = calloc(nwfs, sizeof(dmat *));
    for (int w = 0; w < nwfs; w++) opd[w] = dnew(nloc, 1);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthread)
    for (int w = 0; w < nwfs; w++) {
        for (int s = 0; s < nscr; s++) {
            const double sc = isfinite(hs[w]) ? 1. - ht[s] / hs[w] : 1.;
            prop_grid(maps[s], last_wloc, opd[w]->p, alpha[s], ht[s] * thetax[w] - vx[s] * dt * isim,
                      ht[s] * thetay[w] - vy[s] * dt * isim, sc, wrap[s], 0, 0);
        }
    }
    const long ng = last_gs0->nx;
    for (int w = 0; w < nwfs; w++) {
        dmat *g = dnew(ng, 1);
        dspmm(&g, last_gs0, opd[w], "nn", 1);
        memcpy(grad + w * ng, g->p, sizeof(double) * ng);
        dfree(g);
        dfree(opd[w]);
    }
    free(opd);
    for (int s = 0; s < nscr; s++) mapfree(maps[s]);
    free(maps);
}

/* ------------------------------------------------------------------------
 * Assembled DM fit (fit.square=0, fit.assemble=1): the reference's own
 * create_metapupil (math/loc.c:1471), loc_create_map_npad with its ghost
 * points (math/loc.c:208), mkw_circular (lib/mkw.c:363) and setup_fit
 * (maos/setup_recon_fit.c:303: HXF, HA, genactcpl, act_extrap, low-rank
 * terms, slaving, FR and FL assembly), then muv (lib/muv.c:37) and pcg with
 * muv on FL, as maos/recon.c:93 muv_solve runs them.
 * ---------------------------------------------------------------------- */
static loc_t *g_mp_loc = NULL;
long ref_metapupil(int ndir, const double *dirs, double D, double ht, double dx, double offset, double guard,
                   int square) {
    dmat *d = dnew(3, ndir);
    memcpy(d->p, dirs, sizeof(double) * 3 * ndir);
    map_t *map = NULL;
    create_metapupil(&map, 0, 0, d, D, ht, dx, dx, offset, guard, 0, 0, 0, square);
    if (g_mp_loc) locfree(g_mp_loc);
    g_mp_loc = map2loc(map, 0);
    mapfree(map);
    dfree(d);
    return g_mp_loc->nloc;
}
void ref_metapupil_get(double *x, double *y) {
    memcpy(x, g_mp_loc->locx, sizeof(double) * g_mp_loc->nloc);
    memcpy(y, g_mp_loc->locy, sizeof(double) * g_mp_loc->nloc);
}

static loc_t *mk_loc(long n, const double *x, const double *y, double dx, double ht, int npad) {
    loc_t *l = locnew(n, dx, dx);
    memcpy(l->locx, x, sizeof(double) * n);
    memcpy(l->locy, y, sizeof(double) * n);
    l->ht = ht;
    loc_create_map_npad(l, npad, 0, 0);
    return l;
}

/* the map of a loc: sizes and origin, then the entries (x fastest) */
static loc_t *g_map_loc = NULL;
void ref_loc_map(long n, const double *x, const double *y, double dx, int npad, long *nx, long *ny, double *ox,
                 double *oy) {
    if (g_map_loc) locfree(g_map_loc);
    g_map_loc = mk_loc(n, x, y, dx, 0, npad);
    *nx = g_map_loc->map->nx;
    *ny = g_map_loc->map->ny;
    *ox = g_map_loc->map->ox;
    *oy = g_map_loc->map->oy;
}
void ref_loc_map_get(long *out) {
    long n = g_map_loc->map->nx * g_map_loc->map->ny;
    for (long k = 0; k < n; k++) out[k] = (long)g_map_loc->map->p[k];
}

long ref_mkw_circular(long n, const double *x, const double *y, double dx, int npad, double cx, double cy,
                      double cr) {
    loc_t *loc = mk_loc(n, x, y, dx, 0, npad);
    if (last_w0) dspfree(last_w0);
    if (last_w1) dfree(last_w1);
    mkw_circular(loc, cx, cy, cr, &last_w0, &last_w1);
    locfree(loc);
    return last_w0->p[last_w0->ny];
}

static FIT_T *g_afit = NULL;
static long *g_aaoff = NULL;
static int g_andm = 0;
int ref_fit_assemble(void *hh, int nfit, const double *thetax, const double *thetay, const double *wt,
                     const double *hs, long nf, const double *flocx, const double *flocy, double fdx,
                     const int *w0p, const int *w0i, const double *w0x, const double *w1, int ndm,
                     const double *dmht, const double *dmdx, const int *nact, const double *alocx,
                     const double *alocy, int actslave, int actinterp, double actthres, double tikcr,
                     int lrt_piston, int lrt_tt) {
    refh_t *h = hh;
    FIT_T *fit = calloc(1, sizeof(FIT_T));
    fit->thetax = dnew(nfit, 1);
    fit->thetay = dnew(nfit, 1);
    fit->wt = dnew(nfit, 1);
    fit->hs = dnew(nfit, 1);
    for (int i = 0; i < nfit; i++) {
        fit->thetax->p[i] = thetax[i];
        fit->thetay->p[i] = thetay[i];
        fit->wt->p[i] = wt[i];
        fit->hs->p[i] = hs[i];
    }
    fit->xloc = h->recon->xloc;
    fit->floc = mk_loc(nf, flocx, flocy, fdx, 0, 1);
    fit->W0 = mk_csc(nf, nf, w0p, w0i, w0x);
    fit->W1 = dnew(nf, 1);
    memcpy(fit->W1->p, w1, sizeof(double) * nf);
    fit->aloc = loccellnew(ndm, 1);
    free(g_aaoff);
    g_aaoff = calloc(ndm + 1, sizeof(long));
    g_andm = ndm;
    for (int d = 0; d < ndm; d++) {
        fit->aloc->p[d] = mk_loc(nact[d], alocx + g_aaoff[d], alocy + g_aaoff[d], dmdx[d], dmht[d], 1);
        g_aaoff[d + 1] = g_aaoff[d] + nact[d];
    }
    fit->flag.tikcr = tikcr;
    fit->flag.actthres = actthres;
    fit->flag.actslave = actslave;
    fit->flag.actinterp = actinterp;
    fit->flag.nfit = nfit;
    fit->flag.lrt_piston = lrt_piston;
    fit->flag.lrt_tt = lrt_tt;
    fit->flag.alg = 1;
    fit->flag.assemble = 1;
    fit->flag.maxit = 4;
    fit->flag.cgwarm = 1;
    setup_fit(fit, 0);
    g_afit = fit;
    return 0;
}

static dsp *fitas_sp(int which) {
    switch (which) {
        case 0: return dspcell2sp((dspcell *)g_afit->FR.M);
        case 1: return dspcell2sp((dspcell *)g_afit->FL.M);
        case 2: return g_afit->actinterp ? dspcell2sp(g_afit->actinterp) : NULL;
        case 3: return g_afit->actslave ? dspcell2sp(g_afit->actslave) : NULL;
    }
    return NULL;
}
/* which: 0 FR.M, 1 FL.M, 2 actinterp, 3 actslave; CSC; returns nnz (-1: absent) */
long ref_fitas_sp(int which, int *p, int *i, double *x, long *nrow, long *ncol) {
    dsp *A = fitas_sp(which);
    if (!A) return -1;
    long nnz = A->p[A->ny];
    *nrow = A->nx;
    *ncol = A->ny;
    if (p) {
        for (long k = 0; k <= A->ny; k++) p[k] = A->p[k];
        for (long k = 0; k < nnz; k++) { i[k] = A->i[k]; x[k] = A->x[k]; }
    }
    dspfree(A);
    return nnz;
}
/* which: 0 FR.U, 1 FR.V, 2 FL.U, 3 FL.V, 4 actcpl, 5 NW; column-major */
long ref_fitas_dense(int which, double *out, long *nrow, long *ncol) {
    dcell *c = NULL;
    switch (which) {
        case 0: c = g_afit->FR.U; break;
        case 1: c = g_afit->FR.V; break;
        case 2: c = g_afit->FL.U; break;
        case 3: c = g_afit->FL.V; break;
        case 4: c = g_afit->actcpl; break;
        case 5: c = g_afit->NW; break;
    }
    if (!c) return -1;
    dmat *m = dcell2m(c);
    *nrow = m->nx;
    *ncol = m->ny;
    if (out) memcpy(out, m->p, sizeof(double) * m->nx * m->ny);
    long n = m->nx * m->ny;
    dfree(m);
    return n;
}
static dcell *avec2cell_as(const double *v) {
    dcell *c = dcellnew(g_andm, 1);
    for (int d = 0; d < g_andm; d++) {
        c->p[d] = dnew(g_aaoff[d + 1] - g_aaoff[d], 1);
        if (v) memcpy(c->p[d]->p, v + g_aaoff[d], sizeof(double) * (g_aaoff[d + 1] - g_aaoff[d]));
    }
    return c;
}
/* rhs = muv(FR, x) */
void ref_fitas_rhs(void *hh, const double *xin, double *aout) {
    refh_t *h = hh;
    dcell *x = vec2cell(xin, h->xoff, h->nps);
    dcell *a = NULL;
    muv(&a, &g_afit->FR, x, 1);
    cell2vec(aout, a, g_aaoff, g_andm);
    dcellfree(x);
    dcellfree(a);
}
/* y = muv(FL, a) */
void ref_fitas_L(const double *ain, double *aout) {
    dcell *a = avec2cell_as(ain);
    dcell *y = NULL;
    muv(&y, &g_afit->FL, a, 1);
    cell2vec(aout, y, g_aaoff, g_andm);
    dcellfree(a);
    dcellfree(y);
}
/* pcg on FL (muv) from the warm start in a */
double ref_fitas_pcg(const double *b, double *a, int warm, int maxit) {
    dcell *bb = avec2cell_as(b);
    dcell *aa = avec2cell_as(a);
    double res = pcg(&aa, muv, &g_afit->FL, NULL, NULL, bb, warm, maxit);
    cell2vec(a, aa, g_aaoff, g_andm);
    dcellfree(bb);
    dcellfree(aa);
    return res;
}

/* The grid-form fit's slaving term as the reference builds it for
 * fit.square=1 (maos/setup_recon_fit.c:72 genactcpl on HA and W1, then :165
 * slaving with sclsq = 1/nfloc); FitL then adds it (recon_utils.c:555). */
int ref_fit_setup_slave(double thres) {
    FIT_T *fit = g_fit;
    for (int d = 0; d < fit->aloc->nx; d++) loc_create_map(fit->aloc->p[d]);
    fit->actcpl = genactcpl(fit->HA, fit->W1);
    fit->actslave = slaving(fit->aloc, fit->actcpl, NULL, NULL, NULL, thres, 1. / fit->floc->nloc);
    return fit->actslave != NULL;
}

/* ------------------------------------------------------------------------
 * The gpu_* glue test: PARMS_T / RECON_T / POWFS_T / SIM_T as maos holds them
 * after setup, for the glue (maos_b200/glue/maos_gpu_glue.c) to read, and the
 * reference's own CPU tomofit (maos/recon.c:55) on a second SIM_T for the
 * comparison.  gpu_fit 1: the assembled fit of ref_fit_assemble; 2: the grid
 * fit of ref_fit_setup (+ ref_fit_setup_slave).
 * ---------------------------------------------------------------------- */
static SIM_T *g_cpu_simu = NULL;
static dcell *g_cpu_dm = NULL;
static void glue_simu(refh_t *h, SIM_T *s) {
    s->parms = h->parms;
    s->recon = h->recon;
    s->powfs = h->powfs;
    s->cgres = dcellnew(2, 1);
    s->cgres->p[0] = dnew(100000, 1);
    s->cgres->p[1] = dnew(100000, 1);
    s->isim = s->reconisim = 0;
}
int ref_glue_prepare(void *hh, int gpu_fit, int tomo_maxit, int fit_maxit) {
    refh_t *h = hh;
    PARMS_T *parms = h->parms;
    RECON_T *recon = h->recon;
    FIT_T *fit = gpu_fit == 2 ? g_fit : g_afit;
    if (!fit) return -1;
    const int ndm = (int)fit->aloc->nx;
    parms->recon.alg = 0;
    if (!parms->dbg.tomo_maxit) parms->dbg.tomo_maxit = lnew(0, 1);
    parms->gpu.tomo = 1;
    parms->gpu.fit = gpu_fit;
    parms->tomo.maxit = tomo_maxit;
    parms->fit.maxit = fit_maxit;
    parms->ndm = ndm;
    parms->fit.nfit = (int)fit->thetax->nx;
    parms->fit.thetax = fit->thetax;
    parms->fit.thetay = fit->thetay;
    parms->fit.wt = fit->wt;
    parms->fit.hs = fit->hs;
    recon->fit = fit;
    recon->aloc = fit->aloc;
    recon->anloc = lnew(ndm, 1);
    recon->anx = lnew(ndm, 1);
    recon->any = lnew(ndm, 1);
    recon->amap = mapcellnew(ndm, 1);
    for (int d = 0; d < ndm; d++) {
        loc_create_map(fit->aloc->p[d]);
        recon->amap->p[d] = fit->aloc->p[d]->map;
        recon->amap->p[d]->h = fit->aloc->p[d]->ht;
        recon->anloc->p[d] = fit->aloc->p[d]->nloc;
        recon->anx->p[d] = recon->amap->p[d]->nx;
        recon->any->p[d] = recon->amap->p[d]->ny;
    }
    recon->fmap = recon->pmap;
    recon->W0 = fit->W0;
    recon->W1 = fit->W1;
    /* the CPU path: muv_solve on RL/RR (tomography) and FL/FR (fit) */
    recon->RR.Mfun = TomoR;
    recon->RR.Mdata = recon;
    recon->RL.Mfun = TomoL;
    recon->RL.Mdata = recon;
    recon->RL.pfun = parms->tomo.precond == 1 ? fdpcg_precond : NULL;
    recon->RL.pdata = recon;
    recon->RL.alg = 1;
    recon->RL.warm = 1;
    recon->RL.maxit = tomo_maxit;
    fit->FL.alg = 1;
    fit->FL.warm = 1;
    fit->FL.maxit = fit_maxit;
    if (!fit->FR.M) { /* the grid fit is not assembled: FitR / FitL (recon_utils.c:483,536) */
        fit->FR.Mfun = FitR;
        fit->FR.Mdata = fit;
        fit->FL.Mfun = FitL;
        fit->FL.Mdata = fit;
    }
    glue_simu(h, h->simu);
    g_cpu_simu = calloc(1, sizeof(SIM_T));
    glue_simu(h, g_cpu_simu);
    return ndm;
}
void ref_glue_handles(void *hh, void **out) {
    refh_t *h = hh;
    out[0] = h->parms;
    out[1] = h->powfs;
    out[2] = h->recon;
    out[3] = h->simu;
}
/* gradients as maos hands them: one column of 2 nsa per WFS */
void *ref_glue_grad_cell(void *hh, const double *g) {
    refh_t *h = hh;
    dcell *c = dcellnew(h->nwfs, 1);
    for (int w = 0; w < h->nwfs; w++) {
        c->p[w] = dnew(h->goff[w + 1] - h->goff[w], 1);
        memcpy(c->p[w]->p, g + h->goff[w], sizeof(double) * (h->goff[w + 1] - h->goff[w]));
    }
    return c;
}
void ref_glue_cell_free(void *c) {
    dcell *d = c;
    dcellfree(d);
}
long ref_glue_cell_get(void *c, double *out) {
    dcell *d = c;
    long off = 0;
    for (int i = 0; i < d->nx * d->ny; i++)
        if (d->p[i]) {
            if (out) memcpy(out + off, d->p[i]->p, sizeof(double) * d->p[i]->nx * d->p[i]->ny);
            off += d->p[i]->nx * d->p[i]->ny;
        }
    return off;
}
/* the reference's CPU tomography + fit of one step (its own tomofit) */
double ref_glue_cpu_step(void *grad, double *dmout) {
    tomofit(&g_cpu_dm, g_cpu_simu, (dcell *)grad);
    ref_glue_cell_get(g_cpu_dm, dmout);
    g_cpu_simu->reconisim++;
    return g_cpu_simu->cgres->p[1]->p[g_cpu_simu->reconisim - 1];
}
/* install a control matrix (nact x ngrad, column-major) as recon->MVM */
void ref_glue_set_mvm(void *hh, const double *M, long nact, long ngrad) {
    refh_t *h = hh;
    dfree(h->recon->MVM);
    h->recon->MVM = dnew(nact, ngrad);
    memcpy(h->recon->MVM->p, M, sizeof(double) * nact * ngrad);
}
/* a DM command cell shaped like recon->anloc (or the grid sizes) */
void *ref_glue_dm_cell(void *hh, int grid) {
    refh_t *h = hh;
    RECON_T *r = h->recon;
    return grid ? dcellnew3(h->parms->ndm, 1, r->anx->p, r->any->p) : dcellnew3(h->parms->ndm, 1, r->anloc->p, NULL);
}
