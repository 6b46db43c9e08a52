/*
 * maos_b200 -- B200-native wavefront reconstruction for the MAOS adaptive
 * optics simulator: WFS gradients in, tomography (CG or FDPCG), DM fit (CG),
 * actuator commands out, plus the precomputed control-matrix MVM.
 *
 * C ABI.  Only plain pointers, sizes and POD structs cross it.  Each entry
 * point stands in for one function of the reference's GPU interface
 * (cuda/gpu.h); the citation is given beside each declaration.  The
 * reference passes its simulator structs (PARMS_T, RECON_T, SIM_T); this ABI
 * takes the same information as flat arrays, so the glue a maintainer adds to
 * maos (the gpu_* functions of maos_b200/glue/maos_gpu_glue.c) copies fields out of
 * RECON_T into the descriptors below.
 *
 * Conventions (same as the reference's dmat / map_t / dsp):
 *   - grids: point (ix, iy) sits at (ox + ix*dx, oy + iy*dy), stored at
 *     ix + iy*nx;
 *   - gradients of one WFS: nsa x-slopes then nsa y-slopes;
 *   - sparse matrices: compressed sparse column (p: ncol+1, i, x);
 *   - complex arrays: interleaved (re, im) doubles; matrices column-major.
 *
 * Every call returns MB_OK (0) or a negative MB_E* code; mb_error_string()
 * and mb_last_error_message() describe the last failure.  Nothing aborts the
 * process (the reference aborts on any CUDA error, cuda/common.h:103).
 */
#ifndef MAOS_B200_H
#define MAOS_B200_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define MB_OK 0
#define MB_EINVAL (-1)   /* invalid descriptor or argument */
#define MB_ECUDA (-2)    /* CUDA runtime / library error */
#define MB_ENOMEM (-3)   /* device allocation failed */
#define MB_ESTATE (-4)   /* call not valid in the current state */
#define MB_EUNSUP (-5)   /* geometry the kernels do not support */
#define MB_ENUM (-6)     /* non-finite input or CG breakdown */

typedef struct mb_recon mb_recon; /* one reconstructor bound to one GPU */

/* A square or rectangular sampling grid (map_t). */
typedef struct {
    int nx, ny;
    double dx, dy;
    double ox, oy;
    double ht; /* conjugation height (m) */
} mb_grid;

/* One wavefront sensor as the tomography sees it (RECON_T per-WFS fields). */
typedef struct {
    double thetax, thetay; /* direction (rad) */
    double hs;             /* guide-star range (m); INFINITY for NGS */
    int nsa;               /* subapertures */
    double dsa;            /* subaperture size (m) */
    const double *salocx;  /* [nsa] lower-left corners (m) */
    const double *salocy;  /* [nsa] */
    /* GP: (2*nsa) x (pmap.nx*pmap.ny) average-gradient operator, CSC
       (recon->GP->p[iwfs]). */
    const int *gp_p;
    const int *gp_i;
    const double *gp_x;
    /* inverse NEA per subaperture, [cx, cy, cxy] x nsa, already scaled by
       TOMOSCALE (recon->saneai diagonal block, tomo.cu:111 convert_neai) */
    const double *neai;
    /* 2 x (2*nsa) column-major tip/tilt projector (recon->PTT diagonal
       block), NULL when the WFS has no tip/tilt removal */
    const double *ptt;
} mb_wfs_desc;

/* What the device needs to form the FDPCG block matrices' data term itself
 * (the WFS sum of maos/fdpcg.c:427-480: prop' (gx' sel' sel gx + gy' sel' sel
 * gy) prop / neam^2 per WFS), so a change of the WFS noise is absorbed on the
 * GPU (mb_update_recon_neam).  All of it is geometry fixed at setup except
 * neam. */
typedef struct {
    int nxp, nyp;          /* pupil frequency grid of the data term (nx0/os0 * tomo.pos) */
    double dxp;            /* its sampling (recon->ploc->dx) */
    int pos;               /* pupil frequencies aliasing to one block, per axis (tomo.pos) */
    int adimx, adimy;      /* blocks per axis (nx0/os0, ny0/os0) */
    const double *gx, *gy; /* [nyp][nxp] complex (re, im), fftshifted: average-gradient
                              transfer functions (fdpcg.c:199 fdpcg_g) */
    int nsel;              /* entries of the selection autocorrelation */
    const int *sel_dx, *sel_dy; /* their shifts on the pupil frequency grid (mod nxp, nyp) */
    const double *sel_r;   /* [nsel] complex (re, im): R(d) = sum_s conj(v_{s+d}) v_s over the
                              kept coefficients v of fdpcg_saselect (fdpcg.c:71) */
    int needscale;         /* fdpcg->scale: 0 multiplies the term by nx0*ny0 (fdpcg.c:498) */
    const double *neam;    /* [nwfs] mean NEA per WFS at setup (recon->neam, TOMOSCALE units) */
} mb_fdpcg_geom;

/* Fourier-domain preconditioner tables (recon->fdpcg, maos/fdpcg.c:331). */
typedef struct {
    int nb, bs;          /* blocks and block size */
    int scale;           /* 1: FFTs scaled by 1/sqrt(nx*ny) (fdpcg->scale) */
    const long *perm;    /* [nb*bs] fdpcg->perm (shift=1, full spectrum) */
    const double *mbinv; /* [nb*bs*bs*2] fdpcg->Mbinv, complex, column-major blocks */
    /* Optional (both or neither; no reference counterpart): the block matrix
       before inversion, split into its WFS term [nb*bs*bs*2] (complex,
       column-major blocks) and its diagonal invpsd term [nb*bs] at the l2c
       passed with this descriptor.  With them the device keeps the data term,
       and mb_update_recon_cn2(r, l2c, NULL) rebuilds Mbinv on the GPU (the
       invpsd term scales with each layer's l2c). */
    const double *mdata;
    const double *mdiag;
    /* Optional (needs mdiag; no reference counterpart): the data term's
       geometry; the device then forms the data term itself (mdata may be
       NULL) and mb_update_recon_neam rebuilds the blocks for new noise. */
    const mb_fdpcg_geom *geom;
} mb_fdpcg_desc;

/* A sparse matrix in compressed sparse column form (the reference's dsp). */
typedef struct {
    int nrow, ncol;
    const int *p;          /* [ncol+1] column starts; NULL: no matrix */
    const int *i;          /* [nnz] row indices */
    const double *x;       /* [nnz] values */
} mb_csc;

/* DM fit in grid form (cuda/fit.cu cufit_grid; recon->fit, maos/setup_recon_fit.c):
 *   FitR x = sum_f wt_f HA_f^T (W0 - W1 W1^T) Hxp_f x
 *   FitL a = sum_f wt_f HA_f^T (W0 - W1 W1^T) HA_f a + NW NW^T a
 * HA and Hxp are bilinear ray tracing onto the fit grid, built internally from
 * the grids below (the grid form requires fit.square=1: every point of each
 * DM grid is an actuator, maos/setup_parms.c:3001). */
typedef struct {
    mb_grid floc;          /* fit grid (recon->fmap) */
    int nfit;              /* fit directions */
    const double *thetax;  /* [nfit] (rad) */
    const double *thetay;
    const double *wt;      /* [nfit] fit.wt */
    const double *hs;      /* [nfit] fit.hs (INFINITY for science directions) */
    const int *w0_p;       /* W0: nfloc x nfloc CSC (recon->W0) */
    const int *w0_i;
    const double *w0_x;
    const double *w1;      /* [nfloc] recon->W1 */
    int ndm;
    const mb_grid *amap;   /* [ndm] actuator grids with ht (recon->amap) */
    int nnw;               /* low-rank columns (fit->NW) */
    const double *nw;      /* [nact_total x nnw] column-major, DMs concatenated */
    int maxit;             /* fit.maxit */
    /* Optional slaving term added to FitL (recon->fit->actslave on the DM
       grids, applied by cufit_grid::L, cuda/fit.cu:232-234): nact_total x
       nact_total; p NULL when there is none. */
    mb_csc actslave;
} mb_fit_desc;

/* The assembled DM fit, the reference's default GPU fit (gpu.fit=1:
 * cuda/solve.cu cusolve_sparse over recon->fit->FR and FL, the sparse plus
 * low-rank MUV_T of lib/muv.c:37):
 *   rhs  = FR.M x - FR.U (FR.V^T x)
 *   FL a = FL.M a - FL.U (FL.V^T a)
 * then CG on FL warm-started from the previous commands (curecon_t::fit,
 * cuda/recon.cu:277).  Any actuator set works, in particular fit.square=0
 * (actuators inside the metapupil, the reference default); the actuators of
 * all DMs are concatenated in recon->aloc order.  FL.M carries the Tikhonov
 * and slaving terms, and HA inside FR and FL the extrapolation to weakly
 * coupled actuators, as maos/setup_recon_fit.c:186-293 assembles them. */
typedef struct {
    mb_csc frm;            /* nact x nxtot: fit->FR.M, its DM x layer blocks as one matrix */
    int nfr;               /* columns of FR.U and FR.V (<= 16) */
    const double *fru;     /* [nact x nfr] column-major (fit->FR.U) */
    const double *frv;     /* [nxtot x nfr] column-major (fit->FR.V) */
    mb_csc flm;            /* nact x nact: fit->FL.M */
    int nfl;               /* columns of FL.U and FL.V (<= 16) */
    const double *flu;     /* [nact x nfl] column-major (fit->FL.U) */
    const double *flv;     /* [nact x nfl] column-major (fit->FL.V) */
    int maxit;             /* fit.maxit */
} mb_fit_sparse_desc;

/* Everything gpu_setup_recon (cuda/recon.cu:477) reads. */
typedef struct {
    mb_grid pmap;          /* pupil grid of ploc (tomo.square=1) */
    int nps;               /* reconstructed layers */
    const mb_grid *xmap;   /* [nps] layer grids (ht set) */
    const double *l2c;     /* [nps] biharmonic weight (laplacian_coef/4)^2*cxxscale*TOMOSCALE */
    int nwfs;
    const mb_wfs_desc *wfs;
    int maxit;             /* tomo.maxit */
    int precond;           /* 0: CG, 1: FDPCG (tomo.precond) */
    int split;             /* recon.split: non-zero skips tip/tilt removal in the LHS */
    const mb_fdpcg_desc *fdpcg; /* required when precond==1 */
    int nbatch;            /* independent instances sharing these tables (>=1) */
    const mb_fit_desc *fit; /* optional DM fit in grid form (NULL: none) */
    /* optional assembled DM fit (gpu.fit=1, the reference default); at most
       one of fit and fit_sparse */
    const mb_fit_sparse_desc *fit_sparse;
} mb_recon_desc;

/* gpu_init (cuda/gpu.h:27): select the device for subsequent setups. */
int mb_init(int device);
/* gpu_cleanup (cuda/gpu.h:28). */
void mb_cleanup(void);

/* gpu_setup_recon (cuda/gpu.h:47): build a reconstructor on the current device. */
int mb_setup_recon(const mb_recon_desc *desc, mb_recon **out);
/* gpu_recon_free (declared at cuda/gpu.h:54). */
void mb_recon_free(mb_recon *r);
/* gpu_recon_reset (cuda/gpu.h:52): zero the warm-start state of every instance. */
int mb_recon_reset(mb_recon *r);
/* gpu_update_recon (cuda/gpu.h:49): new NEA (and tip/tilt projector) for one WFS. */
int mb_update_recon_nea(mb_recon *r, int iwfs, const double *neai, const double *ptt);
/* gpu_update_recon_cn2 (cuda/gpu.h:50): new layer weights and FDPCG blocks.
 * fdpcg NULL (FDPCG on): the blocks are rebuilt on the GPU from the data term
 * kept at setup (mb_fdpcg_desc.mdata/mdiag), with invpsd scaled by the new
 * l2c; MB_EINVAL when no data term was given. */
int mb_update_recon_cn2(mb_recon *r, const double *l2c, const mb_fdpcg_desc *fdpcg);

/* The FDPCG part of gpu_update_recon (cuda/gpu.h:49; maos recomputes
 * recon->fdpcg with fdpcg_prepare after the noise changes): new mean NEA per
 * WFS (recon->neam), the data term formed on the device from the geometry of
 * mb_fdpcg_desc.geom, the blocks inverted and folded on the device, in place
 * (the step graphs keep working).  MB_EINVAL when no geometry was given. */
int mb_update_recon_neam(mb_recon *r, const double *neam);
/* The device's FDPCG data term [nb][bs][bs] complex (re, im), column-major
 * blocks, as mb_fdpcg_desc.mdata (for checks). */
int mb_fdpcg_data(mb_recon *r, double *out);

/* gpu_tomo (cuda/gpu.h:55, curecon_t::tomo cuda/recon.cu:259).
 * grad: [nbatch][ngrad] host FP64 gradients.  opdr: optional host output
 * [nbatch][nxtot].  cgres: optional [nbatch] final CG residual |r|/|b|. */
int mb_tomo(mb_recon *r, const double *grad, double *opdr, float *cgres);

/* gpu_tomo with maos's own gradient cells (the dcell gradin of
 * cuda/recon.cu:564, one column per WFS), one instance (nbatch 1): grad[iwfs]
 * points at that WFS's 2*nsa FP64 gradients, x then y (NULL: zeros).  They are
 * converted straight from the columns into a pinned staging buffer, with no
 * concatenated copy.  opdr (may be NULL; NULL entries skipped): per-layer FP64
 * outputs of nx*ny points (the copy to simu->opdr, cuda/recon.cu:574-580).
 * cgres: optional final CG residual. */
int mb_tomo_wfs(mb_recon *r, const double *const *grad, double *const *opdr, float *cgres);

/* gpu_fit when the tomography ran on the CPU (gpu.tomo=0: curecon_t::fit
 * copies simu->opdr to the device first, cuda/recon.cu:278-281), one instance:
 * opdr[ips] the host FP64 layer OPD (NULL: zeros); it replaces the device's
 * layer solution, then the fit runs as in mb_fit.  dmout: [nact] FP64. */
int mb_fit_opdr(mb_recon *r, const double *const *opdr, double *dmout, float *cgres);

/* gpu_fit (cuda/gpu.h:56, curecon_t::fit cuda/recon.cu:277): DM fit of the
 * current tomography solution.  dmout: [nbatch][nact] host FP64 actuator
 * commands (overwritten, like add2cpu(...,0,...) at recon.cu:285).  cgres:
 * optional [nbatch] fit CG residual. */
int mb_fit(mb_recon *r, double *dmout, float *cgres);
/* One whole reconstruction step (tomography then fit) on the device, one
 * graph launch: d_grad [nbatch][ngrad] FP32 device in; the actuator commands
 * stay on the device (mb_fit_solution). */
int mb_recon_step_device(mb_recon *r, const float *d_grad, void *stream);
/* Device pointer to the FP32 DM commands [nbatch][nact]. */
const float *mb_fit_solution(mb_recon *r);

/* Reconstructors of different geometries stepped together (uneven
 * instances: e.g. 8 m SCAO, 8 m LTAO and 30 m MCAO pools).  No counterpart in
 * the reference, which runs one reconstructor per simulation (curecon_t,
 * cuda/recon.cu:477).  One captured graph advances every member by one step
 * (tomography + fit, as mb_recon_step_device): the tomography operators (the
 * RHS and each CG iteration's A p, k_pupil_rows + k_hxt_rows) are one launch
 * over all members' instances, each block reading its member's tables from
 * a per-member argument table; each member's CG vector updates,
 * preconditioner and fit run between them, members overlapping.  A member's
 * result equals its own mb_recon_step_device's.  Members must share the
 * device and the tomography iteration count; at creation their padded list
 * widths are made equal (exact zeros added; their own graphs are
 * recaptured).  A member stays owned by the caller and must outlive the
 * group; after a member's tables change (updates, autotune) the next step
 * recaptures the group's graph.  At most 8 members per grouped launch (more
 * members take more launches). */
typedef struct mb_group mb_group;
int mb_group_create(mb_recon *const *members, int n, mb_group **out);
/* d_grad[i]: member i's FP32 gradients [nbatch_i][ngrad_i] on the device;
 * the commands stay in each member's mb_fit_solution. */
int mb_group_step_device(mb_group *g, const float *const *d_grad, void *stream);
/* Kernel launches of one group step (the captured graph's kernels). */
long mb_group_graph_kernels(const mb_group *g);
void mb_group_free(mb_group *g);
long mb_nact(const mb_recon *r);

/* Device-resident form of mb_tomo for batched serving and benchmarks:
 * d_grad is a device FP32 buffer [nbatch][ngrad]; stream is a cudaStream_t
 * (NULL = the legacy default stream).  Returns after enqueueing. */
int mb_tomo_device(mb_recon *r, const float *d_grad, void *stream);
/* The reconstructor's own stream (a cudaStream_t), used by mb_tomo. */
void *mb_recon_stream(mb_recon *r);
/* Device pointer to the FP32 tomography solution [nbatch][nxtot]. */
const float *mb_tomo_solution(mb_recon *r);
/* Copy the last residuals [nbatch] (synchronises the stream). */
int mb_tomo_residual(mb_recon *r, float *cgres);

/* ---- Serving: instances as slots ----
 * No counterpart in the reference (one curecon_t serves one simulation).
 * Each of the nbatch instances is a slot holding one AO system's warm-start
 * state.  A masked step advances only the slots whose flag is non-zero;
 * every other slot's state is left untouched and no slot's result depends on
 * which other slots ran.  All four calls enqueue on `stream` and return. */
/* Zero one slot's warm-start state (layer OPD and DM commands). */
int mb_recon_reset_slot(mb_recon *r, int slot, void *stream);
/* Copy one slot's FP32 gradients [ngrad] (host, pinned for asynchrony, or
 * device) into the reconstructor. */
int mb_slot_upload(mb_recon *r, int slot, const float *grad, void *stream);
/* Copy one slot's FP32 result out: DM commands [nact] with a fit, else the
 * layer OPD [nxtot]. */
int mb_slot_download(mb_recon *r, int slot, float *out, void *stream);
/* One step (tomography, then the fit if set up) of the slots with
 * active[slot] != 0; active is a host array [nbatch], read before return. */
int mb_recon_step_slots(mb_recon *r, const int *active, void *stream);
/* The three in one call: gradients of the active slots from grad
 * [nbatch][ngrad], one masked step, their results into out [nbatch][nact]
 * (or [nbatch][nxtot] without a fit); rows of inactive slots are neither
 * read nor written.  Pinned host or device buffers; one copy per run of
 * consecutive active slots each way. */
int mb_recon_serve_step(mb_recon *r, const int *active, const float *grad, float *out, void *stream);

/* Autotuner (no counterpart in the reference): times the tomography
 * operator with each admissible row blocking of its pupil-grid kernel (4, 8,
 * 16 pupil rows per CTA, and every even split of the pupil rows into blocks
 * of 1 to 32 rows) and the y-half kernel's CTA size (256, 128 or 64 threads)
 * on this batch size, keeps the fastest, then times whole
 * tomography steps with each form of the FDPCG preconditioner
 * (mb_fdpcg_mode; the three-kernel form at each batch shape of
 * mb_fdpcg_shape) and keeps the fastest, then whole steps with and without
 * programmatic dependent launch between the graph's kernels (faster for one
 * instance, slower for a few), and captures the step graphs again;
 * the instances restart cold.  The row blocking does not change results, the
 * preconditioner's form changes them only at FP32 rounding.  rows (may be
 * NULL): the blocking kept; ms (may be NULL, 3 floats): ms per operator for
 * 4, 8, 16 rows, -1 where a blocking does not fit. */
int mb_autotune(mb_recon *r, int reps, int *rows, float *ms);

/* Form of the FDPCG preconditioner inside the CG step (no counterpart in the
 * reference; mb_autotune picks the faster for the batch size): 1 = three
 * kernels (forward FFTs of every (layer, instance), block solve sharing the
 * blocks over instances, inverse FFTs), 2 = one kernel per step in which the
 * layers of an instance are split over one thread-block cluster of up to 16
 * CTAs that exchange rows, columns and block members through distributed
 * shared memory, 0 = 2 when that cluster fits on the device, -1 = no change
 * (query).  Results agree to FP32 rounding.  The step graphs are captured
 * again.  Returns the form in use (1 or 2) or a negative MB_E* code. */
int mb_fdpcg_mode(mb_recon *r, int mode);

/* Batch shape of the three-kernel FDPCG form (no counterpart in the
 * reference): instances per CTA of the block solve, 2, 4, 8 or 16 (more read
 * the shared block matrices fewer times, fewer give more CTAs), -1 = query.
 * Results do not depend on it.  The step graphs are captured again.  Returns
 * the shape in use or a negative MB_E* code. */
int mb_fdpcg_shape(mb_recon *r, int ni);

/* Servo filter on the device (no GPU counterpart in the reference; the CPU
 * code is lib/servo.c servo_new / servo_filter / servo_reset, used by
 * maos/filter.c filter_dm): the integrator that turns the per-step DM
 * command errors into DM commands, for n values (e.g. nbatch instances x
 * nact actuators) in FP64 on the device.  ap: the integrator history
 * coefficients (NULL: {1}); al: extra latency in steps; ep (column-major
 * ep_nx x ep_ny): ep_nx 1 = type I gain (ep_ny 1, or one per mode with
 * n a multiple of ep_ny), 2 = PID (2 x 1), 3 = type II (gain, a, T per
 * column); dt: the loop period.  mb_servo_filter takes one step: d_merr
 * (device, n doubles) in, d_cmd (device, n doubles) = the new commands
 * (mint[0]) out, on `stream`. */
typedef struct mb_servo mb_servo;
int mb_servo_create(long n, const double *ap, int nap, int al, const double *ep, int ep_nx, int ep_ny, double dt,
                    mb_servo **out);
int mb_servo_filter(mb_servo *s, const double *d_merr, double *d_cmd, void *stream);
int mb_servo_reset(mb_servo *s);
void mb_servo_free(mb_servo *s);

/* ---- Geometric Shack-Hartmann WFS (the simulation side upstream of mb_tomo) ----
 * Replaces the geometric branch of cuda/gpu.h gpu_wfsgrad_queue
 * (cuda/wfsgrad.cu gpu_wfsgrad_iwfs with powfs.gtype_sim = 0: the OPD of the
 * atmosphere, cuda/accphi.cu:508 gpu_atm2loc, minus the DMs, :556
 * gpu_dm2loc, then GS0 * OPD and add_geom_noise_do, cuda/wfsgrad.cu:47),
 * with the screens of cuda/gpu.h gpu_atm2gpu and the DM commands of
 * gpu_dmreal2gpu given as arguments.
 *
 * Each WFS's OPD points lie on a fine square grid (spacing dx, grid index
 * (0, 0) at (gox, goy)); subaperture j's nxsa x nxsa points start at grid
 * index (sa_ix, sa_iy), and its average-gradient stencil (the rows of the
 * reference's GS0 = mkg(loc, loc, amp, saloc, 1, 0, 0, 1),
 * maos/setup_powfs.c:565) is stencils[stencil_off[sa_stencil[j]] ...]: the
 * x weights then the y weights of the (nxsa+2)^2 grid points from
 * (sa_ix-1, sa_iy-1), row-major.  Per-subaperture arrays are concatenated
 * over WFS.  nea (may be NULL): per WFS [3][nsa] sqrt-NEA xx, yy, xy (rad).
 * Atmosphere layer l: an atm_nx x atm_ny map (x fastest) of spacing atm_dx,
 * origin (atm_ox, atm_oy), height atm_ht, wind (atm_vx, atm_vy) m/s, seen
 * with wrap-around.  DM m: a dm_nx x dm_ny actuator map (the commands of one
 * instance are the DM maps concatenated), no wrap-around.  nbatch
 * instances each have their own atmosphere and DM commands. */
typedef struct {
    int nwfs;
    const int *nsa, *nxsa;
    const double *dx, *gox, *goy;
    const double *thetax, *thetay, *hs;    /* rad, rad, m (inf: natural guide star) */
    const int *sa_ix, *sa_iy, *sa_stencil;
    int nstencil;
    const long *stencil_off;
    const double *stencils;
    long stencil_len;
    const double *nea;
    int natm;
    const int *atm_nx, *atm_ny;
    const double *atm_dx, *atm_ox, *atm_oy, *atm_ht, *atm_vx, *atm_vy;
    int ndm;
    const int *dm_nx, *dm_ny;
    const double *dm_dx, *dm_ox, *dm_oy, *dm_ht;
    double dt;                              /* sim.dt: the atmosphere moves v dt per step */
    int nbatch;
} mb_geom_wfs_desc;
typedef struct mb_geom_wfs mb_geom_wfs;
int mb_geom_wfs_create(const mb_geom_wfs_desc *d, mb_geom_wfs **out);
/* Upload one atmosphere layer of one instance (host FP64, stored FP32). */
int mb_geom_wfs_set_atm(mb_geom_wfs *w, int inst, int layer, const double *screen);
/* Wind of one layer of one instance (m/s; the descriptor's atm_vx, atm_vy
 * are every instance's at creation). */
int mb_geom_wfs_set_wind(mb_geom_wfs *w, int inst, int layer, double vx, double vy);
/* Gradients of step isim (atmosphere shifted by v dt isim): d_dm (device
 * FP32 [nbatch][nact], NULL: open loop) is subtracted; d_grad (device FP32
 * [nbatch][ngrad], each WFS x then y) is written; seed != 0 adds the noise,
 * drawn from (seed, subaperture, WFS, isim, instance). */
int mb_geom_wfs_grad(mb_geom_wfs *w, long isim, const float *d_dm, float *d_grad, unsigned long long seed,
                     void *stream);
long mb_geom_wfs_ngrad(const mb_geom_wfs *w);
long mb_geom_wfs_nact(const mb_geom_wfs *w);
void mb_geom_wfs_free(mb_geom_wfs *w);

/* Sizes of the bound geometry. */
long mb_ngrad(const mb_recon *r);
long mb_nxtot(const mb_recon *r);
int mb_nbatch(const mb_recon *r);

/* Single operator applications, for parity tests.  All host FP64, [nbatch][n]. */
int mb_apply_tomo_R(mb_recon *r, const double *grad, double *xout);    /* TomoR */
int mb_apply_tomo_L(mb_recon *r, const double *xin, double *xout);     /* TomoL */
int mb_apply_fdpcg(mb_recon *r, const double *xin, double *xout);      /* fdpcg_precond */
int mb_apply_hx(mb_recon *r, const double *xin, double *opd);          /* Hx: [nbatch][nwfs][np] */
int mb_apply_fit_R(mb_recon *r, const double *xin, double *aout);      /* FitR */
int mb_apply_fit_L(mb_recon *r, const double *ain, double *aout);      /* FitL */

/* ---- Control-matrix MVM (recon.mvm): a = M g ---- */
#define MB_MVM_F32 0   /* FP32 storage */
#define MB_MVM_BF16 1  /* BF16 storage */
#define MB_MVM_FP8 2   /* FP8-E4M3 storage with one FP32 scale per row */
typedef struct mb_mvm mb_mvm;
/* gpu_setup_recon_mvm (cuda/gpu.h:48): install the control matrix.  Mcol is
 * recon->MVM: nact x ngrad, column-major FP64.  It is converted once to the
 * requested storage type; products accumulate in FP32.  nbatch instances
 * share M and are applied together. */
int mb_mvm_create(const double *Mcol, long nact, long ngrad, int dtype, int nbatch, mb_mvm **out);
void mb_mvm_free(mb_mvm *m);
/* Bytes of control-matrix storage on the device (M plus row scales). */
long mb_mvm_bytes(const mb_mvm *m);
/* gpu_recon_mvm (cuda/gpu.h:57): host FP64 gradients [nbatch][ngrad] in,
 * host FP64 DM commands [nbatch][nact] out (overwritten). */
int mb_recon_mvm(mb_mvm *m, const double *grad, double *dmout);
/* Device form: FP32 [nbatch][ngrad] in, FP32 [nbatch][nact] out, on `stream`. */
int mb_mvm_apply_device(mb_mvm *m, const float *d_grad, float *d_out, void *stream);

/* Allocation-free FP32 MVM.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory -- a real-time control loop
 * that must never block on cudaMalloc (which can synchronise the device and
 * take unbounded time), or code that runs where allocation is not allowed.
 * The caller passes M (device, FP32, row-major nact x ngrad with leading
 * dimension ldm: ldm >= ngrad, ldm a multiple of 4, M 16-byte aligned), the
 * gradients d_grad [nbatch][ngrad] and the output d_out [nbatch][nact], all on
 * the device.  The split-K partial sums go to one static device array of
 * MB_NOALLOC_MAX_PARTIALS floats (4 MiB, held by every GPU that loads the
 * library until exit); a call needing more, ceil(ngrad/2048)*nbatch*nact,
 * returns MB_EINVAL with the sizes in the message.  The first call on a device
 * looks up the array's address on that device; make that first call before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * race.  It calls no cudaMalloc/cudaFree. */
#define MB_NOALLOC_MAX_PARTIALS 1048576
int mb_mvm_apply_noalloc(const float *d_M, long nact, long ngrad, long ldm, const float *d_grad,
                         float *d_out, int nbatch, void *stream);

/* Per-stage timing for roofline accounting.  Stages are the kernels of one
 * CG iteration (see mb_stage_name).  For each stage: average device time of
 * one launch over `reps` back-to-back launches on the reconstructor's stream
 * (ms), the algorithmic bytes one launch must move (each operand read or
 * written once), and how many launches one mb_tomo step makes. */
int mb_num_stages(void);
const char *mb_stage_name(int stage);
int mb_time_stages(mb_recon *r, int reps, float *ms, double *bytes, int *launches_per_step);

/* Number of kernels this library enqueued since the last reset of the counter. */
long mb_kernel_launches(int reset);

const char *mb_error_string(int code);
const char *mb_last_error_message(void);
int mb_version(void);

#ifdef __cplusplus
}
#endif
#endif
