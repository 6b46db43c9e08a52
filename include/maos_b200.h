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
 * maos copies fields out of RECON_T into the descriptors
 * below.
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

/* Fourier-domain preconditioner tables (recon->fdpcg, maos/fdpcg.c:331). */
typedef struct {
    int nb, bs;          /* blocks and block size */
    int scale;           /* 1: FFTs scaled by 1/sqrt(nx*ny) (fdpcg->scale) */
    const long *perm;    /* [nb*bs] fdpcg->perm (shift=1, full spectrum) */
    const double *mbinv; /* [nb*bs*bs*2] fdpcg->Mbinv, complex, column-major blocks */
} mb_fdpcg_desc;

/* Everything gpu_setup_recon (cuda/recon.cu:477) reads for tomography. */
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
} mb_tomo_desc;

/* gpu_init (cuda/gpu.h:27): select the device for subsequent setups. */
int mb_init(int device);
/* gpu_cleanup (cuda/gpu.h:28). */
void mb_cleanup(void);

/* gpu_setup_recon (cuda/gpu.h:47): build a reconstructor on the current device. */
int mb_setup_recon(const mb_tomo_desc *desc, mb_recon **out);
/* gpu_recon_free (declared at cuda/gpu.h:54). */
void mb_recon_free(mb_recon *r);
/* gpu_recon_reset (cuda/gpu.h:52): zero the warm-start state of every instance. */
int mb_recon_reset(mb_recon *r);
/* gpu_update_recon (cuda/gpu.h:49): new NEA (and tip/tilt projector) for one WFS. */
int mb_update_recon_nea(mb_recon *r, int iwfs, const double *neai, const double *ptt);
/* gpu_update_recon_cn2 (cuda/gpu.h:50): new layer weights and FDPCG blocks. */
int mb_update_recon_cn2(mb_recon *r, const double *l2c, const mb_fdpcg_desc *fdpcg);

/* gpu_tomo (cuda/gpu.h:55, curecon_t::tomo cuda/recon.cu:259).
 * grad: [nbatch][ngrad] host FP64 gradients.  opdr: optional host output
 * [nbatch][nxtot].  cgres: optional [nbatch] final CG residual |r|/|b|. */
int mb_tomo(mb_recon *r, const double *grad, double *opdr, float *cgres);

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

/* Sizes of the bound geometry. */
long mb_ngrad(const mb_recon *r);
long mb_nxtot(const mb_recon *r);
int mb_nbatch(const mb_recon *r);

/* Single operator applications, for parity tests.  All host FP64, [nbatch][n]. */
int mb_apply_tomo_R(mb_recon *r, const double *grad, double *xout);    /* TomoR */
int mb_apply_tomo_L(mb_recon *r, const double *xin, double *xout);     /* TomoL */
int mb_apply_fdpcg(mb_recon *r, const double *xin, double *xout);      /* fdpcg_precond */
int mb_apply_hx(mb_recon *r, const double *xin, double *opd);          /* Hx: [nbatch][nwfs][np] */

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
