/*
 * Project-written implementation of the FFTW3 API subset declared in
 * fftw3.h, for the reference CPU build only (test infrastructure).
 *
 * Algorithm: recursive mixed-radix decimation in time.  For n = p*m with p the
 * smallest prime factor,
 *     X[k] = sum_{r<p} w_n^{r k} Y_r[k mod m],   Y_r = DFT_m( x[r + p j] ),
 * w_n = exp(sign*2*pi*i/n).  Prime lengths fall back to the direct O(n^2) sum.
 * Twiddles come from one table per transform dim, made when the plan is made
 * and indexed by (r*k mod n); a transform's workspace is allocated once per
 * execution (no allocation per line or per recursion level).
 * Transforms are unnormalised, like FFTW.  Multi-dimensional and "many"
 * transforms are executed line by line over strided views; float plans run
 * through the double-precision kernel.
 */
#include "fftw3.h"
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;
static cplx *twiddles(long n, int sign);

enum { K_CPLX = 0, K_SPLIT = 1, K_R2HC = 2, K_HC2R = 3 };

struct maosref_fft_plan {
    int kind;
    int single;              /* 1 when the user arrays are float */
    int sign;
    int rank;                /* transform dims */
    fftw_iodim dims[3];
    int hrank;               /* loop (howmany) dims */
    fftw_iodim hdims[2];
    void *in, *out;          /* interleaved complex or real arrays */
    void *ri, *ii, *ro, *io; /* split arrays */
    cplx *tw[3];             /* twiddles of each transform dim (made at plan time) */
};

/* x: n points; tw: twiddles of the top-level length N (tw[k] = w_N^k);
 * n divides N and w_n^e = tw[e * (N/n)].  ws: workspace of 2n points (the
 * children of a level reuse its second half). */
static void dft_rec(cplx *x, long n, const cplx *tw, long N, cplx *ws) {
    if (n <= 1) return;
    const long ts = N / n;
    cplx *tmp = ws;
    long p = 0;
    for (long f = 2; f * f <= n; f++) {
        if (n % f == 0) { p = f; break; }
    }
    if (!p) { /* prime: direct sum */
        for (long k = 0; k < n; k++) {
            cplx s = 0;
            for (long j = 0; j < n; j++) s += x[j] * tw[((j * k) % n) * ts];
            tmp[k] = s;
        }
        memcpy(x, tmp, sizeof(cplx) * n);
        return;
    }
    long m = n / p;
    for (long r = 0; r < p; r++)
        for (long j = 0; j < m; j++) tmp[r * m + j] = x[r + p * j];
    for (long r = 0; r < p; r++) dft_rec(tmp + r * m, m, tw, N, ws + n);
    for (long k = 0; k < n; k++) {
        cplx s = 0;
        long km = k % m;
        for (long r = 0; r < p; r++) s += tmp[r * m + km] * tw[((r * k) % n) * ts];
        x[k] = s;
    }
}

/* twiddles w_n^k = exp(sign 2 pi i k / n), computed once per plan and dim */
static cplx *twiddles(long n, int sign) {
    cplx *tw = (cplx *)malloc(sizeof(cplx) * (n > 0 ? n : 1));
    for (long k = 0; k < n; k++) {
        double a = sign * 2.0 * M_PI * (double)k / (double)n;
        tw[k] = cos(a) + I * sin(a);
    }
    return tw;
}

/* one unnormalised line transform with the plan's twiddles; ws: 2n points */
static void dft_line(cplx *buf, long n, const cplx *tw, cplx *ws) {
    if (n <= 1) return;
    dft_rec(buf, n, tw, n, ws);
}

/* element accessors on the four storage forms */
static cplx load_c(const struct maosref_fft_plan *pl, long off) {
    if (pl->kind == K_SPLIT) {
        if (pl->single) return ((float *)pl->ro)[off] + I * ((float *)pl->io)[off];
        return ((double *)pl->ro)[off] + I * ((double *)pl->io)[off];
    }
    if (pl->single) {
        float *q = (float *)pl->out + 2 * off;
        return q[0] + I * q[1];
    }
    double *q = (double *)pl->out + 2 * off;
    return q[0] + I * q[1];
}
static void store_c(const struct maosref_fft_plan *pl, long off, cplx v) {
    if (pl->kind == K_SPLIT) {
        if (pl->single) { ((float *)pl->ro)[off] = (float)creal(v); ((float *)pl->io)[off] = (float)cimag(v); }
        else { ((double *)pl->ro)[off] = creal(v); ((double *)pl->io)[off] = cimag(v); }
        return;
    }
    if (pl->single) { float *q = (float *)pl->out + 2 * off; q[0] = (float)creal(v); q[1] = (float)cimag(v); }
    else { double *q = (double *)pl->out + 2 * off; q[0] = creal(v); q[1] = cimag(v); }
}

/* copy input -> output layout when a plan is out of place */
static void copy_in_to_out(const struct maosref_fft_plan *pl) {
    int nd = pl->rank + pl->hrank;
    fftw_iodim all[5];
    for (int i = 0; i < pl->rank; i++) all[i] = pl->dims[i];
    for (int i = 0; i < pl->hrank; i++) all[pl->rank + i] = pl->hdims[i];
    long total = 1;
    for (int i = 0; i < nd; i++) total *= all[i].n;
    for (long lin = 0; lin < total; lin++) {
        long rem = lin, ioff = 0, ooff = 0;
        for (int i = 0; i < nd; i++) {
            long c = rem % all[i].n; rem /= all[i].n;
            ioff += c * all[i].is; ooff += c * all[i].os;
        }
        cplx v;
        if (pl->kind == K_SPLIT) {
            if (pl->single) v = ((float *)pl->ri)[ioff] + I * ((float *)pl->ii)[ioff];
            else v = ((double *)pl->ri)[ioff] + I * ((double *)pl->ii)[ioff];
        } else if (pl->single) {
            float *q = (float *)pl->in + 2 * ioff; v = q[0] + I * q[1];
        } else {
            double *q = (double *)pl->in + 2 * ioff; v = q[0] + I * q[1];
        }
        store_c(pl, ooff, v);
    }
}

static void exec_complex(const struct maosref_fft_plan *pl) {
    int inplace = (pl->kind == K_SPLIT) ? (pl->ri == pl->ro && pl->ii == pl->io) : (pl->in == pl->out);
    if (!inplace) copy_in_to_out(pl);
    /* loop over every transform dim; for each, transform all lines along it */
    for (int d = 0; d < pl->rank; d++) {
        long n = pl->dims[d].n, st = pl->dims[d].os;
        fftw_iodim others[4];
        int no = 0;
        for (int i = 0; i < pl->rank; i++) if (i != d) others[no++] = pl->dims[i];
        for (int i = 0; i < pl->hrank; i++) others[no++] = pl->hdims[i];
        long nlines = 1;
        for (int i = 0; i < no; i++) nlines *= others[i].n;
        cplx *buf = (cplx *)malloc(sizeof(cplx) * 3 * (n > 0 ? n : 1));
        for (long l = 0; l < nlines; l++) {
            long rem = l, base = 0;
            for (int i = 0; i < no; i++) { long c = rem % others[i].n; rem /= others[i].n; base += c * others[i].os; }
            for (long j = 0; j < n; j++) buf[j] = load_c(pl, base + j * st);
            dft_line(buf, n, pl->tw[d], buf + n);
            for (long j = 0; j < n; j++) store_c(pl, base + j * st, buf[j]);
        }
        free(buf);
    }
}

static void exec_r2r(const struct maosref_fft_plan *pl) {
    long n = pl->dims[0].n;
    cplx *buf = (cplx *)malloc(sizeof(cplx) * 3 * n);
    double *tmp = (double *)malloc(sizeof(double) * n);
    for (long j = 0; j < n; j++)
        tmp[j] = pl->single ? ((float *)pl->in)[j] : ((double *)pl->in)[j];
    if (pl->kind == K_R2HC) {
        for (long j = 0; j < n; j++) buf[j] = tmp[j];
        dft_line(buf, n, pl->tw[0], buf + n);
        /* halfcomplex: r0 r1 .. r_{n/2} i_{(n+1)/2-1} .. i1 */
        for (long k = 0; k <= n / 2; k++) tmp[k] = creal(buf[k]);
        for (long k = 1; k < (n + 1) / 2; k++) tmp[n - k] = cimag(buf[k]);
    } else {
        for (long k = 0; k <= n / 2; k++) {
            double im = (k > 0 && k < (n + 1) / 2) ? tmp[n - k] : 0.0;
            buf[k] = tmp[k] + I * im;
        }
        for (long k = n / 2 + 1; k < n; k++) buf[k] = conj(buf[n - k]);
        dft_line(buf, n, pl->tw[0], buf + n);
        for (long j = 0; j < n; j++) tmp[j] = creal(buf[j]);
    }
    for (long j = 0; j < n; j++) {
        if (pl->single) ((float *)pl->out)[j] = (float)tmp[j];
        else ((double *)pl->out)[j] = tmp[j];
    }
    free(buf);
    free(tmp);
}

static struct maosref_fft_plan *plan_new(int kind, int single, int sign) {
    struct maosref_fft_plan *pl = (struct maosref_fft_plan *)calloc(1, sizeof(*pl));
    pl->kind = kind; pl->single = single; pl->sign = sign;
    return pl;
}

static struct maosref_fft_plan *mk_1d(int n, void *in, void *out, int sign, int single) {
    struct maosref_fft_plan *pl = plan_new(K_CPLX, single, sign);
    pl->rank = 1; pl->dims[0].n = n; pl->dims[0].is = 1; pl->dims[0].os = 1;
    pl->in = in; pl->out = out;
    return pl;
}
static struct maosref_fft_plan *mk_2d(int n0, int n1, void *in, void *out, int sign, int single) {
    /* row major: n1 is contiguous */
    struct maosref_fft_plan *pl = plan_new(K_CPLX, single, sign);
    pl->rank = 2;
    pl->dims[0].n = n1; pl->dims[0].is = 1; pl->dims[0].os = 1;
    pl->dims[1].n = n0; pl->dims[1].is = n1; pl->dims[1].os = n1;
    pl->in = in; pl->out = out;
    return pl;
}
static struct maosref_fft_plan *mk_many(int rank, const int *n, int howmany, void *in,
                                        const int *inembed, int istride, int idist, void *out,
                                        const int *onembed, int ostride, int odist, int sign, int single) {
    if (rank != 1 || inembed || onembed) return NULL;
    struct maosref_fft_plan *pl = plan_new(K_CPLX, single, sign);
    pl->rank = 1;
    pl->dims[0].n = n[0]; pl->dims[0].is = istride; pl->dims[0].os = ostride;
    pl->hrank = 1;
    pl->hdims[0].n = howmany; pl->hdims[0].is = idist; pl->hdims[0].os = odist;
    pl->in = in; pl->out = out;
    return pl;
}
static struct maosref_fft_plan *mk_split(int rank, const fftw_iodim *dims, int hrank,
                                         const fftw_iodim *hdims, void *ri, void *ii, void *ro,
                                         void *io, int single) {
    if (rank > 3 || hrank > 2) return NULL;
    struct maosref_fft_plan *pl = plan_new(K_SPLIT, single, FFTW_FORWARD);
    pl->rank = rank;
    for (int i = 0; i < rank; i++) pl->dims[i] = dims[i];
    pl->hrank = hrank;
    for (int i = 0; i < hrank; i++) pl->hdims[i] = hdims[i];
    pl->ri = ri; pl->ii = ii; pl->ro = ro; pl->io = io;
    return pl;
}
static struct maosref_fft_plan *mk_r2r(int n, void *in, void *out, fftw_r2r_kind kind, int single) {
    struct maosref_fft_plan *pl = plan_new(kind == FFTW_R2HC ? K_R2HC : K_HC2R, single, 0);
    pl->rank = 1; pl->dims[0].n = n; pl->dims[0].is = 1; pl->dims[0].os = 1;
    pl->in = in; pl->out = out;
    return pl;
}
/* the twiddle tables of a finished plan (r2r: forward for R2HC, backward for HC2R) */
static struct maosref_fft_plan *with_twiddles(struct maosref_fft_plan *pl) {
    if (!pl) return pl;
    const int sign = pl->kind == K_R2HC ? -1 : pl->kind == K_HC2R ? 1 : pl->sign;
    for (int d = 0; d < pl->rank; d++) pl->tw[d] = twiddles(pl->dims[d].n, sign);
    return pl;
}
static void plan_free(struct maosref_fft_plan *pl) {
    if (!pl) return;
    for (int d = 0; d < 3; d++) free(pl->tw[d]);
    free(pl);
}
static void execute_any(const struct maosref_fft_plan *pl) {
    if (!pl) return;
    if (pl->kind == K_R2HC || pl->kind == K_HC2R) exec_r2r(pl);
    else exec_complex(pl);
}

/* ---- double API ---- */
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags; return with_twiddles(mk_1d(n, in, out, sign, 0));
}
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags; return with_twiddles(mk_2d(n0, n1, in, out, sign, 0));
}
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed,
                             int istride, int idist, fftw_complex *out, const int *onembed, int ostride,
                             int odist, int sign, unsigned flags) {
    (void)flags;
    return with_twiddles(mk_many(rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, sign, 0));
}
fftw_plan fftw_plan_guru_split_dft(int rank, const fftw_iodim *dims, int howmany_rank,
                                   const fftw_iodim *howmany_dims, double *ri, double *ii, double *ro,
                                   double *io, unsigned flags) {
    (void)flags; return with_twiddles(mk_split(rank, dims, howmany_rank, howmany_dims, ri, ii, ro, io, 0));
}
fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned flags) {
    (void)flags; return with_twiddles(mk_r2r(n, in, out, kind, 0));
}
void fftw_execute(const fftw_plan p) { execute_any(p); }
void fftw_destroy_plan(fftw_plan p) { plan_free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}
int fftw_import_wisdom_from_file(FILE *f) { (void)f; return 0; }
void fftw_export_wisdom_to_file(FILE *f) { (void)f; }

/* ---- float API ---- */
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags) {
    (void)flags; return with_twiddles(mk_1d(n, in, out, sign, 1));
}
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags) {
    (void)flags; return with_twiddles(mk_2d(n0, n1, in, out, sign, 1));
}
fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in, const int *inembed,
                               int istride, int idist, fftwf_complex *out, const int *onembed, int ostride,
                               int odist, int sign, unsigned flags) {
    (void)flags;
    return with_twiddles(mk_many(rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, sign, 1));
}
fftwf_plan fftwf_plan_guru_split_dft(int rank, const fftwf_iodim *dims, int howmany_rank,
                                     const fftwf_iodim *howmany_dims, float *ri, float *ii, float *ro,
                                     float *io, unsigned flags) {
    (void)flags; return with_twiddles(mk_split(rank, dims, howmany_rank, howmany_dims, ri, ii, ro, io, 1));
}
fftwf_plan fftwf_plan_r2r_1d(int n, float *in, float *out, fftwf_r2r_kind kind, unsigned flags) {
    (void)flags; return with_twiddles(mk_r2r(n, in, out, kind, 1));
}
void fftwf_execute(const fftwf_plan p) { execute_any(p); }
void fftwf_destroy_plan(fftwf_plan p) { plan_free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftwf_cleanup_threads(void) {}
void fftwf_cleanup(void) {}
int fftwf_import_wisdom_from_file(FILE *f) { (void)f; return 0; }
void fftwf_export_wisdom_to_file(FILE *f) { (void)f; }
