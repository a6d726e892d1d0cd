/* CPU implementation of the two cuFFT symbols the reference calls.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  The reference runs its spectral
 * active-gel solve through cufftPlan2d(&plan, M, M, CUFFT_C2C) and
 * cufftExecC2C(plan, in, out, CUFFT_FORWARD|CUFFT_INVERSE)
 * (main_code/run_with_active_gels.cpp:87-88, functions/useful_functions.cpp:646-660).
 * Compiled into the oracle builds of the reference, this file stands in for
 * libcufft so that the reference's own sources run serially on the host.
 *
 * Semantics follow cuFFT's documented C2C transform: unnormalised, forward
 * sign -1 (exp(-2 pi i k n / N)), inverse sign +1, row-major (nx slowest).
 * Arithmetic is double precision throughout; the FP32 build rounds the result
 * to float once at the end.  1-D transforms use recursive mixed-radix
 * Cooley-Tukey for lengths whose prime factors are <= 7 and Bluestein's chirp-z
 * algorithm (power-of-two convolution) for any other length (M = 398 = 2*199 at
 * the reference's default zone_size of 200).  Pinned against numpy.fft.fft2 in
 * tests/test_oracle_fft.py.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "cufft.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b) {
    cplx r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re };
    return r;
}

/* ---- 1-D plan: factors, twiddles exp(-2 pi i k / n), Bluestein data ---- */
typedef struct plan1d {
    int n;
    int nfac;
    int fac[40];
    cplx *tw;          /* n twiddles, forward sign */
    int bluestein;     /* 1 when some prime factor exceeds 7 */
    int L;             /* Bluestein convolution length (power of two) */
    cplx *chirp;       /* n values exp(-i pi k^2 / n) */
    cplx *bfft_fwd;    /* FFT_L of the conjugate chirp kernel (forward sign) */
    struct plan1d *sub;/* plan of length L */
} plan1d_t;

#define MAX_PLANS1D 64
static plan1d_t *g_p1[MAX_PLANS1D];
static int g_np1 = 0;

static plan1d_t *get_plan1d(int n);

static void fft_rec(cplx *out, const cplx *in, int n, int istride,
                    const int *fac, const plan1d_t *top, int sign)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = fac[0], m = n / p;
    for (int r = 0; r < p; r++)
        fft_rec(out + (size_t)r * m, in + (size_t)r * istride, m, istride * p, fac + 1, top, sign);
    int step_n = top->n / n;   /* W_n^k = tw[k * step_n] */
    int step_p = top->n / p;   /* W_p^k = tw[k * step_p] */
    cplx t[64];
    cplx *tt = (p <= 64) ? t : (cplx *)malloc(sizeof(cplx) * p);
    for (int q = 0; q < m; q++) {
        for (int r = 0; r < p; r++) {
            cplx w = top->tw[(size_t)((long)r * q % n) * step_n];
            if (sign > 0) w.im = -w.im;
            tt[r] = cmul(out[(size_t)r * m + q], w);
        }
        if (p == 2) {
            out[q].re = tt[0].re + tt[1].re; out[q].im = tt[0].im + tt[1].im;
            out[q + m].re = tt[0].re - tt[1].re; out[q + m].im = tt[0].im - tt[1].im;
        } else {
            for (int s = 0; s < p; s++) {
                double ar = 0.0, ai = 0.0;
                for (int r = 0; r < p; r++) {
                    cplx w = top->tw[(size_t)((long)r * s % p) * step_p];
                    if (sign > 0) w.im = -w.im;
                    ar += tt[r].re * w.re - tt[r].im * w.im;
                    ai += tt[r].re * w.im + tt[r].im * w.re;
                }
                out[q + (size_t)m * s].re = ar; out[q + (size_t)m * s].im = ai;
            }
        }
    }
    if (tt != t) free(tt);
}

static void fft1d(plan1d_t *pl, cplx *data, int sign, cplx *scratch);

static void bluestein(plan1d_t *pl, cplx *data, int sign, cplx *scratch)
{
    int n = pl->n, L = pl->L;
    plan1d_t *sp = (plan1d_t *)pl->sub;
    cplx *a = scratch;            /* L */
    cplx *s2 = scratch + L;       /* L scratch for the inner transform */
    for (int k = 0; k < L; k++) { a[k].re = 0.0; a[k].im = 0.0; }
    /* a[k] = x[k] * chirp_s[k], chirp_s = exp(s i pi k^2/n) */
    for (int k = 0; k < n; k++) {
        cplx c = pl->chirp[k];
        if (sign > 0) c.im = -c.im;
        a[k] = cmul(data[k], c);
    }
    fft1d(sp, a, -1, s2);
    /* multiply by FFT of the kernel conj(chirp_s)[k] (wrapped) */
    for (int k = 0; k < L; k++) {
        cplx b = pl->bfft_fwd[k];
        if (sign > 0) {
            /* kernel for sign +1 is the conjugate of the sign -1 kernel; the FFT of
             * conj(h) at k equals conj(FFT(h) at -k). */
            cplx bb = pl->bfft_fwd[(L - k) % L];
            b.re = bb.re; b.im = -bb.im;
        }
        a[k] = cmul(a[k], b);
    }
    fft1d(sp, a, +1, s2);
    for (int k = 0; k < n; k++) {
        cplx c = pl->chirp[k];
        if (sign > 0) c.im = -c.im;
        cplx v = { a[k].re / L, a[k].im / L };
        data[k] = cmul(v, c);
    }
}

static void fft1d(plan1d_t *pl, cplx *data, int sign, cplx *scratch)
{
    if (pl->n == 1) return;
    if (pl->bluestein) { bluestein(pl, data, sign, scratch); return; }
    memcpy(scratch, data, sizeof(cplx) * pl->n);
    fft_rec(data, scratch, pl->n, 1, pl->fac, pl, sign);
}

static plan1d_t *get_plan1d(int n)
{
    for (int i = 0; i < g_np1; i++) if (g_p1[i]->n == n) return g_p1[i];
    plan1d_t *pl = (plan1d_t *)calloc(1, sizeof(plan1d_t));
    pl->n = n;
    int m = n, big = 0;
    while (m > 1) {
        int f = 0;
        if (m % 2 == 0) f = 2;
        else { for (int d = 3; d <= 7; d += 2) if (m % d == 0) { f = d; break; } }
        if (!f) { big = 1; break; }
        pl->fac[pl->nfac++] = f;
        m /= f;
    }
    pl->tw = (cplx *)malloc(sizeof(cplx) * (n > 0 ? n : 1));
    for (int k = 0; k < n; k++) {
        double ang = -2.0 * M_PI * (double)k / (double)n;
        pl->tw[k].re = cos(ang); pl->tw[k].im = sin(ang);
    }
    if (big) {
        pl->bluestein = 1;
        int L = 1;
        while (L < 2 * n - 1) L <<= 1;
        pl->L = L;
        pl->chirp = (cplx *)malloc(sizeof(cplx) * n);
        for (int k = 0; k < n; k++) {
            long k2 = ((long)k * k) % (2L * n);
            double ang = -M_PI * (double)k2 / (double)n;
            pl->chirp[k].re = cos(ang); pl->chirp[k].im = sin(ang);
        }
        pl->sub = (struct plan1d *)get_plan1d(L);
        cplx *h = (cplx *)calloc(L, sizeof(cplx));
        for (int k = 0; k < n; k++) {
            h[k].re = pl->chirp[k].re; h[k].im = -pl->chirp[k].im;
            if (k) { h[L - k] = h[k]; }
        }
        cplx *scr = (cplx *)malloc(sizeof(cplx) * 2 * L);
        fft1d((plan1d_t *)pl->sub, h, -1, scr);
        free(scr);
        pl->bfft_fwd = h;
    }
    if (g_np1 < MAX_PLANS1D) g_p1[g_np1++] = pl;
    return pl;
}

/* ---- 2-D plans (the cufftHandle is an index into this table) ---- */
#define MAX_PLANS2D 64
static struct { int nx, ny, used; } g_p2[MAX_PLANS2D];

cufftResult cufftPlan2d(cufftHandle *plan, int nx, int ny, cufftType type)
{
    if (!plan || nx < 1 || ny < 1 || type != CUFFT_C2C) return CUFFT_INVALID_VALUE;
    for (int i = 0; i < MAX_PLANS2D; i++) {
        if (!g_p2[i].used) {
            g_p2[i].used = 1; g_p2[i].nx = nx; g_p2[i].ny = ny;
            get_plan1d(nx); get_plan1d(ny);
            *plan = i;
            return CUFFT_SUCCESS;
        }
    }
    return CUFFT_ALLOC_FAILED;
}

cufftResult cufftDestroy(cufftHandle plan)
{
    if (plan < 0 || plan >= MAX_PLANS2D || !g_p2[plan].used) return CUFFT_INVALID_PLAN;
    g_p2[plan].used = 0;
    return CUFFT_SUCCESS;
}

/* Double-precision 2-D transform on an nx*ny row-major array (exported for the
 * oracle restatement and for the FFT unit test). */
void pfag_shim_fft2d_f64(int nx, int ny, double *re_im, int direction)
{
    plan1d_t *px = get_plan1d(nx), *py = get_plan1d(ny);
    int mx = nx > ny ? nx : ny;
    int Lx = px->bluestein ? px->L : 0, Ly = py->bluestein ? py->L : 0;
    int Lm = Lx > Ly ? Lx : Ly;
    size_t scr_n = (size_t)(mx > 2 * Lm ? mx : 2 * Lm) + (size_t)mx;
    cplx *scr = (cplx *)malloc(sizeof(cplx) * (scr_n + (size_t)mx));
    cplx *line = scr + scr_n;
    cplx *d = (cplx *)re_im;
    int sign = (direction == CUFFT_INVERSE) ? +1 : -1;
    for (int i = 0; i < nx; i++) fft1d(py, d + (size_t)i * ny, sign, scr);
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < nx; i++) line[i] = d[(size_t)i * ny + j];
        fft1d(px, line, sign, scr);
        for (int i = 0; i < nx; i++) d[(size_t)i * ny + j] = line[i];
    }
    free(scr);
}

/* Optional capture of inverse-transform outputs (real parts, in call order):
 * the reference keeps each cell's velocity only in FFT scratch
 * (rho_functions.cpp:449-456), so the oracle reads it here. */
static double *g_cap = 0;
static long g_cap_cap = 0, g_cap_len = 0;

void pfag_shim_capture(double *buf, long capacity)
{
    g_cap = buf; g_cap_cap = capacity; g_cap_len = 0;
}

long pfag_shim_capture_len(void) { return g_cap_len; }

cufftResult cufftExecC2C(cufftHandle plan, cufftComplex *idata, cufftComplex *odata, int direction)
{
    if (plan < 0 || plan >= MAX_PLANS2D || !g_p2[plan].used) return CUFFT_INVALID_PLAN;
    int nx = g_p2[plan].nx, ny = g_p2[plan].ny;
    size_t n = (size_t)nx * ny;
    double *buf = (double *)malloc(sizeof(double) * 2 * n);
    for (size_t k = 0; k < n; k++) { buf[2 * k] = idata[k].x; buf[2 * k + 1] = idata[k].y; }
    pfag_shim_fft2d_f64(nx, ny, buf, direction);
    for (size_t k = 0; k < n; k++) { odata[k].x = buf[2 * k]; odata[k].y = buf[2 * k + 1]; }
    if (g_cap && direction == CUFFT_INVERSE && g_cap_len + (long)n <= g_cap_cap) {
        for (size_t k = 0; k < n; k++) g_cap[g_cap_len + (long)k] = (double)odata[k].x;
        g_cap_len += (long)n;
    }
    free(buf);
    return CUFFT_SUCCESS;
}
