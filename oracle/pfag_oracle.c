/* pfag_oracle.c — CPU restatement of the reference's time step (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
 * bench.py's CPU baseline leg as the checker; never part of the product path.
 *
 * It restates, on an explicit state struct instead of the reference's
 * globals, the loop body of main_code/run_with_active_gels.cpp:123-182 and the
 * functions it calls.  Each function cites the reference lines it follows and
 * keeps the reference's operation order and literal types, so that the FP64
 * build (-DPFAG_REF_DOUBLE) reproduces the reference's own FP64 build
 * (oracle/_ref/libref_fp64.so) bit for bit when both use oracle/cufft_shim.c
 * for the transforms; tests/test_oracle.py pins that, and the golden fixtures
 * of tests/golden/.  Single thread, plain C11.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "cufft.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#ifdef PFAG_REF_DOUBLE
typedef double real;
#define FABS fabs
#else
typedef float real;
#define FABS fabsf
#endif

typedef struct {
    int N_s, Ntot, zone_size, N_current, rdev_threshold, rimax;
    double dx, dt, R, s0, sigma, coupling_PF_AG, tau, alpha, beta, eta;
    double tau_lum, beta_lum_cells, eta_lum_cells, xi_lum;
    double alpha_ECM, tau_ECM, beta_ECM_cells, eta_ECM_cells, xi_ECM, beta_lum_ECM;
    double wi, rtol, rdt, friction;
    double a_tan_apical, a_tan_basal, a_tan_lateral, a_ort_apical, a_ort_basal, a_ort_lateral;
    double b_ap, b_bas, b_lat, matgenrate_apical, matgenrate_basal, matgenrate_lateral;
    double degrate_apical, degrate_basal, degrate_lateral, viscosity_ap, viscosity_bas, viscosity_lat;
} pfo_params;

/* Parameters are stored in the state's precision, as the reference's globals are. */
typedef struct {
    real dx, dt, R, s0, sigma, cpl, tau, alpha, beta, eta;
    real tau_lum, beta_lum_cells, eta_lum_cells, xi_lum;
    real alpha_ECM, tau_ECM, beta_ECM_cells, eta_ECM_cells, xi_ECM, beta_lum_ECM;
    real wi, rtol, rdt, friction;
    real deg[3], gen[3], aort[3], atan_[3], visc[3], bmap[3];   /* 0 apical, 1 basal, 2 lateral */
    int rdev_threshold, rimax, N_current;
} rparams;

typedef struct {
    int N, Ntot, z, M;
    rparams q;
    real *phi, *phin, *rho, *rhon, *lum, *lumn, *ecm, *ecmn;
    real *hcell, *hlum, *hecm, *psi, *g, *pnd, *jx, *jy, *ngl;
    real *deg, *gen, *at, *ao, *visc, *bm, *pxx, *pxy, *pyy;
    real *s, *f0;
    int *xc, *yc;
    cufftComplex *tf, *tfr, *frho, *freact, *fxx, *fxy, *fyy, *fvx, *fvy, *frvx, *frvy;
    cufftHandle planf, planr;
    int iters_cells_max, iters_cells_sum, iters_lum, iters_ecm;
    int *iters_cell;
    double *rdev_trace;     /* per cell: the last two rdev values of the latest reshaping loop (diagnostics) */
} pfo_state;

#define C3(n, i, j) ((size_t)(n) * N * N + (size_t)(i) * N + (size_t)(j))
#define C2(i, j) ((size_t)(i) * N + (size_t)(j))

static real *zalloc(size_t n) { return (real *)calloc(n ? n : 1, sizeof(real)); }

pfo_state *pfo_create(const pfo_params *p)
{
    pfo_state *st = (pfo_state *)calloc(1, sizeof(pfo_state));
    const int N = p->N_s;
    st->N = N; st->Ntot = p->Ntot; st->z = p->zone_size; st->M = 2 * p->zone_size - 2;
    rparams *q = &st->q;
    q->dx = (real)p->dx; q->dt = (real)p->dt; q->R = (real)p->R; q->s0 = (real)p->s0; q->sigma = (real)p->sigma;
    q->cpl = (real)p->coupling_PF_AG; q->tau = (real)p->tau; q->alpha = (real)p->alpha; q->beta = (real)p->beta;
    q->eta = (real)p->eta; q->tau_lum = (real)p->tau_lum; q->beta_lum_cells = (real)p->beta_lum_cells;
    q->eta_lum_cells = (real)p->eta_lum_cells; q->xi_lum = (real)p->xi_lum; q->alpha_ECM = (real)p->alpha_ECM;
    q->tau_ECM = (real)p->tau_ECM; q->beta_ECM_cells = (real)p->beta_ECM_cells; q->eta_ECM_cells = (real)p->eta_ECM_cells;
    q->xi_ECM = (real)p->xi_ECM; q->beta_lum_ECM = (real)p->beta_lum_ECM; q->wi = (real)p->wi;
    q->rtol = (real)p->rtol; q->rdt = (real)p->rdt; q->friction = (real)p->friction;
    q->deg[0] = (real)p->degrate_apical; q->deg[1] = (real)p->degrate_basal; q->deg[2] = (real)p->degrate_lateral;
    q->gen[0] = (real)p->matgenrate_apical; q->gen[1] = (real)p->matgenrate_basal; q->gen[2] = (real)p->matgenrate_lateral;
    q->aort[0] = (real)p->a_ort_apical; q->aort[1] = (real)p->a_ort_basal; q->aort[2] = (real)p->a_ort_lateral;
    q->atan_[0] = (real)p->a_tan_apical; q->atan_[1] = (real)p->a_tan_basal; q->atan_[2] = (real)p->a_tan_lateral;
    q->visc[0] = (real)p->viscosity_ap; q->visc[1] = (real)p->viscosity_bas; q->visc[2] = (real)p->viscosity_lat;
    q->bmap[0] = (real)p->b_ap; q->bmap[1] = (real)p->b_bas; q->bmap[2] = (real)p->b_lat;
    q->rdev_threshold = p->rdev_threshold; q->rimax = p->rimax; q->N_current = p->N_current;
    const size_t nc = (size_t)p->Ntot * N * N, ng = (size_t)N * N, mm = (size_t)st->M * st->M;
    real **cellf[] = {&st->phi, &st->phin, &st->rho, &st->rhon, &st->hcell, &st->g, &st->pnd, &st->jx, &st->jy,
                      &st->deg, &st->gen, &st->at, &st->ao, &st->visc, &st->bm, &st->pxx, &st->pxy, &st->pyy};
    for (size_t k = 0; k < sizeof(cellf) / sizeof(cellf[0]); k++) *cellf[k] = zalloc(nc);
    real **gridf[] = {&st->lum, &st->lumn, &st->ecm, &st->ecmn, &st->hlum, &st->hecm, &st->psi, &st->ngl};
    for (size_t k = 0; k < sizeof(gridf) / sizeof(gridf[0]); k++) *gridf[k] = zalloc(ng);
    st->s = zalloc(p->Ntot); st->f0 = zalloc(p->Ntot);
    st->xc = (int *)calloc(p->Ntot, sizeof(int)); st->yc = (int *)calloc(p->Ntot, sizeof(int));
    st->iters_cell = (int *)calloc(p->Ntot, sizeof(int));
    st->rdev_trace = (double *)calloc(2 * (size_t)p->Ntot, sizeof(double));
    cufftComplex **ff[] = {&st->tf, &st->tfr, &st->frho, &st->freact, &st->fxx, &st->fxy, &st->fyy,
                           &st->fvx, &st->fvy, &st->frvx, &st->frvy};
    for (size_t k = 0; k < sizeof(ff) / sizeof(ff[0]); k++) *ff[k] = (cufftComplex *)calloc(mm, sizeof(cufftComplex));
    cufftPlan2d(&st->planf, st->M, st->M, CUFFT_C2C);
    cufftPlan2d(&st->planr, st->M, st->M, CUFFT_C2C);
    return st;
}

void pfo_destroy(pfo_state *st)
{
    if (!st) return;
    real *a[] = {st->phi, st->phin, st->rho, st->rhon, st->hcell, st->g, st->pnd, st->jx, st->jy, st->deg, st->gen,
                 st->at, st->ao, st->visc, st->bm, st->pxx, st->pxy, st->pyy, st->lum, st->lumn, st->ecm, st->ecmn,
                 st->hlum, st->hecm, st->psi, st->ngl, st->s, st->f0};
    for (size_t k = 0; k < sizeof(a) / sizeof(a[0]); k++) free(a[k]);
    cufftComplex *b[] = {st->tf, st->tfr, st->frho, st->freact, st->fxx, st->fxy, st->fyy, st->fvx, st->fvy,
                         st->frvx, st->frvy};
    for (size_t k = 0; k < sizeof(b) / sizeof(b[0]); k++) free(b[k]);
    free(st->xc); free(st->yc); free(st->iters_cell); free(st->rdev_trace);
    cufftDestroy(st->planf); cufftDestroy(st->planr);
    free(st);
}

/* state in, then the copies of run_with_active_gels.cpp:92-98; hfunc_cell,
 * phin and rhon start at zero (:70-75) */
void pfo_load(pfo_state *st, const real *phi, const real *rho, const real *lum, const real *ecm)
{
    const int N = st->N;
    const size_t nc = (size_t)st->Ntot * N * N, ng = (size_t)N * N;
    memcpy(st->phi, phi, nc * sizeof(real)); memcpy(st->rho, rho, nc * sizeof(real));
    memcpy(st->lum, lum, ng * sizeof(real)); memcpy(st->ecm, ecm, ng * sizeof(real));
    memset(st->hcell, 0, nc * sizeof(real));
    memcpy(st->ecmn, st->ecm, ng * sizeof(real)); memcpy(st->lumn, st->lum, ng * sizeof(real));
    memcpy(st->phin, st->phi, nc * sizeof(real)); memcpy(st->rhon, st->rho, nc * sizeof(real));
}

/* useful_functions.cpp:193-227: integer centroid of the sites with phi > 0.5 */
static int centres(pfo_state *st)
{
    const int N = st->N;
    for (int n = 0; n < st->Ntot; n++) {
        int sx = 0, sy = 0, cnt = 0;
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++)
                if (st->phi[C3(n, i, j)] > 0.5) { sx += i; sy += j; cnt += 1; }
        if (cnt == 0) return -4;
        st->xc[n] = (int)(sx / cnt);
        st->yc[n] = (int)(sy / cnt);
        if (st->xc[n] - st->z < 1 || st->xc[n] + st->z > N - 1 || st->yc[n] - st->z < 1 || st->yc[n] + st->z > N - 1)
            return -3;
    }
    return 0;
}

/* rho_functions.cpp:286-405: apical / basal / lateral winner per zone site */
static void maps(pfo_state *st)
{
    const int N = st->N, z = st->z;
    const rparams *q = &st->q;
    for (int n = 0; n < st->Ntot; n++) {
        int n1, n2;
        if (n == 0) { n1 = st->Ntot - 1; n2 = n + 1; }
        else if (n == st->Ntot - 1) { n1 = n - 1; n2 = 0; }
        else { n1 = n - 1; n2 = n + 1; }
        if (n2 >= st->Ntot) n2 = 0;   /* Ntot == 1: the reference reads past the array here */
        for (int i = st->xc[n] - z; i < st->xc[n] + z; i++)
            for (int j = st->yc[n] - z; j < st->yc[n] + z; j++) {
                const real f = st->phi[C3(n, i, j)];
                real mx;
                int idx;
                real a = f * st->lum[C2(i, j)], b = f * st->ecm[C2(i, j)];
                if (a > b) { idx = 0; mx = a; } else { idx = 1; mx = b; }
                real c = f * st->phi[C3(n1, i, j)];
                if (c > mx) { idx = 2; mx = c; }
                real d = f * st->phi[C3(n2, i, j)];
                if (d > mx) { idx = 3; mx = d; }
                const int k = (idx == 3) ? 2 : idx;
                const size_t o = C3(n, i, j);
                st->deg[o] = q->deg[k]; st->gen[o] = q->gen[k]; st->ao[o] = q->aort[k];
                st->at[o] = q->atan_[k]; st->visc[o] = q->visc[k]; st->bm[o] = q->bmap[k];
            }
    }
}

/* useful_functions.cpp:391-420 on the first `ncells` slices */
static void bc_cells(pfo_state *st, real *t, int ncells)
{
    const int N = st->N;
    for (int n = 0; n < ncells; n++) {
        real *p = t + (size_t)n * N * N;
        for (int i = 1; i < N - 1; i++) {
            p[C2(i, 0)] = p[C2(i, N - 2)];
            p[C2(i, N - 1)] = p[C2(i, 1)];
            p[C2(0, i)] = p[C2(N - 2, i)];
            p[C2(N - 1, i)] = p[C2(1, i)];
        }
        p[C2(0, 0)] = p[C2(N - 2, N - 2)];
        p[C2(0, N - 1)] = p[C2(N - 2, 1)];
        p[C2(N - 1, 0)] = p[C2(1, N - 2)];
        p[C2(N - 1, N - 1)] = p[C2(1, 1)];
    }
}

/* |grad u| on the interior: useful_functions.cpp:347-349 (cells), cell_phase_functions.cpp:734-736 (lumen) */
static void norm_grad(pfo_state *st, const real *u, real *out, int ncells)
{
    const int N = st->N;
    const real dx = st->q.dx;
    for (int n = 0; n < ncells; n++) {
        const real *a = u + (size_t)n * N * N;
        real *o = out + (size_t)n * N * N;
        for (int i = 1; i < N - 1; i++)
            for (int j = 1; j < N - 1; j++)
                o[C2(i, j)] = sqrt((1.0 / dx / dx / 4.0) *
                                   ((a[C2(i + 1, j)] - a[C2(i - 1, j)]) * (a[C2(i + 1, j)] - a[C2(i - 1, j)]) +
                                    (a[C2(i, j + 1)] - a[C2(i, j - 1)]) * (a[C2(i, j + 1)] - a[C2(i, j - 1)])));
    }
}

static inline real hfun(real v) { return v * v * (3.0 - 2.0 * v); }   /* useful_functions.cpp:247 */

/* useful_functions.cpp:168-190 */
static void areas(pfo_state *st)
{
    const int N = st->N;
    const real dx = st->q.dx;
    for (int n = 0; n < st->Ntot; n++) {
        real sum = 0.0;
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) sum += (st->hcell[C3(n, i, j)]) * dx * dx;
        st->s[n] = sum;
        st->f0[n] = st->q.alpha * (st->q.s0 - st->s[n]);
    }
}

/* one cell of update_all_cortices, rho_functions.cpp:413-466 */
static void cortex_cell(pfo_state *st, int nc)
{
    const int N = st->N, z = st->z, M = st->M;
    const rparams *q = &st->q;
    const int i0 = st->xc[nc] - z + 1, j0 = st->yc[nc] - z + 1;
    /* load_temp_fft (useful_functions.cpp:605-625) of rho, forward */
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) { st->tf[i * M + j].x = st->rho[C3(nc, i + i0, j + j0)]; st->tf[i * M + j].y = 0.0; }
    cufftExecC2C(st->planf, st->tf, st->frho, CUFFT_FORWARD);
    /* create_deg_gen (rho_functions.cpp:193-209), forward */
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) {
            const size_t o = C3(nc, i + i0, j + j0);
            st->tf[i * M + j].x = -st->deg[o] * st->rho[o] + st->gen[o] * st->pnd[o];
            st->tf[i * M + j].y = 0.0;
        }
    cufftExecC2C(st->planf, st->tf, st->freact, CUFFT_FORWARD);
    /* compute_pi_xx, compute_pi_xy, compute_pi_yy (rho_functions.cpp:32-115) on the zone */
    for (int i = st->xc[nc] - z; i < st->xc[nc] + z; i++)
        for (int j = st->yc[nc] - z; j < st->yc[nc] + z; j++) {
            const size_t o = C3(nc, i, j);
            const real r = st->rho[o], at = st->at[o], ao = st->ao[o], gg = st->g[o];
            const real dxp = st->phi[C3(nc, i + 1, j)] - st->phi[C3(nc, i - 1, j)];
            const real dyp = st->phi[C3(nc, i, j + 1)] - st->phi[C3(nc, i, j - 1)];
            st->pxx[o] = -at * r * r * r + st->bm[o] * r * r * r * r;
            if (gg > 0.0) st->pxx[o] += (at - ao) * r * r * r * (1.0 / (4.0 * q->dx * q->dx)) * dxp * dxp / gg / gg;
            st->pxy[o] = 0.0;
            if (gg > 0.0) st->pxy[o] += (at - ao) * r * r * r * (1.0 / (4.0 * q->dx * q->dx)) * dxp * dyp / gg / gg;
            st->pyy[o] = -at * r * r * r + st->bm[o] * r * r * r * r;
            if (gg > 0.0) st->pyy[o] += (at - ao) * r * r * r * (1.0 / (4.0 * q->dx * q->dx)) * dyp * dyp / gg / gg;
        }
    real *pis[3] = {st->pxx, st->pxy, st->pyy};
    cufftComplex *fpis[3] = {st->fxx, st->fxy, st->fyy};
    for (int k = 0; k < 3; k++) {
        for (int i = 0; i < M; i++)
            for (int j = 0; j < M; j++) { st->tf[i * M + j].x = pis[k][C3(nc, i + i0, j + j0)]; st->tf[i * M + j].y = 0.0; }
        cufftExecC2C(st->planf, st->tf, fpis[k], CUFFT_FORWARD);
    }
    /* update_rho_velocity (rho_functions.cpp:133-190) */
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) {
            const int b = i * M + j;
            const int ir = (i < M / 2) ? i : i - M, jr = (j < M / 2) ? j : j - M;
            const real kx = (2.0 * M_PI / (M * q->dx)) * ir, ky = (2.0 * M_PI / (M * q->dx)) * jr;
            const real et = st->visc[C3(nc, i + i0, j + j0)];
            const real fr = q->friction;
            const cufftComplex pxx = st->fxx[b], pyy = st->fyy[b], pxy = st->fxy[b];
            const double den = -(4.0 * et * et * kx * kx * ky * ky + fr * fr + 3.0 * et * fr * (kx * kx + ky * ky) +
                               2.0 * et * et * (kx * kx * kx * kx + ky * ky * ky * ky));
            cufftComplex vx = {0.0, 0.0}, vy = {0.0, 0.0};
            vy.x += et * kx * ky * (kx * pxx.y + ky * pxy.y);
            vy.x -= (fr + 2.0 * et * (kx * kx + ky * ky / 2.0)) * (ky * pyy.y + kx * pxy.y);
            vy.x /= den;
            vy.y -= et * kx * ky * (kx * pxx.x + ky * pxy.x);
            vy.y += (fr + 2.0 * et * (kx * kx + ky * ky / 2.0)) * (ky * pyy.x + kx * pxy.x);
            vy.y /= den;
            vx.x += kx * pxx.y + ky * pxy.y - et * kx * ky * vy.x;
            vx.x /= fr + 2.0 * et * (kx * kx + ky * ky / 2.0);
            vx.y += -kx * pxx.x - ky * pxy.x - et * kx * ky * vy.y;
            vx.y /= fr + 2.0 * et * (kx * kx + ky * ky / 2.0);
            st->fvx[b] = vx;
            st->fvy[b] = vy;
        }
    /* IFFT(v), load_fft_rho_v (rho_functions.cpp:267-284), FFT(rho v) for x then y */
    cufftComplex *fv[2] = {st->fvx, st->fvy}, *frv[2] = {st->frvx, st->frvy};
    for (int k = 0; k < 2; k++) {
        cufftExecC2C(st->planr, fv[k], st->tfr, CUFFT_INVERSE);
        for (int i = 0; i < M; i++)
            for (int j = 0; j < M; j++) {
                st->tf[i * M + j].x = st->rho[C3(nc, i + i0, j + j0)] * st->tfr[i * M + j].x / (M * M);
                st->tf[i * M + j].y = 0.0;
            }
        cufftExecC2C(st->planf, st->tf, frv[k], CUFFT_FORWARD);
    }
    /* update_fft_rho (rho_functions.cpp:213-251) */
    for (int b = 0; b < M * M; b++) {
        st->frho[b].x += q->dt * st->freact[b].x;
        st->frho[b].y += q->dt * st->freact[b].y;
    }
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) {
            const int b = i * M + j;
            const int ir = (i < M / 2) ? i : i - M, jr = (j < M / 2) ? j : j - M;
            st->frho[b].x += q->dt * (2.0 * M_PI / (M * q->dx)) * (ir * st->frvx[b].y + jr * st->frvy[b].y);
            st->frho[b].y -= q->dt * (2.0 * M_PI / (M * q->dx)) * (ir * st->frvx[b].x + jr * st->frvy[b].x);
        }
    cufftExecC2C(st->planr, st->frho, st->tf, CUFFT_INVERSE);
    /* copy_to_rhon (rho_functions.cpp:253-265) */
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) st->rhon[C3(nc, i + i0, j + j0)] = st->tf[i * M + j].x / (M * M);
}

/* one relaxation increment of the reshaping scheme at (i, j) of field p with
 * normals X, Y (cell_phase_functions.cpp:511-547 and :802-838, same terms) */
static real resh_increment(const real *p, const real *X, const real *Y, int N, int i, int j, real pn, real wi,
                           real rdt, real dx)
{
    const int ip = i + 1, im = i - 1, jp = j + 1, jm = j - 1;
#define P(a, b) p[C2(a, b)]
#define JX(a, b) X[C2(a, b)]
#define JY(a, b) Y[C2(a, b)]
    pn += 0.5 * (JX(ip, j) + JX(i, j)) *
          (wi * wi * (rdt / dx / dx) * (P(ip, j) - P(i, j)) * 0.5 * (JX(ip, j) + JX(i, j)) +
           wi * wi * (rdt / dx / dx) * 0.25 * (P(ip, jp) + P(i, jp) - P(ip, jm) - P(i, jm)) * 0.5 * (JY(ip, j) + JY(i, j)) -
           rdt * wi * sqrt(2.0) / dx * 0.5 * (P(ip, j) * (1.0 - P(ip, j)) + P(i, j) * (1.0 - P(i, j))));
    pn += 0.5 * (JY(i, jp) + JY(i, j)) *
          (wi * wi * (rdt / dx / dx) * (P(i, jp) - P(i, j)) * 0.5 * (JY(i, jp) + JY(i, j)) +
           wi * wi * (rdt / dx / dx) * 0.25 * (P(ip, jp) + P(ip, j) - P(im, jp) - P(im, j)) * 0.5 * (JX(i, jp) + JX(i, j)) -
           rdt * wi * sqrt(2.0) / dx * 0.5 * (P(i, jp) * (1.0 - P(i, jp)) + P(i, j) * (1.0 - P(i, j))));
    pn -= 0.5 * (JX(i, j) + JX(im, j)) *
          (wi * wi * (rdt / dx / dx) * (P(i, j) - P(im, j)) * 0.5 * (JX(i, j) + JX(im, j)) +
           wi * wi * (rdt / dx / dx) * 0.25 * (P(i, jp) + P(im, jp) - P(i, jm) - P(im, jm)) * 0.5 * (JY(i, j) + JY(im, j)) -
           rdt * wi * sqrt(2.0) / dx * 0.5 * (P(i, j) * (1.0 - P(i, j)) + P(im, j) * (1.0 - P(im, j))));
    pn -= 0.5 * (JY(i, j) + JY(i, jm)) *
          (wi * wi * (rdt / dx / dx) * (P(i, j) - P(i, jm)) * 0.5 * (JY(i, j) + JY(i, jm)) +
           wi * wi * (rdt / dx / dx) * 0.25 * (P(ip, j) + P(ip, jm) - P(im, j) - P(im, jm)) * 0.5 * (JX(i, j) + JX(i, jm)) -
           rdt * wi * sqrt(2.0) / dx * 0.5 * (P(i, j) * (1.0 - P(i, j)) + P(i, jm) * (1.0 - P(i, jm))));
#undef P
#undef JX
#undef JY
    return pn;
}

/* useful_functions.cpp:422-437 (corners to 0) and :439-462 (corners to the side value) */
static void dirichlet(pfo_state *st, real *t, real side, real corner)
{
    const int N = st->N;
    for (int i = 1; i < N - 1; i++) { t[C2(i, 0)] = side; t[C2(i, N - 1)] = side; t[C2(0, i)] = side; t[C2(N - 1, i)] = side; }
    t[C2(0, 0)] = corner; t[C2(0, N - 1)] = corner; t[C2(N - 1, 0)] = corner; t[C2(N - 1, N - 1)] = corner;
}

/* cell_phase_functions.cpp:709-871 */
static int reshape_field(pfo_state *st, real *f, real *fn, real side)
{
    const int N = st->N;
    const rparams *q = &st->q;
    real rdev = (2 * q->rdev_threshold) * q->rtol * q->rdt;   /* rdev_ini*rtol*rdt, constants_template.cpp:7 */
    norm_grad(st, f, st->ngl, 1);
    bc_cells(st, st->ngl, 1);
    for (int i = 1; i < N - 1; i++)
        for (int j = 1; j < N - 1; j++) {
            const real g = st->ngl[C2(i, j)];
            st->jx[C2(i, j)] = (g != 0.0) ? (1.0 / (2.0 * q->dx)) * (fn[C2(i + 1, j)] - fn[C2(i - 1, j)]) / g : 0.0;
            st->jy[C2(i, j)] = (g != 0.0) ? (1.0 / (2.0 * q->dx)) * (fn[C2(i, j + 1)] - fn[C2(i, j - 1)]) / g : 0.0;
        }
    bc_cells(st, st->jx, 1);
    bc_cells(st, st->jy, 1);
    int ri = 0;
    while (rdev > q->rdev_threshold * q->rtol * q->rdt) {
        memcpy(f, fn, (size_t)N * N * sizeof(real));
        for (int i = 1; i < N - 1; i++)
            for (int j = 1; j < N - 1; j++)
                fn[C2(i, j)] = resh_increment(f, st->jx, st->jy, N, i, j, fn[C2(i, j)], q->wi, q->rdt, q->dx);
        dirichlet(st, fn, side, 0.0);
        rdev = 0.0;
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) rdev += FABS(fn[C2(i, j)] - f[C2(i, j)]) * q->dx * q->dx;
        if (ri > q->rimax) break;
        ri++;
    }
    return ri;
}

/* The loop body of run_with_active_gels.cpp:123-182 (without the snapshot). */
int pfo_step(pfo_state *st, int it)
{
    (void)it;
    const int N = st->N, z = st->z, Nt = st->Ntot;
    const rparams *q = &st->q;
    int rc = centres(st);
    if (rc) return rc;
    maps(st);
    /* compute_hfunc_3d_tables_kernels_loop_n (useful_functions.cpp:233-251) */
    for (int n = 0; n < Nt; n++)
        for (int i = st->xc[n] - z; i < st->xc[n] + z; i++)
            for (int j = st->yc[n] - z; j < st->yc[n] + z; j++) st->hcell[C3(n, i, j)] = hfun(st->phi[C3(n, i, j)]);
    /* compute_all_hfunc_2d_tables_kernels (:272-285) */
    for (size_t k = 0; k < (size_t)N * N; k++) { st->hlum[k] = hfun(st->lum[k]); st->hecm[k] = hfun(st->ecm[k]); }
    norm_grad(st, st->phi, st->g, Nt);
    bc_cells(st, st->g, Nt);
    /* compute_prod_norm_delta (rho_functions.cpp:13-30) */
    for (int n = 0; n < Nt; n++)
        for (int i = st->xc[n] - z; i < st->xc[n] + z; i++)
            for (int j = st->yc[n] - z; j < st->yc[n] + z; j++) {
                const size_t o = C3(n, i, j);
                st->pnd[o] = st->g[o] * exp(-(st->phi[o] - 0.5) * (st->phi[o] - 0.5) / 2.0 / q->sigma / q->sigma) /
                             sqrt(2.0 * M_PI) / q->sigma;
            }
    /* compute_psi_kernels (useful_functions.cpp:305-322) */
    for (size_t k = 0; k < (size_t)N * N; k++) {
        st->psi[k] = 0.0;
        for (int n = 0; n < Nt; n++) st->psi[k] += st->hcell[(size_t)n * N * N + k];
    }
    areas(st);
    for (int n = 0; n < Nt; n++) cortex_cell(st, n);
    bc_cells(st, st->rhon, Nt);
    /* update_lumen_and_ECM (cell_phase_functions.cpp:372-444) */
    real sum_ecm = 0.0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) sum_ecm += (st->hecm[C2(i, j)]) * q->dx * q->dx;
    for (int i = 1; i < N - 1; i++)
        for (int j = 1; j < N - 1; j++) {
            const real *s = st->psi;
            const real L = -12.0 * s[C2(i, j)] + 2.0 * (s[C2(i + 1, j)] + s[C2(i - 1, j)] + s[C2(i, j + 1)] + s[C2(i, j - 1)]) +
                           s[C2(i + 1, j + 1)] + s[C2(i + 1, j - 1)] + s[C2(i - 1, j - 1)] + s[C2(i - 1, j + 1)];
            const real l = st->lum[C2(i, j)], e = st->ecm[C2(i, j)];
            st->lumn[C2(i, j)] = l;
            st->lumn[C2(i, j)] += (1.0 / q->tau_lum) * l * (1.0 - l) * q->dt *
                                  (q->xi_lum - q->beta_lum_cells * s[C2(i, j)] + q->eta_lum_cells * (L) / (4.0 * q->dx * q->dx) -
                                   q->beta_lum_ECM * st->hecm[C2(i, j)]);
            st->ecmn[C2(i, j)] = e;
            st->ecmn[C2(i, j)] += (1.0 / q->tau_ECM) * e * (1.0 - e) * q->dt *
                                  (q->alpha_ECM * (N * N * q->dx * q->dx - sum_ecm) + q->xi_ECM - q->beta_ECM_cells * s[C2(i, j)] +
                                   q->eta_ECM_cells * (L) / (4.0 * q->dx * q->dx) - q->beta_lum_ECM * st->hlum[C2(i, j)]);
        }
    dirichlet(st, st->lumn, 0.0, 0.0);
    dirichlet(st, st->ecmn, 1.0, 1.0);
    st->iters_lum = reshape_field(st, st->lum, st->lumn, 0.0);
    st->iters_ecm = reshape_field(st, st->ecm, st->ecmn, 1.0);
    /* compute_normal_to_phi (useful_functions.cpp:356-388) + boundary conditions */
    for (int n = 0; n < Nt; n++)
        for (int i = 1; i < N - 1; i++)
            for (int j = 1; j < N - 1; j++) {
                const size_t o = C3(n, i, j);
                st->jx[o] = (st->g[o] > 0.00) ? (1.0 / (2.0 * q->dx)) * (st->phi[C3(n, i + 1, j)] - st->phi[C3(n, i - 1, j)]) / st->g[o] : 0.0;
                st->jy[o] = (st->g[o] > 0.00) ? (1.0 / (2.0 * q->dx)) * (st->phi[C3(n, i, j + 1)] - st->phi[C3(n, i, j - 1)]) / st->g[o] : 0.0;
            }
    bc_cells(st, st->jx, Nt);
    bc_cells(st, st->jy, Nt);
    /* update_all_cells (cell_phase_functions.cpp:126-217); temp_phase = psi - hfunc_cell */
    for (int n = 0; n < Nt; n++)
        for (int i = st->xc[n] - z; i < st->xc[n] + z; i++)
            for (int j = st->yc[n] - z; j < st->yc[n] + z; j++) {
                const size_t o = C3(n, i, j);
#define T(a, b) (st->psi[C2(a, b)] - st->hcell[C3(n, a, b)])
#define L9(u) (-12.0 * u(i, j) + 2.0 * (u(i + 1, j) + u(i - 1, j) + u(i, j + 1) + u(i, j - 1)) + u(i + 1, j + 1) + u(i + 1, j - 1) + u(i - 1, j - 1) + u(i - 1, j + 1))
#define HL(a, b) (st->hlum[C2(a, b)])
#define HE(a, b) (st->hecm[C2(a, b)])
                const real f = st->phi[o];
                const real Tv[9] = {T(i, j), T(i + 1, j), T(i - 1, j), T(i, j + 1), T(i, j - 1), T(i + 1, j + 1),
                                    T(i + 1, j - 1), T(i - 1, j - 1), T(i - 1, j + 1)};
                const real LT = -12.0 * Tv[0] + 2.0 * (Tv[1] + Tv[2] + Tv[3] + Tv[4]) + Tv[5] + Tv[6] + Tv[7] + Tv[8];
                st->phin[o] = f;
                if (st->g[o] > 0.0)
                    st->phin[o] -= q->cpl / q->tau * (q->dt / q->dx / q->dx / 4.0) *
                                   exp(-(f - 0.5) * (f - 0.5) / 2.0 / q->sigma / q->sigma) / sqrt(2.0 * M_PI) / q->sigma *
                                   ((st->rho[C3(n, i + 1, j)] - st->rho[C3(n, i - 1, j)]) * (st->phi[C3(n, i + 1, j)] - st->phi[C3(n, i - 1, j)]) +
                                    (st->rho[C3(n, i, j + 1)] - st->rho[C3(n, i, j - 1)]) * (st->phi[C3(n, i, j + 1)] - st->phi[C3(n, i, j - 1)])) /
                                   st->g[o];
                st->phin[o] += (1.0 / q->tau) * f * (1.0 - f) * q->dt *
                               (st->f0[n] - q->beta * Tv[0] + q->eta * (LT) / (4.0 * q->dx * q->dx) -
                                q->beta_lum_cells * HL(i, j) + q->eta_lum_cells * (L9(HL)) / (4.0 * q->dx * q->dx) -
                                q->beta_ECM_cells * HE(i, j) + q->eta_ECM_cells * (L9(HE)) / (4.0 * q->dx * q->dx));
#undef T
#undef L9
#undef HL
#undef HE
            }
    bc_cells(st, st->phin, Nt);
    /* reshaping_cells (cell_phase_functions.cpp:447-580) */
    st->iters_cells_max = 0; st->iters_cells_sum = 0;
    for (int n = 0; n < Nt; n++) {
        real *ph = st->phi + (size_t)n * N * N, *pn = st->phin + (size_t)n * N * N;
        const real *X = st->jx + (size_t)n * N * N, *Y = st->jy + (size_t)n * N * N;
        int ri = 0, cnt = 0;
        real rdev = 2.0 * q->rtol * 2.0 * M_PI * q->R * q->wi * q->rdt;
        while (rdev > q->rtol * 2.0 * M_PI * q->R * q->wi * q->rdt) {
            for (int i = st->xc[n] - z; i < st->xc[n] + z; i++)
                for (int j = st->yc[n] - z; j < st->yc[n] + z; j++) ph[C2(i, j)] = pn[C2(i, j)];
            for (int i = st->xc[n] - z; i < st->xc[n] + z; i++)
                for (int j = st->yc[n] - z; j < st->yc[n] + z; j++)
                    pn[C2(i, j)] = resh_increment(ph, X, Y, N, i, j, pn[C2(i, j)], q->wi, q->rdt, q->dx);
            rdev = 0.0;
            for (int i = st->xc[n] - z; i < st->xc[n] + z; i++)
                for (int j = st->yc[n] - z; j < st->yc[n] + z; j++)
                    rdev += (FABS(pn[C2(i, j)] - ph[C2(i, j)])) * q->dx * q->dx / q->N_current;
            st->rdev_trace[2 * n] = st->rdev_trace[2 * n + 1];
            st->rdev_trace[2 * n + 1] = (double)rdev;
            if (ri > q->rimax) break;
            ri++;
            cnt++;
        }
        st->iters_cell[n] = cnt;
        st->iters_cells_sum += cnt;
        if (cnt > st->iters_cells_max) st->iters_cells_max = cnt;
    }
    /* run_with_active_gels.cpp:175-182 */
    memcpy(st->rho, st->rhon, (size_t)Nt * N * N * sizeof(real));
    memcpy(st->ecm, st->ecmn, (size_t)N * N * sizeof(real));
    memcpy(st->lum, st->lumn, (size_t)N * N * sizeof(real));
    return 0;
}

/* accessors for the ctypes harness */
real *pfo_field(pfo_state *st, const char *name)
{
    struct { const char *n; real *p; } t[] = {{"phi", st->phi}, {"rho", st->rho}, {"lum", st->lum}, {"ECM", st->ecm},
                                              {"psi", st->psi}, {"hfunc_cell", st->hcell}, {"s", st->s}, {"f0", st->f0}};
    for (size_t k = 0; k < sizeof(t) / sizeof(t[0]); k++) if (strcmp(t[k].n, name) == 0) return t[k].p;
    return 0;
}
int *pfo_centres(pfo_state *st, int which) { return which ? st->yc : st->xc; }
int *pfo_cell_iters(pfo_state *st) { return st->iters_cell; }
double *pfo_rdev_trace(pfo_state *st) { return st->rdev_trace; }
int pfo_iters(pfo_state *st, int which) { return which == 0 ? st->iters_lum : st->iters_ecm; }
int pfo_real_size(void) { return (int)sizeof(real); }
