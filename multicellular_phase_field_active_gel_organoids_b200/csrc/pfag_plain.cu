// Plain path: one kernel per reference function, full-grid passes wherever the
// reference makes them, cuFFT for the per-cell spectral solve (batched over
// cells).  This is the FP64 comparison path and what the drop-in layer calls
// function by function.  Each kernel cites the reference loop it computes.
#include "pfag_internal.cuh"
#include <cmath>

namespace {

constexpr int TBX = 32, TBY = 8;

inline dim3 grid2d(int nx, int ny, int nz) {
    return dim3((unsigned)((ny + TBX - 1) / TBX), (unsigned)((nx + TBY - 1) / TBY), (unsigned)nz);
}

// ---- find_centres_cells (useful_functions.cpp:193-227) ---------------------
template <typename real>
__global__ void k_centres_accum(const real *__restrict__ phi, int N, long long *__restrict__ acc) {
    const int n = blockIdx.y;
    long long cnt = 0, sx = 0, sy = 0;
    const size_t base = (size_t)n * N * N;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < (size_t)N * N;
         k += (size_t)gridDim.x * blockDim.x) {
        if (phi[base + k] > (real)0.5) {
            cnt++;
            sx += (long long)(k / N);
            sy += (long long)(k % N);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        sx += __shfl_down_sync(0xffffffffu, sx, o);
        sy += __shfl_down_sync(0xffffffffu, sy, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd((unsigned long long *)&acc[3 * n + 0], (unsigned long long)cnt);
        atomicAdd((unsigned long long *)&acc[3 * n + 1], (unsigned long long)sx);
        atomicAdd((unsigned long long *)&acc[3 * n + 2], (unsigned long long)sy);
    }
}

// xcenters = (int)(x_barycentre/count): integer division, as the reference.
// Zone / box bounds: the reference indexes phi[n][i+-1][j+-1] for i in
// [xc-z, xc+z) without checks, so it needs xc-z >= 1 and xc+z <= N-1.
__global__ void k_centres_finalize(const long long *__restrict__ acc, int Ntot, int N, int zone,
                                   int *__restrict__ xc, int *__restrict__ yc, unsigned *__restrict__ err) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Ntot) return;
    long long c = acc[3 * n];
    if (c == 0) {
        atomicOr(err, ERRBIT_EMPTY_CELL);
        xc[n] = N / 2;
        yc[n] = N / 2;
        return;
    }
    int x = (int)(acc[3 * n + 1] / c), y = (int)(acc[3 * n + 2] / c);
    if (x - zone < 1 || x + zone > N - 1 || y - zone < 1 || y + zone > N - 1) {
        // flag it and clamp, so that no zone kernel can index outside the grid
        atomicOr(err, ERRBIT_ZONE);
        x = min(max(x, zone + 1), N - 1 - zone);
        y = min(max(y, zone + 1), N - 1 - zone);
    }
    xc[n] = x;
    yc[n] = y;
}

// ---- create_turnover_rates_tensions (rho_functions.cpp:286-405) -------------
// Winner among phi*lum (apical, 0), phi*ECM (basal, 1), phi*phi_{n-1},
// phi*phi_{n+1} (lateral, 2 and 3); index neighbours are cyclic.
template <typename real>
__device__ __forceinline__ int map_class(real ph, real l, real e, real pm, real pp) {
    real c1l = ph * l, c1e = ph * e;
    int index;
    real mx;
    if (c1l > c1e) { index = 0; mx = c1l; } else { index = 1; mx = c1e; }
    real c1c2 = ph * pm;
    if (c1c2 > mx) { index = 2; mx = c1c2; }
    real c1c3 = ph * pp;
    if (c1c3 > mx) { index = 3; }
    return index == 3 ? 2 : index;   // 2 and 3 both lateral
}

template <typename real>
__global__ void k_maps(const real *__restrict__ phi, const real *__restrict__ lum, const real *__restrict__ ecm,
                       const int *__restrict__ xc, const int *__restrict__ yc, DevParams P,
                       real *__restrict__ deg, real *__restrict__ gen, real *__restrict__ atan_,
                       real *__restrict__ aort, real *__restrict__ visc, real *__restrict__ bm) {
    const int n = blockIdx.z, N = P.N, z = P.zone;
    const int i = xc[n] - z + blockIdx.y * TBY + threadIdx.y;
    const int j = yc[n] - z + blockIdx.x * TBX + threadIdx.x;
    if (i >= xc[n] + z || j >= yc[n] + z) return;
    const int n1 = (n == 0) ? P.Ntot - 1 : n - 1;
    const int n2 = (n == P.Ntot - 1) ? 0 : n + 1;
    const size_t s = (size_t)i * N + j;
    const real ph = phi[(size_t)n * N * N + s];
    int c = map_class<real>(ph, lum[s], ecm[s], phi[(size_t)n1 * N * N + s], phi[(size_t)n2 * N * N + s]);
    // reference index order: 0 apical, 1 basal, 2/3 lateral; P arrays: 0 ap, 1 bas, 2 lat
    const size_t o = (size_t)n * N * N + s;
    deg[o] = (real)P.deg[c];
    gen[o] = (real)P.gen[c];
    aort[o] = (real)P.a_ort[c];
    atan_[o] = (real)P.a_tan[c];
    visc[o] = (real)P.visc[c];
    bm[o] = (real)P.bb[c];
}

// ---- compute_hfunc_3d_tables_kernels_loop_n (useful_functions.cpp:233-251) --
template <typename real>
__global__ void k_hfunc_zone(const real *__restrict__ phi, real *__restrict__ h, const int *__restrict__ xc,
                             const int *__restrict__ yc, int N, int z) {
    const int n = blockIdx.z;
    const int i = xc[n] - z + blockIdx.y * TBY + threadIdx.y;
    const int j = yc[n] - z + blockIdx.x * TBX + threadIdx.x;
    if (i >= xc[n] + z || j >= yc[n] + z) return;
    const size_t o = cidx(n, i, j, N);
    real f = phi[o];
    h[o] = f * f * ((real)3.0 - (real)2.0 * f);
}

// ---- compute_all_hfunc_2d_tables_kernels (useful_functions.cpp:272-285) -----
template <typename real>
__global__ void k_hfunc_2d(const real *__restrict__ lum, const real *__restrict__ ecm, real *__restrict__ hl,
                           real *__restrict__ he, size_t ng) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < ng; k += (size_t)gridDim.x * blockDim.x) {
        real a = lum[k], b = ecm[k];
        hl[k] = a * a * ((real)3.0 - (real)2.0 * a);
        he[k] = b * b * ((real)3.0 - (real)2.0 * b);
    }
}

// ---- compute_normal_grad_phi (useful_functions.cpp:326-354) -----------------
template <typename real>
__global__ void k_norm_grad(const real *__restrict__ phi, real *__restrict__ g, int N, real c4) {
    const int n = blockIdx.z;
    const int i = 1 + blockIdx.y * TBY + threadIdx.y;
    const int j = 1 + blockIdx.x * TBX + threadIdx.x;
    if (i > N - 2 || j > N - 2) return;
    const real *p = phi + (size_t)n * N * N;
    real a = p[(size_t)(i + 1) * N + j] - p[(size_t)(i - 1) * N + j];
    real b = p[(size_t)i * N + j + 1] - p[(size_t)i * N + j - 1];
    g[cidx(n, i, j, N)] = sqrt(c4 * (a * a + b * b));
}

// ---- boundary_conditions_cells (useful_functions.cpp:391-420) --------------
// All reads are interior sites, so the ghost ring can be written in any order.
template <typename real>
__global__ void k_bc_cells(real *__restrict__ t, int N, int ncells) {
    const int n = blockIdx.y;
    if (n >= ncells) return;
    real *p = t + (size_t)n * N * N;
    const int perim = 4 * N;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < perim; k += gridDim.x * blockDim.x) {
        int i, j;
        if (k < N) { i = 0; j = k; }
        else if (k < 2 * N) { i = N - 1; j = k - N; }
        else if (k < 3 * N) { i = k - 2 * N; j = 0; }
        else { i = k - 3 * N; j = N - 1; }
        if ((k >= 2 * N) && (i == 0 || i == N - 1)) continue;  // corners written once
        p[(size_t)i * N + j] = p[(size_t)ghost_src(i, N) * N + ghost_src(j, N)];
    }
}

// ---- compute_prod_norm_delta (rho_functions.cpp:13-30) ----------------------
template <typename real>
__global__ void k_prod_norm_delta(const real *__restrict__ g, const real *__restrict__ phi, real *__restrict__ pnd,
                                  const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, real sigma) {
    const int n = blockIdx.z;
    const int i = xc[n] - z + blockIdx.y * TBY + threadIdx.y;
    const int j = yc[n] - z + blockIdx.x * TBX + threadIdx.x;
    if (i >= xc[n] + z || j >= yc[n] + z) return;
    const size_t o = cidx(n, i, j, N);
    real f = phi[o];
    pnd[o] = g[o] * exp(-(f - (real)0.5) * (f - (real)0.5) / (real)2.0 / sigma / sigma) /
             sqrt((real)(2.0 * M_PI)) / sigma;
}

// ---- compute_psi_kernels (useful_functions.cpp:305-322) ---------------------
template <typename real>
__global__ void k_psi(const real *__restrict__ h, real *__restrict__ psi, size_t ng, int ncells) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < ng; k += (size_t)gridDim.x * blockDim.x) {
        real s = (real)0.0;
        for (int n = 0; n < ncells; n++) s += h[(size_t)n * ng + k];
        psi[k] = s;
    }
}

// ---- sum_s_kernels (useful_functions.cpp:168-190): FP64 accumulation --------
// Deterministic: fixed-size per-block partials, then a fixed-order final sum.
constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 128;

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) r += sh[k];
    return r;
}

template <typename real>
__global__ void k_sum_cells(const real *__restrict__ h, size_t ng, double scale, double *__restrict__ part) {
    const int n = blockIdx.y;
    double acc = 0.0;
    const real *p = h + (size_t)n * ng;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < ng; k += (size_t)gridDim.x * blockDim.x)
        acc += (double)p[k] * scale;
    double r = block_sum(acc);
    if (threadIdx.x == 0) part[(size_t)n * gridDim.x + blockIdx.x] = r;
}

__global__ void k_sum_s_finalize(const double *__restrict__ part, int nblk, int ncells, double alpha, double s0,
                                 double *__restrict__ s, double *__restrict__ f0) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ncells) return;
    double a = 0.0;
    for (int b = 0; b < nblk; b++) a += part[(size_t)n * nblk + b];
    s[n] = a;
    f0[n] = alpha * (s0 - a);
}

// Serial-order sums (pfag_set_serial_sums): one thread per cell adds the terms
// in the order and with the expression of the reference's host loops, i-major
// with j inner.  sum_s_kernels (useful_functions.cpp:179-184):
// sum += h*dx*dx over the full grid; the reshaping check
// (cell_phase_functions.cpp:556-561): rdev += |phin-phi|*dx*dx/N_current over
// the zone; update_lumen_and_ECM's sum_ecm (:380-386) and the lumen/ECM check
// (:848-854): sum += v*dx*dx over the full grid.  Compiled without
// contraction, each partial sum then rounds as the host build's does.
template <typename real>
__global__ void k_serial_sum_cells(const real *__restrict__ h, int N, int ncells, double dx,
                                   double *__restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ncells) return;
    const real *p = h + (size_t)n * N * N;
    double acc = 0.0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) acc += (double)p[(size_t)i * N + j] * dx * dx;
    out[n] = acc;
}

template <typename real>
__global__ void k_serial_absdiff(const real *__restrict__ a, const real *__restrict__ b, int N, double dx,
                                 double *__restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double acc = 0.0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            const size_t o = (size_t)i * N + j;
            acc += fabs((double)a[o] - (double)b[o]) * dx * dx;
        }
    *out = acc;
}

template <typename real>
__global__ void k_serial_cell_rdev(const real *__restrict__ pn, const real *__restrict__ p,
                                   const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, int ncells,
                                   double dx, double ncur, const int *__restrict__ active,
                                   double *__restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ncells) return;
    double acc = 0.0;
    if (active[n])
        for (int i = xc[n] - z; i < xc[n] + z; i++)
            for (int j = yc[n] - z; j < yc[n] + z; j++) {
                const size_t o = cidx(n, i, j, N);
                acc += fabs((double)pn[o] - (double)p[o]) * dx * dx / ncur;
            }
    out[n] = acc;
}

// ---- update_all_cortices helpers (rho_functions.cpp:32-284, useful_functions.cpp:605-625)
template <typename real>
__global__ void k_pi(const real *__restrict__ rho, const real *__restrict__ g, const real *__restrict__ phi,
                     const real *__restrict__ atan_, const real *__restrict__ aort, const real *__restrict__ bm,
                     const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, real c4,
                     real *__restrict__ pxx, real *__restrict__ pxy, real *__restrict__ pyy) {
    const int n = blockIdx.z;
    const int i = xc[n] - z + blockIdx.y * TBY + threadIdx.y;
    const int j = yc[n] - z + blockIdx.x * TBX + threadIdx.x;
    if (i >= xc[n] + z || j >= yc[n] + z) return;
    const size_t o = cidx(n, i, j, N);
    const real r = rho[o], at = atan_[o], ao = aort[o], b = bm[o], gg = g[o];
    const real *p = phi + (size_t)n * N * N;
    const real dxp = p[(size_t)(i + 1) * N + j] - p[(size_t)(i - 1) * N + j];
    const real dyp = p[(size_t)i * N + j + 1] - p[(size_t)i * N + j - 1];
    real xx = -at * r * r * r + b * r * r * r * r;
    real yy = xx;
    real xy = (real)0.0;
    if (gg > (real)0.0) {
        xx += (at - ao) * r * r * r * c4 * dxp * dxp / gg / gg;   // rho_functions.cpp:51
        yy += (at - ao) * r * r * r * c4 * dyp * dyp / gg / gg;   // :79
        xy += (at - ao) * r * r * r * c4 * dxp * dyp / gg / gg;   // :109
    }
    pxx[o] = xx;
    pxy[o] = xy;
    pyy[o] = yy;
}

// load_temp_fft: box[i][j] = table[n][i+1+xc-z][j+1+yc-z] + 0i
template <typename real>
__global__ void k_box_load(const real *__restrict__ t, typename Cplx<real>::type *__restrict__ box,
                           const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, int M) {
    const int n = blockIdx.z;
    const int i = blockIdx.y * TBY + threadIdx.y, j = blockIdx.x * TBX + threadIdx.x;
    if (i >= M || j >= M) return;
    const int gi = i + 1 + xc[n] - z, gj = j + 1 + yc[n] - z;
    typename Cplx<real>::type v;
    v.x = t[cidx(n, gi, gj, N)];
    v.y = (real)0.0;
    box[((size_t)n * M + i) * M + j] = v;
}

// create_deg_gen (rho_functions.cpp:193-209): -deg*rho + gen*prod_norm_delta
template <typename real>
__global__ void k_box_deg_gen(const real *__restrict__ deg, const real *__restrict__ rho, const real *__restrict__ gen,
                              const real *__restrict__ pnd, typename Cplx<real>::type *__restrict__ box,
                              const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, int M) {
    const int n = blockIdx.z;
    const int i = blockIdx.y * TBY + threadIdx.y, j = blockIdx.x * TBX + threadIdx.x;
    if (i >= M || j >= M) return;
    const size_t o = cidx(n, i + 1 + xc[n] - z, j + 1 + yc[n] - z, N);
    typename Cplx<real>::type v;
    v.x = -deg[o] * rho[o] + gen[o] * pnd[o];
    v.y = (real)0.0;
    box[((size_t)n * M + i) * M + j] = v;
}

// update_rho_velocity (rho_functions.cpp:133-190); viscosity is read at the
// real-space box site with the same (i, j) as the wavevector.
template <typename real>
__global__ void k_velocity(const typename Cplx<real>::type *__restrict__ fxx,
                           const typename Cplx<real>::type *__restrict__ fyy,
                           const typename Cplx<real>::type *__restrict__ fxy,
                           typename Cplx<real>::type *__restrict__ fvx, typename Cplx<real>::type *__restrict__ fvy,
                           const real *__restrict__ visc, const int *__restrict__ xc, const int *__restrict__ yc,
                           int N, int z, int M, double kfac, real friction) {
    const int n = blockIdx.z;
    const int i = blockIdx.y * TBY + threadIdx.y, j = blockIdx.x * TBX + threadIdx.x;
    if (i >= M || j >= M) return;
    const size_t b = ((size_t)n * M + i) * M + j;
    const int ir = (i < M / 2) ? i : i - M;
    const int jr = (j < M / 2) ? j : j - M;
    const real kx = (real)(kfac * ir), ky = (real)(kfac * jr);
    const real et = visc[cidx(n, i + 1 + xc[n] - z, j + 1 + yc[n] - z, N)];
    const auto pxx = fxx[b], pyy = fyy[b], pxy = fxy[b];
    const real A = friction + (real)2.0 * et * (kx * kx + ky * ky / (real)2.0);
    const real D = -((real)4.0 * et * et * kx * kx * ky * ky + friction * friction +
                     (real)3.0 * et * friction * (kx * kx + ky * ky) +
                     (real)2.0 * et * et * (kx * kx * kx * kx + ky * ky * ky * ky));
    typename Cplx<real>::type vx, vy;
    vy.x = (real)0.0 + et * kx * ky * (kx * pxx.y + ky * pxy.y);
    vy.x -= A * (ky * pyy.y + kx * pxy.y);
    vy.x /= D;
    vy.y = (real)0.0 - et * kx * ky * (kx * pxx.x + ky * pxy.x);
    vy.y += A * (ky * pyy.x + kx * pxy.x);
    vy.y /= D;
    vx.x = (real)0.0 + (kx * pxx.y + ky * pxy.y - et * kx * ky * vy.x);
    vx.x /= A;
    vx.y = (real)0.0 + (-kx * pxx.x - ky * pxy.x - et * kx * ky * vy.y);
    vx.y /= A;
    fvx[b] = vx;
    fvy[b] = vy;
}

// load_fft_rho_v (rho_functions.cpp:267-284): rho * Re(v) / (M*M) + 0i
template <typename real>
__global__ void k_load_rho_v(const real *__restrict__ rho, const typename Cplx<real>::type *__restrict__ tr,
                             typename Cplx<real>::type *__restrict__ box, const int *__restrict__ xc,
                             const int *__restrict__ yc, int N, int z, int M, real *__restrict__ vdbg) {
    const int n = blockIdx.z;
    const int i = blockIdx.y * TBY + threadIdx.y, j = blockIdx.x * TBX + threadIdx.x;
    if (i >= M || j >= M) return;
    const size_t b = ((size_t)n * M + i) * M + j;
    const real mm = (real)((double)M * (double)M);
    typename Cplx<real>::type v;
    v.x = rho[cidx(n, i + 1 + xc[n] - z, j + 1 + yc[n] - z, N)] * tr[b].x / mm;
    v.y = (real)0.0;
    box[b] = v;
    if (vdbg) vdbg[b] = tr[b].x / mm;
}

// update_fft_rho (rho_functions.cpp:213-251)
template <typename real>
__global__ void k_update_fft_rho(typename Cplx<real>::type *__restrict__ fr,
                                 const typename Cplx<real>::type *__restrict__ freact,
                                 const typename Cplx<real>::type *__restrict__ frvx,
                                 const typename Cplx<real>::type *__restrict__ frvy, int M, real dt, double kfac) {
    const int n = blockIdx.z;
    const int i = blockIdx.y * TBY + threadIdx.y, j = blockIdx.x * TBX + threadIdx.x;
    if (i >= M || j >= M) return;
    const size_t b = ((size_t)n * M + i) * M + j;
    const int ir = (i < M / 2) ? i : i - M;
    const int jr = (j < M / 2) ? j : j - M;
    auto r = fr[b];
    const auto q = freact[b];
    r.x += dt * q.x;
    r.y += dt * q.y;
    const real dk = (real)((double)dt * kfac);
    const auto a = frvx[b], c = frvy[b];
    r.x += dk * ((real)ir * a.y + (real)jr * c.y);
    r.y -= dk * ((real)ir * a.x + (real)jr * c.x);
    fr[b] = r;
}

// copy_to_rhon (rho_functions.cpp:253-265)
template <typename real>
__global__ void k_copy_to_rhon(const typename Cplx<real>::type *__restrict__ box, real *__restrict__ rhon,
                               const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, int M) {
    const int n = blockIdx.z;
    const int i = blockIdx.y * TBY + threadIdx.y, j = blockIdx.x * TBX + threadIdx.x;
    if (i >= M || j >= M) return;
    rhon[cidx(n, i + 1 + xc[n] - z, j + 1 + yc[n] - z, N)] =
        box[((size_t)n * M + i) * M + j].x / (real)((double)M * (double)M);
}

// ---- update_lumen_and_ECM (cell_phase_functions.cpp:372-444) ---------------
template <typename real>
__global__ void k_lum_ecm_update(const real *__restrict__ lum, const real *__restrict__ ecm,
                                 const real *__restrict__ psi, const real *__restrict__ hl, const real *__restrict__ he,
                                 real *__restrict__ lumn, real *__restrict__ ecmn, DevParams P,
                                 const double *__restrict__ sum_ecm) {
    const int N = P.N;
    const int i = 1 + blockIdx.y * TBY + threadIdx.y, j = 1 + blockIdx.x * TBX + threadIdx.x;
    if (i > N - 2 || j > N - 2) return;
    const size_t c = (size_t)i * N + j;
    const real s = psi[c];
    const real L = lap9<real>(s, psi[c + N], psi[c - N], psi[c + 1], psi[c - 1], psi[c + N + 1], psi[c + N - 1],
                              psi[c - N - 1], psi[c - N + 1]);
    const real dx = (real)P.dx, dt = (real)P.dt;
    const real l = lum[c], e = ecm[c];
    real ln = l;
    ln += ((real)1.0 / (real)P.tau_lum) * l * ((real)1.0 - l) * dt *
          ((real)P.xi_lum - (real)P.beta_lum_cells * s + (real)P.eta_lum_cells * L / ((real)4.0 * dx * dx) -
           (real)P.beta_lum_ECM * he[c]);
    real en = e;
    const real elastic = (real)(P.alpha_ECM * ((double)N * (double)N * P.dx * P.dx - *sum_ecm));
    en += ((real)1.0 / (real)P.tau_ECM) * e * ((real)1.0 - e) * dt *
          (elastic + (real)P.xi_ECM - (real)P.beta_ECM_cells * s + (real)P.eta_ECM_cells * L / ((real)4.0 * dx * dx) -
           (real)P.beta_lum_ECM * hl[c]);
    lumn[c] = ln;
    ecmn[c] = en;
}

// boundary_conditions_lumen_and_ECM (useful_functions.cpp:439-462) and
// boundary_conditions_dirichlet (:422-437): sides to the side value, corners
// to `corner` (0 for the Dirichlet helper, the side value for the first one).
template <typename real>
__global__ void k_dirichlet(real *__restrict__ t, int N, real side, real corner) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 4 * N; k += gridDim.x * blockDim.x) {
        int i, j;
        if (k < N) { i = 0; j = k; }
        else if (k < 2 * N) { i = N - 1; j = k - N; }
        else if (k < 3 * N) { i = k - 2 * N; j = 0; }
        else { i = k - 3 * N; j = N - 1; }
        if ((k >= 2 * N) && (i == 0 || i == N - 1)) continue;
        bool corner_site = (i == 0 || i == N - 1) && (j == 0 || j == N - 1);
        t[(size_t)i * N + j] = corner_site ? corner : side;
    }
}

// reshaping_lumen_or_ECM prologue (cell_phase_functions.cpp:722-771)
template <typename real>
__global__ void k_norm_grad_2d(const real *__restrict__ f, real *__restrict__ g, int N, real c4) {
    const int i = 1 + blockIdx.y * TBY + threadIdx.y, j = 1 + blockIdx.x * TBX + threadIdx.x;
    if (i > N - 2 || j > N - 2) return;
    const size_t c = (size_t)i * N + j;
    real a = f[c + N] - f[c - N], b = f[c + 1] - f[c - 1];
    g[c] = sqrt(c4 * (a * a + b * b));
}

template <typename real>
__global__ void k_lum_normals(const real *__restrict__ lumn, const real *__restrict__ ngl, real *__restrict__ jx,
                              real *__restrict__ jy, int N, real inv2dx) {
    const int i = 1 + blockIdx.y * TBY + threadIdx.y, j = 1 + blockIdx.x * TBX + threadIdx.x;
    if (i > N - 2 || j > N - 2) return;
    const size_t c = (size_t)i * N + j;
    const real g = ngl[c];
    jx[c] = (g != (real)0.0) ? inv2dx * (lumn[c + N] - lumn[c - N]) / g : (real)0.0;
    jy[c] = (g != (real)0.0) ? inv2dx * (lumn[c + 1] - lumn[c - 1]) / g : (real)0.0;
}

// one relaxation update of the lumen/ECM field (interior), :802-838
template <typename real>
__global__ void k_lum_relax(const real *__restrict__ p, real *__restrict__ pn, const real *__restrict__ jx,
                            const real *__restrict__ jy, int N, real A, real B) {
    const int i = 1 + blockIdx.y * TBY + threadIdx.y, j = 1 + blockIdx.x * TBX + threadIdx.x;
    if (i > N - 2 || j > N - 2) return;
    const size_t c = (size_t)i * N + j;
    real q[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) q[a][b] = p[c + (size_t)(a - 1) * N + (b - 1)];
    pn[c] = resh_update<real>(A, B, q, jx[c], jx[c + N], jx[c - N], jx[c + 1], jx[c - 1], jy[c], jy[c + N],
                              jy[c - N], jy[c + 1], jy[c - 1], pn[c]);
}

template <typename real>
__global__ void k_absdiff_sum(const real *__restrict__ a, const real *__restrict__ b, size_t ng, double scale,
                              double *__restrict__ part) {
    double acc = 0.0;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < ng; k += (size_t)gridDim.x * blockDim.x)
        acc += fabs((double)a[k] - (double)b[k]) * scale;
    double r = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void k_sum_partials(const double *__restrict__ part, int nblk, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0.0;
        for (int b = 0; b < nblk; b++) a += part[b];
        *out = a;
    }
}

// ---- compute_normal_to_phi (useful_functions.cpp:356-388) -------------------
template <typename real>
__global__ void k_normals(const real *__restrict__ phi, const real *__restrict__ g, real *__restrict__ jx,
                          real *__restrict__ jy, int N, real inv2dx) {
    const int n = blockIdx.z;
    const int i = 1 + blockIdx.y * TBY + threadIdx.y, j = 1 + blockIdx.x * TBX + threadIdx.x;
    if (i > N - 2 || j > N - 2) return;
    const real *p = phi + (size_t)n * N * N;
    const size_t c = (size_t)i * N + j, o = (size_t)n * N * N + c;
    const real gg = g[o];
    jx[o] = (gg > (real)0.0) ? inv2dx * (p[c + N] - p[c - N]) / gg : (real)0.0;
    jy[o] = (gg > (real)0.0) ? inv2dx * (p[c + 1] - p[c - 1]) / gg : (real)0.0;
}

// ---- update_all_cells (cell_phase_functions.cpp:126-217) --------------------
// temp_phase = psi - hfunc_cell is formed on the fly at each stencil point.
template <typename real>
__global__ void k_update_cells(const real *__restrict__ phi, real *__restrict__ phin, const real *__restrict__ g,
                               const real *__restrict__ rho, const real *__restrict__ h, const double *__restrict__ f0,
                               const real *__restrict__ psi, const int *__restrict__ xc, const int *__restrict__ yc,
                               const real *__restrict__ hl, const real *__restrict__ he, DevParams P) {
    const int n = blockIdx.z, N = P.N, z = P.zone;
    const int i = xc[n] - z + blockIdx.y * TBY + threadIdx.y;
    const int j = yc[n] - z + blockIdx.x * TBX + threadIdx.x;
    if (i >= xc[n] + z || j >= yc[n] + z) return;
    const size_t c = (size_t)i * N + j, base = (size_t)n * N * N, o = base + c;
    const real dx = (real)P.dx, dt = (real)P.dt, tau = (real)P.tau, sigma = (real)P.sigma;
    const real f = phi[o];
    real pn = f;
    const real gg = g[o];
    if (gg > (real)0.0) {
        const real *p = phi + base, *r = rho + base;
        pn -= (real)P.cpl / tau * (dt / dx / dx / (real)4.0) *
              exp(-(f - (real)0.5) * (f - (real)0.5) / (real)2.0 / sigma / sigma) / sqrt((real)(2.0 * M_PI)) / sigma *
              ((r[c + N] - r[c - N]) * (p[c + N] - p[c - N]) + (r[c + 1] - r[c - 1]) * (p[c + 1] - p[c - 1])) / gg;
    }
    const real *hh = h + base;
    auto T = [&](size_t k) { return psi[k] - hh[k]; };
    const real Tc = T(c);
    const real LT = lap9<real>(Tc, T(c + N), T(c - N), T(c + 1), T(c - 1), T(c + N + 1), T(c + N - 1),
                               T(c - N - 1), T(c - N + 1));
    const real Ll = lap9<real>(hl[c], hl[c + N], hl[c - N], hl[c + 1], hl[c - 1], hl[c + N + 1], hl[c + N - 1],
                               hl[c - N - 1], hl[c - N + 1]);
    const real Le = lap9<real>(he[c], he[c + N], he[c - N], he[c + 1], he[c - 1], he[c + N + 1], he[c + N - 1],
                               he[c - N - 1], he[c - N + 1]);
    const real q4 = (real)4.0 * dx * dx;
    pn += ((real)1.0 / tau) * f * ((real)1.0 - f) * dt *
          ((real)f0[n] - (real)P.beta * Tc + (real)P.eta * LT / q4 - (real)P.beta_lum_cells * hl[c] +
           (real)P.eta_lum_cells * Ll / q4 - (real)P.beta_ECM_cells * he[c] + (real)P.eta_ECM_cells * Le / q4);
    phin[o] = pn;
}

// ---- reshaping_cells (cell_phase_functions.cpp:447-580) ---------------------
// active[n] != 0 while cell n is still iterating.
template <typename real>
__global__ void k_zone_copy(real *__restrict__ dst, const real *__restrict__ src, const int *__restrict__ xc,
                            const int *__restrict__ yc, int N, int z, const int *__restrict__ active) {
    const int n = blockIdx.z;
    if (!active[n]) return;
    const int i = xc[n] - z + blockIdx.y * TBY + threadIdx.y;
    const int j = yc[n] - z + blockIdx.x * TBX + threadIdx.x;
    if (i >= xc[n] + z || j >= yc[n] + z) return;
    dst[cidx(n, i, j, N)] = src[cidx(n, i, j, N)];
}

template <typename real>
__global__ void k_cell_relax(const real *__restrict__ p, real *__restrict__ pn, const real *__restrict__ jx,
                             const real *__restrict__ jy, const int *__restrict__ xc, const int *__restrict__ yc,
                             int N, int z, real A, real B, const int *__restrict__ active) {
    const int n = blockIdx.z;
    if (!active[n]) return;
    const int i = xc[n] - z + blockIdx.y * TBY + threadIdx.y;
    const int j = yc[n] - z + blockIdx.x * TBX + threadIdx.x;
    if (i >= xc[n] + z || j >= yc[n] + z) return;
    const size_t base = (size_t)n * N * N, c = (size_t)i * N + j;
    const real *q = p + base, *X = jx + base, *Y = jy + base;
    real w[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) w[a][b] = q[c + (size_t)(a - 1) * N + (b - 1)];
    pn[base + c] = resh_update<real>(A, B, w, X[c], X[c + N], X[c - N], X[c + 1], X[c - 1], Y[c], Y[c + N],
                                     Y[c - N], Y[c + 1], Y[c - 1], pn[base + c]);
}

// rdev per active cell: sum over the zone of |phin - phi| dx^2 / N_current
template <typename real>
__global__ void k_cell_rdev(const real *__restrict__ pn, const real *__restrict__ p, const int *__restrict__ xc,
                            const int *__restrict__ yc, int N, int z, double scale, const int *__restrict__ active,
                            double *__restrict__ part) {
    const int n = blockIdx.y;
    double acc = 0.0;
    if (active[n]) {
        const int w = 2 * z;
        const size_t tot = (size_t)w * w;
        for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += (size_t)gridDim.x * blockDim.x) {
            const int i = xc[n] - z + (int)(k / w), j = yc[n] - z + (int)(k % w);
            const size_t o = cidx(n, i, j, N);
            acc += fabs((double)pn[o] - (double)p[o]) * scale;
        }
    }
    double r = block_sum(acc);
    if (threadIdx.x == 0) part[(size_t)n * gridDim.x + blockIdx.x] = r;
}

// Convergence bookkeeping of the while loop at cell_phase_functions.cpp:475-574:
// after an iteration, the loop ends when rdev <= thr, or (ri > rimax) breaks.
__global__ void k_cell_check(const double *__restrict__ part, int nblk, int ncells, double thr, int rimax,
                             int *__restrict__ active, int *__restrict__ ri, int *__restrict__ nactive,
                             unsigned *__restrict__ err) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ncells) return;
    if (!active[n]) return;
    double a = 0.0;
    for (int b = 0; b < nblk; b++) a += part[(size_t)n * nblk + b];
    bool stop = false;
    if (ri[n] > rimax) { atomicOr(err, ERRBIT_RELAX); stop = true; }
    else ri[n]++;
    if (a <= thr) stop = true;
    if (stop) active[n] = 0;
    else atomicAdd(nactive, 1);
}

template <typename real>
__global__ void k_copy(real *__restrict__ dst, const real *__restrict__ src, size_t n) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = src[k];
}

// ---------------------------------------------------------------------------
// ---- initial-condition generator (initialisation_code/prepare_initial_files.cpp:53-117)

// ini_phi (functions/initialisation_functions.cpp:116-160): N_ini cells on a
// ring of radius rcyst about the grid centre (one cell: at the centre), each a
// logistic profile 1/(1 + exp((dx r - R0)/wi)).  The float build computes the
// centre in double and stores it as float, r, the exponent and exp in float.
template <typename real>
__global__ void k_ini_phi(real *__restrict__ phi, int N, int N_ini, real dx, real R0, real wi, real rcyst) {
    const int n = blockIdx.z;
    const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || j >= N) return;
    real xcen, ycen;
    if (N_ini > 1) {
        xcen = (real)((double)(N / 2) + (double)rcyst * cos((double)n * 2.0 * M_PI / (double)N_ini));
        ycen = (real)((double)(N / 2) + (double)rcyst * sin((double)n * 2.0 * M_PI / (double)N_ini));
    } else {
        xcen = (real)(N / 2);
        ycen = (real)(N / 2);
    }
    const real di = (real)i - xcen, dj = (real)j - ycen;
    const real e = exp((dx * sqrt(di * di + dj * dj) - R0) / wi);
    phi[(size_t)n * N * N + (size_t)i * N + j] = (real)(1.0 / (1.0 + (double)e));
}

// ini_ECM_lumen (initialisation_functions.cpp:72-110): the space the cells
// leave free, 1 - sum phi, is lumen inside the ring radius and ECM outside;
// zero where the cells fill the site.  Sites not assigned stay zero.
template <typename real>
__global__ void k_ini_lum_ecm(const real *__restrict__ phi, real *__restrict__ lum, real *__restrict__ ecm, int N,
                              int N_ini, real rcyst) {
    const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || j >= N) return;
    const size_t k = (size_t)i * N + j, NN = (size_t)N * N;
    real all = (real)0.0;
    for (int n = 0; n < N_ini; n++) all += phi[(size_t)n * NN + k];
    real l = (real)0.0, e = (real)0.0;
    if (1.0 - (double)all > 0.0) {
        const int a = i - N / 2, b = j - N / 2;
        const double d = sqrt((double)(a * a + b * b));
        if (d < (double)rcyst) l = (real)(1.0 - (double)all);
        else e = (real)(1.0 - (double)all);
    }
    lum[k] = l;
    ecm[k] = e;
}

// The cortex density of a phase value (initialisation_functions.cpp:62-70 and
// update_rho_to_shape, cell_phase_functions.cpp:42-62), in double as both
// builds evaluate it: rho0 exp(-1/(4 h (1 - h) + tol) + 1/(1 + tol)),
// h = phi^2 (3 - 2 phi), and 0 below the floor rho0 exp(-1/(2 tol) + 1/(1 + tol)).
// set_everywhere: ini_rho assigns every site; update_rho_to_shape only sites
// with phi != 0 (then applies the floor to every site).
template <typename real>
__global__ void k_rho_shape(const real *__restrict__ phi, real *__restrict__ rho, size_t n, double rho0, double tol,
                            int set_everywhere) {
    // rho0 and tol are parameters of the build's precision
    rho0 = (double)(real)rho0;
    tol = (double)(real)tol;
    const double floor_v = rho0 * exp(-1.0 / (2.0 * tol) + 1.0 / (1.0 + tol));
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const real p = phi[k];
        const double f = (double)p;
        const double pp = (double)(p * p);     // phi*phi is a product in the build's precision there
        real r = rho[k];
        if (set_everywhere || p != (real)0.0)
            r = (real)(rho0 * exp(-1.0 / (4.0 * f * f * (3.0 - 2.0 * f) * (1.0 - pp * (3.0 - 2.0 * f)) + tol) +
                                  1.0 / (1.0 + tol)));
        if ((double)r < floor_v) r = (real)0.0;
        rho[k] = r;
    }
}

template <typename real> struct FFTX;
template <> struct FFTX<double> {
    static cufftResult exec(cufftHandle p, void *in, void *out, int dir) {
        return cufftExecZ2Z(p, (cufftDoubleComplex *)in, (cufftDoubleComplex *)out, dir);
    }
    static constexpr cufftType type = CUFFT_Z2Z;
};
template <> struct FFTX<float> {
    static cufftResult exec(cufftHandle p, void *in, void *out, int dir) {
        return cufftExecC2C(p, (cufftComplex *)in, (cufftComplex *)out, dir);
    }
    static constexpr cufftType type = CUFFT_C2C;
};

template <typename real>
struct Plain {
    typedef typename Cplx<real>::type cx;
    pfag_ctx *c;
    explicit Plain(pfag_ctx *ctx) : c(ctx) {}
    real *R(void *p) { return (real *)p; }
    dim3 zone_grid() { return grid2d(2 * c->zone, 2 * c->zone, c->Ntot); }
    dim3 interior_grid(int ncells) { return grid2d(c->N - 2, c->N - 2, ncells); }
    dim3 box_grid() { return grid2d(c->M, c->M, c->Ntot); }
    cx *fb(int k) { return (cx *)c->fftbuf + (size_t)k * c->Ntot * c->M * c->M; }

    int centres() {
        const int N = c->N;
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_cacc, 0, sizeof(long long) * 3 * c->Ntot, c->stream));
        int nb = (int)std::min<size_t>(64, ((size_t)N * N + 255) / 256);
        k_centres_accum<real><<<dim3(nb, c->Ntot), 256, 0, c->stream>>>(R(c->phi), N, c->d_cacc);
        PFAG_LAUNCHED(c);
        k_centres_finalize<<<(c->Ntot + 127) / 128, 128, 0, c->stream>>>(c->d_cacc, c->Ntot, N, c->zone, c->d_xc,
                                                                           c->d_yc, c->d_err);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int maps() {
        void **m = c->maps;
        k_maps<real><<<zone_grid(), dim3(TBX, TBY), 0, c->stream>>>(
            R(c->phi), R(c->lum), R(c->ecm), c->d_xc, c->d_yc, c->dp, R(m[0]), R(m[1]), R(m[2]), R(m[3]), R(m[4]),
            R(m[5]));
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int hfunc3d() {
        k_hfunc_zone<real><<<zone_grid(), dim3(TBX, TBY), 0, c->stream>>>(R(c->phi), R(c->hfunc), c->d_xc, c->d_yc,
                                                                           c->N, c->zone);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int hfunc2d() {
        k_hfunc_2d<real><<<592, 256, 0, c->stream>>>(R(c->lum), R(c->ecm), R(c->hlum), R(c->hecm), c->ng);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int bc_cells(void *t, int ncells) {
        k_bc_cells<real><<<dim3((4 * c->N + 255) / 256, ncells), 256, 0, c->stream>>>(R(t), c->N, ncells);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    real c4() { return (real)(1.0 / c->dp.dx / c->dp.dx / 4.0); }
    int norm_grad() {
        k_norm_grad<real><<<interior_grid(c->Ntot), dim3(TBX, TBY), 0, c->stream>>>(R(c->phi), R(c->g), c->N, c4());
        PFAG_LAUNCHED(c);
        return bc_cells(c->g, c->Ntot);
    }
    int prod_norm_delta() {
        k_prod_norm_delta<real><<<zone_grid(), dim3(TBX, TBY), 0, c->stream>>>(
            R(c->g), R(c->phi), R(c->pnd), c->d_xc, c->d_yc, c->N, c->zone, (real)c->dp.sigma);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int psi() {
        k_psi<real><<<592, 256, 0, c->stream>>>(R(c->hfunc), R(c->psi), c->ng, c->Ntot);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int sum_s() {
        int nblk = RED_BLOCKS;
        if (c->serial_sums) {
            nblk = 1;
            k_serial_sum_cells<real><<<(c->Ntot + 63) / 64, 64, 0, c->stream>>>(R(c->hfunc), c->N, c->Ntot,
                                                                                c->dp.dx, c->d_part);
        } else {
            k_sum_cells<real><<<dim3(RED_BLOCKS, c->Ntot), RED_THREADS, 0, c->stream>>>(R(c->hfunc), c->ng,
                                                                                       c->dp.dx * c->dp.dx, c->d_part);
        }
        PFAG_LAUNCHED(c);
        k_sum_s_finalize<<<(c->Ntot + 127) / 128, 128, 0, c->stream>>>(c->d_part, nblk, c->Ntot, c->dp.alpha,
                                                                         c->dp.s0, c->d_s, c->d_f0);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int fft(cx *in, cx *out, int dir) {
        PFAG_CUFFT_CHECK(FFTX<real>::exec(c->plan, in, out, dir));
        c->launches += 2;   // cuFFT library launches (row and column passes)
        return PFAG_OK;
    }
    int cortices() {
        const int N = c->N, z = c->zone, M = c->M;
        cx *T = fb(0), *TR = fb(1), *Frho = fb(2), *Freact = fb(3), *Fxx = fb(4), *Fxy = fb(5), *Fyy = fb(6),
           *Fvx = fb(7), *Fvy = fb(8), *Frvx = fb(9), *Frvy = fb(10);
        dim3 bg = box_grid(), tb(TBX, TBY);
        cudaStream_t s = c->stream;
        k_box_load<real><<<bg, tb, 0, s>>>(R(c->rho), T, c->d_xc, c->d_yc, N, z, M); PFAG_LAUNCHED(c);
        PFAG_TRY(fft(T, Frho, CUFFT_FORWARD));
        k_box_deg_gen<real><<<bg, tb, 0, s>>>(R(c->maps[0]), R(c->rho), R(c->maps[1]), R(c->pnd), T, c->d_xc,
                                               c->d_yc, N, z, M);
        PFAG_LAUNCHED(c);
        PFAG_TRY(fft(T, Freact, CUFFT_FORWARD));
        k_pi<real><<<zone_grid(), tb, 0, s>>>(R(c->rho), R(c->g), R(c->phi), R(c->maps[2]), R(c->maps[3]),
                                              R(c->maps[5]), c->d_xc, c->d_yc, N, z, c4(), R(c->pixx), R(c->pixy),
                                              R(c->piyy));
        PFAG_LAUNCHED(c);
        k_box_load<real><<<bg, tb, 0, s>>>(R(c->pixx), T, c->d_xc, c->d_yc, N, z, M); PFAG_LAUNCHED(c);
        PFAG_TRY(fft(T, Fxx, CUFFT_FORWARD));
        k_box_load<real><<<bg, tb, 0, s>>>(R(c->pixy), T, c->d_xc, c->d_yc, N, z, M); PFAG_LAUNCHED(c);
        PFAG_TRY(fft(T, Fxy, CUFFT_FORWARD));
        k_box_load<real><<<bg, tb, 0, s>>>(R(c->piyy), T, c->d_xc, c->d_yc, N, z, M); PFAG_LAUNCHED(c);
        PFAG_TRY(fft(T, Fyy, CUFFT_FORWARD));
        k_velocity<real><<<bg, tb, 0, s>>>(Fxx, Fyy, Fxy, Fvx, Fvy, R(c->maps[4]), c->d_xc, c->d_yc, N, z, M,
                                           c->dp.kfac, (real)c->dp.friction);
        PFAG_LAUNCHED(c);
        PFAG_TRY(fft(Fvx, TR, CUFFT_INVERSE));
        k_load_rho_v<real><<<bg, tb, 0, s>>>(R(c->rho), TR, T, c->d_xc, c->d_yc, N, z, M,
                                             c->debug ? R(c->d_vx) : nullptr);
        PFAG_LAUNCHED(c);
        PFAG_TRY(fft(T, Frvx, CUFFT_FORWARD));
        PFAG_TRY(fft(Fvy, TR, CUFFT_INVERSE));
        k_load_rho_v<real><<<bg, tb, 0, s>>>(R(c->rho), TR, T, c->d_xc, c->d_yc, N, z, M,
                                             c->debug ? R(c->d_vy) : nullptr);
        PFAG_LAUNCHED(c);
        PFAG_TRY(fft(T, Frvy, CUFFT_FORWARD));
        k_update_fft_rho<real><<<bg, tb, 0, s>>>(Frho, Freact, Frvx, Frvy, M, (real)c->dp.dt, c->dp.kfac);
        PFAG_LAUNCHED(c);
        PFAG_TRY(fft(Frho, T, CUFFT_INVERSE));
        k_copy_to_rhon<real><<<bg, tb, 0, s>>>(T, R(c->rhon), c->d_xc, c->d_yc, N, z, M); PFAG_LAUNCHED(c);
        return bc_cells(c->rhon, c->Ntot);
    }
    int sum_reduce_2d(const void *a, const void *b, double scale, double *out) {
        if (c->serial_sums) {
            k_serial_absdiff<real><<<1, 32, 0, c->stream>>>(R((void *)a), R((void *)b), c->N, c->dp.dx, out);
            PFAG_LAUNCHED(c);
            return PFAG_OK;
        }
        k_absdiff_sum<real><<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(R((void *)a), R((void *)b), c->ng, scale,
                                                                      c->d_part);
        PFAG_LAUNCHED(c);
        k_sum_partials<<<1, 32, 0, c->stream>>>(c->d_part, RED_BLOCKS, out);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int lum_ecm_update() {
        const int N = c->N;
        // sum_ecm = sum h(ECM) dx^2 over the full grid (FP64)
        if (c->serial_sums) {
            k_serial_sum_cells<real><<<1, 32, 0, c->stream>>>(R(c->hecm), N, 1, c->dp.dx, c->d_scal + 0);
            PFAG_LAUNCHED(c);
        } else {
            k_sum_cells<real><<<dim3(RED_BLOCKS, 1), RED_THREADS, 0, c->stream>>>(R(c->hecm), c->ng,
                                                                                 c->dp.dx * c->dp.dx, c->d_part);
            PFAG_LAUNCHED(c);
            k_sum_partials<<<1, 32, 0, c->stream>>>(c->d_part, RED_BLOCKS, c->d_scal + 0);
            PFAG_LAUNCHED(c);
        }
        k_lum_ecm_update<real><<<interior_grid(1), dim3(TBX, TBY), 0, c->stream>>>(
            R(c->lum), R(c->ecm), R(c->psi), R(c->hlum), R(c->hecm), R(c->lumn), R(c->ecmn), c->dp, c->d_scal + 0);
        PFAG_LAUNCHED(c);
        k_dirichlet<real><<<(4 * N + 255) / 256, 256, 0, c->stream>>>(R(c->lumn), N, (real)0.0, (real)0.0);
        PFAG_LAUNCHED(c);
        k_dirichlet<real><<<(4 * N + 255) / 256, 256, 0, c->stream>>>(R(c->ecmn), N, (real)1.0, (real)1.0);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int reshape_lum(int which, int *iters_out) {
        const int N = c->N;
        void *f = which ? c->ecm : c->lum, *fn = which ? c->ecmn : c->lumn;
        const real side = which ? (real)1.0 : (real)0.0;
        k_norm_grad_2d<real><<<interior_grid(1), dim3(TBX, TBY), 0, c->stream>>>(R(f), R(c->ngl), N, c4());
        PFAG_LAUNCHED(c);
        PFAG_TRY(bc_cells(c->ngl, 1));
        // J_x, J_y: cell 0's slices of the normal arrays serve as scratch (:743)
        k_lum_normals<real><<<interior_grid(1), dim3(TBX, TBY), 0, c->stream>>>(
            R(fn), R(c->ngl), R(c->jx), R(c->jy), N, (real)(1.0 / (2.0 * c->dp.dx)));
        PFAG_LAUNCHED(c);
        PFAG_TRY(bc_cells(c->jx, 1));
        PFAG_TRY(bc_cells(c->jy, 1));
        double rdev = c->dp.rdev0_lum;
        int ri = 0;
        const real A = (real)c->dp.A_resh, B = (real)c->dp.B_resh;
        while (rdev > c->dp.thr_lum) {
            k_copy<real><<<592, 256, 0, c->stream>>>(R(f), R(fn), c->ng); PFAG_LAUNCHED(c);
            k_lum_relax<real><<<interior_grid(1), dim3(TBX, TBY), 0, c->stream>>>(R(f), R(fn), R(c->jx), R(c->jy), N,
                                                                                  A, B);
            PFAG_LAUNCHED(c);
            k_dirichlet<real><<<(4 * N + 255) / 256, 256, 0, c->stream>>>(R(fn), N, side, (real)0.0);
            PFAG_LAUNCHED(c);
            PFAG_TRY(sum_reduce_2d(fn, f, c->dp.dx * c->dp.dx, c->d_scal + 1));
            PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_scal + 1, c->d_scal + 1, sizeof(double), cudaMemcpyDeviceToHost,
                                            c->stream));
            PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
            rdev = c->h_scal[1];
            if (ri > c->p.rimax) { c->stats.relax_failures++; break; }
            ri++;
        }
        if (iters_out) *iters_out = ri;
        return PFAG_OK;
    }
    int normals() {
        k_normals<real><<<interior_grid(c->Ntot), dim3(TBX, TBY), 0, c->stream>>>(
            R(c->phi), R(c->g), R(c->jx), R(c->jy), c->N, (real)(1.0 / (2.0 * c->dp.dx)));
        PFAG_LAUNCHED(c);
        PFAG_TRY(bc_cells(c->jx, c->Ntot));
        return bc_cells(c->jy, c->Ntot);
    }
    int update_cells() {
        k_update_cells<real><<<zone_grid(), dim3(TBX, TBY), 0, c->stream>>>(
            R(c->phi), R(c->phin), R(c->g), R(c->rho), R(c->hfunc), c->d_f0, R(c->psi), c->d_xc, c->d_yc,
            R(c->hlum), R(c->hecm), c->dp);
        PFAG_LAUNCHED(c);
        return bc_cells(c->phin, c->Ntot);
    }
    int reshape_cells() {
        const int Nt = c->Ntot;
        int *active = c->d_iflags, *ri = c->d_iflags + Nt, *nact = c->d_iflags + 2 * Nt;
        // all cells start active with ri = 0
        std::fill(c->h_iflags, c->h_iflags + Nt, 1);
        std::fill(c->h_iflags + Nt, c->h_iflags + 2 * Nt + 1, 0);
        PFAG_CUDA_CHECK(cudaMemcpyAsync(c->d_iflags, c->h_iflags, sizeof(int) * (2 * Nt + 1), cudaMemcpyHostToDevice,
                                        c->stream));
        const real A = (real)c->dp.A_resh, B = (real)c->dp.B_resh;
        const double scale = c->dp.dx * c->dp.dx / (double)c->dp.Ncur;
        const int nblk = c->serial_sums ? 1 : 32;
        for (;;) {
            k_zone_copy<real><<<zone_grid(), dim3(TBX, TBY), 0, c->stream>>>(R(c->phi), R(c->phin), c->d_xc, c->d_yc,
                                                                             c->N, c->zone, active);
            PFAG_LAUNCHED(c);
            k_cell_relax<real><<<zone_grid(), dim3(TBX, TBY), 0, c->stream>>>(
                R(c->phi), R(c->phin), R(c->jx), R(c->jy), c->d_xc, c->d_yc, c->N, c->zone, A, B, active);
            PFAG_LAUNCHED(c);
            if (c->serial_sums)
                k_serial_cell_rdev<real><<<(Nt + 63) / 64, 64, 0, c->stream>>>(
                    R(c->phin), R(c->phi), c->d_xc, c->d_yc, c->N, c->zone, Nt, c->dp.dx, (double)c->dp.Ncur, active,
                    c->d_part);
            else
                k_cell_rdev<real><<<dim3(nblk, Nt), RED_THREADS, 0, c->stream>>>(
                    R(c->phin), R(c->phi), c->d_xc, c->d_yc, c->N, c->zone, scale, active, c->d_part);
            PFAG_LAUNCHED(c);
            PFAG_CUDA_CHECK(cudaMemsetAsync(nact, 0, sizeof(int), c->stream));
            k_cell_check<<<(Nt + 127) / 128, 128, 0, c->stream>>>(c->d_part, nblk, Nt, c->dp.thr_cells, c->p.rimax,
                                                                   active, ri, nact, c->d_err);
            PFAG_LAUNCHED(c);
            PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_iflags + 2 * Nt, nact, sizeof(int), cudaMemcpyDeviceToHost,
                                            c->stream));
            PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
            if (c->h_iflags[2 * Nt] == 0) break;
        }
        PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_iflags + Nt, ri, sizeof(int) * Nt, cudaMemcpyDeviceToHost, c->stream));
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        int mx = 0, sm = 0;
        for (int n = 0; n < Nt; n++) {
            // the loop body increments ri once per iteration that does not break
            int it = c->h_iflags[Nt + n];
            c->h_iflags[4 * Nt + n] = it;   // per-cell counts, read by pfag_get_cell_iters
            mx = std::max(mx, it);
            sm += it;
        }
        c->stats.cell_iters_max = mx;
        c->stats.cell_iters_sum = sm;
        return PFAG_OK;
    }
    int copy_back() {
        k_copy<real><<<1184, 256, 0, c->stream>>>(R(c->rho), R(c->rhon), c->nc); PFAG_LAUNCHED(c);
        k_copy<real><<<592, 256, 0, c->stream>>>(R(c->ecm), R(c->ecmn), c->ng); PFAG_LAUNCHED(c);
        k_copy<real><<<592, 256, 0, c->stream>>>(R(c->lum), R(c->lumn), c->ng); PFAG_LAUNCHED(c);
        return PFAG_OK;
    }
    int check_zone() {
        // the reference reads xcenters on the host here (acc update host); so do we
        PFAG_TRY(pfag_check_device_error(c));
        return PFAG_OK;
    }
    // prepare_initial_files.cpp:53-117: the initial fields (when make_fields),
    // then centres, phin <- phi, |grad phi| and normals, the cells' reshaping,
    // rho fitted to the reshaped cells, the lumen/ECM update and their
    // reshaping.  The reference reads hfunc_lum, hfunc_ECM and psi there before
    // anything writes them (fresh, zero-filled allocations); they are zeroed.
    int generate(double rho0, double tol, int make_fields) {
        const int N = c->N, Nt = c->Ntot;
        cudaStream_t s = c->stream;
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), s));
        const real rcyst = (real)((double)Nt * 0.9 * c->p.R / c->p.dx / M_PI);
        if (make_fields) {
            const dim3 tb(TBX, TBY), gb((N + TBX - 1) / TBX, (N + TBY - 1) / TBY, Nt);
            PFAG_CUDA_CHECK(cudaMemsetAsync(c->lum, 0, c->ng * c->rsz, s));
            PFAG_CUDA_CHECK(cudaMemsetAsync(c->ecm, 0, c->ng * c->rsz, s));
            k_ini_phi<real><<<gb, tb, 0, s>>>(R(c->phi), N, Nt, (real)c->p.dx, (real)c->p.R, (real)c->p.wi, rcyst);
            PFAG_LAUNCHED(c);
            k_ini_lum_ecm<real><<<dim3(gb.x, gb.y), tb, 0, s>>>(R(c->phi), R(c->lum), R(c->ecm), N, Nt, rcyst);
            PFAG_LAUNCHED(c);
            k_rho_shape<real><<<1184, 256, 0, s>>>(R(c->phi), R(c->rho), c->nc, rho0, tol, 1);
            PFAG_LAUNCHED(c);
        }
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->hfunc, 0, c->nc * c->rsz, s));
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->psi, 0, c->ng * c->rsz, s));
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->hlum, 0, c->ng * c->rsz, s));
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->hecm, 0, c->ng * c->rsz, s));
        PFAG_TRY(centres());
        PFAG_TRY(check_zone());
        k_copy<real><<<1184, 256, 0, s>>>(R(c->phin), R(c->phi), c->nc); PFAG_LAUNCHED(c);
        PFAG_TRY(norm_grad());
        PFAG_TRY(normals());
        PFAG_TRY(reshape_cells());
        k_rho_shape<real><<<1184, 256, 0, s>>>(R(c->phi), R(c->rho), c->nc, rho0, tol, 0);
        PFAG_LAUNCHED(c);
        PFAG_TRY(lum_ecm_update());
        PFAG_TRY(reshape_lum(0, &c->stats.lum_iters));
        PFAG_TRY(reshape_lum(1, &c->stats.ecm_iters));
        PFAG_CUDA_CHECK(cudaStreamSynchronize(s));
        return pfag_check_device_error(c);
    }
    int step(int it) {
        (void)it;
        PFAG_TRY(centres());
        PFAG_TRY(check_zone());
        PFAG_TRY(maps());
        PFAG_TRY(hfunc3d());
        PFAG_TRY(hfunc2d());
        PFAG_TRY(norm_grad());
        PFAG_TRY(prod_norm_delta());
        PFAG_TRY(psi());
        PFAG_TRY(sum_s());
        PFAG_TRY(cortices());
        PFAG_TRY(lum_ecm_update());
        PFAG_TRY(reshape_lum(0, &c->stats.lum_iters));
        PFAG_TRY(reshape_lum(1, &c->stats.ecm_iters));
        PFAG_TRY(normals());
        PFAG_TRY(update_cells());
        PFAG_TRY(reshape_cells());
        PFAG_TRY(copy_back());
        return PFAG_OK;
    }
};

}  // namespace

int pfag_plain_alloc(pfag_ctx *c) {
    const size_t rs = c->rsz, nc = c->nc, ng = c->ng;
    PFAG_CUDA_CHECK(cudaMalloc(&c->g, nc * rs));
    PFAG_CUDA_CHECK(cudaMalloc(&c->pnd, nc * rs));
    PFAG_CUDA_CHECK(cudaMalloc(&c->jx, nc * rs));
    PFAG_CUDA_CHECK(cudaMalloc(&c->jy, nc * rs));
    PFAG_CUDA_CHECK(cudaMalloc(&c->ngl, ng * rs));
    for (int k = 0; k < 6; k++) PFAG_CUDA_CHECK(cudaMalloc(&c->maps[k], nc * rs));
    PFAG_CUDA_CHECK(cudaMalloc(&c->pixx, nc * rs));
    PFAG_CUDA_CHECK(cudaMalloc(&c->pixy, nc * rs));
    PFAG_CUDA_CHECK(cudaMalloc(&c->piyy, nc * rs));
    PFAG_CUDA_CHECK(cudaMemset(c->g, 0, nc * rs));
    PFAG_CUDA_CHECK(cudaMemset(c->jx, 0, nc * rs));
    PFAG_CUDA_CHECK(cudaMemset(c->jy, 0, nc * rs));
    const size_t mm = (size_t)c->M * c->M;
    PFAG_CUDA_CHECK(cudaMalloc(&c->fftbuf, 11 * (size_t)c->Ntot * mm * 2 * rs));
    int dims[2] = {c->M, c->M};
    PFAG_CUFFT_CHECK(cufftPlanMany(&c->plan, 2, dims, nullptr, 1, (int)mm, nullptr, 1, (int)mm,
                                   c->prec == 64 ? CUFFT_Z2Z : CUFFT_C2C, c->Ntot));
    PFAG_CUFFT_CHECK(cufftSetStream(c->plan, c->stream));
    c->plan_ok = true;
    return PFAG_OK;
}

void pfag_plain_free(pfag_ctx *c) {
    void *bufs[] = {c->g, c->pnd, c->jx, c->jy, c->ngl, c->pixx, c->pixy, c->piyy, c->fftbuf};
    for (void *b : bufs) if (b) cudaFree(b);
    for (int k = 0; k < 6; k++) if (c->maps[k]) cudaFree(c->maps[k]);
    if (c->plan_ok) cufftDestroy(c->plan);
    c->plan_ok = false;
}

int pfag_plain_step(pfag_ctx *c, int it, bool) {
    return c->prec == 64 ? Plain<double>(c).step(it) : Plain<float>(c).step(it);
}

int pfag_plain_generate(pfag_ctx *c, double rho0, double tol, int make_fields) {
    return c->prec == 64 ? Plain<double>(c).generate(rho0, tol, make_fields)
                         : Plain<float>(c).generate(rho0, tol, make_fields);
}

// Per-function entry points (the drop-in layer's targets).
#define PLAIN_DISPATCH(ctx, call) \
    ((ctx)->prec == 64 ? Plain<double>(ctx).call : Plain<float>(ctx).call)

int pfag_plain_fn(pfag_ctx *c, const char *which, int arg) {
    std::string w(which);
    if (w == "centres") { PFAG_TRY(PLAIN_DISPATCH(c, centres())); return pfag_check_device_error(c); }
    if (w == "maps") return PLAIN_DISPATCH(c, maps());
    if (w == "hfunc3d") return PLAIN_DISPATCH(c, hfunc3d());
    if (w == "hfunc2d") return PLAIN_DISPATCH(c, hfunc2d());
    if (w == "norm_grad") return PLAIN_DISPATCH(c, norm_grad());
    if (w == "pnd") return PLAIN_DISPATCH(c, prod_norm_delta());
    if (w == "psi") return PLAIN_DISPATCH(c, psi());
    if (w == "sum_s") return PLAIN_DISPATCH(c, sum_s());
    if (w == "cortices") return PLAIN_DISPATCH(c, cortices());
    if (w == "lum_ecm_update") return PLAIN_DISPATCH(c, lum_ecm_update());
    if (w == "reshape_lum") return PLAIN_DISPATCH(c, reshape_lum(arg, arg ? &c->stats.ecm_iters : &c->stats.lum_iters));
    if (w == "normals") return PLAIN_DISPATCH(c, normals());
    if (w == "update_cells") return PLAIN_DISPATCH(c, update_cells());
    if (w == "reshape_cells") return PLAIN_DISPATCH(c, reshape_cells());
    if (w == "copy_back") return PLAIN_DISPATCH(c, copy_back());
    pfag_set_error("unknown plain function %s", which);
    return PFAG_E_ARG;
}
