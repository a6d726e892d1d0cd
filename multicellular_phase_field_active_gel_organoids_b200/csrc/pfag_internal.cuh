// Internal definitions shared by the plain and fused paths of libpfag.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include "../../include/pfag.h"

#define PFAG_VERSION 1

void pfag_set_error(const char *fmt, ...);

#define PFAG_CUDA_CHECK(expr)                                                            \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess) {                                                         \
            pfag_set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
            return PFAG_E_CUDA;                                                          \
        }                                                                                \
    } while (0)

#define PFAG_CUFFT_CHECK(expr)                                                           \
    do {                                                                                 \
        cufftResult _r = (expr);                                                         \
        if (_r != CUFFT_SUCCESS) {                                                       \
            pfag_set_error("%s:%d %s: cufft error %d", __FILE__, __LINE__, #expr, (int)_r); \
            return PFAG_E_CUDA;                                                          \
        }                                                                                \
    } while (0)

#define PFAG_TRY(expr)                 \
    do {                               \
        int _rc = (expr);              \
        if (_rc != PFAG_OK) return _rc; \
    } while (0)

// Device error word bits (ctx->d_err).
enum : unsigned {
    ERRBIT_EMPTY_CELL = 1u,
    ERRBIT_ZONE = 2u,
    ERRBIT_RELAX = 4u,
    ERRBIT_ITER_CAP = 8u,
    ERRBIT_TIMEOUT = 16u,     // a bounded device wait (a TMA copy's completion) gave up
};

// Scalars the kernels read, precomputed on the host in double with the
// reference's operation order.
struct DevParams {
    int N, Ntot, zone, M, Ncur;
    double dx, dt, s0, alpha, sigma, beta, eta, tau;
    double cpl;                 // coupling_PF_AG
    double beta_lum_cells, eta_lum_cells, beta_ECM_cells, eta_ECM_cells;
    double tau_lum, xi_lum, beta_lum_ECM, alpha_ECM, tau_ECM, xi_ECM;
    double friction;
    double wi, rdt;
    double A_resh;              // wi*wi*(rdt/dx/dx)
    double B_resh;              // rdt*wi*sqrt(2.0)/dx
    double thr_cells;           // rtol*2.0*M_PI*R*wi*rdt
    double thr_lum;             // rdev_threshold*rtol*rdt
    double rdev0_lum;           // rdev_ini*rtol*rdt
    double kfac;                // 2.0*M_PI/((2*zone_size-2)*dx)
    // folded constants of the FP32 fused kernels
    double k_cpl;               // coupling_PF_AG/tau*(dt/dx/dx/4)/sqrt(2 pi)/sigma
    double inv_2s2;             // 1/(2 sigma^2)
    double dt_tau;              // dt/tau
    double inv_q4;              // 1/(4 dx^2)
    double inv_norm;            // 1/(M*M) as the reference divides: x/((2z-2)*(2z-2))
    // parameter maps, index 0 apical, 1 basal, 2 lateral
    double deg[3], gen[3], a_ort[3], a_tan[3], visc[3], bb[3];
};

struct pfag_ctx {
    pfag_params p;
    DevParams dp;
    int prec;       // 32 or 64
    int path;       // PFAG_PATH_*
    int rsz;        // sizeof(real)
    cudaStream_t stream;
    int N, Ntot, zone, M;
    size_t ng, nc;  // N*N, Ntot*N*N
    // state (reference layout)
    void *phi, *phin, *rho, *rhon, *lum, *lumn, *ecm, *ecmn;
    void *hfunc, *hlum, *hecm, *psi;
    // plain-path full-grid work arrays
    void *g, *pnd, *jx, *jy, *ngl;
    void *maps[6];  // deg, gen, a_tan, a_ort, visc, b
    void *pixx, *pixy, *piyy;
    void *fftbuf;   // 11 * Ntot * M*M complex
    cufftHandle plan;
    bool plan_ok;
    // small device arrays
    int *d_xc, *d_yc;
    long long *d_cacc;    // Ntot*3 centroid accumulators
    double *d_s, *d_f0;
    double *d_part;       // reduction partials
    size_t part_cap;
    double *d_scal;       // misc device scalars
    int *d_iflags;        // per-cell flags / counters (Ntot*4)
    unsigned *d_err;
    // host mirrors
    int *h_xc, *h_yc;
    double *h_s, *h_f0;
    int *h_iflags;        // pinned
    double *h_scal;       // pinned
    unsigned *h_err;      // pinned
    pfag_stats stats;
    long launches;
    int debug;
    int relax_cap;        // device-side loop bound (fused path)
    int serial_sums;      // plain path: reductions in the reference's serial host order
    void *d_vx, *d_vy;
    // fused-path resources (opaque, owned by pfag_fused.cu)
    void *fused;
    void *prof;           // per-kernel event timing (pfag_prof.cu)
    void *snap;           // asynchronous snapshot staging (pfag_snapshot.cu)
};

void pfag_prof_begin(pfag_ctx *ctx, const char *name);
void pfag_prof_end(pfag_ctx *ctx);
void pfag_prof_free(pfag_ctx *ctx);
void pfag_snapshot_free(pfag_ctx *ctx);
bool pfag_prof_on(pfag_ctx *ctx);

// Launch accounting helper; closes the profiling bracket of the launch.
#define PFAG_LAUNCHED(ctx) ((ctx)->launches++, pfag_prof_end(ctx))

int pfag_plain_alloc(pfag_ctx *ctx);
void pfag_plain_free(pfag_ctx *ctx);
int pfag_plain_step(pfag_ctx *ctx, int it, bool sync_host);
int pfag_plain_generate(pfag_ctx *ctx, double rho0, double tol, int make_fields);
int pfag_fused_alloc(pfag_ctx *ctx);
void pfag_fused_free(pfag_ctx *ctx);
int pfag_fused_upload_hook(pfag_ctx *ctx);
int pfag_fused_step(pfag_ctx *ctx, int it, bool sync_host);
int pfag_check_device_error(pfag_ctx *ctx);
int pfag_after_upload(pfag_ctx *ctx);
int pfag_fused_recentre(pfag_ctx *ctx);
int pfag_fused_stats(pfag_ctx *c);        // reshaping iteration counts of the last step into c->stats
int pfag_fetch_observables(pfag_ctx *ctx);

// ---------------------------------------------------------------------------
// Device helpers shared by both paths.
template <typename real> struct Cplx;
template <> struct Cplx<double> { typedef double2 type; };
template <> struct Cplx<float> { typedef float2 type; };

__device__ __forceinline__ size_t cidx(int n, int i, int j, int N) {
    return ((size_t)n * N + i) * N + j;
}

// Periodic ghost map of boundary_conditions_cells / boundary_conditions_periodic
// (useful_functions.cpp:391-420, :505-526): ghost row/column 0 holds row/column
// N-2, ghost N-1 holds 1.
__device__ __forceinline__ int ghost_src(int i, int N) {
    return i == 0 ? N - 2 : (i == N - 1 ? 1 : i);
}

// 9-point stencil of the reference: -12 u_c + 2 (u_ip + u_im + u_jp + u_jm)
// + u_ip,jp + u_ip,jm + u_im,jm + u_im,jp   (cell_phase_functions.cpp:198)
template <typename real>
__device__ __forceinline__ real lap9(real c, real ip, real im, real jp, real jm,
                                     real ipjp, real ipjm, real imjm, real imjp) {
    return -(real)12.0 * c + (real)2.0 * (ip + im + jp + jm) + ipjp + ipjm + imjm + imjp;
}

// One face term of the reshaping flux (cell_phase_functions.cpp:511-547, :802-838):
// 0.5*(Jn_a+Jn_b) * ( A*(pa-pb)*0.5*(Jn_a+Jn_b) + A*0.25*tang*0.5*(Jt_a+Jt_b)
//                     - B*0.5*(pa*(1-pa) + pb*(1-pb)) )
template <typename real>
__device__ __forceinline__ real resh_face(real A, real B, real jn_a, real jn_b, real pa, real pb,
                                          real tang, real jt_a, real jt_b) {
    real jn = (real)0.5 * (jn_a + jn_b);
    return jn * (A * (pa - pb) * jn + A * (real)0.25 * tang * ((real)0.5 * (jt_a + jt_b)) -
                 B * (real)0.5 * (pa * ((real)1.0 - pa) + pb * ((real)1.0 - pb)));
}

// Full reshaping increment at one site given the 3x3 neighbourhood of the
// phase p and the 3x3 cross of the normals.  Order of the four face terms
// follows the reference (x+, y+, x-, y-).
template <typename real>
__device__ __forceinline__ real resh_update(real A, real B,
                                            // p[di][dj], di,dj in {0,1,2} = {-1,0,+1}
                                            const real p[3][3],
                                            real jx_c, real jx_ip, real jx_im, real jx_jp, real jx_jm,
                                            real jy_c, real jy_ip, real jy_im, real jy_jp, real jy_jm,
                                            real pn) {
    // x+ face: tangential (p[ip,jp]+p[i,jp]-p[ip,jm]-p[i,jm])
    pn += resh_face(A, B, jx_ip, jx_c, p[2][1], p[1][1],
                    p[2][2] + p[1][2] - p[2][0] - p[1][0], jy_ip, jy_c);
    // y+ face: tangential (p[ip,jp]+p[ip,j]-p[im,jp]-p[im,j])
    pn += resh_face(A, B, jy_jp, jy_c, p[1][2], p[1][1],
                    p[2][2] + p[2][1] - p[0][2] - p[0][1], jx_jp, jx_c);
    // x- face: 0.5*(Jx_c+Jx_im)*(A*(p_c-p_im)*... tangential (p[i,jp]+p[im,jp]-p[i,jm]-p[im,jm]))
    pn -= resh_face(A, B, jx_c, jx_im, p[1][1], p[0][1],
                    p[1][2] + p[0][2] - p[1][0] - p[0][0], jy_c, jy_im);
    // y- face: tangential (p[ip,j]+p[ip,jm]-p[im,j]-p[im,jm])
    pn -= resh_face(A, B, jy_c, jy_jm, p[1][1], p[1][0],
                    p[2][1] + p[2][0] - p[0][1] - p[0][0], jx_c, jx_jm);
    return pn;
}

// The same increment for the fused FP32 path with the constants folded:
// with s = Jn_a + Jn_b, t = Jt_a + Jt_b and h(p) = p (1 - p) a face is
//   s * ( (A/4)(pa - pb) s + (A/16) tang t - (B/4)(h_a + h_b) ),
// h is formed once per site of the cross and the tangential differences once
// per row / column.  FP64 keeps the reference's operation order (resh_update).
struct ReshConst {
    float a4, a16, b4;
};
__device__ __forceinline__ ReshConst resh_const(double A, double B) {
    return ReshConst{(float)(A * 0.25), (float)(A * 0.0625), (float)(B * 0.25)};
}
__device__ __forceinline__ float resh_face_f(const ReshConst &k, float s, float pa, float pb, float ha, float hb,
                                             float tang, float t) {
    return s * fmaf(k.a4 * (pa - pb), s, fmaf(k.a16 * tang, t, -k.b4 * (ha + hb)));
}
__device__ __forceinline__ float resh_update_f(const ReshConst &k, const float p[3][3], float jx_c, float jx_ip,
                                               float jx_im, float jx_jp, float jx_jm, float jy_c, float jy_ip,
                                               float jy_im, float jy_jp, float jy_jm, float pn) {
    const float hc = fmaf(-p[1][1], p[1][1], p[1][1]);
    const float hip = fmaf(-p[2][1], p[2][1], p[2][1]), him = fmaf(-p[0][1], p[0][1], p[0][1]);
    const float hjp = fmaf(-p[1][2], p[1][2], p[1][2]), hjm = fmaf(-p[1][0], p[1][0], p[1][0]);
    const float cd0 = p[0][2] - p[0][0], cd1 = p[1][2] - p[1][0], cd2 = p[2][2] - p[2][0];
    const float rd0 = p[2][0] - p[0][0], rd1 = p[2][1] - p[0][1], rd2 = p[2][2] - p[0][2];
    pn += resh_face_f(k, jx_ip + jx_c, p[2][1], p[1][1], hip, hc, cd2 + cd1, jy_ip + jy_c);
    pn += resh_face_f(k, jy_jp + jy_c, p[1][2], p[1][1], hjp, hc, rd2 + rd1, jx_jp + jx_c);
    pn -= resh_face_f(k, jx_c + jx_im, p[1][1], p[0][1], hc, him, cd1 + cd0, jy_c + jy_im);
    pn -= resh_face_f(k, jy_c + jy_jm, p[1][1], p[1][0], hc, hjm, rd1 + rd0, jx_c + jx_jm);
    return pn;
}
