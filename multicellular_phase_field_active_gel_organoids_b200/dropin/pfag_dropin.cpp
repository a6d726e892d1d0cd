// Drop-in replacement of the reference's step functions, with their exact C++
// signatures, implemented over the C ABI of libpfag (include/pfag.h).
//
// The reference's main (main_code/run_with_active_gels.cpp) is linked against
// this library instead of functions/useful_functions.cpp, rho_functions.cpp
// and cell_phase_functions.cpp; its remaining host files (constants.cpp,
// declare_tables.cpp, declare_fft_tables.cpp, initialisation_functions.cpp)
// stay as they are.  Declarations followed: functions/useful_functions.h:10-48,
// rho_functions.h:10-26, cell_phase_functions.h:18-39.  Built twice: `float`
// for the shipped reference and `double` (PFAG_DROPIN_DOUBLE) for its
// float -> double rewrite.
//
// Device residency.  main's OpenACC data region (run_with_active_gels.cpp:83)
// is inert once main is compiled by a host compiler, so the first call made
// here creates the device context from the parameter globals of
// functions/constants.h and copies in phi, rho, lum and ECM from the table
// globals of functions/declare_tables.h (the region's copyin).  Every table then
// lives on the device; the host copies are refreshed where the host reads them:
// xcenters/ycenters after find_centres_cells, s/f0 after sum_s_kernels, and the
// phiout/rhoout/lumout/ECMout slots in saving_out_functions.
//
// Paths.  PFAG_DROPIN_PATH=plain (default): every function runs its own
// per-function entry point (one kernel set per reference function).
// PFAG_DROPIN_PATH=fused: find_centres_cells, the first call of each time step
// (run_with_active_gels.cpp:124), runs the whole fused step; the step's later
// calls only check their arguments, and its table copies (:175-182) are part of
// that step.  Observable outputs are the same in both paths.
//
// Errors.  The reference functions return void.  A failing C-ABI call prints
// the library's message and aborts; a reshaping loop past rimax prints the
// reference's "Relaxation failure!" line and goes on, as the reference does
// (cell_phase_functions.cpp:563-567).  An argument that is not the table the
// reference passes at that position aborts: the drop-in keeps exactly the
// reference's tables on the device and no others.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "pfag.h"

#ifdef PFAG_DROPIN_DOUBLE
typedef double real_t;
#define PFAG_DROPIN_PRECISION 64
#else
typedef float real_t;
#define PFAG_DROPIN_PRECISION 32
#endif

// Parameter globals (functions/constants.h:3-124), defined by the program's
// constants.cpp.
extern const int N_s;
extern const int Ntot;
extern int zone_size, N_current, N_ini, rdev_threshold, rimax, nsaving, Ntotsave;
extern real_t dx, dt, R, s0, sigma, coupling_PF_AG;
extern real_t tau, alpha, beta, eta;
extern real_t tau_lum, beta_lum_cells, eta_lum_cells, xi_lum;
extern real_t alpha_ECM, tau_ECM, beta_ECM_cells, eta_ECM_cells, xi_ECM, beta_lum_ECM;
extern real_t wi, rtol, rdt, friction;
extern real_t a_tan_apical, a_tan_basal, a_tan_lateral;
extern real_t a_ort_apical, a_ort_basal, a_ort_lateral;
extern real_t b_ap, b_bas, b_lat;
extern real_t matgenrate_apical, matgenrate_basal, matgenrate_lateral;
extern real_t degrate_apical, degrate_basal, degrate_lateral;
extern real_t viscosity_ap, viscosity_bas, viscosity_lat;

// Table globals (functions/declare_tables.h:10-78), allocated by malloc_all.
extern real_t *phi, *phin, *rho, *rhon, *lum, *ECM, *lumn, *ECMn, *psi;
extern real_t *hfunc_cell, *hfunc_lum, *hfunc_ECM;
extern real_t *norm_grad_phi, *prod_norm_delta, *J_x, *J_y;
extern real_t *a_tan_1, *a_ort_1, *b, *viscosity, *matgenrates, *degrates;
extern real_t *phiout, *rhoout, *lumout, *ECMout;
extern int *xcenters, *ycenters;

namespace {

struct DropinState {
    pfag_ctx *ctx = nullptr;
    bool fused = false;
    int steps = 0;          // time steps started (calls of find_centres_cells)
    int relax_seen = 0;     // relaxation failures already reported
};
DropinState g;

[[noreturn]] void fail(const char *fn, const char *what) {
    std::fprintf(stderr, "pfag drop-in: %s: %s\n", fn, what);
    std::abort();
}

void check(int rc, const char *fn) {
    if (rc != PFAG_OK) fail(fn, pfag_last_error());
}

// Reshaping loops that passed rimax since the last look: the reference prints
// its message and goes on (cell_phase_functions.cpp:563-567, :859-863).
void report_relax_failures(pfag_ctx *c, const char *fn) {
    check(pfag_sync(c), fn);
    pfag_stats st;
    check(pfag_get_stats(c, &st), fn);
    for (; g.relax_seen < st.relax_failures; g.relax_seen++)
        std::fprintf(stderr, "Relaxation failure! at i=%d ri=%d \n", g.steps - 1, rimax + 1);
}

void destroy_ctx() {
    if (g.ctx) pfag_destroy(g.ctx);
    g.ctx = nullptr;
}

pfag_params params_from_globals() {
    pfag_params p;
    std::memset(&p, 0, sizeof p);
    p.N_s = N_s; p.Ntot = Ntot; p.zone_size = zone_size; p.N_current = N_current;
    p.rdev_threshold = rdev_threshold; p.rimax = rimax;
    p.dx = dx; p.dt = dt; p.R = R; p.s0 = s0; p.sigma = sigma; p.coupling_PF_AG = coupling_PF_AG;
    p.tau = tau; p.alpha = alpha; p.beta = beta; p.eta = eta;
    p.tau_lum = tau_lum; p.beta_lum_cells = beta_lum_cells; p.eta_lum_cells = eta_lum_cells; p.xi_lum = xi_lum;
    p.alpha_ECM = alpha_ECM; p.tau_ECM = tau_ECM; p.beta_ECM_cells = beta_ECM_cells;
    p.eta_ECM_cells = eta_ECM_cells; p.xi_ECM = xi_ECM; p.beta_lum_ECM = beta_lum_ECM;
    p.wi = wi; p.rtol = rtol; p.rdt = rdt; p.friction = friction;
    p.a_tan_apical = a_tan_apical; p.a_tan_basal = a_tan_basal; p.a_tan_lateral = a_tan_lateral;
    p.a_ort_apical = a_ort_apical; p.a_ort_basal = a_ort_basal; p.a_ort_lateral = a_ort_lateral;
    p.b_ap = b_ap; p.b_bas = b_bas; p.b_lat = b_lat;
    p.matgenrate_apical = matgenrate_apical; p.matgenrate_basal = matgenrate_basal;
    p.matgenrate_lateral = matgenrate_lateral;
    p.degrate_apical = degrate_apical; p.degrate_basal = degrate_basal; p.degrate_lateral = degrate_lateral;
    p.viscosity_ap = viscosity_ap; p.viscosity_bas = viscosity_bas; p.viscosity_lat = viscosity_lat;
    return p;
}

// The data region's entry (run_with_active_gels.cpp:83-98), on first use.
pfag_ctx *ctx(const char *fn) {
    if (g.ctx) return g.ctx;
    const char *path = std::getenv("PFAG_DROPIN_PATH");
    if (path && std::strcmp(path, "fused") != 0 && std::strcmp(path, "plain") != 0)
        fail(fn, "PFAG_DROPIN_PATH must be plain or fused");
    g.fused = path && std::strcmp(path, "fused") == 0;
    const pfag_params p = params_from_globals();
    check(pfag_create(&p, PFAG_DROPIN_PRECISION, g.fused ? PFAG_PATH_FUSED : PFAG_PATH_PLAIN, &g.ctx), fn);
    check(pfag_upload(g.ctx, phi, rho, lum, ECM), fn);
    std::atexit(destroy_ctx);
    return g.ctx;
}

// The argument must be the reference's table for this position.
void expect(const void *arg, const void *table, const char *fn, const char *name) {
    if (arg != table) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "argument %s is not the table the reference passes here", name);
        fail(fn, msg);
    }
}

// Device mirror of a host table: (field name, per-cell or shared).
struct Mirror { const char *field; bool per_cell; };
bool mirror_of(const void *host, Mirror &m) {
    const struct { const void *h; Mirror m; } tab[] = {
        {phi, {"phi", true}}, {phin, {"phin", true}}, {rho, {"rho", true}}, {rhon, {"rhon", true}},
        {hfunc_cell, {"hfunc_cell", true}}, {psi, {"psi", false}}, {lum, {"lum", false}},
        {lumn, {"lumn", false}}, {ECM, {"ECM", false}}, {ECMn, {"ECMn", false}},
        {hfunc_lum, {"hfunc_lum", false}}, {hfunc_ECM, {"hfunc_ECM", false}}};
    for (const auto &e : tab)
        if (e.h == host) { m = e.m; return true; }
    return false;
}

real_t *device_table(const void *host, bool per_cell, const char *fn) {
    Mirror m;
    if (!mirror_of(host, m) || m.per_cell != per_cell) fail(fn, "table is not resident on the device");
    void *p = nullptr;
    long cnt = 0;
    check(pfag_device_field(ctx(fn), m.field, &p, &cnt), fn);
    return static_cast<real_t *>(p);
}

void device_copy(real_t *dst, const real_t *src, size_t elems, const char *fn) {
    cudaStream_t s = static_cast<cudaStream_t>(pfag_stream(ctx(fn)));
    if (cudaMemcpyAsync(dst, src, elems * sizeof(real_t), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        fail(fn, "device copy failed");
}

// In the fused path the step's own calls after find_centres_cells are done.
bool step_done_by_fused() { return g.fused && g.steps > 0; }

void fetch_centres(const char *fn) {
    check(pfag_get_centres(ctx(fn), xcenters, ycenters), fn);
}

}  // namespace

// ---- functions/useful_functions.cpp ---------------------------------------

// useful_functions.cpp:66-99: slot it/nsaving of the out tables (N_ini cells).
void saving_out_functions(int it, real_t *phi_, real_t *rho_, real_t *ECM_, real_t *lum_, real_t *phiout_,
                          real_t *rhoout_, real_t *lumout_, real_t *ECMout_) {
    const char *fn = "saving_out_functions";
    expect(phi_, phi, fn, "phi"); expect(rho_, rho, fn, "rho");
    expect(ECM_, ECM, fn, "ECM"); expect(lum_, lum, fn, "lum");
    const int slot = it / nsaving;
    if (slot < 0 || slot >= Ntotsave) fail(fn, "snapshot slot it/nsaving outside [0, Ntotsave)");
    const size_t NN = (size_t)N_s * N_s;
    const real_t *d_phi = device_table(phi, true, fn), *d_rho = device_table(rho, true, fn);
    const real_t *d_lum = device_table(lum, false, fn), *d_ecm = device_table(ECM, false, fn);
    cudaStream_t s = static_cast<cudaStream_t>(pfag_stream(ctx(fn)));
    const size_t cells = (size_t)N_ini * NN * sizeof(real_t);
    if (cudaMemcpyAsync(phiout_ + (size_t)slot * NN * Ntot, d_phi, cells, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(rhoout_ + (size_t)slot * NN * Ntot, d_rho, cells, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(lumout_ + (size_t)slot * NN, d_lum, NN * sizeof(real_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(ECMout_ + (size_t)slot * NN, d_ecm, NN * sizeof(real_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        fail(fn, "device to host copy failed");
}

// useful_functions.cpp:193-227; first call of a time step (run_with_active_gels.cpp:124).
void find_centres_cells(real_t *phi_, int *xc, int *yc) {
    const char *fn = "find_centres_cells";
    expect(phi_, phi, fn, "phi"); expect(xc, xcenters, fn, "xcenters"); expect(yc, ycenters, fn, "ycenters");
    pfag_ctx *c = ctx(fn);
    const int it = g.steps++;
    if (g.fused) {
        check(pfag_step(c, it, 1), fn);
        report_relax_failures(c, fn);
    } else {
        check(pfag_fn_find_centres_cells(c), fn);
        check(pfag_sync(c), fn);            // device errors and the host copies of the centres
    }
    fetch_centres(fn);
}

// useful_functions.cpp:233-251
void compute_hfunc_3d_tables_kernels_loop_n(real_t *hfunc, real_t *phi_, int *xc, int *yc) {
    const char *fn = "compute_hfunc_3d_tables_kernels_loop_n";
    expect(hfunc, hfunc_cell, fn, "hfunc_cell"); expect(phi_, phi, fn, "phi");
    expect(xc, xcenters, fn, "xcenters"); expect(yc, ycenters, fn, "ycenters");
    if (step_done_by_fused()) return;
    check(pfag_fn_compute_hfunc_3d_tables_kernels_loop_n(ctx(fn)), fn);
}

// useful_functions.cpp:272-285
void compute_all_hfunc_2d_tables_kernels(real_t *hl, real_t *lum_, real_t *he, real_t *ecm_) {
    const char *fn = "compute_all_hfunc_2d_tables_kernels";
    expect(hl, hfunc_lum, fn, "hfunc_lum"); expect(lum_, lum, fn, "lum");
    expect(he, hfunc_ECM, fn, "hfunc_ECM"); expect(ecm_, ECM, fn, "ECM");
    if (step_done_by_fused()) return;
    check(pfag_fn_compute_all_hfunc_2d_tables_kernels(ctx(fn)), fn);
}

// useful_functions.cpp:326-354 (the periodic ghosts of :391-420 included)
void compute_normal_grad_phi(real_t *g_, real_t *phi_) {
    const char *fn = "compute_normal_grad_phi";
    expect(g_, norm_grad_phi, fn, "norm_grad_phi"); expect(phi_, phi, fn, "phi");
    if (step_done_by_fused()) return;
    check(pfag_fn_compute_normal_grad_phi(ctx(fn)), fn);
}

// useful_functions.cpp:391-420.  main applies it right after the producers of
// these tables (run_with_active_gels.cpp:136,167-168,172), which already apply it.
void boundary_conditions_cells(real_t *table) {
    const char *fn = "boundary_conditions_cells";
    if (table != norm_grad_phi && table != J_x && table != J_y && table != phin)
        fail(fn, "only norm_grad_phi, J_x, J_y and phin (as main calls it) are supported");
    (void)ctx(fn);
}

// rho_functions.cpp:13-30
void compute_prod_norm_delta(real_t *pnd, real_t *g_, real_t *phi_, int *xc, int *yc) {
    const char *fn = "compute_prod_norm_delta";
    expect(pnd, prod_norm_delta, fn, "prod_norm_delta"); expect(g_, norm_grad_phi, fn, "norm_grad_phi");
    expect(phi_, phi, fn, "phi"); expect(xc, xcenters, fn, "xcenters"); expect(yc, ycenters, fn, "ycenters");
    if (step_done_by_fused()) return;
    check(pfag_fn_compute_prod_norm_delta(ctx(fn)), fn);
}

// useful_functions.cpp:305-322
void compute_psi_kernels(real_t *psi_, real_t *hfunc) {
    const char *fn = "compute_psi_kernels";
    expect(psi_, psi, fn, "psi"); expect(hfunc, hfunc_cell, fn, "hfunc_cell");
    if (step_done_by_fused()) return;
    check(pfag_fn_compute_psi_kernels(ctx(fn)), fn);
}

// useful_functions.cpp:168-190; writes the host s and f0 (the host reads s at
// run_with_active_gels.cpp:146-151).
void sum_s_kernels(real_t *hfunc, real_t *s, real_t *f0) {
    const char *fn = "sum_s_kernels";
    expect(hfunc, hfunc_cell, fn, "hfunc_cell");
    if (!s || !f0) fail(fn, "null s or f0");
    pfag_ctx *c = ctx(fn);
    double sd[1024], fd[1024];
    if (Ntot > 1024) fail(fn, "more than 1024 cells");
    if (step_done_by_fused()) check(pfag_get_areas(c, sd, fd), fn);
    else check(pfag_fn_sum_s_kernels(c, sd, fd), fn);
    for (int n = 0; n < Ntot; n++) { s[n] = (real_t)sd[n]; f0[n] = (real_t)fd[n]; }
}

// useful_functions.cpp:679-693 (phase <- phasen for cell n)
void copy_cell_tables_1_by_1(int n, real_t *phase, real_t *phasen) {
    const char *fn = "copy_cell_tables_1_by_1";
    if (n < 0 || n >= Ntot) fail(fn, "cell index outside [0, Ntot)");
    real_t *d = device_table(phase, true, fn);
    const real_t *s = device_table(phasen, true, fn);
    if (step_done_by_fused()) return;
    const size_t NN = (size_t)N_s * N_s;
    device_copy(d + (size_t)n * NN, s + (size_t)n * NN, NN, fn);
}

// useful_functions.cpp:695-709 (phase <- phasen)
void copy_tables_ECM_or_lumen(real_t *phase, real_t *phasen) {
    const char *fn = "copy_tables_ECM_or_lumen";
    real_t *d = device_table(phase, false, fn);
    const real_t *s = device_table(phasen, false, fn);
    if (step_done_by_fused()) return;
    device_copy(d, s, (size_t)N_s * N_s, fn);
}

// useful_functions.cpp:356-388 (ghosts of :391-420 included)
void compute_normal_to_phi(real_t *phi_, real_t *g_, real_t *jx, real_t *jy) {
    const char *fn = "compute_normal_to_phi";
    expect(phi_, phi, fn, "phi"); expect(g_, norm_grad_phi, fn, "norm_grad_phi");
    expect(jx, J_x, fn, "J_x"); expect(jy, J_y, fn, "J_y");
    if (step_done_by_fused()) return;
    check(pfag_fn_compute_normal_to_phi(ctx(fn)), fn);
}

// useful_functions.cpp:439-462: applied by update_lumen_and_ECM below.
void boundary_conditions_lumen_and_ECM(real_t *lumn_, real_t *ecmn_) {
    const char *fn = "boundary_conditions_lumen_and_ECM";
    expect(lumn_, lumn, fn, "lumn"); expect(ecmn_, ECMn, fn, "ECMn");
    (void)ctx(fn);
}

// ---- functions/rho_functions.cpp ------------------------------------------

// rho_functions.cpp:286-405
void create_turnover_rates_tensions(real_t *deg, real_t *gen, real_t *at, real_t *ao, real_t *visc, real_t *bb,
                                    real_t *phi_, real_t *lum_, real_t *ecm_, int *xc, int *yc) {
    const char *fn = "create_turnover_rates_tensions";
    expect(deg, degrates, fn, "degrates"); expect(gen, matgenrates, fn, "matgenrates");
    expect(at, a_tan_1, fn, "a_tan_1"); expect(ao, a_ort_1, fn, "a_ort_1");
    expect(visc, viscosity, fn, "viscosity"); expect(bb, b, fn, "b");
    expect(phi_, phi, fn, "phi"); expect(lum_, lum, fn, "lum"); expect(ecm_, ECM, fn, "ECM");
    expect(xc, xcenters, fn, "xcenters"); expect(yc, ycenters, fn, "ycenters");
    if (step_done_by_fused()) return;
    check(pfag_fn_create_turnover_rates_tensions(ctx(fn)), fn);
}

// rho_functions.cpp:409-471.  The plans and the cufftComplex scratch of
// declare_fft_tables.cpp are the host program's; the library uses its own.
void update_all_cortices(real_t *phi_, real_t *rho_, real_t *rhon_, int *xc, int *yc, real_t *deg, real_t *gen,
                         real_t *at, real_t *ao, real_t *visc, real_t *bb, real_t *g_, real_t *pnd,
                         cufftHandle planf, cufftHandle planr, cufftComplex *temp_fft, cufftComplex *temp_fft_real,
                         cufftComplex *fft_rho, cufftComplex *fft_pi_xx, cufftComplex *fft_pi_xy,
                         cufftComplex *fft_pi_yy, cufftComplex *fft_vx, cufftComplex *fft_vy,
                         cufftComplex *fft_react, cufftComplex *fft_rho_vx, cufftComplex *fft_rho_vy) {
    const char *fn = "update_all_cortices";
    expect(phi_, phi, fn, "phi"); expect(rho_, rho, fn, "rho"); expect(rhon_, rhon, fn, "rhon");
    expect(xc, xcenters, fn, "xcenters"); expect(yc, ycenters, fn, "ycenters");
    expect(deg, degrates, fn, "degrates"); expect(gen, matgenrates, fn, "matgenrates");
    expect(at, a_tan_1, fn, "a_tan_1"); expect(ao, a_ort_1, fn, "a_ort_1");
    expect(visc, viscosity, fn, "viscosity"); expect(bb, b, fn, "b");
    expect(g_, norm_grad_phi, fn, "norm_grad_phi"); expect(pnd, prod_norm_delta, fn, "prod_norm_delta");
    (void)planf; (void)planr; (void)temp_fft; (void)temp_fft_real; (void)fft_rho; (void)fft_pi_xx;
    (void)fft_pi_xy; (void)fft_pi_yy; (void)fft_vx; (void)fft_vy; (void)fft_react; (void)fft_rho_vx;
    (void)fft_rho_vy;
    if (step_done_by_fused()) return;
    check(pfag_fn_update_all_cortices(ctx(fn)), fn);
}

// ---- functions/cell_phase_functions.cpp -----------------------------------

// cell_phase_functions.cpp:372-444 (+ the Dirichlet sides of useful_functions.cpp:439-462)
void update_lumen_and_ECM(real_t *lum_, real_t *lumn_, real_t *ecm_, real_t *ecmn_, real_t *hl, real_t *he,
                          real_t *psi_) {
    const char *fn = "update_lumen_and_ECM";
    expect(lum_, lum, fn, "lum"); expect(lumn_, lumn, fn, "lumn");
    expect(ecm_, ECM, fn, "ECM"); expect(ecmn_, ECMn, fn, "ECMn");
    expect(hl, hfunc_lum, fn, "hfunc_lum"); expect(he, hfunc_ECM, fn, "hfunc_ECM"); expect(psi_, psi, fn, "psi");
    if (step_done_by_fused()) return;
    check(pfag_fn_update_lumen_and_ECM(ctx(fn)), fn);
}

// cell_phase_functions.cpp:709-871; side_value 0 for the lumen, 1 for the ECM.
void reshaping_lumen_or_ECM(int it, real_t *phase, real_t *phasen, real_t side_value) {
    const char *fn = "reshaping_lumen_or_ECM";
    (void)it;
    int which;
    if (phase == lum && phasen == lumn && side_value == (real_t)0.0) which = 0;
    else if (phase == ECM && phasen == ECMn && side_value == (real_t)1.0) which = 1;
    else fail(fn, "expects (lum, lumn, 0.0) or (ECM, ECMn, 1.0)");
    if (step_done_by_fused()) return;
    check(pfag_fn_reshaping_lumen_or_ECM(ctx(fn), which), fn);
    report_relax_failures(ctx(fn), fn);
}

// cell_phase_functions.cpp:126-217 (+ the ghosts of phin, run_with_active_gels.cpp:172)
void update_all_cells(int it, real_t *phi_, real_t *phin_, real_t *g_, real_t *rho_, real_t *hfunc, real_t *f0,
                      real_t *psi_, int *xc, int *yc, real_t *hl, real_t *he) {
    const char *fn = "update_all_cells";
    (void)it;
    expect(phi_, phi, fn, "phi"); expect(phin_, phin, fn, "phin"); expect(g_, norm_grad_phi, fn, "norm_grad_phi");
    expect(rho_, rho, fn, "rho"); expect(hfunc, hfunc_cell, fn, "hfunc_cell"); expect(psi_, psi, fn, "psi");
    expect(xc, xcenters, fn, "xcenters"); expect(yc, ycenters, fn, "ycenters");
    expect(hl, hfunc_lum, fn, "hfunc_lum"); expect(he, hfunc_ECM, fn, "hfunc_ECM");
    if (!f0) fail(fn, "null f0");   // f0 as written by sum_s_kernels; the library keeps its own copy
    if (step_done_by_fused()) return;
    check(pfag_fn_update_all_cells(ctx(fn)), fn);
}

// cell_phase_functions.cpp:447-580
void reshaping_cells(int it, real_t *phase, real_t *phasen, real_t *g_, real_t *jx, real_t *jy, int *xc, int *yc) {
    const char *fn = "reshaping_cells";
    (void)it;
    expect(phase, phi, fn, "phi"); expect(phasen, phin, fn, "phin"); expect(g_, norm_grad_phi, fn, "norm_grad_phi");
    expect(jx, J_x, fn, "J_x"); expect(jy, J_y, fn, "J_y");
    expect(xc, xcenters, fn, "xcenters"); expect(yc, ycenters, fn, "ycenters");
    if (step_done_by_fused()) return;
    check(pfag_fn_reshaping_cells(ctx(fn)), fn);
    report_relax_failures(ctx(fn), fn);
}
