/* Library harness around the reference's own step functions.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  Compiled together with the
 * reference's functions/*.cpp (unmodified for the FP32 build, float->double
 * rewritten for the FP64 build), ref_params.cpp and cufft_shim.c into
 * oracle/_ref/libref_fp{32,64}.so.  It exposes, with C linkage, the set-up and
 * the loop body of main_code/run_with_active_gels.cpp so that tests can run the
 * reference step on arbitrary in-memory state:
 *   pfag_ref_init      <- run_with_active_gels.cpp:46-75 and :87-88
 *   pfag_ref_prepare   <- run_with_active_gels.cpp:92-98
 *   pfag_ref_step      <- run_with_active_gels.cpp:110-184 (one pass of the loop)
 * Every numerical operation is performed by the reference's own functions; this
 * file only calls them in the driver's order and moves data in and out.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cufft.h>
#include "constants.h"
#include "declare_tables.h"
#include "declare_fft_tables.h"
#include "initialisation_functions.h"
#include "useful_functions.h"
#include "rho_functions.h"
#include "cell_phase_functions.h"

#ifdef PFAG_REF_DOUBLE
typedef double real;
#else
typedef float real;
#endif

static real *g_s = nullptr;
static real *g_f0 = nullptr;

extern "C" int pfag_ref_real_size(void) { return (int)sizeof(real); }

/* run_with_active_gels.cpp:46-75 (allocation, zeroed phin/rhon/hfunc_cell) and :87-88 (plans) */
extern "C" int pfag_ref_init(void)
{
    malloc_all();
    ini_fft_all();
    g_s = (real *)std::malloc(Ntot * sizeof(real));
    g_f0 = (real *)std::malloc(Ntot * sizeof(real));
    if (!phi || !g_s || !g_f0) return -1;
    for (int n = 0; n < N_ini; n++) {
        ini_phin(phin, n);
        ini_rhon(rhon, n);
        ini_phin(hfunc_cell, n);
    }
    if (cufftPlan2d(&planf, 2 * zone_size - 2, 2 * zone_size - 2, CUFFT_C2C) != CUFFT_SUCCESS) return -2;
    if (cufftPlan2d(&planr, 2 * zone_size - 2, 2 * zone_size - 2, CUFFT_C2C) != CUFFT_SUCCESS) return -2;
    return 0;
}

/* Copy a state (phi, rho: Ntot*N_s*N_s; lum, ECM: N_s*N_s) into the reference's globals. */
extern "C" void pfag_ref_load(const real *phi_in, const real *rho_in, const real *lum_in, const real *ecm_in)
{
    const size_t nc = (size_t)Ntot * N_s * N_s, ng = (size_t)N_s * N_s;
    std::memcpy(phi, phi_in, nc * sizeof(real));
    std::memcpy(rho, rho_in, nc * sizeof(real));
    std::memcpy(lum, lum_in, ng * sizeof(real));
    std::memcpy(ECM, ecm_in, ng * sizeof(real));
}

/* run_with_active_gels.cpp:92-98 */
extern "C" void pfag_ref_prepare(void)
{
    copy_tables_ECM_or_lumen(ECMn, ECM);
    copy_tables_ECM_or_lumen(lumn, lum);
    for (int n = 0; n < Ntot; n++) {
        copy_cell_tables_1_by_1(n, phin, phi);
        copy_cell_tables_1_by_1(n, rhon, rho);
    }
}

/* One pass of the loop body, run_with_active_gels.cpp:110-184 (the snapshot at
 * :110-116 only when `save` is non-zero, the stderr print of :144-151 omitted). */
extern "C" void pfag_ref_step(int it_, int save)
{
    if (save && it_ % nsaving == 0)
        saving_out_functions(it_, phi, rho, ECM, lum, phiout, rhoout, lumout, ECMout);
    find_centres_cells(phi, xcenters, ycenters);
    create_turnover_rates_tensions(degrates, matgenrates, a_tan_1, a_ort_1, viscosity, b, phi, lum, ECM, xcenters, ycenters);
    compute_hfunc_3d_tables_kernels_loop_n(hfunc_cell, phi, xcenters, ycenters);
    compute_all_hfunc_2d_tables_kernels(hfunc_lum, lum, hfunc_ECM, ECM);
    compute_normal_grad_phi(norm_grad_phi, phi);
    boundary_conditions_cells(norm_grad_phi);
    compute_prod_norm_delta(prod_norm_delta, norm_grad_phi, phi, xcenters, ycenters);
    compute_psi_kernels(psi, hfunc_cell);
    sum_s_kernels(hfunc_cell, g_s, g_f0);
    update_all_cortices(phi, rho, rhon, xcenters, ycenters, degrates, matgenrates, a_tan_1, a_ort_1, viscosity, b,
                        norm_grad_phi, prod_norm_delta, planf, planr, temp_fft, temp_fft_real, fft_rho, fft_pi_xx,
                        fft_pi_xy, fft_pi_yy, fft_vx, fft_vy, fft_react, fft_rho_vx, fft_rho_vy);
    update_lumen_and_ECM(lum, lumn, ECM, ECMn, hfunc_lum, hfunc_ECM, psi);
    boundary_conditions_lumen_and_ECM(lumn, ECMn);
    reshaping_lumen_or_ECM(it_, lum, lumn, 0.0);
    reshaping_lumen_or_ECM(it_, ECM, ECMn, 1.0);
    compute_normal_to_phi(phi, norm_grad_phi, J_x, J_y);
    boundary_conditions_cells(J_x);
    boundary_conditions_cells(J_y);
    update_all_cells(it_, phi, phin, norm_grad_phi, rho, hfunc_cell, g_f0, psi, xcenters, ycenters, hfunc_lum, hfunc_ECM);
    boundary_conditions_cells(phin);
    reshaping_cells(it_, phi, phin, norm_grad_phi, J_x, J_y, xcenters, ycenters);
    for (int n = 0; n < Ntot; n++) copy_cell_tables_1_by_1(n, rho, rhon);
    copy_tables_ECM_or_lumen(ECM, ECMn);
    copy_tables_ECM_or_lumen(lum, lumn);
}

/* Read access to the reference's arrays by name (size in elements in *count). */
extern "C" void *pfag_ref_array(const char *name, long *count)
{
    const long nc = (long)Ntot * N_s * N_s, ng = (long)N_s * N_s;
    struct { const char *n; void *p; long c; } tab[] = {
        {"phi", phi, nc}, {"phin", phin, nc}, {"rho", rho, nc}, {"rhon", rhon, nc},
        {"lum", lum, ng}, {"lumn", lumn, ng}, {"ECM", ECM, ng}, {"ECMn", ECMn, ng},
        {"psi", psi, ng}, {"hfunc_cell", hfunc_cell, nc}, {"hfunc_lum", hfunc_lum, ng},
        {"hfunc_ECM", hfunc_ECM, ng}, {"norm_grad_phi", norm_grad_phi, nc},
        {"prod_norm_delta", prod_norm_delta, nc}, {"J_x", J_x, nc}, {"J_y", J_y, nc},
        {"temp_phase", temp_phase, nc}, {"norm_grad_lum", norm_grad_lum, ng},
        {"degrates", degrates, nc}, {"matgenrates", matgenrates, nc}, {"a_tan_1", a_tan_1, nc},
        {"a_ort_1", a_ort_1, nc}, {"viscosity", viscosity, nc}, {"b", b, nc},
        {"pi_xx", pi_xx, nc}, {"pi_xy", pi_xy, nc}, {"pi_yy", pi_yy, nc},
        {"xcenters", xcenters, Ntot}, {"ycenters", ycenters, Ntot}, {"s", g_s, Ntot}, {"f0", g_f0, Ntot},
        {"phiout", phiout, nc * Ntotsave}, {"rhoout", rhoout, nc * Ntotsave},
        {"lumout", lumout, ng * Ntotsave}, {"ECMout", ECMout, ng * Ntotsave},
    };
    for (auto &e : tab) if (std::strcmp(e.n, name) == 0) { if (count) *count = e.c; return e.p; }
    if (count) *count = 0;
    return nullptr;
}
