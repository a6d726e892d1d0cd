/* Definitions of the reference's global parameter set for the oracle builds.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference declares its parameters as extern
 * globals in functions/constants.h:1-124 and defines them in a jinja2-rendered
 * functions/constants_template.cpp:4-129, where N_s and Ntot are compile-time
 * `const int`.  This file defines the same symbols (same names, same storage
 * types; `REAL` is float for the shipped build and double for the
 * float->double rewritten build) but leaves every one of them writable, so a
 * single oracle binary serves every grid size and cell count.  Values are
 * loaded before main() from the key/value text file named by the environment
 * variable PFAG_REF_PARAMS (one "name value" pair per line), or set at run time
 * with pfag_ref_param_set().  Derived values (a_tan_* = a_ort_* * epsilon_*,
 * Ntotsave, ...) are computed by the generator of that file, following
 * constants_template.cpp:14,27,61-63,74-75,88,94,102.
 *
 * The reference header is deliberately not included: it declares N_s, Ntot
 * and L as `extern const int`, and these writable definitions carry the same
 * unmangled symbol names.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>

#ifdef PFAG_REF_DOUBLE
typedef double REAL;
#else
typedef float REAL;
#endif

int threshold_reshaping_steps = 100000;
int riprint = 100000;
int rdev_threshold = 5;
int rdev_ini = 10;
int Nsteps = 11;
int ncontinue = 0;
int ndisplay = 5;
int nsaving = 10;
int Ntotsave = 2;
REAL dx = 0.01;
REAL dt = 0.002;
int N_s = 1200;
int L = 120;
REAL R0 = 1.0;
REAL R = 1.0;
REAL s0 = 3.15159265359;
REAL Rint = 1.0;
REAL Rout = 1.0;
REAL sigma = 0.2;
int N_ini = 6;
int Ntot = 6;
int N_current = 6;
int zone_size = 200;
REAL coupling_PF_AG = 1.0;
int random_ontime = 12;
REAL seuil_gel = 0.1;
int gen_ontime = 0;
int active_gel_ontime = 0;
int contract_ontime = 0;
REAL epsilon_ap = 1.0, epsilon_bas = 1.0, epsilon_lat = 1.0;
REAL a_ort_lateral = 100.0, a_ort_apical = 100.0, a_ort_basal = 100.0;
REAL a_tan_lateral = 100.0, a_tan_apical = 100.0, a_tan_basal = 100.0;
REAL b_ap = 1.0, b_bas = 1.0, b_lat = 1.0;
REAL matgenrate_apical = 1.0, degrate_apical = 100.0;
REAL matgenrate_lateral = 1.0, degrate_lateral = 100.0;
REAL matgenrate_basal = 1.0, degrate_basal = 100.0;
REAL friction = 1.0;
REAL viscosity_ap = 1.0, viscosity_bas = 1.0, viscosity_lat = 1.0;
REAL tau = 1.0, alpha = 1.0, beta = 1.0, eta = 0.03, gamma_cell = 0.045;
REAL tau_lum = 1.0, beta_lum_cells = 1.0, eta_lum_cells = 0.0, gamma_lum_cells = 0.0, xi_lum = 0.15;
REAL alpha_ECM = 0.002, tau_ECM = 1.0, beta_ECM_cells = 1.0, eta_ECM_cells = 0.001,
     gamma_ECM_cells = 0.0011, xi_ECM = 0.0;
REAL beta_lum_ECM = 1.0;
REAL wi = 0.07, rho0 = 0.001, tol = 0.01;
int ri;
int rimax = 1000000;
REAL rdev;
REAL rtol = 0.001, rdt = 0.001;
REAL ans = 0.0, sum_s = 0.0;
int it, k, l, ir, jr, c;
int nelse;
int ip, im, jp, jm;
/* declared extern in constants.h:207,215,224,252 but never defined by the template */
REAL D0, D_lum, D_ECM;
int i, j, n;

struct ParamEntry { const char *name; void *ptr; int is_int; };

#define PR(x) { #x, (void *)&x, 0 }
#define PI_(x) { #x, (void *)&x, 1 }
static const ParamEntry g_params[] = {
    PI_(threshold_reshaping_steps), PI_(riprint), PI_(rdev_threshold), PI_(rdev_ini),
    PI_(Nsteps), PI_(ncontinue), PI_(ndisplay), PI_(nsaving), PI_(Ntotsave),
    PR(dx), PR(dt), PI_(N_s), PI_(L), PR(R0), PR(R), PR(s0), PR(Rint), PR(Rout), PR(sigma),
    PI_(N_ini), PI_(Ntot), PI_(N_current), PI_(zone_size), PR(coupling_PF_AG),
    PI_(random_ontime), PR(seuil_gel), PI_(gen_ontime), PI_(active_gel_ontime), PI_(contract_ontime),
    PR(epsilon_ap), PR(epsilon_bas), PR(epsilon_lat),
    PR(a_ort_lateral), PR(a_ort_apical), PR(a_ort_basal),
    PR(a_tan_lateral), PR(a_tan_apical), PR(a_tan_basal),
    PR(b_ap), PR(b_bas), PR(b_lat),
    PR(matgenrate_apical), PR(degrate_apical), PR(matgenrate_lateral), PR(degrate_lateral),
    PR(matgenrate_basal), PR(degrate_basal),
    PR(friction), PR(viscosity_ap), PR(viscosity_bas), PR(viscosity_lat),
    PR(tau), PR(alpha), PR(beta), PR(eta), PR(gamma_cell),
    PR(tau_lum), PR(beta_lum_cells), PR(eta_lum_cells), PR(gamma_lum_cells), PR(xi_lum),
    PR(alpha_ECM), PR(tau_ECM), PR(beta_ECM_cells), PR(eta_ECM_cells), PR(gamma_ECM_cells), PR(xi_ECM),
    PR(beta_lum_ECM), PR(wi), PR(rho0), PR(tol), PI_(rimax), PR(rtol), PR(rdt),
};

extern "C" int pfag_ref_param_set(const char *name, double value)
{
    for (const ParamEntry &e : g_params) {
        if (std::strcmp(e.name, name) == 0) {
            if (e.is_int) *(int *)e.ptr = (int)value;
            else *(REAL *)e.ptr = (REAL)value;
            return 0;
        }
    }
    return -1;
}

extern "C" double pfag_ref_param_get(const char *name)
{
    for (const ParamEntry &e : g_params)
        if (std::strcmp(e.name, name) == 0)
            return e.is_int ? (double)*(int *)e.ptr : (double)*(REAL *)e.ptr;
    return 0.0 / 0.0;
}

extern "C" int pfag_ref_param_load(const char *path)
{
    FILE *f = std::fopen(path, "r");
    if (!f) { std::fprintf(stderr, "pfag oracle: cannot open parameter file %s\n", path); return -1; }
    char key[128];
    double v;
    int bad = 0;
    while (std::fscanf(f, "%127s %lf", key, &v) == 2) {
        if (pfag_ref_param_set(key, v) != 0) {
            std::fprintf(stderr, "pfag oracle: unknown parameter %s\n", key);
            bad = 1;
        }
    }
    std::fclose(f);
    return bad ? -1 : 0;
}

__attribute__((constructor)) static void pfag_ref_param_autoload()
{
    const char *p = std::getenv("PFAG_REF_PARAMS");
    if (p && *p && pfag_ref_param_load(p) != 0) std::exit(3);
}
