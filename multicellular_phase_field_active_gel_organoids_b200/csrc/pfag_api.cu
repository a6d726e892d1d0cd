// C ABI of libpfag (declared in include/pfag.h): contexts, state transfer,
// the step, and one entry point per reference function on the step path.
#include "pfag_internal.cuh"
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <new>

static thread_local char g_err[1024] = "";

void pfag_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int pfag_plain_fn(pfag_ctx *c, const char *which, int arg);

extern "C" const char *pfag_last_error(void) { return g_err; }
extern "C" int pfag_version(void) { return PFAG_VERSION; }

static int validate(const pfag_params *p) {
    if (!p) { pfag_set_error("null params"); return PFAG_E_ARG; }
    if (p->N_s < 8 || p->Ntot < 1 || p->zone_size < 3) {
        pfag_set_error("invalid sizes N_s=%d Ntot=%d zone_size=%d", p->N_s, p->Ntot, p->zone_size);
        return PFAG_E_ARG;
    }
    if (2 * p->zone_size + 2 > p->N_s) {
        pfag_set_error("zone 2*%d does not fit a %d grid", p->zone_size, p->N_s);
        return PFAG_E_ZONE;
    }
    if (!(p->dx > 0) || p->N_current <= 0) { pfag_set_error("dx and N_current must be positive"); return PFAG_E_ARG; }
    if (!(p->friction > 0)) {
        pfag_set_error("friction must be positive (the k=0 velocity mode divides by it)");
        return PFAG_E_ARG;
    }
    return PFAG_OK;
}

// Scalars in the reference's own operation order (double).
static DevParams make_devparams(const pfag_params &p) {
    DevParams d{};
    d.N = p.N_s; d.Ntot = p.Ntot; d.zone = p.zone_size; d.M = 2 * p.zone_size - 2; d.Ncur = p.N_current;
    d.dx = p.dx; d.dt = p.dt; d.s0 = p.s0; d.alpha = p.alpha; d.sigma = p.sigma; d.beta = p.beta;
    d.eta = p.eta; d.tau = p.tau; d.cpl = p.coupling_PF_AG;
    d.beta_lum_cells = p.beta_lum_cells; d.eta_lum_cells = p.eta_lum_cells;
    d.beta_ECM_cells = p.beta_ECM_cells; d.eta_ECM_cells = p.eta_ECM_cells;
    d.tau_lum = p.tau_lum; d.xi_lum = p.xi_lum; d.beta_lum_ECM = p.beta_lum_ECM;
    d.alpha_ECM = p.alpha_ECM; d.tau_ECM = p.tau_ECM; d.xi_ECM = p.xi_ECM;
    d.friction = p.friction; d.wi = p.wi; d.rdt = p.rdt;
    d.A_resh = p.wi * p.wi * (p.rdt / p.dx / p.dx);                 // cell_phase_functions.cpp:512
    d.B_resh = p.rdt * p.wi * std::sqrt(2.0) / p.dx;                 // :516
    d.thr_cells = p.rtol * 2.0 * M_PI * p.R * p.wi * p.rdt;          // :475
    d.thr_lum = (double)p.rdev_threshold * p.rtol * p.rdt;          // :774
    d.rdev0_lum = (double)(2 * p.rdev_threshold) * p.rtol * p.rdt;  // :720 (rdev_ini = 2*rdev_threshold)
    d.kfac = 2.0 * M_PI / ((2 * p.zone_size - 2) * p.dx);           // rho_functions.cpp:164
    d.inv_norm = 1.0 / ((double)d.M * (double)d.M);
    d.k_cpl = p.coupling_PF_AG / p.tau * (p.dt / p.dx / p.dx / 4.0) / std::sqrt(2.0 * M_PI) / p.sigma;
    d.inv_2s2 = 1.0 / (2.0 * p.sigma * p.sigma);
    d.dt_tau = p.dt / p.tau;
    d.inv_q4 = 1.0 / (4.0 * p.dx * p.dx);
    // rho_functions.cpp:355-397: 0 apical, 1 basal, 2 lateral
    d.deg[0] = p.degrate_apical; d.deg[1] = p.degrate_basal; d.deg[2] = p.degrate_lateral;
    d.gen[0] = p.matgenrate_apical; d.gen[1] = p.matgenrate_basal; d.gen[2] = p.matgenrate_lateral;
    d.a_ort[0] = p.a_ort_apical; d.a_ort[1] = p.a_ort_basal; d.a_ort[2] = p.a_ort_lateral;
    d.a_tan[0] = p.a_tan_apical; d.a_tan[1] = p.a_tan_basal; d.a_tan[2] = p.a_tan_lateral;
    d.visc[0] = p.viscosity_ap; d.visc[1] = p.viscosity_bas; d.visc[2] = p.viscosity_lat;
    d.bb[0] = p.b_ap; d.bb[1] = p.b_bas; d.bb[2] = p.b_lat;
    return d;
}

static void free_ctx(pfag_ctx *c) {
    if (!c) return;
    cudaStreamSynchronize(c->stream);
    pfag_plain_free(c);
    pfag_fused_free(c);
    pfag_prof_free(c);
    pfag_snapshot_free(c);
    void *bufs[] = {c->phi, c->phin, c->rho, c->rhon, c->lum, c->lumn, c->ecm, c->ecmn, c->hfunc, c->hlum,
                    c->hecm, c->psi, c->d_xc, c->d_yc, c->d_cacc, c->d_s, c->d_f0, c->d_part, c->d_scal,
                    c->d_iflags, c->d_err, c->d_vx, c->d_vy};
    for (void *b : bufs) if (b) cudaFree(b);
    void *hb[] = {c->h_iflags, c->h_scal, c->h_err};
    for (void *b : hb) if (b) cudaFreeHost(b);
    delete[] c->h_xc; delete[] c->h_yc; delete[] c->h_s; delete[] c->h_f0;
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int pfag_create(const pfag_params *p, int precision, int path, pfag_ctx **out) {
    if (!out) { pfag_set_error("null out"); return PFAG_E_ARG; }
    *out = nullptr;
    PFAG_TRY(validate(p));
    if (precision != 32 && precision != 64) { pfag_set_error("precision must be 32 or 64"); return PFAG_E_ARG; }
    if (path != PFAG_PATH_PLAIN && path != PFAG_PATH_FUSED) { pfag_set_error("unknown path %d", path); return PFAG_E_ARG; }
    pfag_ctx *c = new (std::nothrow) pfag_ctx();
    if (!c) { pfag_set_error("out of host memory"); return PFAG_E_ARG; }
    std::memset((void *)c, 0, sizeof(*c));
    c->p = *p;
    c->dp = make_devparams(*p);
    c->prec = precision;
    c->path = path;
    c->rsz = precision == 64 ? 8 : 4;
    c->relax_cap = p->rimax + 2;
    c->N = p->N_s; c->Ntot = p->Ntot; c->zone = p->zone_size; c->M = 2 * p->zone_size - 2;
    c->ng = (size_t)c->N * c->N;
    c->nc = (size_t)c->Ntot * c->ng;
    int rc = PFAG_OK;
#define ALLOC(ptr, bytes)                                                   \
    do {                                                                    \
        cudaError_t e_ = cudaMalloc((void **)&(ptr), (bytes));              \
        if (e_ != cudaSuccess) {                                            \
            pfag_set_error("cudaMalloc %zu bytes: %s", (size_t)(bytes), cudaGetErrorString(e_)); \
            rc = PFAG_E_CUDA;                                               \
            goto fail;                                                      \
        }                                                                   \
    } while (0)
    {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { pfag_set_error("stream: %s", cudaGetErrorString(e)); rc = PFAG_E_CUDA; goto fail; }
        const size_t rs = c->rsz;
        ALLOC(c->phi, c->nc * rs); ALLOC(c->phin, c->nc * rs); ALLOC(c->rho, c->nc * rs); ALLOC(c->rhon, c->nc * rs);
        ALLOC(c->hfunc, c->nc * rs);
        ALLOC(c->lum, c->ng * rs); ALLOC(c->lumn, c->ng * rs); ALLOC(c->ecm, c->ng * rs); ALLOC(c->ecmn, c->ng * rs);
        ALLOC(c->hlum, c->ng * rs); ALLOC(c->hecm, c->ng * rs); ALLOC(c->psi, c->ng * rs);
        ALLOC(c->d_xc, sizeof(int) * c->Ntot); ALLOC(c->d_yc, sizeof(int) * c->Ntot);
        ALLOC(c->d_cacc, sizeof(long long) * 3 * c->Ntot);
        ALLOC(c->d_s, sizeof(double) * c->Ntot); ALLOC(c->d_f0, sizeof(double) * c->Ntot);
        c->part_cap = std::max<size_t>((size_t)c->Ntot * 128, 4096);
        ALLOC(c->d_part, sizeof(double) * c->part_cap);
        ALLOC(c->d_scal, sizeof(double) * 64);
        ALLOC(c->d_iflags, sizeof(int) * (8 * c->Ntot + 64));
        ALLOC(c->d_err, sizeof(unsigned) * 4);
        cudaMemset(c->d_err, 0, sizeof(unsigned) * 4);
        cudaMemset(c->d_scal, 0, sizeof(double) * 64);
        if (cudaMallocHost((void **)&c->h_iflags, sizeof(int) * (8 * c->Ntot + 64)) != cudaSuccess ||
            cudaMallocHost((void **)&c->h_scal, sizeof(double) * 64) != cudaSuccess ||
            cudaMallocHost((void **)&c->h_err, sizeof(unsigned) * 4) != cudaSuccess) {
            pfag_set_error("pinned host allocation failed");
            rc = PFAG_E_CUDA;
            goto fail;
        }
        c->h_xc = new int[c->Ntot]();
        c->h_yc = new int[c->Ntot]();
        c->h_s = new double[c->Ntot]();
        c->h_f0 = new double[c->Ntot]();
        if (path == PFAG_PATH_PLAIN) rc = pfag_plain_alloc(c);
        else rc = pfag_fused_alloc(c);
        if (rc != PFAG_OK) goto fail;
    }
#undef ALLOC
    *out = c;
    return PFAG_OK;
fail:
    free_ctx(c);
    return rc;
}

extern "C" int pfag_destroy(pfag_ctx *ctx) {
    free_ctx(ctx);
    return PFAG_OK;
}

int pfag_check_device_error(pfag_ctx *c) {
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_err, c->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    unsigned e = c->h_err[0];
    if (e & ERRBIT_EMPTY_CELL) { pfag_set_error("a cell has no site with phi > 0.5"); return PFAG_E_EMPTY_CELL; }
    if (e & ERRBIT_ZONE) {
        pfag_set_error("a cell's zone [xc-%d, xc+%d) leaves the grid interior", c->zone, c->zone);
        return PFAG_E_ZONE;
    }
    if (e & ERRBIT_TIMEOUT) {
        // reported once and cleared: the kernel returned, the context stays usable
        pfag_set_error("a device wait for a TMA copy gave up after its iteration limit");
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        return PFAG_E_CUDA;
    }
    if (e & ERRBIT_ITER_CAP) { pfag_set_error("a device relaxation loop hit its iteration cap"); return PFAG_E_RELAX; }
    if (e & ERRBIT_RELAX) {
        // a cell loop passed rimax: the reference prints and goes on
        // (cell_phase_functions.cpp:563-567); counted, then cleared
        c->stats.relax_failures++;
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    }
    return PFAG_OK;
}

extern "C" int pfag_upload(pfag_ctx *c, const void *phi, const void *rho, const void *lum, const void *ecm) {
    if (!c || !phi || !rho || !lum || !ecm) { pfag_set_error("null argument"); return PFAG_E_ARG; }
    const size_t rs = c->rsz;
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->phi, phi, c->nc * rs, cudaMemcpyHostToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->rho, rho, c->nc * rs, cudaMemcpyHostToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->lum, lum, c->ng * rs, cudaMemcpyHostToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->ecm, ecm, c->ng * rs, cudaMemcpyHostToDevice, c->stream));
    return pfag_after_upload(c);
}

extern "C" int pfag_upload_device(pfag_ctx *c, const void *phi, const void *rho, const void *lum, const void *ecm) {
    if (!c || !phi || !rho || !lum || !ecm) { pfag_set_error("null argument"); return PFAG_E_ARG; }
    const size_t rs = c->rsz;
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->phi, phi, c->nc * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->rho, rho, c->nc * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->lum, lum, c->ng * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->ecm, ecm, c->ng * rs, cudaMemcpyDeviceToDevice, c->stream));
    return pfag_after_upload(c);
}

// The state phi, rho, lum, ECM is on the device: the rest of the set-up
// main does before its loop (run_with_active_gels.cpp:70-75 zero phin, rhon,
// hfunc_cell; :92-98 then copy), the fused path's upload checks; synchronous.
int pfag_after_upload(pfag_ctx *c) {
    const size_t rs = c->rsz;
    PFAG_CUDA_CHECK(cudaMemsetAsync(c->hfunc, 0, c->nc * rs, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->phin, c->phi, c->nc * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->rhon, c->rho, c->nc * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->lumn, c->lum, c->ng * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->ecmn, c->ecm, c->ng * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemsetAsync(c->psi, 0, c->ng * rs, c->stream));
    PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
    if (c->path == PFAG_PATH_FUSED) PFAG_TRY(pfag_fused_upload_hook(c));
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return PFAG_OK;
}

extern "C" int pfag_download(pfag_ctx *c, void *phi, void *rho, void *lum, void *ecm) {
    if (!c) { pfag_set_error("null ctx"); return PFAG_E_ARG; }
    const size_t rs = c->rsz;
    if (phi) PFAG_CUDA_CHECK(cudaMemcpyAsync(phi, c->phi, c->nc * rs, cudaMemcpyDeviceToHost, c->stream));
    if (rho) PFAG_CUDA_CHECK(cudaMemcpyAsync(rho, c->rho, c->nc * rs, cudaMemcpyDeviceToHost, c->stream));
    if (lum) PFAG_CUDA_CHECK(cudaMemcpyAsync(lum, c->lum, c->ng * rs, cudaMemcpyDeviceToHost, c->stream));
    if (ecm) PFAG_CUDA_CHECK(cudaMemcpyAsync(ecm, c->ecm, c->ng * rs, cudaMemcpyDeviceToHost, c->stream));
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return PFAG_OK;
}

int pfag_fetch_observables(pfag_ctx *c) {
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_s, c->d_s, sizeof(double) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_f0, c->d_f0, sizeof(double) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_xc, c->d_xc, sizeof(int) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_yc, c->d_yc, sizeof(int) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return PFAG_OK;
}

static int run_steps(pfag_ctx *c, int it0, int nsteps, bool sync) {
    if (!c || nsteps < 0) { pfag_set_error("bad arguments"); return PFAG_E_ARG; }
    c->launches = 0;
    for (int k = 0; k < nsteps; k++) {
        int rc = (c->path == PFAG_PATH_PLAIN) ? pfag_plain_step(c, it0 + k, sync) : pfag_fused_step(c, it0 + k, sync);
        if (rc != PFAG_OK) return rc;
    }
    if (sync) {
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        PFAG_TRY(pfag_check_device_error(c));
        PFAG_TRY(pfag_fetch_observables(c));
    }
    return PFAG_OK;
}

extern "C" int pfag_step(pfag_ctx *c, int it0, int nsteps) { return run_steps(c, it0, nsteps, true); }
extern "C" int pfag_step_async(pfag_ctx *c, int it0, int nsteps) { return run_steps(c, it0, nsteps, false); }
extern "C" int pfag_sync(pfag_ctx *c) {
    if (!c) return PFAG_E_ARG;
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    PFAG_TRY(pfag_check_device_error(c));
    if (c->path == PFAG_PATH_FUSED && c->fused) PFAG_TRY(pfag_fused_stats(c));
    return pfag_fetch_observables(c);
}

extern "C" int pfag_observables_async(pfag_ctx *c, double *s, double *f0, int *xc, int *yc) {
    if (!c) { pfag_set_error("null ctx"); return PFAG_E_ARG; }
    if (s) PFAG_CUDA_CHECK(cudaMemcpyAsync(s, c->d_s, sizeof(double) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    if (f0) PFAG_CUDA_CHECK(cudaMemcpyAsync(f0, c->d_f0, sizeof(double) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    if (xc) PFAG_CUDA_CHECK(cudaMemcpyAsync(xc, c->d_xc, sizeof(int) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    if (yc) PFAG_CUDA_CHECK(cudaMemcpyAsync(yc, c->d_yc, sizeof(int) * c->Ntot, cudaMemcpyDeviceToHost, c->stream));
    return PFAG_OK;
}

extern "C" int pfag_get_areas(pfag_ctx *c, double *s, double *f0) {
    if (!c) return PFAG_E_ARG;
    if (s) std::memcpy(s, c->h_s, sizeof(double) * c->Ntot);
    if (f0) std::memcpy(f0, c->h_f0, sizeof(double) * c->Ntot);
    return PFAG_OK;
}

extern "C" int pfag_get_centres(pfag_ctx *c, int *xc, int *yc) {
    if (!c) return PFAG_E_ARG;
    if (xc) std::memcpy(xc, c->h_xc, sizeof(int) * c->Ntot);
    if (yc) std::memcpy(yc, c->h_yc, sizeof(int) * c->Ntot);
    return PFAG_OK;
}

extern "C" int pfag_get_stats(pfag_ctx *c, pfag_stats *st) {
    if (!c || !st) return PFAG_E_ARG;
    *st = c->stats;
    return PFAG_OK;
}

extern "C" int pfag_set_relax_cap(pfag_ctx *c, int cap) {
    if (!c || cap < 1) { pfag_set_error("relax cap must be >= 1"); return PFAG_E_ARG; }
    c->relax_cap = cap;
    return PFAG_OK;
}

extern "C" int pfag_set_serial_sums(pfag_ctx *c, int on) {
    if (!c) return PFAG_E_ARG;
    if (on && c->path != PFAG_PATH_PLAIN) {
        pfag_set_error("serial-order sums exist on the plain path only");
        return PFAG_E_UNSUPPORTED;
    }
    c->serial_sums = on ? 1 : 0;
    return PFAG_OK;
}

extern "C" int pfag_get_cell_iters(pfag_ctx *c, int *iters) {
    if (!c || !iters) return PFAG_E_ARG;
    std::memcpy(iters, c->h_iflags + 4 * c->Ntot, sizeof(int) * c->Ntot);
    return PFAG_OK;
}

extern "C" int pfag_set_debug(pfag_ctx *c, int flags) {
    if (!c) return PFAG_E_ARG;
    c->debug = flags;
    if (flags && !c->d_vx) {
        const size_t n = (size_t)c->Ntot * c->M * c->M * c->rsz;
        PFAG_CUDA_CHECK(cudaMalloc(&c->d_vx, n));
        PFAG_CUDA_CHECK(cudaMalloc(&c->d_vy, n));
        PFAG_CUDA_CHECK(cudaMemset(c->d_vx, 0, n));
        PFAG_CUDA_CHECK(cudaMemset(c->d_vy, 0, n));
    }
    return PFAG_OK;
}

extern "C" int pfag_get_velocity(pfag_ctx *c, void *vx, void *vy) {
    if (!c || !c->d_vx) { pfag_set_error("velocity capture needs pfag_set_debug(ctx, 1) before the step"); return PFAG_E_ARG; }
    const size_t n = (size_t)c->Ntot * c->M * c->M * c->rsz;
    if (vx) PFAG_CUDA_CHECK(cudaMemcpyAsync(vx, c->d_vx, n, cudaMemcpyDeviceToHost, c->stream));
    if (vy) PFAG_CUDA_CHECK(cudaMemcpyAsync(vy, c->d_vy, n, cudaMemcpyDeviceToHost, c->stream));
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return PFAG_OK;
}

extern "C" int pfag_device_state(pfag_ctx *c, void **phi, void **rho, void **lum, void **ecm) {
    if (!c) return PFAG_E_ARG;
    if (phi) *phi = c->phi;
    if (rho) *rho = c->rho;
    if (lum) *lum = c->lum;
    if (ecm) *ecm = c->ecm;
    return PFAG_OK;
}

extern "C" int pfag_device_field(pfag_ctx *c, const char *name, void **ptr, long *elements) {
    if (!c || !name || !ptr) { pfag_set_error("null argument"); return PFAG_E_ARG; }
    struct { const char *n; void *p; size_t cnt; } tab[] = {
        {"phi", c->phi, c->nc}, {"phin", c->phin, c->nc}, {"rho", c->rho, c->nc}, {"rhon", c->rhon, c->nc},
        {"hfunc_cell", c->hfunc, c->nc}, {"psi", c->psi, c->ng}, {"lum", c->lum, c->ng},
        {"lumn", c->lumn, c->ng}, {"ECM", c->ecm, c->ng}, {"ECMn", c->ecmn, c->ng},
        {"hfunc_lum", c->hlum, c->ng}, {"hfunc_ECM", c->hecm, c->ng}};
    for (auto &e : tab) {
        if (std::strcmp(e.n, name) == 0) {
            *ptr = e.p;
            if (elements) *elements = (long)e.cnt;
            return PFAG_OK;
        }
    }
    pfag_set_error("unknown field %s", name);
    return PFAG_E_ARG;
}

extern "C" void *pfag_stream(pfag_ctx *c) { return c ? (void *)c->stream : nullptr; }
extern "C" long pfag_launch_count(pfag_ctx *c) { return c ? c->launches : -1; }

// ---- per-function entry points (plain-path kernels) ------------------------
static int need_plain(pfag_ctx *c) {
    if (!c) { pfag_set_error("null ctx"); return PFAG_E_ARG; }
    if (c->path != PFAG_PATH_PLAIN) {
        pfag_set_error("per-function entry points need a context created with PFAG_PATH_PLAIN");
        return PFAG_E_UNSUPPORTED;
    }
    return PFAG_OK;
}

#define FN(name, which, arg)                          \
    extern "C" int name(pfag_ctx *c) {                \
        PFAG_TRY(need_plain(c));                      \
        PFAG_TRY(pfag_plain_fn(c, which, arg));       \
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream)); \
        return PFAG_OK;                               \
    }
FN(pfag_fn_find_centres_cells, "centres", 0)
FN(pfag_fn_create_turnover_rates_tensions, "maps", 0)
FN(pfag_fn_compute_hfunc_3d_tables_kernels_loop_n, "hfunc3d", 0)
FN(pfag_fn_compute_all_hfunc_2d_tables_kernels, "hfunc2d", 0)
FN(pfag_fn_compute_normal_grad_phi, "norm_grad", 0)
FN(pfag_fn_compute_prod_norm_delta, "pnd", 0)
FN(pfag_fn_compute_psi_kernels, "psi", 0)
FN(pfag_fn_update_all_cortices, "cortices", 0)
FN(pfag_fn_update_lumen_and_ECM, "lum_ecm_update", 0)
FN(pfag_fn_compute_normal_to_phi, "normals", 0)
FN(pfag_fn_update_all_cells, "update_cells", 0)
FN(pfag_fn_reshaping_cells, "reshape_cells", 0)
FN(pfag_fn_copy_back, "copy_back", 0)
#undef FN

extern "C" int pfag_fn_reshaping_lumen_or_ECM(pfag_ctx *c, int which) {
    PFAG_TRY(need_plain(c));
    PFAG_TRY(pfag_plain_fn(c, "reshape_lum", which ? 1 : 0));
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return PFAG_OK;
}

extern "C" int pfag_fn_sum_s_kernels(pfag_ctx *c, double *s_host, double *f0_host) {
    PFAG_TRY(need_plain(c));
    PFAG_TRY(pfag_plain_fn(c, "sum_s", 0));
    PFAG_TRY(pfag_fetch_observables(c));
    return pfag_get_areas(c, s_host, f0_host);
}

extern "C" int pfag_generate_initial(pfag_ctx *c, double rho0, double tol, int make_fields) {
    PFAG_TRY(need_plain(c));
    if (!(tol > 0.0) || !(rho0 >= 0.0)) { pfag_set_error("rho0 must be >= 0 and tol > 0"); return PFAG_E_ARG; }
    PFAG_TRY(pfag_plain_generate(c, rho0, tol, make_fields));
    return pfag_fetch_observables(c);
}

extern "C" int pfag_fn_saving_out_functions(pfag_ctx *c, void *phi_out, void *rho_out, void *lum_out, void *ecm_out) {
    return pfag_download(c, phi_out, rho_out, lum_out, ecm_out);
}
