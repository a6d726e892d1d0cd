/* pfag.h — C ABI of the B200 time step of the multicellular phase-field /
 * active-gel organoid model (drop-in for the step that
 * main_code/run_with_active_gels.cpp:101-185 of the reference drives).
 *
 * Plain pointers and sizes only.  All state arrays use the reference layout:
 * per-cell fields [Ntot][N_s][N_s] row-major (index n*N_s*N_s + i*N_s + j),
 * shared fields [N_s][N_s].  The element type is double for a context created
 * with precision 64 and float for precision 32; `const void *` arguments carry
 * that type.  Every function returns PFAG_OK (0) or a negative PFAG_E* code;
 * pfag_last_error() gives the message of the last failure on this thread.
 */
#ifndef PFAG_H
#define PFAG_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PFAG_OK = 0,
    PFAG_E_ARG = -1,          /* invalid argument or parameter */
    PFAG_E_CUDA = -2,         /* CUDA runtime / cuFFT failure */
    PFAG_E_ZONE = -3,         /* a cell's zone or FFT box leaves the grid (the reference reads out of bounds there) */
    PFAG_E_EMPTY_CELL = -4,   /* a cell has no site with phi > 0.5 (the reference divides by zero there) */
    PFAG_E_UNSUPPORTED = -5,  /* configuration outside what the selected path supports */
    PFAG_E_RELAX = -6         /* a reshaping loop passed rimax (the reference prints "Relaxation failure!" and goes on) */
};

/* Execution paths. */
enum {
    PFAG_PATH_PLAIN = 0,  /* one kernel per reference function, full-grid passes where the reference makes them, cuFFT */
    PFAG_PATH_FUSED = 1   /* zone-restricted fused kernels, hand-written batched FFT, device-side convergence loops */
};

/* The parameter set of functions/constants_template.cpp:4-129 that the step
 * reads (the same names; derived values already derived). */
typedef struct pfag_params {
    int N_s, Ntot, zone_size, N_current;
    int rdev_threshold, rimax;
    double dx, dt, R, s0, sigma, coupling_PF_AG;
    double tau, alpha, beta, eta;
    double tau_lum, beta_lum_cells, eta_lum_cells, xi_lum;
    double alpha_ECM, tau_ECM, beta_ECM_cells, eta_ECM_cells, xi_ECM, beta_lum_ECM;
    double wi, rtol, rdt, friction;
    double a_tan_apical, a_tan_basal, a_tan_lateral;
    double a_ort_apical, a_ort_basal, a_ort_lateral;
    double b_ap, b_bas, b_lat;
    double matgenrate_apical, matgenrate_basal, matgenrate_lateral;
    double degrate_apical, degrate_basal, degrate_lateral;
    double viscosity_ap, viscosity_bas, viscosity_lat;
} pfag_params;

/* Per-step diagnostics of the last pfag_step call (its final step). */
typedef struct pfag_stats {
    int cell_iters_max;     /* largest reshaping iteration count over cells (cell_phase_functions.cpp:475-574) */
    int cell_iters_sum;     /* sum over cells */
    int lum_iters;          /* lumen reshaping iterations (cell_phase_functions.cpp:774-869, side 0) */
    int ecm_iters;          /* ECM reshaping iterations (side 1) */
    int relax_failures;     /* loops that passed rimax */
    double sum_ecm;         /* sum of h(ECM) dx^2 (cell_phase_functions.cpp:376-386) */
} pfag_stats;

typedef struct pfag_ctx pfag_ctx;

const char *pfag_last_error(void);
int pfag_version(void);

/* Create a context on the current CUDA device; allocates the device state.
 * precision: 64 (double) or 32 (float).  path: PFAG_PATH_*. */
int pfag_create(const pfag_params *p, int precision, int path, pfag_ctx **out);
int pfag_destroy(pfag_ctx *ctx);

/* Host -> device state (run_with_active_gels.cpp:65-75 then :92-98):
 * phi, rho [Ntot][N][N], lum, ECM [N][N]; phin, rhon, hfunc_cell start at zero
 * and are then set to phi, rho (the copies at :92-98).  Synchronous. */
int pfag_upload(pfag_ctx *ctx, const void *phi, const void *rho, const void *lum, const void *ecm);
/* The same from device buffers of the current device (element type by the
 * context's precision).  Synchronous. */
int pfag_upload_device(pfag_ctx *ctx, const void *phi, const void *rho, const void *lum, const void *ecm);
/* Device -> host state; any pointer may be NULL.  Synchronous. */
int pfag_download(pfag_ctx *ctx, void *phi, void *rho, void *lum, void *ecm);

/* Advance nsteps steps from step index it0 (the loop body of
 * run_with_active_gels.cpp:110-184 without the snapshot).  Synchronous. */
int pfag_step(pfag_ctx *ctx, int it0, int nsteps);
/* The same, enqueued on the context's stream without a final synchronisation
 * (device-resident benchmarking); errors surface at the next synchronous call. */
int pfag_step_async(pfag_ctx *ctx, int it0, int nsteps);
/* Wait for the context's stream, report device-side errors, and refresh the
 * host copies of the observables and (fused path) the reshaping statistics. */
int pfag_sync(pfag_ctx *ctx);

/* Observables of the last step: s (Ntot doubles, cell areas), xc, yc (Ntot ints). */
int pfag_get_areas(pfag_ctx *ctx, double *s, double *f0);
/* The areas s, f0 and centres of the last enqueued step (sum_s_kernels and
 * find_centres_cells results), copied to the given host buffers in stream
 * order after it, without waiting: valid after pfag_sync (or any later
 * synchronising call).  Any pointer may be NULL; pinned buffers make the copy
 * asynchronous.  With pfag_step_async this streams every step's observables
 * back without a host round trip per step. */
int pfag_observables_async(pfag_ctx *ctx, double *s, double *f0, int *xc, int *yc);
int pfag_get_centres(pfag_ctx *ctx, int *xc, int *yc);
int pfag_get_stats(pfag_ctx *ctx, pfag_stats *st);
/* Per-cell reshaping iteration counts of the last step (Ntot ints). */
int pfag_get_cell_iters(pfag_ctx *ctx, int *iters);
/* Per-cell velocity of the last step's spectral solve, Re(IFFT(v))/M^2 on the
 * FFT box (rho_functions.cpp:449-456): vx, vy [Ntot][M][M], M = 2*zone_size-2.
 * Requires pfag_set_debug(ctx, 1) before the step.  Any nonzero flags keep
 * the fused path eager (no graph).  Bit 2 (flags & 2) is a test hook of the
 * device-side wait limits: the TMA-staged lumen tiles (pfag_set_lumen_tiles)
 * then wait for copies that are never issued, so their bounded waits run out
 * with nothing in flight; the next synchronising call returns PFAG_E_CUDA
 * once ("a device wait ... gave up") and the context stays usable. */
int pfag_set_debug(pfag_ctx *ctx, int flags);
int pfag_get_velocity(pfag_ctx *ctx, void *vx, void *vy);

/* Bound on the device-side relaxation loops of the fused path (default
 * rimax + 2, the bound the reference's loops have).  A loop that reaches the
 * cap stops with PFAG_E_RELAX reported at the next synchronisation. */
int pfag_set_relax_cap(pfag_ctx *ctx, int cap);

/* Plain path only: on != 0 takes the cell areas (sum_s_kernels,
 * useful_functions.cpp:179-184), sum_ecm (cell_phase_functions.cpp:380-386)
 * and the reshaping loops' rdev sums (cell_phase_functions.cpp:556-561,
 * :848-854) in the reference's serial host order, one thread per sum adding
 * the terms i-major with the reference's expression, so each sum rounds as
 * the host build's does on the same state.  Slow (a thread walks the grid);
 * for parity studies.  The fused path returns PFAG_E_UNSUPPORTED. */
int pfag_set_serial_sums(pfag_ctx *ctx, int on);

/* A seeded synthetic organoid generated on the device instead of uploaded:
 * phi_n = 0.5 (1 - tanh((r_n - radius)/2)) about centres[2n], centres[2n+1]
 * (grid coordinates i, j; host array of Ntot pairs), rho_n = 1 where
 * 0.05 < phi_n < 0.95 times (1 + 0.01 u) with u uniform in [-1, 1) from a
 * hash of (seed, site), lumen 0, ECM 0.5 (1 + tanh((r - env_radius)/2))
 * about the mean centre; then everything pfag_upload does after its copies.
 * For workloads whose state is too large to build on the host.  Synchronous.
 * No counterpart in the reference (it reads ini_*.bin files). */
int pfag_seed_organoid(pfag_ctx *ctx, const double *centres, double radius, double env_radius,
                       unsigned long long seed);

/* Fused path: launch shapes of the step's persistent relaxation kernel and
 * phi update (the knobs the batched sweep's autotuner sets).  coop_blocks > 0
 * caps the persistent kernel's grid (0: the default, every co-resident block
 * up to the loops' task count); update_warps > 0 is the warp budget the phi
 * update sizes its row tasks for (0: the default, one full wave of the GPU).
 * The next step recaptures its graph.  No counterpart in the reference (its
 * OpenACC runtime picks the launch shapes). */
int pfag_set_launch_shape(pfag_ctx *ctx, int coop_blocks, long update_warps);
/* Fused path, FP32: tma != 0 runs the lumen / ECM relaxation iterations that
 * precede the persistent kernel (reshaping_lumen_or_ECM,
 * cell_phase_functions.cpp:774-869) on tiles staged by TMA (kl_relax_tma)
 * instead of per-thread copies (kl_relax); the same arithmetic per site, the
 * rdev tile partials in another grouping.  Off by default: faster alone, but
 * slower inside the step, where it runs beside the spectral passes.  A knob of
 * the batched sweep's autotuner.  PFAG_E_UNSUPPORTED unless N_s >= 128 and
 * N_s % 4 == 0 (FP32 contexts only). */
int pfag_set_lumen_tiles(pfag_ctx *ctx, int tma);

/* ---- Batches: several organoids (fused-path contexts on the current device)
 * advanced together, the in-process form of the reference's parameter sweep
 * (main_code/setup_simulation.py:206-312 writes one folder and one batch job
 * per member).  After each member's first two steps (the first eager, the
 * second captured as its step graph) a batch step is ONE graph launch whose
 * child graphs are the members' step graphs, with no dependencies between
 * members, so the GPU runs them side by side.  Member order is the caller's
 * (group members of one box size together: the autotuner's buckets).
 * pfag_batch_step is synchronous and refreshes every member's observables
 * and statistics; pfag_batch_step_async enqueues only (the members' streams
 * wait for it, so per-member calls stay ordered after it).  A member whose
 * step graph changes (a new relaxation cap, launch shape, debug flag) makes
 * the next batch step rebuild the parent graph. */
typedef struct pfag_batch pfag_batch;
int pfag_batch_create(pfag_ctx *const *ctxs, int n, pfag_batch **out);
int pfag_batch_step(pfag_batch *b, int it0, int nsteps);
int pfag_batch_step_async(pfag_batch *b, int it0, int nsteps);
int pfag_batch_sync(pfag_batch *b);
void *pfag_batch_stream(pfag_batch *b);       /* cudaStream_t the parent graph is launched on */
long pfag_batch_launch_count(pfag_batch *b);  /* kernel launches of the last step call */
int pfag_batch_destroy(pfag_batch *b);

/* ---- Cell sharding: one organoid's cells split over contexts by contiguous
 * ranges (one context per GPU, or several on one GPU).  Cells couple only
 * through psi = sum_n h(phi_n) (useful_functions.cpp:305-322) and the index
 * neighbours' phi in the class map (rho_functions.cpp:297-311, cyclic over
 * the organoid); lum and ECM are updated redundantly by every shard from the
 * full psi.  A shard is a fused-path context created with Ntot = its cell
 * count and the organoid's N_current.
 * pfag_shard_enable allocates the context's two neighbour planes (N_s^2
 * values each, the context's precision) and returns their device pointers:
 * *lo holds phi of the cell before local cell 0, *hi phi of the cell after
 * local cell Ntot-1; the host writes them before each step (they start as
 * the context's own cells Ntot-1 and 0, i.e. an unsharded organoid).
 * pfag_step_head enqueues the step up to this context's partial psi (over
 * its own cells, in cell order; pfag_device_field "psi"); the host then
 * completes psi on every shard (the sum over shards, the same values on
 * every shard) and pfag_step_tail enqueues the rest of the step.  Both are
 * asynchronous on the context's stream and replay CUDA graphs from the
 * second step on; pfag_sync afterwards refreshes the observables.  Fused
 * path only (PFAG_E_UNSUPPORTED otherwise); a tail without its head, or a
 * whole-step call between them, returns PFAG_E_ARG.
 * pfag_sum_planes: out[i] = parts[0][i] + parts[1][i] + ... in that order
 * (1 <= nparts <= 64; precision 32 or 64; out may be one of the parts), on
 * `stream` (cudaStream_t); with one part it is a device copy. */
int pfag_shard_enable(pfag_ctx *ctx, void **lo, void **hi);
int pfag_step_head(pfag_ctx *ctx, int it);
int pfag_step_tail(pfag_ctx *ctx, int it);
int pfag_sum_planes(void *out, const void *const *parts, int nparts, long count, int precision, void *stream);

/* Per-kernel CUDA-event timing of the fused path on the context's stream.
 * pfag_profile_read synchronises and returns the number of kernels (<= cap):
 * names (64 bytes each), accumulated milliseconds and launch counts since the
 * previous read. */
int pfag_set_profile(pfag_ctx *ctx, int on);
int pfag_profile_read(pfag_ctx *ctx, char *names, double *ms, long *launches, int cap);

/* Device pointers of the state (phi, rho: [Ntot][N][N]; lum, ECM: [N][N]). */
int pfag_device_state(pfag_ctx *ctx, void **phi, void **rho, void **lum, void **ecm);
/* Device pointer of one named state array of the context: "phi", "phin",
 * "rho", "rhon", "hfunc_cell", "psi", "lum", "lumn", "ECM", "ECMn",
 * "hfunc_lum", "hfunc_ECM" (reference names, declare_tables.h:20-60);
 * *elements receives its length.  The context keeps ownership. */
int pfag_device_field(pfag_ctx *ctx, const char *name, void **ptr, long *elements);
/* CUDA stream (cudaStream_t) the context enqueues on. */
void *pfag_stream(pfag_ctx *ctx);
/* Number of kernel launches the last pfag_step / pfag_step_async enqueued. */
long pfag_launch_count(pfag_ctx *ctx);

/* ---- One entry point per reference function on the step path. ----------
 * Each operates on the context's device state, exactly as the reference
 * function of the same name does on its OpenACC-present arrays.  They are
 * what the C++ drop-in layer (reference signatures) forwards to. */
int pfag_fn_find_centres_cells(pfag_ctx *ctx);                 /* useful_functions.cpp:193-227 */
int pfag_fn_create_turnover_rates_tensions(pfag_ctx *ctx);     /* rho_functions.cpp:286-405 */
int pfag_fn_compute_hfunc_3d_tables_kernels_loop_n(pfag_ctx *ctx); /* useful_functions.cpp:233-251 */
int pfag_fn_compute_all_hfunc_2d_tables_kernels(pfag_ctx *ctx);   /* useful_functions.cpp:272-285 */
int pfag_fn_compute_normal_grad_phi(pfag_ctx *ctx);            /* useful_functions.cpp:326-354 + :391-420 */
int pfag_fn_compute_prod_norm_delta(pfag_ctx *ctx);            /* rho_functions.cpp:13-30 */
int pfag_fn_compute_psi_kernels(pfag_ctx *ctx);                /* useful_functions.cpp:305-322 */
int pfag_fn_sum_s_kernels(pfag_ctx *ctx, double *s_host, double *f0_host); /* useful_functions.cpp:168-190 */
int pfag_fn_update_all_cortices(pfag_ctx *ctx);                /* rho_functions.cpp:409-471 */
int pfag_fn_update_lumen_and_ECM(pfag_ctx *ctx);               /* cell_phase_functions.cpp:372-444 + useful_functions.cpp:439-462 */
int pfag_fn_reshaping_lumen_or_ECM(pfag_ctx *ctx, int which);  /* cell_phase_functions.cpp:709-871; which 0 lumen, 1 ECM */
int pfag_fn_compute_normal_to_phi(pfag_ctx *ctx);              /* useful_functions.cpp:356-388 + :391-420 */
int pfag_fn_update_all_cells(pfag_ctx *ctx);                   /* cell_phase_functions.cpp:126-217 + useful_functions.cpp:391-420 */
int pfag_fn_reshaping_cells(pfag_ctx *ctx);                    /* cell_phase_functions.cpp:447-580 */
int pfag_fn_copy_back(pfag_ctx *ctx);                          /* run_with_active_gels.cpp:175-182 */
/* Cell areas s[n] = sum of hfunc_cell[n] dx^2 over the grid and
 * f0[n] = alpha (s0 - s[n]), computed the way pfag_fn_sum_s_kernels computes
 * them, for callers that cannot allocate device memory: a host program whose
 * device memory already belongs to another allocator (an OpenACC data region,
 * a framework's caching allocator, a pool reserved up front), or a
 * latency-critical loop that must not pay cudaMalloc's device
 * synchronisation.  This entry point has no counterpart in the reference.
 * It allocates nothing: its scratch is a 1 MiB static device array that each
 * GPU loading the library holds until exit, so Ntot may be at most 1024
 * (larger values return PFAG_E_ARG).  hfunc_cell ([Ntot][N_s][N_s], element
 * type by precision 32/64), s and f0 (Ntot doubles) are device pointers the
 * caller owns; the work is enqueued on `stream` (a cudaStream_t, NULL for the
 * default stream) and not synchronised.  The first call on a device resolves
 * the scratch address there (cudaGetSymbolAddress) and should be made before
 * any stream capture.  The resolved address belongs to the device's current
 * primary context: a process that resets the device (cudaDeviceReset) must
 * not call this entry point on that device afterwards.  All calls share the one scratch array, so calls that
 * overlap on the GPU (different streams, no ordering) race; order them on one
 * stream.  Every scratch value a call reads it first writes, so no clearing
 * is needed between calls. */
int pfag_areas_noalloc(const void *hfunc_cell, int precision, int Ntot, int N_s, double dx, double alpha,
                       double s0, double *s, double *f0, void *stream);

/* The initial-condition generator, initialisation_code/prepare_initial_files.cpp:53-117,
 * on the device (a context created with PFAG_PATH_PLAIN).  make_fields != 0:
 * first the initial fields of functions/initialisation_functions.cpp:62-160
 * (ini_phi: Ntot cells on a ring of radius Ntot*0.9*R/dx/pi about the centre,
 * logistic profiles of width wi; ini_ECM_lumen; ini_rho with rho0, tol;
 * phin = 0); make_fields == 0: the uploaded state stands for them.  Then the
 * one-shot shaping: centres, phin <- phi, |grad phi| and normals, the cells'
 * reshaping loops, rho refitted to the cells (update_rho_to_shape,
 * cell_phase_functions.cpp:42-62), the lumen/ECM update and reshaping.
 * pfag_download then returns what the reference saves in snapshot slot 1
 * (the ini_*.bin files it writes, :139-213). */
int pfag_generate_initial(pfag_ctx *ctx, double rho0, double tol, int make_fields);

/* saving_out_functions (useful_functions.cpp:66-99) without stalling the
 * steps: the state (phi, rho: Ntot*N*N; lum, ecm: N*N elements) is copied into
 * a device staging area on the context's stream, then into the given host
 * buffers on a copy stream while later steps run.  Returns a ticket (>= 0) or
 * an error code (< 0).  Host buffers should be pinned (cudaHostAlloc) and must
 * stay untouched until pfag_snapshot_wait(ticket) has returned.  The first call
 * allocates the staging area (2 Ntot N^2 + 2 N^2 reals). */
long pfag_snapshot_async(pfag_ctx *ctx, void *phi, void *rho, void *lum, void *ecm);
int pfag_snapshot_wait(pfag_ctx *ctx, long ticket);

/* One N x N table (precision 32 or 64) written in the reference's text layout,
 * "%.15f\n" per value and a blank line after each row
 * (run_with_active_gels.cpp:215-229); host only, several threads. */
int pfag_write_text_snapshot(const void *table, int precision, int N, const char *path);

/* saving_out_functions (useful_functions.cpp:66-99): device state -> host
 * snapshot slot; phi_out/rho_out get Ntot*N*N, lum_out/ecm_out N*N elements. */
int pfag_fn_saving_out_functions(pfag_ctx *ctx, void *phi_out, void *rho_out, void *lum_out, void *ecm_out);

/* ---- Learned coarse-grid corrector: convolution kernels on tcgen05 ----------
 * No counterpart in the reference (its step has no learned part).  Tensors are
 * device buffers.  An activation is BF16 [B][H+2][W+2][C] (channels last,
 * with a one-site zero halo that is the convolution's zero padding; the
 * caller zeroes a buffer once, the kernels keep its halo zero); weights are
 * BF16 [Cout][9][Cin], tap t = (dy+1)*3 + (dx+1); biases and gradients FP32.
 * All work is enqueued on `stream` (a cudaStream_t, NULL for the default
 * stream).  `err` is a device word: bit 0 is set when a kernel's bounded
 * wait for its tensor-core work runs out (its outputs are then invalid). */
/* y = act(conv3x3(x, w) + bias), act = GELU when gelu_on; pre (optional)
 * receives the pre-activation.  (cin, cout) in {(16,32), (32,32), (32,16),
 * (16,16)}; W up to about 1500. */
int pfag_conv3x3(const void *x, const void *w, const float *bias, void *y, void *pre, int B, int H, int W,
                 int cin, int cout, int gelu_on, unsigned *err, void *stream);
/* dw[co][t][ci] += sum over sites of dz[q][co] x[q + off_t][ci]; db[co] +=
 * sum of dz[q][co] (accumulates: zero dw, db first). */
int pfag_conv3x3_wgrad(const void *x, const void *dz, float *dw, float *db, int B, int H, int W, int cin,
                       int cout, unsigned *err, void *stream);
/* dz = dy * GELU'(pre) (gelu_on) or dy, zero on the halo. */
int pfag_conv_act_bwd(const void *dy, const void *pre, void *dz, int B, int H, int W, int c, int gelu_on,
                      void *stream);
/* wt[ci][t][co] = w[co][8-t][ci]: the input gradient is pfag_conv3x3 of dz with wt. */
int pfag_conv_flip(const void *w, void *wt, int cin, int cout, void *stream);
/* One Adam step (bias-corrected, step t >= 1) on FP32 parameters p with
 * gradient g and moments m, v; pb (optional) receives BF16 copies; mask
 * (optional) multiplies each update. */
int pfag_adam(float *p, const float *g, float *m, float *v, void *pb, const float *mask, int n, float lr,
              float b1, float b2, float eps, int t, void *stream);
/* Squared error of the first nout channels of out (C = 16 channels) against
 * target [B][H][W][nout] (FP32): *loss += the sum, dout = 2 scale (out -
 * target) on those channels and sites, zero elsewhere. */
int pfag_conv_mse(const void *out, const float *target, void *dout, float *loss, int B, int H, int W, int c,
                  int nout, float scale, void *stream);
/* The corrector's input on every cell's FFT box (M = 2 zone_size - 2) of a
 * context: x0 [Ntot][M+2][M+2][16] BF16 gets (s_phi phi, s_rho rho,
 * s_v vx, s_v vy, 0...) of the last step (the velocity needs
 * pfag_set_debug(ctx, 1) before that step; without it those channels are
 * zero); enqueued on the context's stream. */
int pfag_corrector_gather(pfag_ctx *ctx, void *x0, float s_phi, float s_rho, float s_v);
/* phi += s_phi out[..0], rho += s_rho out[..1] on every cell's FFT box of a
 * fused-path context, then the centroid sums the next step starts from are
 * taken again from the corrected phi; enqueued on the context's stream. */
int pfag_corrector_apply(pfag_ctx *ctx, const void *out, float s_phi, float s_rho);

#ifdef __cplusplus
}
#endif
#endif
