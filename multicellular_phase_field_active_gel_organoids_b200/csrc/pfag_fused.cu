// Fused path: precision dispatch and resource release (kernels in pfag_fused_impl.cuh,
// instantiated in pfag_fused_f64.cu and pfag_fused_f32.cu).
#include "pfag_fused_impl.cuh"
#include <cstring>

int pfag_fused_alloc_f64(pfag_ctx *c);
int pfag_fused_alloc_f32(pfag_ctx *c);
int pfag_fused_upload_f64(pfag_ctx *c);
int pfag_fused_upload_f32(pfag_ctx *c);
int pfag_fused_step_f64(pfag_ctx *c, bool sync_host);
int pfag_fused_step_f32(pfag_ctx *c, bool sync_host);
int pfag_fused_stats_f64(pfag_ctx *c);
int pfag_fused_stats_f32(pfag_ctx *c);
int pfag_fused_recentre_f64(pfag_ctx *c);
int pfag_fused_recentre_f32(pfag_ctx *c);
int pfag_fused_step_part_f64(pfag_ctx *c, int part, bool sync_host);
int pfag_fused_step_part_f32(pfag_ctx *c, int part, bool sync_host);

int pfag_fused_stats(pfag_ctx *c) {
    return c->prec == 64 ? pfag_fused_stats_f64(c) : pfag_fused_stats_f32(c);
}

int pfag_fused_recentre(pfag_ctx *c) {
    return c->prec == 64 ? pfag_fused_recentre_f64(c) : pfag_fused_recentre_f32(c);
}

int pfag_fused_alloc(pfag_ctx *c) {
    c->fused = new FusedRes();
    std::memset(c->fused, 0, sizeof(FusedRes));
    return c->prec == 64 ? pfag_fused_alloc_f64(c) : pfag_fused_alloc_f32(c);
}

void pfag_fused_free(pfag_ctx *c) {
    FusedRes *r = F(c);
    if (!r) return;
    fused_drop_graph(r);
    if (r->side) { cudaStreamSynchronize(r->side); cudaStreamDestroy(r->side); }
    cudaEvent_t evs[] = {r->ev_psi, r->ev_area, r->ev_boxA, r->ev_lum};
    for (cudaEvent_t e : evs) if (e) cudaEventDestroy(e);
    void *bufs[] = {r->Y1, r->Y2, r->Rb, r->clsT, r->Jc, r->Jl, r->rect, r->part_r, r->part_e, r->part_l,
                    r->part_lt, r->part_a, r->cK, r->G, r->Gsp, r->btw, r->bcw, r->bwf,
                    r->bhdi, r->bh, r->nb_lo};
    for (void *b : bufs) if (b) cudaFree(b);
    delete r->lmaps;
    delete r;
    c->fused = nullptr;
}

int pfag_fused_upload_hook(pfag_ctx *c) {
    return c->prec == 64 ? pfag_fused_upload_f64(c) : pfag_fused_upload_f32(c);
}

int pfag_fused_step(pfag_ctx *c, int, bool sync_host) {
    return c->prec == 64 ? pfag_fused_step_f64(c, sync_host) : pfag_fused_step_f32(c, sync_host);
}

// ---- launch shapes (the autotuner's knobs) ---------------------------------
extern "C" int pfag_set_launch_shape(pfag_ctx *c, int coop_blocks, long update_warps) {
    if (!c || coop_blocks < 0 || update_warps < 0) { pfag_set_error("bad launch shape"); return PFAG_E_ARG; }
    if (c->path != PFAG_PATH_FUSED) { pfag_set_error("launch shapes exist on the fused path only"); return PFAG_E_UNSUPPORTED; }
    FusedRes *r = F(c);
    r->coop_r = coop_blocks > 0 ? std::min(coop_blocks, r->coop_default) : r->coop_default;
    r->upd_warps = update_warps > 0 ? update_warps : r->upd_default;
    fused_drop_graph(r);      // the captured step holds the old grid sizes
    r->graph_state = 0;
    return PFAG_OK;
}

extern "C" int pfag_set_lumen_tiles(pfag_ctx *c, int tma) {
    if (!c) { pfag_set_error("null ctx"); return PFAG_E_ARG; }
    if (c->path != PFAG_PATH_FUSED) { pfag_set_error("the lumen tiles are a fused-path knob"); return PFAG_E_UNSUPPORTED; }
    FusedRes *r = F(c);
    if (tma && !r->lmaps) {
        pfag_set_error("TMA-staged lumen tiles need FP32, N_s >= %d and N_s %% 4 == 0", LT_W);
        return PFAG_E_UNSUPPORTED;
    }
    if (r->lum_tma != (tma != 0)) {
        r->lum_tma = tma != 0;
        fused_drop_graph(r);      // the captured step holds the other kernel
        r->graph_state = 0;
    }
    return PFAG_OK;
}

// ---- batches of contexts stepped as one graph ---------------------------------
struct pfag_batch {
    std::vector<pfag_ctx *> m;
    std::vector<cudaGraph_t> built_from;   // member step graphs the parent graph was built from
    std::vector<cudaEvent_t> mev;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long launches = 0;                      // kernel launches of the last pfag_batch_step call
    long per_step = 0;                      // kernel launches in one replay of the parent graph
};

static void batch_drop_graph(pfag_batch *b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
    b->built_from.clear();
}

extern "C" int pfag_batch_create(pfag_ctx *const *ctxs, int n, pfag_batch **out) {
    if (!out || !ctxs || n < 1) { pfag_set_error("pfag_batch_create: bad arguments"); return PFAG_E_ARG; }
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!ctxs[i] || ctxs[i]->path != PFAG_PATH_FUSED) {
            pfag_set_error("pfag_batch_create: member %d is not a fused-path context", i);
            return PFAG_E_ARG;
        }
        for (int j = 0; j < i; j++)
            if (ctxs[j] == ctxs[i]) { pfag_set_error("pfag_batch_create: member %d repeats member %d", i, j); return PFAG_E_ARG; }
    }
    pfag_batch *b = new pfag_batch();
    b->m.assign(ctxs, ctxs + n);
    b->mev.assign(n, nullptr);
    int rc = PFAG_OK;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) rc = PFAG_E_CUDA;
    for (int i = 0; i < n && rc == PFAG_OK; i++)
        if (cudaEventCreateWithFlags(&b->mev[i], cudaEventDisableTiming) != cudaSuccess) rc = PFAG_E_CUDA;
    if (rc != PFAG_OK) {
        pfag_set_error("pfag_batch_create: %s", cudaGetErrorString(cudaGetLastError()));
        for (cudaEvent_t e : b->mev) if (e) cudaEventDestroy(e);
        if (b->ev) cudaEventDestroy(b->ev);
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return rc;
    }
    *out = b;
    return PFAG_OK;
}

extern "C" int pfag_batch_destroy(pfag_batch *b) {
    if (!b) return PFAG_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    for (cudaEvent_t e : b->mev) if (e) cudaEventDestroy(e);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return PFAG_OK;
}

static bool member_ready(pfag_ctx *c) {
    const FusedRes *r = F(c);
    return r->graph_ok && !r->ring_pending;
}

// the parent graph: one child node per member step graph, no edges between them
static int batch_build(pfag_batch *b) {
    batch_drop_graph(b);
    PFAG_CUDA_CHECK(cudaGraphCreate(&b->graph, 0));
    b->per_step = 0;
    for (pfag_ctx *c : b->m) {
        FusedRes *r = F(c);
        cudaGraphNode_t node;
        PFAG_CUDA_CHECK(cudaGraphAddChildGraphNode(&node, b->graph, nullptr, 0, r->graph));
        b->built_from.push_back(r->graph);
        b->per_step += r->graph_launches;
    }
    PFAG_CUDA_CHECK(cudaGraphInstantiate(&b->gexec, b->graph, 0));
    return PFAG_OK;
}

extern "C" int pfag_batch_step_async(pfag_batch *b, int it0, int nsteps) {
    if (!b || nsteps < 0) { pfag_set_error("pfag_batch_step: bad arguments"); return PFAG_E_ARG; }
    b->launches = 0;
    int k = 0;
    // members step on their own streams until each has captured its step graph
    // (the first step after an upload runs eagerly, the next one is captured)
    for (; k < nsteps; k++) {
        bool ready = true;
        for (pfag_ctx *c : b->m) ready = ready && member_ready(c);
        if (ready) break;
        for (pfag_ctx *c : b->m) {
            const long l0 = c->launches;
            PFAG_TRY(pfag_fused_step(c, it0 + k, false));
            b->launches += c->launches - l0;
        }
    }
    if (k == nsteps) return PFAG_OK;
    bool stale = !b->gexec || b->built_from.size() != b->m.size();
    for (size_t i = 0; !stale && i < b->m.size(); i++) stale = F(b->m[i])->graph != b->built_from[i];
    if (stale) PFAG_TRY(batch_build(b));
    // the batch stream after every member's pending work, every member stream after the batch
    for (size_t i = 0; i < b->m.size(); i++) {
        PFAG_CUDA_CHECK(cudaEventRecord(b->mev[i], b->m[i]->stream));
        PFAG_CUDA_CHECK(cudaStreamWaitEvent(b->stream, b->mev[i], 0));
    }
    for (; k < nsteps; k++) {
        PFAG_CUDA_CHECK(cudaGraphLaunch(b->gexec, b->stream));
        b->launches += b->per_step;
    }
    PFAG_CUDA_CHECK(cudaEventRecord(b->ev, b->stream));
    for (pfag_ctx *c : b->m) PFAG_CUDA_CHECK(cudaStreamWaitEvent(c->stream, b->ev, 0));
    return PFAG_OK;
}

extern "C" int pfag_batch_sync(pfag_batch *b) {
    if (!b) { pfag_set_error("null batch"); return PFAG_E_ARG; }
    PFAG_CUDA_CHECK(cudaStreamSynchronize(b->stream));
    for (pfag_ctx *c : b->m) {
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        PFAG_TRY(pfag_check_device_error(c));
        PFAG_TRY(c->prec == 64 ? pfag_fused_stats_f64(c) : pfag_fused_stats_f32(c));
        PFAG_TRY(pfag_fetch_observables(c));
    }
    return PFAG_OK;
}

extern "C" int pfag_batch_step(pfag_batch *b, int it0, int nsteps) {
    PFAG_TRY(pfag_batch_step_async(b, it0, nsteps));
    return pfag_batch_sync(b);
}

extern "C" void *pfag_batch_stream(pfag_batch *b) { return b ? (void *)b->stream : nullptr; }
extern "C" long pfag_batch_launch_count(pfag_batch *b) { return b ? b->launches : -1; }

// ---- cell sharding: one organoid's cells split over contexts ------------------
// (contiguous cell ranges; cells couple through psi and the index neighbours'
// phi, rho_functions.cpp:297-311, useful_functions.cpp:305-322)
extern "C" int pfag_shard_enable(pfag_ctx *c, void **lo, void **hi) {
    if (!c || !lo || !hi) { pfag_set_error("null argument"); return PFAG_E_ARG; }
    if (c->path != PFAG_PATH_FUSED) { pfag_set_error("cell sharding runs on the fused path"); return PFAG_E_UNSUPPORTED; }
    FusedRes *r = F(c);
    if (!r->nb_lo) {
        const size_t plane = (size_t)c->N * c->N * (c->prec == 64 ? 8 : 4);
        PFAG_CUDA_CHECK(cudaMalloc(&r->nb_lo, 2 * plane));
        r->nb_hi = (char *)r->nb_lo + plane;
        // until the host writes them: this context's own cyclic neighbours
        PFAG_CUDA_CHECK(cudaMemcpyAsync(r->nb_lo, (const char *)c->phi + (size_t)(c->Ntot - 1) * plane, plane,
                                        cudaMemcpyDeviceToDevice, c->stream));
        PFAG_CUDA_CHECK(cudaMemcpyAsync(r->nb_hi, c->phi, plane, cudaMemcpyDeviceToDevice, c->stream));
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        fused_drop_graph(r);          // captured steps read the previous neighbour planes
        r->graph_state = 0;
    }
    *lo = r->nb_lo;
    *hi = r->nb_hi;
    return PFAG_OK;
}

static int step_part(pfag_ctx *c, int part) {
    if (!c) { pfag_set_error("null ctx"); return PFAG_E_ARG; }
    if (c->path != PFAG_PATH_FUSED) { pfag_set_error("the split step runs on the fused path"); return PFAG_E_UNSUPPORTED; }
    if (part == 1) c->launches = 0;
    return c->prec == 64 ? pfag_fused_step_part_f64(c, part, false) : pfag_fused_step_part_f32(c, part, false);
}
extern "C" int pfag_step_head(pfag_ctx *c, int) { return step_part(c, 1); }
extern "C" int pfag_step_tail(pfag_ctx *c, int) { return step_part(c, 2); }

// out[i] = ((parts[0][i] + parts[1][i]) + parts[2][i]) + ...: the shards' psi
// partials in shard order (out may be one of the parts)
constexpr int SUM_MAX_PARTS = 64;
template <typename real> struct PartList { const real *p[SUM_MAX_PARTS]; };
template <typename real>
__global__ void k_sum_planes(real *out, PartList<real> L, int nparts, long count) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        real v = L.p[0][i];
        for (int k = 1; k < nparts; k++) v += L.p[k][i];
        out[i] = v;
    }
}

template <typename real>
static int sum_planes_t(void *out, const void *const *parts, int nparts, long count, cudaStream_t s) {
    PartList<real> L{};
    for (int k = 0; k < nparts; k++) L.p[k] = (const real *)parts[k];
    const long blocks = std::min<long>((count + 255) / 256, 148L * 8);
    k_sum_planes<real><<<(unsigned)std::max(1L, blocks), 256, 0, s>>>((real *)out, L, nparts, count);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

extern "C" int pfag_sum_planes(void *out, const void *const *parts, int nparts, long count, int precision,
                               void *stream) {
    if (!out || !parts || nparts < 1 || nparts > SUM_MAX_PARTS || count < 0 || (precision != 32 && precision != 64)) {
        pfag_set_error("pfag_sum_planes: bad arguments");
        return PFAG_E_ARG;
    }
    for (int k = 0; k < nparts; k++)
        if (!parts[k]) { pfag_set_error("pfag_sum_planes: null part"); return PFAG_E_ARG; }
    if (count == 0) return PFAG_OK;
    cudaStream_t s = (cudaStream_t)stream;
    return precision == 64 ? sum_planes_t<double>(out, parts, nparts, count, s)
                           : sum_planes_t<float>(out, parts, nparts, count, s);
}
