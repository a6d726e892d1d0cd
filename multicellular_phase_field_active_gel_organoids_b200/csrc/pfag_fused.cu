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
                    r->bhdi, r->bh};
    for (void *b : bufs) if (b) cudaFree(b);
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
