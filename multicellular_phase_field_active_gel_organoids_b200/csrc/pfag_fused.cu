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

int pfag_fused_alloc(pfag_ctx *c) {
    c->fused = new FusedRes();
    std::memset(c->fused, 0, sizeof(FusedRes));
    return c->prec == 64 ? pfag_fused_alloc_f64(c) : pfag_fused_alloc_f32(c);
}

void pfag_fused_free(pfag_ctx *c) {
    FusedRes *r = F(c);
    if (!r) return;
    fused_drop_graph(r);
    if (r->gplan_ok) cufftDestroy(r->gplan);
    if (r->gplan_xy_ok) cufftDestroy(r->gplan_xy);
    if (r->gplan_r2c_ok) cufftDestroy(r->gplan_r2c);
    if (r->gplan_c2r_ok) cufftDestroy(r->gplan_c2r);
    if (r->side) { cudaStreamSynchronize(r->side); cudaStreamDestroy(r->side); }
    cudaEvent_t evs[] = {r->ev_psi, r->ev_area, r->ev_boxA, r->ev_lum};
    for (cudaEvent_t e : evs) if (e) cudaEventDestroy(e);
    void *bufs[] = {r->Y1, r->Y2, r->Rb, r->clsT, r->Jc, r->Jl, r->rect, r->part_r, r->part_e, r->part_l,
                    r->part_lt, r->part_a, r->cK, r->G, r->Gsp};
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
