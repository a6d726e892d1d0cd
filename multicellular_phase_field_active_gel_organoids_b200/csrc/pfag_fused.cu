// Fused path (zone-restricted kernels); filled in below the plain path.
#include "pfag_internal.cuh"

int pfag_fused_alloc(pfag_ctx *) { pfag_set_error("fused path not built yet"); return PFAG_E_UNSUPPORTED; }
void pfag_fused_free(pfag_ctx *) {}
int pfag_fused_upload_hook(pfag_ctx *) { return PFAG_E_UNSUPPORTED; }
int pfag_fused_step(pfag_ctx *, int, bool) { return PFAG_E_UNSUPPORTED; }
