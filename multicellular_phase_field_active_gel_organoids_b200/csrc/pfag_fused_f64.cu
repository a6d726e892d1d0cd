// FP64 instantiation of the fused path (kernels in pfag_fused_impl.cuh).
#include "pfag_fused_impl.cuh"

int pfag_fused_alloc_f64(pfag_ctx *c) { return fused_alloc_t<double>(c); }
int pfag_fused_upload_f64(pfag_ctx *c) { return fused_upload_t<double>(c); }
int pfag_fused_step_f64(pfag_ctx *c, bool sync_host) { return fused_step_t<double>(c, sync_host); }
int pfag_fused_stats_f64(pfag_ctx *c) { return fused_stats_t<double>(c); }
int pfag_fused_recentre_f64(pfag_ctx *c) { return fused_recentre_t<double>(c); }
int pfag_fused_step_part_f64(pfag_ctx *c, int part, bool sync_host) { return fused_step_part_t<double>(c, part, sync_host); }
