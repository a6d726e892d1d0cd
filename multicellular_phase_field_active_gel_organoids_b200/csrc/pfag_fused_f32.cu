// FP32 instantiation of the fused path (kernels in pfag_fused_impl.cuh).
#include "pfag_fused_impl.cuh"

int pfag_fused_alloc_f32(pfag_ctx *c) { return fused_alloc_t<float>(c); }
int pfag_fused_upload_f32(pfag_ctx *c) { return fused_upload_t<float>(c); }
int pfag_fused_step_f32(pfag_ctx *c, bool sync_host) { return fused_step_t<float>(c, sync_host); }
int pfag_fused_stats_f32(pfag_ctx *c) { return fused_stats_t<float>(c); }
int pfag_fused_recentre_f32(pfag_ctx *c) { return fused_recentre_t<float>(c); }
int pfag_fused_step_part_f32(pfag_ctx *c, int part, bool sync_host) { return fused_step_part_t<float>(c, part, sync_host); }
