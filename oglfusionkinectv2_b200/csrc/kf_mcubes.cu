// kf_mcubes.cu — marching-cubes extraction (placeholder until the kernels land).
#include "kf_internal.cuh"

int kf_mc_run(kf_session* s, float, int, uint32_t*) {
  s->last_error = "marching cubes not built yet";
  return KF_ERR_STATE;
}

extern "C" {
int kf_mc_extract(kf_session* s, float iso, int method, uint32_t* n) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  return kf_mc_run(s, iso, method, n);
}
int kf_mc_copy_vertices(kf_session* s, float*, uint64_t) { return s ? KF_ERR_STATE : KF_ERR_INVALID_ARGUMENT; }
int kf_mc_copy_base_level(kf_session* s, uint32_t*, uint64_t) { return s ? KF_ERR_STATE : KF_ERR_INVALID_ARGUMENT; }
int kf_mc_export_stl(kf_session* s, const char*) { return s ? KF_ERR_STATE : KF_ERR_INVALID_ARGUMENT; }
int kf_mc_export_ply(kf_session* s, const char*) { return s ? KF_ERR_STATE : KF_ERR_INVALID_ARGUMENT; }
int kf_prefix_sum_u32(const uint32_t*, uint32_t*, uint64_t, uint32_t*, void*) { return KF_ERR_STATE; }
}
