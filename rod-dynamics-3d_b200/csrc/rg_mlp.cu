// rg_mlp.cu - learned PSOR warm start (placeholder until the kernels land).
#include "rg_internal.cuh"

namespace rg {
void mlp_warm_launch(rg_system*) {}
void mlp_record_launch(rg_system*) {}
}  // namespace rg

extern "C" {
size_t rg_mlp_param_count(void) { return 0; }
int rg_mlp_set_params(rg_system*, const float*, size_t) { return RG_ERR_STATE; }
int rg_mlp_get_params(const rg_system*, float*, size_t) { return RG_ERR_STATE; }
int rg_mlp_record(rg_system*, int, size_t) { return RG_ERR_STATE; }
int rg_mlp_records(const rg_system*, float*, float*, size_t, size_t*) { return RG_ERR_STATE; }
int rg_mlp_train(rg_system*, const float*, const float*, size_t, int, int, float, uint64_t, float*) {
  return RG_ERR_STATE;
}
int rg_mlp_infer(rg_system*, const float*, float*, size_t) { return RG_ERR_STATE; }
int rg_batch_create(const rg_config*, int, rg_batch**) { return RG_ERR_STATE; }
int rg_batch_destroy(rg_batch*) { return RG_ERR_STATE; }
int rg_batch_set_bodies(rg_batch*, int, const double*, const double*, const double*, const double*,
                        const double*) { return RG_ERR_STATE; }
int rg_batch_set_state(rg_batch*, int, const double*, const double*, const double*, const double*) {
  return RG_ERR_STATE;
}
int rg_batch_get_state(const rg_batch*, int, double*, double*, double*, double*) { return RG_ERR_STATE; }
int rg_batch_step(rg_batch*, int, rg_step_stats*) { return RG_ERR_STATE; }
int rg_batch_set_mlp(rg_batch*, const float*, size_t) { return RG_ERR_STATE; }
}
