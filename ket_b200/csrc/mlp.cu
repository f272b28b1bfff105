// mlp.cu -- the learned fusion cost model.
#include <cuda_runtime.h>

#include "internal.h"

#define KB_API extern "C" __attribute__((visibility("default")))

namespace kb {
bool learned_model_attached() { return false; }
float learned_block_cost(int, const std::vector<const ketgpu_op*>&, const int*, int) { return 0.f; }
void block_features(int, const std::vector<const ketgpu_op*>&, const int*, int, float*) {}
}  // namespace kb

KB_API int ketgpu_mlp_create(uint64_t, ketgpu_mlp**) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_mlp_destroy(ketgpu_mlp*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_mlp_get_weights(const ketgpu_mlp*, float*, float*, float*, float*, float*, float*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_mlp_set_weights(ketgpu_mlp*, const float*, const float*, const float*, const float*, const float*, const float*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_mlp_forward(ketgpu_mlp*, const float*, uint64_t, float*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_mlp_gradients(ketgpu_mlp*, const float*, const float*, uint64_t, float*, float*, float*, float*, float*, float*, float*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_mlp_train(ketgpu_mlp*, const float*, const float*, uint64_t, uint64_t, uint64_t, float, float*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_planner_set_model(ketgpu_mlp*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_block_features(int32_t, const ketgpu_op*, uint64_t, const int32_t*, int32_t, float*) { return KETGPU_ERR_LOGIC; }
KB_API int ketgpu_time_block(ketgpu_state*, const int32_t*, int32_t, int32_t, int32_t, float*) { return KETGPU_ERR_LOGIC; }
