// plan_model.cpp -- weights of the plan-variant network used by
// sparsep_opts.autotune = 1.  No model is built in: the learned choice falls
// back to timing every variant.
#include <cstdint>

namespace sparsep {
const uint16_t *plan_model_weights() { return nullptr; }
const float *plan_model_mean() { return nullptr; }
const float *plan_model_std() { return nullptr; }
}  // namespace sparsep
