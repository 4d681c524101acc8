// k_tensor.cu -- K2 placeholder (replaced by the tcgen05 implementation).
#include <cstdio>
#include "ltl_kernels.h"
namespace ltl {
struct TensorPlan { unsigned int* err; };
bool tensor_supported(int, int, char* why, size_t n) { snprintf(why, n, "not built yet"); return false; }
TensorPlan* tensor_plan_create(const Frame&, const Frame&, const Rule&, int, char* why, size_t n) {
    snprintf(why, n, "not built yet"); return nullptr; }
void tensor_plan_destroy(TensorPlan*) {}
int tensor_plan_depth(const TensorPlan*) { return 1; }
int tensor_plan_operand_bits(const TensorPlan*) { return 0; }
int tensor_plan_halo_needed(int r) { return halo_for(r, 1); }
cudaError_t launch_tensor_pass(TensorPlan*, bool, cudaStream_t) { return cudaErrorNotSupported; }
unsigned int* tensor_plan_error_flag(TensorPlan* p) { return p ? p->err : nullptr; }
}
