// Tensor-core factored point predict (tcgen05).  Placeholder until the
// kernel lands: the form is rejected at construction.
#include "modeller.cuh"

namespace hdc {
int Modeller::tensor_setup() {
    set_error("predict form HDC_PREDICT_TENSOR is not available in this build");
    return HDC_ERR_UNSUPPORTED;
}
int Modeller::tensor_points(double, void*, bool, cudaStream_t) { return HDC_ERR_UNSUPPORTED; }
void Modeller::tensor_release() {}
}  // namespace hdc
