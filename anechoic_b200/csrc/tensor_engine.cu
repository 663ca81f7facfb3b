// Batched SCA engine for replicas sharing J. (Interface only in this revision: tensor_supported() is false, so the
// auto engine always selects the plain engine.)
#include "anc_tensor.cuh"

namespace anc {

bool tensor_supported(int, int, int) { return false; }
bool tensor_prefer(int, int, int, int) { return false; }

int tensor_build_instance(const int8_t*, int, TensorInstance*, std::string* why) {
    if (why) *why = "tensor engine not built";
    return -1;
}

int tensor_run(TensorInstance*, const TensorRun&, cudaStream_t, std::string* why) {
    if (why) *why = "tensor engine not built";
    return -1;
}

void tensor_free_instance(TensorInstance* ti) {
    if (ti && ti->d_J) cudaFree(ti->d_J);
    if (ti) ti->d_J = nullptr;
}

}  // namespace anc
