// Tensor-core form of the Fourier sum (placeholder until the tcgen05 kernel
// lands): reports that no group can use it, so callers take the plain form.
#include "mv_internal.h"

namespace mv {

int tensor_sum_available(const SumRequest&) { return 0; }

int launch_tensor_sum(const SumRequest&, Workspace&, KernelTimer*) {
    return set_error(kUnsupported, "tensor-core form not available");
}

}  // namespace mv
