// k_trace_mixed.cu -- mixed-precision tracer (FP32 far from the critical curve, FP64 in the band).
#include <cuda_runtime.h>

#include "so_launch.h"

namespace so {

cudaError_t launch_trace_mixed(const TraceLaunch&, int, int, cudaStream_t) { return cudaErrorNotSupported; }

}  // namespace so
