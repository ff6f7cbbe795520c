// FP64 instantiation of the kernels: the all-FP64 path, compiled with
// -fmad=false so its products and sums round like the reference's x86 code.
#include "ofg_launch.cuh"
namespace ofg {
int launch_task_f64(ofg_ctx *c, int task, cudaStream_t s) { return launch_task<double>(c, task, s); }
}  // namespace ofg
