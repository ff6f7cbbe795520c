// Mixed-precision instantiation: FP32 face arithmetic (fluxes, gradients,
// limiters), FP64 residual accumulation, update and norms.
#include "ofg_launch.cuh"
namespace ofg {
int launch_task_f32(ofg_ctx *c, int task, cudaStream_t s) { return launch_task<float>(c, task, s); }
}  // namespace ofg
