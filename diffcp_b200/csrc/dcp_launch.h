// Host-side launchers of the kernels in kernels.cu (internal).
#pragma once
#include <cuda_runtime.h>

#include "dcp_internal.cuh"

namespace dcp {

struct LaunchCfg {
  int block;      // threads per CTA = particles per chunk
  int grid_ctas;  // CTAs of the persistent grid-update kernels
};

cudaError_t configure_kernels(const BatchDev& B);
cudaError_t launch_init(const BatchDev& B, const float* x0v, const float* x0o, const float* x0c, float* state, float* rest,
                        cudaStream_t s);
cudaError_t launch_forward(const BatchDev& B, const LaunchCfg& L, const float* params, const float* traj, const float* rest,
                           int step, int window, const float* sin, float* sout, cudaStream_t s);
cudaError_t launch_backward(const BatchDev& B, const LaunchCfg& L, const float* params, const float* traj,
                            const float* rest, int step, int window, const float* sin, const float* aout, float* ain,
                            double* gparams, double* gtraj, cudaStream_t s);
cudaError_t launch_chamfer_forward(const BatchDev& B, int max_nq, const float* state, const float* targets, int* qarg,
                                   float* loss, cudaStream_t s);
cudaError_t launch_chamfer_backward(const BatchDev& B, int max_nq, const float* state, const float* targets,
                                    const int* qarg, const float* gloss, float* adj, cudaStream_t s);

}  // namespace dcp
