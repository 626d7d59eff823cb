// Host-side launchers of the kernels in kernels.cu (internal).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "dcp_internal.cuh"

namespace dcp {

enum KernelId {
  KID_TRI_FORWARD = 0, KID_POINT_P2G, KID_GRID, KID_G2P, KID_G2P_ADJ, KID_GRID_ADJ, KID_POINT_ADJ, KID_TRI_ADJ,
  KID_VERTEX_COLLECT, KID_CHAMFER_FWD, KID_CHAMFER_LOSS, KID_CHAMFER_BWD, KID_INIT, KID_TAPE, KID_RESET, KID_ALLOC,
  KID_RELEASE, KID_COUNT
};
extern const char* const kKernelNames[KID_COUNT];

// Launch accounting: counts every kernel issued and, when `timing` is on,
// brackets each launch with a pair of CUDA events on its stream.
struct Profiler {
  bool timing = false;
  long long launches = 0;
  struct Rec {
    int id;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t take() {
    if (pool.empty()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
};

struct ProfScope {
  Profiler* p;
  cudaStream_t s;
  int id;
  cudaEvent_t a = nullptr;
  ProfScope(Profiler* p_, int id_, cudaStream_t s_) : p(p_), s(s_), id(id_) {
    if (p) {
      ++p->launches;
      if (p->timing) {
        a = p->take();
        cudaEventRecord(a, s);
      }
    }
  }
  ~ProfScope() {
    if (p && p->timing) {
      cudaEvent_t b = p->take();
      cudaEventRecord(b, s);
      p->recs.push_back(Profiler::Rec{id, a, b});
    }
  }
};

struct LaunchCfg {
  int block;      // threads per CTA = particles per chunk
  int grid_ctas;  // CTAs of the persistent grid-update kernels
  int sm_count = 0;   // multiprocessors of the batch's device (dcp_create queries it)
  int min_blocks[3] = {2, 2, 1};  // register-cap levels of k_tri_forward, k_g2p_adj, k_tri_adj (1..6)
  Profiler* prof = nullptr;
};

cudaError_t configure_kernels(const BatchDev& B, const LaunchCfg& L);
cudaError_t launch_init(const BatchDev& B, const LaunchCfg& L, const float* x0v, const float* x0o, const float* x0c,
                        float* state, float* rest, cudaStream_t s);
// T (optional): the rollout's grid tape; forward substeps record into it,
// adjoint substeps restore from it and skip the P2G recompute.
// fdev (optional): F - I per triangle ([9][nt]) that replaces the one formed
// from the state in this substep's stress (the substep after a replay reset).
cudaError_t launch_forward(const BatchDev& B, const LaunchCfg& L, const float* params, const float* traj, const float* rest,
                           int step, int window, const float* sin, float* sout, cudaStream_t s,
                           const TapeP* T = nullptr, const float* fdev = nullptr);
cudaError_t launch_reset(const BatchDev& B, const LaunchCfg& L, float* rest, float* state, float* fdev,
                         cudaStream_t s);
// snext (optional): the state after this substep, as the forward produced it;
// the triangles' damped C is read from it instead of being gathered again.
// collect = false leaves the triangles' per-vertex adjoint sums of this
// substep out of ain; the next adjoint substep, given fold = true, adds them
// to the vertex adjoints it reads (its aout) and clears them.  A chain of
// substeps folds in every substep after the first and collects in the last.
cudaError_t launch_backward(const BatchDev& B, const LaunchCfg& L, const float* params, const float* traj,
                            const float* rest, int step, int window, const float* sin, const float* aout, float* ain,
                            double* gparams, double* gtraj, cudaStream_t s, const TapeP* T = nullptr,
                            const float* snext = nullptr, bool fold = false, bool collect = true);
cudaError_t launch_chamfer_forward(const BatchDev& B, const LaunchCfg& L, int max_nq, const float* rest,
                                   const float* state, const float* targets, int* qarg, float* loss, cudaStream_t s);
cudaError_t launch_chamfer_backward(const BatchDev& B, const LaunchCfg& L, int max_nq, const float* rest,
                                    const float* state, const float* targets, const int* qarg, const float* gloss,
                                    float* adj, cudaStream_t s);

}  // namespace dcp
