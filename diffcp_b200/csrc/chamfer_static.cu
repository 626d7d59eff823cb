// dcp_chamfer_forward_static: the one-sided Chamfer loss of one cloth for
// callers that cannot allocate device memory.
//
// Some callers have no way to call cudaMalloc: a plugin running inside a host
// application whose allocator already owns the GPU's memory and grants the
// plugin none, or a control loop with a hard latency budget in which an
// allocation (and the device synchronisation it can cause) is not allowed.
// The batched entry points need caller-provided scratch (dcp_plan sizes it);
// this entry point needs none: its only scratch, the per-target minima, lives
// in a file-scope device array of fixed size that every GPU loading this
// library holds until the process exits.
//
// The caller still provides every input and output buffer.  A __device__
// array has one address per CUDA context, so the address is looked up with
// cudaGetSymbolAddress the first time a call runs in a context (the primary
// context of a device, or a context the host application created with the
// driver API and made current) and cached under that context's unique id
// (cuCtxGetId), which the driver never hands out twice in a process.  A
// context destroyed and created again (cudaDeviceReset, for example) gets a
// new id, so its first call looks the address up afresh.  The first call in a
// context should therefore come before any stream capture in it.  All calls in
// a context share the one array: two calls that overlap on the GPU (for
// example on two streams) race on it.  Nothing in it needs to start at zero:
// each call writes the entries it later reads.
#include <cuda.h>  // driver API types only; the two functions used are fetched with cudaGetDriverEntryPoint
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/diffcp_b200.h"

namespace dcp {
void set_last_error(const std::string& msg);  // api.cu
}

static __device__ __align__(256) float g_chamfer_scratch[DCP_STATIC_MAX_TARGETS];

namespace {

// Scratch address per CUDA context, keyed by the context's unique id.  Ids
// are never reused, so an entry of a destroyed context is never matched again;
// the table keeps the most recent kMaxContexts entries.
constexpr int kMaxContexts = 64;
struct ScratchEntry {
  unsigned long long ctx_id;
  float* addr;
};
ScratchEntry g_scratch[kMaxContexts];
int g_scratch_n = 0, g_scratch_next = 0;
std::mutex g_scratch_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Per target: min over vertices of |x - t|^2 / 3 (parameter_fitting_functions.py:7-14),
// first vertex index on ties.  The difference x - t is formed rest-relative,
// (x0 - t) + u, with explicitly rounded float32 operations; the reference
// subtracts the target from a stored absolute position, so the two round
// differently.  NaN distances are skipped; a target with no distance below
// +inf (every vertex non-finite) gets a NaN minimum and argmin -1, so the
// loss becomes NaN.
__global__ void __launch_bounds__(128) k_static_min(const float* __restrict__ x0, const float* __restrict__ u, int nv,
                                                    const float* __restrict__ targets, int nq,
                                                    float* __restrict__ qmin, int* __restrict__ argmin) {
  __shared__ float sx[256], sy[256], sz[256], ux[256], uy[256], uz[256];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = q < nq;
  float tx = 0.f, ty = 0.f, tz = 0.f;
  if (valid) {
    tx = targets[q];
    ty = targets[nq + q];
    tz = targets[2 * (long long)nq + q];
  }
  float best = __int_as_float(0x7f800000);
  int bv = -1;
  for (int base = 0; base < nv; base += 256) {
    for (int j = threadIdx.x; j < 256; j += blockDim.x) {
      const int v = base + j;
      if (v < nv) {
        sx[j] = x0[v];
        sy[j] = x0[nv + v];
        sz[j] = x0[2 * (long long)nv + v];
        ux[j] = u ? u[v] : 0.f;
        uy[j] = u ? u[nv + v] : 0.f;
        uz[j] = u ? u[2 * (long long)nv + v] : 0.f;
      }
    }
    __syncthreads();
    const int cnt = min(256, nv - base);
    if (valid) {
      for (int j = 0; j < cnt; ++j) {
        const float dx = __fadd_rn(__fsub_rn(sx[j], tx), ux[j]);
        const float dy = __fadd_rn(__fsub_rn(sy[j], ty), uy[j]);
        const float dz = __fadd_rn(__fsub_rn(sz[j], tz), uz[j]);
        const float dd = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)), 3.f);
        if (dd < best) {
          best = dd;
          bv = base + j;
        }
      }
    }
    __syncthreads();
  }
  if (valid) {
    qmin[q] = bv >= 0 ? best : __int_as_float(0x7fc00000);
    argmin[q] = bv;
  }
}

// loss = sum_q qmin[q] / nq, accumulated in double by one CTA.
__global__ void k_static_sum(const float* __restrict__ qmin, int nq, float* __restrict__ loss) {
  __shared__ double red[32];
  double s = 0.0;
  for (int q = threadIdx.x; q < nq; q += blockDim.x) s += (double)(qmin[q] / (float)nq);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    loss[0] = (float)t;
  }
}

int fail_cuda(const char* what, cudaError_t e) {
  dcp::set_last_error(std::string("dcp_chamfer_forward_static: ") + what + ": " + cudaGetErrorString(e));
  return DCP_ERR_CUDA;
}

// Unique id of the calling thread's current context; 0 when none is current.
int current_context_id(unsigned long long* id) {
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) {
    dcp::set_last_error("dcp_chamfer_forward_static: cuCtxGetCurrent failed");
    return DCP_ERR_CUDA;
  }
  *id = 0;
  if (ctx && g_ctx_get_id(ctx, id) != CUDA_SUCCESS) {
    dcp::set_last_error("dcp_chamfer_forward_static: cuCtxGetId failed");
    return DCP_ERR_CUDA;
  }
  return DCP_OK;
}

int scratch_for_current_context(float** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_ctx_get_current || !g_ctx_get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
    if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
    if (e != cudaSuccess) return fail_cuda("cudaGetDriverEntryPoint", e);
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      dcp::set_last_error("dcp_chamfer_forward_static: the driver lacks cuCtxGetCurrent / cuCtxGetId");
      return DCP_ERR_CUDA;
    }
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  if (rc != DCP_OK) return rc;
  if (id) {
    for (int k = 0; k < g_scratch_n; ++k)
      if (g_scratch[k].ctx_id == id) {
        *out = g_scratch[k].addr;
        return DCP_OK;
      }
  }
  // first call in this context (or no context yet: the runtime then makes the
  // current device's primary context current while it looks the symbol up)
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_chamfer_scratch);
  if (e != cudaSuccess || !p) return fail_cuda("cudaGetSymbolAddress", e);
  if (!id) {
    rc = current_context_id(&id);
    if (rc != DCP_OK) return rc;
  }
  if (id) {
    g_scratch[g_scratch_next] = ScratchEntry{id, static_cast<float*>(p)};
    g_scratch_next = (g_scratch_next + 1) % kMaxContexts;
    if (g_scratch_n < kMaxContexts) ++g_scratch_n;
  }
  *out = static_cast<float*>(p);
  return DCP_OK;
}

}  // namespace

extern "C" int dcp_chamfer_forward_static(const float* x0, const float* u, int32_t n_vertex, const float* targets,
                                          int32_t n_target, int32_t* argmin, float* loss, void* stream) {
  if (!x0 || !targets || !argmin || !loss) {
    dcp::set_last_error("dcp_chamfer_forward_static: NULL argument");
    return DCP_ERR_INVALID;
  }
  if (n_vertex <= 0 || n_target <= 0) {
    dcp::set_last_error("dcp_chamfer_forward_static: n_vertex and n_target must be positive");
    return DCP_ERR_INVALID;
  }
  if (n_target > DCP_STATIC_MAX_TARGETS) {
    dcp::set_last_error("dcp_chamfer_forward_static: n_target exceeds DCP_STATIC_MAX_TARGETS (" +
                        std::to_string(DCP_STATIC_MAX_TARGETS) + "); use dcp_chamfer_forward");
    return DCP_ERR_INVALID;
  }
  float* scratch = nullptr;
  const int rc = scratch_for_current_context(&scratch);
  if (rc != DCP_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  k_static_min<<<(n_target + 127) / 128, 128, 0, s>>>(x0, u, n_vertex, targets, n_target, scratch, argmin);
  k_static_sum<<<1, 256, 0, s>>>(scratch, n_target, loss);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    dcp::set_last_error(std::string("dcp_chamfer_forward_static: ") + cudaGetErrorString(e));
    return DCP_ERR_CUDA;
  }
  return DCP_OK;
}
