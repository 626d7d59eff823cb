// C ABI of libdiffcp_b200 (declared in include/diffcp_b200.h): batch planning,
// launch-table construction, substep / Chamfer entry points and the native
// rollout driver with substep checkpointing and CUDA-graph replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/diffcp_b200.h"
#include "dcp_internal.cuh"
#include "dcp_launch.h"

using namespace dcp;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* where) {
  return fail(DCP_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

namespace dcp {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace dcp

namespace {

struct Layout {
  std::vector<InstDev> inst;
  std::vector<Chunk> chunks;
  int n_tri_chunks = 0, n_point_chunks = 0;
  long long nv = 0, nt = 0, no = 0, nc = 0, nq = 0, total_nodes = 0, traj = 0;
  long long grid_blocks = 0;  // blocks of each grid array (dense: all; paged: pool + spare)
  int pool_cap = 0;
  int max_nq = 0;
  // static buffer offsets
  size_t off_inst, off_triv, off_chunks, off_rank, static_bytes;
  // workspace offsets
  size_t off_pm, off_v, off_adj, off_flags, off_page, off_lblk, off_linst, off_cnt, off_force, off_contrib, off_barf,
      off_tmp, off_status, off_qmin, ws_bytes;
};

int validate(const DcpInstance* in, int n, const DcpOptions* opt) {
  if (!in || n <= 0) return fail(DCP_ERR_INVALID, "n_inst must be positive");
  if (!opt) return fail(DCP_ERR_INVALID, "options missing");
  if (opt->chunk < 32 || opt->chunk > 256 || opt->chunk % 32) return fail(DCP_ERR_INVALID, "chunk must be 32..256, multiple of 32");
  if (!(opt->dt > 0.f)) return fail(DCP_ERR_INVALID, "dt must be positive");
  if (opt->scatter_mode < 0 || opt->scatter_mode > 2) return fail(DCP_ERR_INVALID, "scatter_mode must be 0, 1 or 2");
  if (opt->adj_scatter_mode < 0 || opt->adj_scatter_mode > 2)
    return fail(DCP_ERR_INVALID, "adj_scatter_mode must be 0, 1 or 2");
  for (int k = 0; k < 3; ++k)
    if (opt->min_blocks[k] < 0 || opt->min_blocks[k] > 6) return fail(DCP_ERR_INVALID, "min_blocks must be 0..6");
  if (opt->pool_blocks < 0 || opt->pool_blocks > (1 << 24))
    return fail(DCP_ERR_INVALID, "pool_blocks must be 0..2^24");
  for (int i = 0; i < n; ++i) {
    const DcpInstance& I = in[i];
    char buf[160];
    snprintf(buf, sizeof buf, "instance %d: ", i);
    std::string p(buf);
    if (I.n_vertex < 0 || I.n_tri < 0 || I.n_operator < 0 || I.n_cube < 0 || I.n_target < 0)
      return fail(DCP_ERR_INVALID, p + "negative count");
    if (I.n_grid < 4 || I.n_grid > 2048) return fail(DCP_ERR_INVALID, p + "n_grid out of range");
    if (I.bound < 0) return fail(DCP_ERR_INVALID, p + "bound negative");
    if (I.gripper_mode == DCP_GRIP_OPERATOR) {
      if (I.n_grippers <= 0 || I.group_size <= 0 || I.n_operator != I.n_grippers * I.group_size)
        return fail(DCP_ERR_INVALID, p + "operator mode needs n_operator == n_grippers * group_size");
      if (!(I.keyframe_interval > 0.f) || I.n_actions < 1) return fail(DCP_ERR_INVALID, p + "bad keyframes");
    } else if (I.gripper_mode == DCP_GRIP_KINEMATIC) {
      if (I.n_grippers <= 0 || I.n_traj_steps <= 0) return fail(DCP_ERR_INVALID, p + "kinematic mode needs grippers and steps");
      if (I.n_operator != 0) return fail(DCP_ERR_INVALID, p + "kinematic mode has no operator particles");
    } else if (I.gripper_mode == DCP_GRIP_NONE) {
      if (I.n_operator != 0) return fail(DCP_ERR_INVALID, p + "operator particles need gripper_mode 1");
    } else {
      return fail(DCP_ERR_INVALID, p + "unknown gripper_mode");
    }
  }
  return DCP_OK;
}

void make_layout(const DcpInstance* in, int n, const DcpOptions* opt, Layout& L) {
  L.inst.resize(n);
  const int ch = opt->chunk;
  long long node = 0;
  for (int i = 0; i < n; ++i) {
    const DcpInstance& S = in[i];
    InstDev& I = L.inst[i];
    I.v_off = (int)L.nv; I.nv = S.n_vertex;
    I.t_off = (int)L.nt; I.nt = S.n_tri;
    I.o_off = (int)L.no; I.no = S.n_operator;
    I.c_off = (int)L.nc; I.nc = S.n_cube;
    I.q_off = (int)L.nq; I.nq = S.n_target;
    L.nv += S.n_vertex; L.nt += S.n_tri; L.no += S.n_operator; L.nc += S.n_cube; L.nq += S.n_target;
    L.max_nq = std::max(L.max_nq, S.n_target);
    I.G = S.n_grid;
    I.bound = S.bound;
    I.nb = (S.n_grid + 3) / 4;
    I.node_off = node;
    node += (long long)I.nb * I.nb * I.nb * 64;
    I.dx = 1.f / (float)S.n_grid;
    I.inv_dx = (float)S.n_grid;
    I.m_v = S.vertex_p_mass; I.m_q = S.quadrature_p_mass; I.vol_q = S.quadrature_p_vol;
    I.m_o = S.operator_p_mass; I.m_c = S.cube_p_mass; I.gravity_dv = S.gravity_dv;
    I.grip_mode = S.gripper_mode; I.n_grip = S.n_grippers; I.group_size = S.group_size;
    I.n_actions = S.n_actions; I.interval = S.keyframe_interval; I.frames_per_window = S.frames_per_window;
    I.grip_radius = S.gripper_radius; I.n_traj_steps = S.n_traj_steps;
    I.traj_off = L.traj;
    if (S.gripper_mode == DCP_GRIP_OPERATOR) L.traj += (long long)S.n_actions * S.n_grippers * 3;
    else if (S.gripper_mode == DCP_GRIP_KINEMATIC) L.traj += 2LL * S.n_traj_steps * S.n_grippers * 3;
  }
  L.total_nodes = node;
  // chunks: all triangle chunks first, then vertex / operator / cube chunks
  for (int i = 0; i < n; ++i)
    for (int s = 0; s < in[i].n_tri; s += ch)
      L.chunks.push_back(Chunk{CHUNK_TRI, i, L.inst[i].t_off + s, std::min(ch, in[i].n_tri - s)});
  L.n_tri_chunks = (int)L.chunks.size();
  for (int i = 0; i < n; ++i) {
    for (int s = 0; s < in[i].n_vertex; s += ch)
      L.chunks.push_back(Chunk{CHUNK_VERTEX, i, L.inst[i].v_off + s, std::min(ch, in[i].n_vertex - s)});
    for (int s = 0; s < in[i].n_operator; s += ch)
      L.chunks.push_back(Chunk{CHUNK_OPERATOR, i, L.inst[i].o_off + s, std::min(ch, in[i].n_operator - s)});
    for (int s = 0; s < in[i].n_cube; s += ch)
      L.chunks.push_back(Chunk{CHUNK_CUBE, i, L.inst[i].c_off + s, std::min(ch, in[i].n_cube - s)});
  }
  L.n_point_chunks = (int)L.chunks.size() - L.n_tri_chunks;
  size_t o = 0;
  L.off_inst = o; o = align256(o + sizeof(InstDev) * n);
  L.off_triv = o; o = align256(o + sizeof(int) * 3 * L.nt);
  L.off_chunks = o; o = align256(o + sizeof(Chunk) * L.chunks.size());
  L.off_rank = o; o = align256(o + sizeof(int) * L.nv);
  L.static_bytes = o;
  const long long blocks = L.total_nodes / 64;
  L.pool_cap = opt->pool_blocks;
  L.grid_blocks = L.pool_cap > 0 ? L.pool_cap + 1LL : blocks;
  const long long grid_nodes = 64 * L.grid_blocks;
  o = 0;
  L.off_pm = o; o = align256(o + 16 * grid_nodes);
  L.off_v = o; o = align256(o + 16 * grid_nodes);
  L.off_adj = o; o = align256(o + 16 * grid_nodes);
  // block flags (dense) or page table (paged), one word per block of the batch
  L.off_flags = o; o = align256(o + 4 * blocks);
  L.off_page = L.off_flags;
  L.off_lblk = o; o = align256(o + 4 * blocks);
  L.off_linst = o; o = align256(o + 4 * blocks);
  L.off_cnt = o; o = align256(o + 64);
  L.off_force = o; o = align256(o + 16 * L.nv);
  L.off_contrib = o; o = align256(o + 32 * L.nv);
  L.off_barf = o; o = align256(o + 4 * 3 * L.nv);
  L.off_tmp = o; o = align256(o + 4 * 3 * L.nt);
  L.off_status = o; o = align256(o + 4 * n);
  L.off_qmin = o; o = align256(o + 4 * L.nq);
  L.ws_bytes = o;
}

}  // namespace

struct GraphCache {
  bool valid = false;
  std::vector<long long> key;
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;  // kernels per replay
};

struct DcpBatch {
  BatchDev B;
  LaunchCfg L;
  Layout lay;
  DcpSizes sizes;
  DcpOptions opt;
  int n_inst;
  cudaStream_t cap_stream = nullptr;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  GraphCache gfwd, gbwd;
  Profiler prof;
};

static void fill_sizes(const Layout& L, int n, DcpSizes* s) {
  s->n_vertex = L.nv; s->n_tri = L.nt; s->n_operator = L.no; s->n_cube = L.nc; s->n_target = L.nq;
  s->state_floats = kPointState * (L.nv + L.no + L.nc) + kTriState * L.nt;
  s->rest_floats = kTriRest * L.nt + 3 * (L.nv + L.no + L.nc);
  s->traj_floats = L.traj;
  s->param_floats = (long long)PRM_STRIDE * n;
  s->static_bytes = (long long)L.static_bytes;
  s->workspace_bytes = (long long)L.ws_bytes;
  s->n_tri_chunks = L.n_tri_chunks;
  s->n_point_chunks = L.n_point_chunks;
  s->total_nodes = L.total_nodes;
  s->grid_blocks = L.grid_blocks;
}

extern "C" {

const char* dcp_last_error(void) { return g_err.c_str(); }

int32_t dcp_kernel_count(void) { return KID_COUNT; }
const char* dcp_kernel_name(int32_t id) { return (id >= 0 && id < KID_COUNT) ? kKernelNames[id] : ""; }

int dcp_plan(const DcpInstance* inst, int32_t n_inst, const DcpOptions* opt, DcpSizes* out) {
  int rc = validate(inst, n_inst, opt);
  if (rc) return rc;
  if (!out) return fail(DCP_ERR_INVALID, "sizes pointer is NULL");
  Layout L;
  make_layout(inst, n_inst, opt, L);
  fill_sizes(L, n_inst, out);
  return DCP_OK;
}

int dcp_create(const DcpInstance* inst, int32_t n_inst, const DcpOptions* opt, const int32_t* tri_vertices,
               const int32_t* vertex_rank, void* static_dev, void* workspace_dev, void* stream, DcpBatch** out) {
  int rc = validate(inst, n_inst, opt);
  if (rc) return rc;
  if (!out || !static_dev || !workspace_dev) return fail(DCP_ERR_INVALID, "NULL buffer");
  if (((uintptr_t)static_dev & 255) || ((uintptr_t)workspace_dev & 255))
    return fail(DCP_ERR_INVALID, "device buffers must be 256-byte aligned");
  DcpBatch* b = new DcpBatch();
  b->n_inst = n_inst;
  b->opt = *opt;
  Layout& L = b->lay;
  make_layout(inst, n_inst, opt, L);
  fill_sizes(L, n_inst, &b->sizes);
  // host tables
  std::vector<int> triv(3 * L.nt), rank(L.nv);
  for (int i = 0; i < n_inst; ++i) {
    const InstDev& I = L.inst[i];
    for (int t = 0; t < I.nt; ++t)
      for (int c = 0; c < 3; ++c) {
        const int v = tri_vertices[3LL * (I.t_off + t) + c];
        if (v < 0 || v >= I.nv) {
          delete b;
          return fail(DCP_ERR_INVALID, "triangle vertex index out of range");
        }
        triv[(long long)c * L.nt + I.t_off + t] = I.v_off + v;
      }
  }
  for (int i = 0; i < n_inst; ++i)
    for (int v = 0; v < L.inst[i].nv; ++v)
      rank[L.inst[i].v_off + v] = vertex_rank ? vertex_rank[L.inst[i].v_off + v] : v;
  std::vector<unsigned char> host(L.static_bytes, 0);
  memcpy(host.data() + L.off_inst, L.inst.data(), sizeof(InstDev) * n_inst);
  memcpy(host.data() + L.off_triv, triv.data(), sizeof(int) * triv.size());
  memcpy(host.data() + L.off_chunks, L.chunks.data(), sizeof(Chunk) * L.chunks.size());
  memcpy(host.data() + L.off_rank, rank.data(), sizeof(int) * rank.size());
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(static_dev, host.data(), L.static_bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(workspace_dev, 0, L.ws_bytes, s);
  if (e == cudaSuccess && L.pool_cap > 0)  // every page entry -1: no block has a slot
    e = cudaMemsetAsync((unsigned char*)workspace_dev + L.off_page, 0xff, 4 * (size_t)(L.total_nodes / 64), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e, "dcp_create upload");
  }
  unsigned char* sd = (unsigned char*)static_dev;
  unsigned char* wd = (unsigned char*)workspace_dev;
  BatchDev& B = b->B;
  B.inst = (const InstDev*)(sd + L.off_inst);
  B.n_inst = n_inst;
  B.nv = (int)L.nv; B.nt = (int)L.nt; B.no = (int)L.no; B.nc = (int)L.nc; B.nq = (int)L.nq;
  B.tri_v = (const int*)(sd + L.off_triv);
  B.chunks = (const Chunk*)(sd + L.off_chunks);
  B.n_tri_chunks = L.n_tri_chunks;
  B.n_point_chunks = L.n_point_chunks;
  B.vertex_rank = (const int*)(sd + L.off_rank);
  B.dt = opt->dt;
  B.svd_grad = opt->svd_grad;
  B.scatter_mode = opt->scatter_mode;
  B.adj_scatter_mode = opt->adj_scatter_mode;
  B.grid_pm = (float4*)(wd + L.off_pm);
  B.grid_v = (float4*)(wd + L.off_v);
  B.grid_adj = (float4*)(wd + L.off_adj);
  B.flags = (unsigned*)(wd + L.off_flags);
  B.list_blk = (int*)(wd + L.off_lblk);
  B.list_inst = (int*)(wd + L.off_linst);
  B.counters = (int*)(wd + L.off_cnt);
  B.fvert = (float4*)(wd + L.off_force);
  B.vadj = (float4*)(wd + L.off_contrib);
  B.barf = (float*)(wd + L.off_barf);
  B.tri_tmp = (float*)(wd + L.off_tmp);
  B.status = (int*)(wd + L.off_status);
  B.qmin = (float*)(wd + L.off_qmin);
  B.total_nodes = L.total_nodes;
  B.total_blocks = L.total_nodes / 64;
  B.page = L.pool_cap > 0 ? (int*)(wd + L.off_page) : nullptr;
  B.pool_cap = L.pool_cap;
  b->L.block = opt->chunk;
  // streaming multiprocessors of the current device: the grid-stride kernels
  // launch a multiple of this count
  int dev = 0, sms = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess || sms <= 0) {
    delete b;
    return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidValue, "dcp_create: multiprocessor count");
  }
  b->L.sm_count = sms;
  // k_grid / k_grid_adj are capped to 40 registers (6 resident 256-thread CTAs
  // per SM): one resident wave of CTAs striding over the active blocks
  b->L.grid_ctas = opt->grid_ctas > 0 ? opt->grid_ctas : sms * 6;
  const int default_minb[3] = {2, 2, 1};
  for (int k = 0; k < 3; ++k) b->L.min_blocks[k] = opt->min_blocks[k] > 0 ? opt->min_blocks[k] : default_minb[k];
  b->L.prof = &b->prof;
  e = configure_kernels(B, b->L);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e, "dcp_create configure");
  }
  *out = b;
  return DCP_OK;
}

int dcp_sizes(const DcpBatch* b, DcpSizes* out) {
  if (!b || !out) return fail(DCP_ERR_INVALID, "NULL argument");
  *out = b->sizes;
  return DCP_OK;
}

int dcp_destroy(DcpBatch* b) {
  if (!b) return DCP_OK;
  if (b->gfwd.exec) cudaGraphExecDestroy(b->gfwd.exec);
  if (b->gbwd.exec) cudaGraphExecDestroy(b->gbwd.exec);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->ev_a) cudaEventDestroy(b->ev_a);
  if (b->ev_b) cudaEventDestroy(b->ev_b);
  for (auto& r : b->prof.recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : b->prof.pool) cudaEventDestroy(e);
  delete b;
  return DCP_OK;
}

int dcp_init_state(DcpBatch* b, const float* x0v, const float* x0o, const float* x0c, float* state0, float* rest,
                   void* stream) {
  if (!b || !state0 || !rest || (!x0v && b->B.nv) || (!x0o && b->B.no) || (!x0c && b->B.nc))
    return fail(DCP_ERR_INVALID, "NULL argument");
  cudaError_t e = launch_init(b->B, b->L, x0v, x0o, x0c, state0, rest, (cudaStream_t)stream);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "dcp_init_state");
}

int dcp_substep_forward(DcpBatch* b, const float* params, const float* traj, const float* rest, int32_t step,
                        int32_t window, const float* sin, float* sout, void* stream) {
  if (!b || !params || !rest || !sin || !sout) return fail(DCP_ERR_INVALID, "NULL argument");
  if (sin == sout) return fail(DCP_ERR_INVALID, "state_in and state_out must differ");
  cudaError_t e = launch_forward(b->B, b->L, params, traj, rest, step, window, sin, sout, (cudaStream_t)stream);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "dcp_substep_forward");
}

int dcp_reset_quadrature(DcpBatch* b, float* rest, float* state, float* fdev, void* stream) {
  if (!b || !rest || !state || (!fdev && b->B.nt)) return fail(DCP_ERR_INVALID, "NULL argument");
  cudaError_t e = launch_reset(b->B, b->L, rest, state, fdev, (cudaStream_t)stream);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "dcp_reset_quadrature");
}

int dcp_replay(DcpBatch* b, const float* params, const float* traj, float* rest, float* state, float* work,
               float* fdev, int32_t first_step, int32_t n_blocks, int32_t block_steps, int32_t fdev_pending,
               void* stream) {
  if (!b || !params || !rest || !state || !work || (!fdev && b->B.nt)) return fail(DCP_ERR_INVALID, "NULL argument");
  if (state == work) return fail(DCP_ERR_INVALID, "state and work must differ");
  if (first_step < 0 || n_blocks < 0 || block_steps < 1) return fail(DCP_ERR_INVALID, "bad replay counts");
  cudaStream_t s = (cudaStream_t)stream;
  float* cur = state;
  float* nxt = work;
  int step = first_step;
  bool pending = fdev_pending != 0;
  for (int blk = 0; blk < n_blocks; ++blk) {
    for (int k = 0; k < block_steps; ++k, ++step) {
      cudaError_t e = launch_forward(b->B, b->L, params, traj, rest, step, 0, cur, nxt, s, nullptr,
                                     pending ? fdev : nullptr);
      if (e != cudaSuccess) return cuda_fail(e, "dcp_replay");
      pending = false;
      std::swap(cur, nxt);
    }
    cudaError_t e = launch_reset(b->B, b->L, rest, cur, fdev, s);
    if (e != cudaSuccess) return cuda_fail(e, "dcp_replay reset");
    pending = true;
  }
  if (cur != state) {
    cudaError_t e = cudaMemcpyAsync(state, cur, sizeof(float) * b->sizes.state_floats, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "dcp_replay copy");
  }
  return DCP_OK;
}

int dcp_substep_backward(DcpBatch* b, const float* params, const float* traj, const float* rest, int32_t step,
                         int32_t window, const float* sin, const float* aout, float* ain, double* gparams,
                         double* gtraj, void* stream) {
  if (!b || !params || !rest || !sin || !aout || !ain || !gparams) return fail(DCP_ERR_INVALID, "NULL argument");
  if (aout == ain) return fail(DCP_ERR_INVALID, "adj_out and adj_in must differ");
  if (b->sizes.traj_floats > 0 && (!traj || !gtraj)) return fail(DCP_ERR_INVALID, "trajectory buffers required");
  cudaError_t e = launch_backward(b->B, b->L, params, traj, rest, step, window, sin, aout, ain, gparams, gtraj,
                                  (cudaStream_t)stream);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "dcp_substep_backward");
}

int dcp_chamfer_forward(DcpBatch* b, const float* rest, const float* state, const float* targets, int32_t* argmin,
                        float* loss, void* stream) {
  if (!b || !rest || !state || !loss || (b->B.nq && (!targets || !argmin))) return fail(DCP_ERR_INVALID, "NULL argument");
  cudaError_t e =
      launch_chamfer_forward(b->B, b->L, b->lay.max_nq, rest, state, targets, argmin, loss, (cudaStream_t)stream);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "dcp_chamfer_forward");
}

int dcp_chamfer_backward(DcpBatch* b, const float* rest, const float* state, const float* targets,
                         const int32_t* argmin, const float* gloss, float* adj, void* stream) {
  if (!b || !rest || !state || !gloss || !adj || (b->B.nq && (!targets || !argmin)))
    return fail(DCP_ERR_INVALID, "NULL argument");
  cudaError_t e = launch_chamfer_backward(b->B, b->L, b->lay.max_nq, rest, state, targets, argmin, gloss, adj,
                                          (cudaStream_t)stream);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "dcp_chamfer_backward");
}

// ------------------------------------------------------------- rollouts
// Buffer: checkpoint slots for states 0, K, 2K, ... and the final state, then
// max(K-1, 2) segment slots (forward ping-pong / backward recompute).
static long long n_ckpt_slots(int n, int K) { return n / K + 1 + (n % K ? 1 : 0); }
static long long seg_slots(int K) { return std::max(K - 1, 2); }

int64_t dcp_rollout_floats(const DcpBatch* b, int32_t n_steps, int32_t K) {
  if (!b || n_steps < 0 || K < 1) return -1;
  return (n_ckpt_slots(n_steps, K) + seg_slots(K)) * b->sizes.state_floats;
}

static long long ckpt_slot(int f, int n, int K) {
  if (f % K == 0) return f / K;
  if (f == n) return n_ckpt_slots(n, K) - 1;
  return -1;
}

int64_t dcp_rollout_state_offset(const DcpBatch* b, int32_t n, int32_t K, int32_t f) {
  if (!b || K < 1 || f < 0 || f > n) return -1;
  const long long s = ckpt_slot(f, n, K);
  return s < 0 ? -1 : s * b->sizes.state_floats;
}

}  // extern "C"

template <class F>
static int run_maybe_graph(DcpBatch* b, GraphCache& gc, const std::vector<long long>& key, int use_graph, void* stream,
                           F&& body) {
  cudaStream_t us = (cudaStream_t)stream;
  if (!use_graph || b->prof.timing) {  // per-kernel timing needs eager launches
    cudaError_t e = body(us);
    return e == cudaSuccess ? DCP_OK : cuda_fail(e, "rollout");
  }
  cudaError_t e;
  if (!b->cap_stream) {
    e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_a, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_b, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "graph stream");
  }
  cudaStream_t cs = b->cap_stream;
  if (!gc.valid || gc.key != key) {
    if (gc.exec) {
      cudaGraphExecDestroy(gc.exec);
      gc.exec = nullptr;
    }
    gc.valid = false;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "begin capture");
    const long long before = b->prof.launches;
    cudaError_t eb = body(cs);
    gc.launches = b->prof.launches - before;
    b->prof.launches = before;
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    if (eb != cudaSuccess || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();  // a failed capture must not surface in a later, unrelated call
      return cuda_fail(eb != cudaSuccess ? eb : e, eb != cudaSuccess ? "captured launch" : "end capture");
    }
    e = cudaGraphInstantiate(&gc.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
    gc.key = key;
    gc.valid = true;
  }
  e = cudaEventRecord(b->ev_a, us);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, b->ev_a, 0);
  if (e == cudaSuccess) e = cudaGraphLaunch(gc.exec, cs);
  b->prof.launches += gc.launches;
  if (e == cudaSuccess) e = cudaEventRecord(b->ev_b, cs);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(us, b->ev_b, 0);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "graph launch");
}

// Grid tape layout: [256 B header: int top][meta int2 n][fv float 3*nv*n]
// [blk int cap][inst int cap][data float4 64*cap], each part 256-B aligned.
static size_t tape_fixed(const DcpBatch* b, int n) {
  return 256 + align256(8ull * n) + align256(12ull * n * b->lay.nv);
}
static size_t tape_size(const DcpBatch* b, int n, long long cap) {
  return tape_fixed(b, n) + 2 * align256(4ull * cap) + 1024ull * cap;
}

// Carves the tape; returns false when it is too small for its fixed part.
static bool tape_layout(const DcpBatch* b, int n, void* tape, long long bytes, TapeP& T) {
  const size_t fixed = tape_fixed(b, n);
  if (!tape || bytes < 0 || (size_t)bytes < fixed) return false;
  long long cap = ((long long)bytes - (long long)fixed - 512) / 1032;
  if (cap < 0) cap = 0;
  while (cap > 0 && tape_size(b, n, cap) > (size_t)bytes) --cap;
  char* p = (char*)tape;
  T.top = (int*)p;
  T.meta = (int2*)(p + 256);
  T.fv = (float*)(p + 256 + align256(8ull * n));
  T.blk = (int*)(p + fixed);
  T.inst = (int*)(p + fixed + align256(4ull * cap));
  T.data = (float4*)(p + fixed + 2 * align256(4ull * cap));
  T.cap = std::min<long long>(cap, 0x7fffffffLL);
  return true;
}

extern "C" {

int64_t dcp_tape_bytes(const DcpBatch* b, int32_t n, int64_t blocks) {
  if (!b || n < 0 || blocks < 0) return -1;
  return (int64_t)tape_size(b, n, blocks);
}

int dcp_rollout_forward(DcpBatch* b, const float* params, const float* traj, const float* rest, int32_t window,
                        int32_t n, int32_t K, float* buf, void* tape, int64_t tape_bytes, int32_t use_graph,
                        void* stream) {
  if (!b || !params || !rest || !buf || n < 0 || K < 1) return fail(DCP_ERR_INVALID, "bad rollout arguments");
  TapeP T;
  if (tape && !tape_layout(b, n, tape, tape_bytes, T)) return fail(DCP_ERR_INVALID, "tape smaller than its fixed part");
  const long long S = b->sizes.state_floats;
  const long long seg0 = n_ckpt_slots(n, K) * S;
  std::vector<long long> key = {(long long)params, (long long)traj, (long long)rest, (long long)buf, window, n, K,
                                (long long)tape, tape_bytes};
  return run_maybe_graph(b, b->gfwd, key, use_graph, stream, [&](cudaStream_t s) -> cudaError_t {
    if (tape && n > 0) {
      cudaError_t e = cudaMemsetAsync(T.top, 0, sizeof(int), s);
      if (e == cudaSuccess) e = cudaMemsetAsync(T.meta, 0xff, 8ull * n, s);
      if (e != cudaSuccess) return e;
    }
    const float* cur = buf;
    for (int f = 0; f < n; ++f) {
      const long long slot = ckpt_slot(f + 1, n, K);
      float* nxt = slot >= 0 ? buf + slot * S : buf + seg0 + ((f + 1) % 2) * S;
      cudaError_t e = launch_forward(b->B, b->L, params, traj, rest, f, window, cur, nxt, s, tape ? &T : nullptr);
      if (e != cudaSuccess) return e;
      cur = nxt;
    }
    return cudaSuccess;
  });
}

int dcp_rollout_backward(DcpBatch* b, const float* params, const float* traj, const float* rest, int32_t window,
                         int32_t n, int32_t Lstep, int32_t K, float* buf, float* adj, double* gparams,
                         double* gtraj, void* tape, int64_t tape_bytes, int32_t use_graph, void* stream) {
  if (!b || !params || !rest || !buf || !adj || !gparams || n < 0 || K < 1 || Lstep < 0 || Lstep > n)
    return fail(DCP_ERR_INVALID, "bad rollout arguments");
  if (b->sizes.traj_floats > 0 && (!traj || !gtraj)) return fail(DCP_ERR_INVALID, "trajectory buffers required");
  TapeP T;
  if (tape && !tape_layout(b, n, tape, tape_bytes, T)) return fail(DCP_ERR_INVALID, "tape smaller than its fixed part");
  const TapeP* tp = tape ? &T : nullptr;
  const long long S = b->sizes.state_floats;
  const long long seg0 = n_ckpt_slots(n, K) * S;
  std::vector<long long> key = {(long long)params, (long long)traj, (long long)rest, (long long)buf, (long long)adj,
                                (long long)gparams, (long long)gtraj, window, n, Lstep, K, (long long)tape,
                                tape_bytes};
  return run_maybe_graph(b, b->gbwd, key, use_graph, stream, [&](cudaStream_t s) -> cudaError_t {
    if (Lstep == 0) return cudaSuccess;
    for (int seg = (Lstep - 1) / K; seg >= 0; --seg) {
      const int f0 = seg * K;
      const int last = std::min(f0 + K - 1, Lstep - 1);
      auto state_at = [&](int f) -> float* { return f == f0 ? buf + ckpt_slot(f0, n, K) * S : buf + seg0 + (f - f0 - 1) * S; };
      for (int f = f0; f < last; ++f) {
        cudaError_t e = launch_forward(b->B, b->L, params, traj, rest, f, window, state_at(f), state_at(f + 1), s);
        if (e != cudaSuccess) return e;
      }
      for (int f = last; f >= f0; --f) {
        const int so = (Lstep - 1 - f) % 2;
        // state f + 1: inside the segment, or the next checkpoint / final state
        const long long nslot = f < last ? -2 : ckpt_slot(f + 1, n, K);
        const float* snext = f < last ? state_at(f + 1) : (nslot >= 0 ? buf + nslot * S : nullptr);
        // the triangles' per-vertex adjoint sums pass to the next adjoint
        // substep, which adds them to the vertex adjoints it reads; the last
        // substep (f = 0) adds them to the returned adjoint
        cudaError_t e = launch_backward(b->B, b->L, params, traj, rest, f, window, state_at(f), adj + so * S,
                                        adj + (1 - so) * S, gparams, gtraj, s, tp, snext, f != Lstep - 1, f == 0);
        if (e != cudaSuccess) return e;
      }
    }
    return cudaSuccess;
  });
}

int64_t dcp_launch_count(const DcpBatch* b) { return b ? b->prof.launches : -1; }

int dcp_profile(DcpBatch* b, int32_t enable) {
  if (!b) return fail(DCP_ERR_INVALID, "NULL batch");
  for (auto& r : b->prof.recs) {
    b->prof.pool.push_back(r.a);
    b->prof.pool.push_back(r.b);
  }
  b->prof.recs.clear();
  b->prof.timing = enable != 0;
  return DCP_OK;
}

int dcp_profile_read(DcpBatch* b, double* total_ms, int64_t* launches) {
  if (!b || !total_ms || !launches) return fail(DCP_ERR_INVALID, "NULL argument");
  for (int k = 0; k < KID_COUNT; ++k) {
    total_ms[k] = 0.0;
    launches[k] = 0;
  }
  for (auto& r : b->prof.recs) {
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e != cudaSuccess) return cuda_fail(e, "dcp_profile_read");
    float ms = 0.f;
    e = cudaEventElapsedTime(&ms, r.a, r.b);
    if (e != cudaSuccess) return cuda_fail(e, "dcp_profile_read");
    total_ms[r.id] += ms;
    launches[r.id] += 1;
  }
  return DCP_OK;
}

int64_t dcp_profile_launches(DcpBatch* b, int32_t id, double* ms, int64_t cap) {
  if (!b || id < 0 || id >= KID_COUNT || (cap > 0 && !ms)) {
    fail(DCP_ERR_INVALID, "dcp_profile_launches: bad argument");
    return -1;
  }
  int64_t n = 0;
  for (auto& r : b->prof.recs) {
    if (r.id != id) continue;
    if (n < cap) {
      cudaError_t e = cudaEventSynchronize(r.b);
      float t = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
      if (e != cudaSuccess) {
        cuda_fail(e, "dcp_profile_launches");
        return -1;
      }
      ms[n] = t;
    }
    ++n;
  }
  return n;
}

int dcp_read_status(DcpBatch* b, int32_t* host_status, int32_t clear, void* stream) {
  if (!b || !host_status) return fail(DCP_ERR_INVALID, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(host_status, b->B.status, sizeof(int) * b->n_inst, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && clear) e = cudaMemsetAsync(b->B.status, 0, sizeof(int) * b->n_inst, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? DCP_OK : cuda_fail(e, "dcp_read_status");
}

}  // extern "C"
