// Internal device-side layout of a batch of cloth instances and the helpers
// shared by the substep kernels.
//
// HBM layout (all instances concatenated, structure of arrays):
//   state snapshot   [15][Nv] vertex  u(3) v(3) C(9)    u = x - x0 (displacement)
//                    [12][Nt] triangle C(9) delta3(3)   delta3 = d3 - n0
//                    [15][No] operator u v C
//                    [15][Nc] cube     u v C
//   rest             [9][Nt] D0^-1, [3][Nt] n0 (rest normal), [3][Nv], [3][No],
//                    [3][Nc] rest positions x0
// Positions and the triangle's third column are stored relative to the rest
// configuration so that float32 keeps the small strains that drive the stress
// (absolute positions near 0.5 would leave ~1e-5 strain resolution).
//   grid             block-major per instance: 4x4x4-node blocks of 64 nodes,
//                    float4 (p.xyz, m) / (v_out.xyz, 0) / adjoint per node
//   topology         [3][Nt] global vertex ids, vertex->(corner, triangle) CSR
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cloth_math.cuh"

namespace dcp {

enum ChunkKind { CHUNK_VERTEX = 0, CHUNK_OPERATOR = 1, CHUNK_CUBE = 2, CHUNK_TRI = 3 };
enum GripMode { GRIP_NONE = 0, GRIP_OPERATOR = 1, GRIP_KINEMATIC = 2 };
enum Status { STATUS_OUT_OF_DOMAIN = 1, STATUS_NONFINITE = 2, STATUS_TILE_FALLBACK = 4 };
enum GridMode { GRID_FORWARD = 0, GRID_RECOMPUTE = 1 };

// Parameter table row (floats): E, nu, shearing k_s, contact k_c, ground friction, damping.
enum { PRM_E = 0, PRM_NU = 1, PRM_KS = 2, PRM_KC = 3, PRM_FRICTION = 4, PRM_DAMPING = 5, PRM_STRIDE = 8 };

struct InstDev {
  int v_off, nv, t_off, nt, o_off, no, c_off, nc, q_off, nq;
  int G, bound, nb;
  long long node_off;  // first node of this instance's grid (multiple of 64)
  float dx, inv_dx;
  float m_v, m_q, vol_q, m_o, m_c, gravity_dv;
  int grip_mode, n_grip, group_size, n_actions;
  float interval;
  int frames_per_window;
  float grip_radius;
  int n_traj_steps;
  long long traj_off;
};

struct Chunk {
  int kind, inst, start, count;
};

struct BatchDev {
  const InstDev* inst;
  int n_inst;
  int nv, nt, no, nc, nq;
  const int* tri_v;     // [3][nt]
  const int* inc_ptr;   // [nv + 1]
  const int* inc_e;     // [3 nt], e = corner * nt + t
  const Chunk* chunks;  // tri chunks then point chunks
  int n_tri_chunks, n_point_chunks;
  const int* vertex_rank;  // [nv] tie-break rank for the Chamfer argmin
  float dt;
  int svd_grad;
  int tile_nodes;  // shared-memory tile capacity (float4 nodes)
  // workspace
  float4* grid_pm;
  float4* grid_v;
  float4* grid_adj;
  unsigned* flags;
  int* list_blk;
  int* list_inst;
  int* counters;  // [0] active blocks
  float* force;   // [3][3 nt]
  float* contrib; // [6][3 nt]
  float* barf;    // [3][nv]
  float* tri_tmp; // [3][nt]
  int* status;    // [n_inst]
  float* qmin;    // [nq]
  long long total_nodes, total_blocks;
};

struct StateP {
  float* v;
  float* t;
  float* o;
  float* c;
};
__host__ __device__ inline StateP state_ptrs(float* base, int nv, int nt, int no) {
  StateP s;
  s.v = base;
  s.t = base + 15LL * nv;
  s.o = s.t + 12LL * nt;
  s.c = s.o + 15LL * no;
  return s;
}

struct RestP {
  const float* Di;  // [9][nt]
  const float* n0;  // [3][nt]
  const float* xv;  // [3][nv]
  const float* xo;  // [3][no]
  const float* xc;  // [3][nc]
};
__host__ __device__ inline RestP rest_ptrs(const float* rest, int nv, int nt, int no) {
  RestP r;
  r.Di = rest;
  r.n0 = rest + 9LL * nt;
  r.xv = rest + 12LL * nt;
  r.xo = r.xv + 3LL * nv;
  r.xc = r.xo + 3LL * no;
  return r;
}

__device__ __forceinline__ long long node_index(const InstDev& I, int i, int j, int k) {
  const int blk = ((i >> 2) * I.nb + (j >> 2)) * I.nb + (k >> 2);
  const int within = ((i & 3) << 4) | ((j & 3) << 2) | (k & 3);
  return I.node_off + (long long)blk * 64 + within;
}

// Quadratic B-spline stencil of one particle (simulation.py:140-142): base node
// = trunc(x/dx - 0.5) per axis, fractional offset fx, 1-D weights and slopes.
// Out-of-domain bases are clamped so every access stays inside the instance's
// grid, and the instance is flagged.
struct Sten {
  int base[3];
  float fx[3];
  float w[3][3];
  float dw[3][3];
};
__device__ __forceinline__ void make_stencil(const float p[3], const InstDev& I, Sten& s, int* status, int inst) {
  bool bad = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float sx = p[a] * I.inv_dx;
    const float t = sx - 0.5f;
    int b = (int)t;
    if (!(t >= 0.f) || b > I.G - 3) {
      bad = true;
      b = b < 0 ? 0 : (b > I.G - 3 ? I.G - 3 : b);
      if (!(t == t)) b = 0;
    }
    s.base[a] = b;
    s.fx[a] = sx - (float)b;
    bspline(s.fx[a], s.w[a], s.dw[a]);
  }
  if (bad) atomicOr(status + inst, STATUS_OUT_OF_DOMAIN);
}

__device__ __forceinline__ void mark_block(long long node, unsigned* flags, int* list_blk, int* list_inst, int* counter,
                                           int inst) {
  const long long b = node >> 6;
  if (*((volatile unsigned*)(flags + b)) == 0u) {
    if (atomicExch(flags + b, 1u) == 0u) {
      const int slot = atomicAdd(counter, 1);
      list_blk[slot] = (int)b;
      list_inst[slot] = inst;
    }
  }
}

// ------------------------------------------------------------------ tiles
// A CTA scatters its particles' 27-node stencils into a shared-memory tile
// that covers the bounding box of the CTA's stencils, then flushes the tile to
// the global grid with one vector atomic per touched node.  Particles of one
// CTA are a contiguous, spatially coherent range of one instance (mesh order),
// so the box is compact; when it exceeds the tile capacity the CTA falls back
// to direct global atomics.
struct TileHdr {
  int lo[3];
  int dim[3];
  int vol;
  int use;
  int any;
};

__device__ __forceinline__ void tile_setup(TileHdr& T, const int base[3], bool valid, int capacity) {
  __shared__ int red[6][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  int v[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    v[a] = valid ? base[a] : 0x3fffffff;
    v[3 + a] = valid ? base[a] : -0x3fffffff;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    v[a] = __reduce_min_sync(0xffffffffu, v[a]);
    v[3 + a] = __reduce_max_sync(0xffffffffu, v[3 + a]);
  }
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < 6; ++a) red[a][warp] = v[a];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = red[a][0];
      hi[a] = red[3 + a][0];
      for (int w = 1; w < nw; ++w) {
        lo[a] = min(lo[a], red[a][w]);
        hi[a] = max(hi[a], red[3 + a][w]);
      }
    }
    T.any = hi[0] >= lo[0];
    long long vol = 1;
    for (int a = 0; a < 3; ++a) {
      T.lo[a] = lo[a];
      T.dim[a] = T.any ? hi[a] - lo[a] + 3 : 1;
      vol *= T.dim[a];
    }
    T.use = T.any && vol <= capacity;
    T.vol = T.use ? (int)vol : 0;
  }
  __syncthreads();
}

__device__ __forceinline__ void tile_zero(float4* tile, const TileHdr& T) {
  for (int n = threadIdx.x; n < T.vol; n += blockDim.x) tile[n] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Add one node contribution (p.xyz, m) into the tile, or straight into the grid
// when the CTA has no tile.  MARK registers the node's block as active.
template <bool MARK>
__device__ __forceinline__ void emit(float4* tile, const TileHdr& T, const BatchDev& B, const InstDev& I, int inst, int i,
                                     int j, int k, float4 v) {
  if (T.use) {
    float* t = reinterpret_cast<float*>(tile + ((i - T.lo[0]) * T.dim[1] + (j - T.lo[1])) * T.dim[2] + (k - T.lo[2]));
    atomicAdd(t + 0, v.x);
    atomicAdd(t + 1, v.y);
    atomicAdd(t + 2, v.z);
    if (MARK) atomicAdd(t + 3, v.w);
  } else {
    const long long n = node_index(I, i, j, k);
    float4* dst = (MARK ? B.grid_pm : B.grid_adj) + n;
    atomicAdd(dst, v);
    if (MARK && v.w != 0.f) mark_block(n, B.flags, B.list_blk, B.list_inst, B.counters, inst);
  }
}

template <bool MARK>
__device__ __forceinline__ void tile_flush(const float4* tile, const TileHdr& T, const BatchDev& B, const InstDev& I,
                                           int inst) {
  float4* grid = MARK ? B.grid_pm : B.grid_adj;
  const int d12 = T.dim[1] * T.dim[2];
  for (int n = threadIdx.x; n < T.vol; n += blockDim.x) {
    const float4 v = tile[n];
    const bool nz = MARK ? (v.w != 0.f) : (v.x != 0.f || v.y != 0.f || v.z != 0.f);
    if (nz) {
      const int i = n / d12, r = n - i * d12, j = r / T.dim[2], k = r - j * T.dim[2];
      const long long g = node_index(I, i + T.lo[0], j + T.lo[1], k + T.lo[2]);
      atomicAdd(grid + g, v);
      if (MARK) mark_block(g, B.flags, B.list_blk, B.list_inst, B.counters, inst);
    }
  }
}

// Warp + CTA sum of up to 8 doubles, one atomic per value per CTA.
template <int N>
__device__ __forceinline__ void block_sum_atomic(float (&vals)[N], double* dst) {
  __shared__ float red[N][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int a = 0; a < N; ++a) {
    float v = vals[a];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[a][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += (double)red[threadIdx.x][w];
    if (s != 0.0) atomicAdd(dst + threadIdx.x, s);
  }
  __syncthreads();
}

__device__ __forceinline__ float ld(const float* p) { return __ldg(p); }

}  // namespace dcp
