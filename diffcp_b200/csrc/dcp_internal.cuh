// Internal device-side layout of a batch of cloth instances and the helpers
// shared by the substep kernels.
//
// HBM layout (all instances concatenated, structure of arrays):
//   state snapshot   [15][Nv] vertex  u(3) v(3) C(9)    u = x - x0 (displacement)
//                    [18][Nt] triangle C(9) delta3(3) xc(3) vc(3)
//                             delta3 = d3 - n0; xc, vc the centroid position
//                             (absolute) and velocity, kept so that the
//                             triangle kernels read them coalesced instead of
//                             gathering three vertices
//                    [15][No] operator u v C
//                    [15][Nc] cube     u v C
//   rest             [9][Nt] D0^-1, [3][Nt] n0 (rest normal), [6][Nt] rest
//                    edges e1 = x0b - x0a, e2 = x0c - x0a (D0's first two
//                    columns), [3][Nt] rest centroid, [3][Nv], [3][No], [3][Nc]
//                    rest positions x0
// Positions and the triangle's third column are stored relative to the rest
// configuration so that float32 keeps the small strains that drive the stress
// (absolute positions near 0.5 would leave ~1e-5 strain resolution).
//   grid             4x4x4-node blocks of 64 nodes, float4 (p.xyz, m) /
//                    (v_out.xyz, 0) / adjoint per node.  Dense: every block of
//                    every instance's grid, block-major per instance.  Paged:
//                    a pool of blocks shared by the batch; a page table maps a
//                    block (instance's first block + block-major index) to its
//                    pool slot for the current substep, and the slots are the
//                    positions in the substep's active-block list
//   topology         [3][Nt] global vertex ids
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cloth_math.cuh"

namespace dcp {

enum ChunkKind { CHUNK_VERTEX = 0, CHUNK_OPERATOR = 1, CHUNK_CUBE = 2, CHUNK_TRI = 3 };
enum GripMode { GRIP_NONE = 0, GRIP_OPERATOR = 1, GRIP_KINEMATIC = 2 };
enum Status { STATUS_OUT_OF_DOMAIN = 1, STATUS_NONFINITE = 2, STATUS_POOL_FULL = 4 };
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
  const Chunk* chunks;  // tri chunks then point chunks
  int n_tri_chunks, n_point_chunks;
  const int* vertex_rank;  // [nv] tie-break rank for the Chamfer argmin
  float dt;
  int svd_grad;
  int scatter_mode;      // P2G kernels: 0 warp-aggregated runs, 1 one atomic per lane and node, 2 lane pairs
  int adj_scatter_mode;  // k_g2p_adj, same values
  // workspace
  float4* grid_pm;
  float4* grid_v;
  float4* grid_adj;
  unsigned* flags;
  int* list_blk;
  int* list_inst;
  int* counters;  // [0] active blocks
  float4* fvert;  // [nv] summed in-plane corner forces of each vertex (xyz, w unused)
  float4* vadj;   // [2][nv] per-vertex sums of the triangles' position / velocity adjoints
  float* barf;    // [3][nv]
  float* tri_tmp; // [3][nt]
  int* status;    // [n_inst]
  float* qmin;    // [nq]
  long long total_nodes, total_blocks;
  // paged grids (pool_cap > 0): the grid arrays hold pool_cap + 1 blocks, the
  // last one a spare that absorbs the accesses of blocks without a slot
  int* page;      // [total_blocks] pool slot of each block, -1 when it has none
  int pool_cap;   // 0: dense grids
};

// Floats per particle of a state snapshot and of the rest buffer.
constexpr int kPointState = 15, kTriState = 18, kTriRest = 21;
// Rows of a triangle's state: C 0-8, delta3 9-11, centroid 12-14, its velocity 15-17.
enum { TRI_C = 0, TRI_D3 = 9, TRI_XC = 12, TRI_VC = 15 };

struct StateP {
  float* v;
  float* t;
  float* o;
  float* c;
};
__host__ __device__ inline StateP state_ptrs(float* base, int nv, int nt, int no) {
  StateP s;
  s.v = base;
  s.t = base + (long long)kPointState * nv;
  s.o = s.t + (long long)kTriState * nt;
  s.c = s.o + (long long)kPointState * no;
  return s;
}

// Grid tape of a rollout: per substep, the active blocks' (p, m) and every
// vertex's summed corner force, so that the adjoint substep can restore the
// grid instead of recomputing P2G.  Substeps that do not fit the block pool
// are marked (meta.x = -1) and recomputed.
struct TapeP {
  int* top;        // [1] next free block slot
  int2* meta;      // [n_steps] (first slot or -1, active block count)
  int* blk;        // [cap] global block ids
  int* inst;       // [cap] instances
  float4* data;    // [cap][64] (p, m)
  float* fv;       // [n_steps][3][nv] summed corner forces
  long long cap;   // block capacity
};

struct RestP {
  const float* Di;  // [9][nt]
  const float* n0;  // [3][nt]
  const float* e;   // [6][nt] rest edges e1 (rows 0-2), e2 (rows 3-5)
  const float* tc;  // [3][nt] rest centroid
  const float* xv;  // [3][nv]
  const float* xo;  // [3][no]
  const float* xc;  // [3][nc]
};
__host__ __device__ inline RestP rest_ptrs(const float* rest, int nv, int nt, int no) {
  RestP r;
  r.Di = rest;
  r.n0 = rest + 9LL * nt;
  r.e = rest + 12LL * nt;
  r.tc = rest + 18LL * nt;
  r.xv = rest + (long long)kTriRest * nt;
  r.xo = r.xv + 3LL * nv;
  r.xc = r.xo + 3LL * no;
  return r;
}

__device__ __forceinline__ long long node_index(const InstDev& I, int i, int j, int k) {
  const int blk = ((i >> 2) * I.nb + (j >> 2)) * I.nb + (k >> 2);
  const int within = ((i & 3) << 4) | ((j & 3) << 2) | (k & 3);
  return I.node_off + (long long)blk * 64 + within;
}

// Addresses of a stencil's 27 nodes: node (base + (oi, oj, ok)) sits at
// grid_base<PAGED>(grid, I)[at(oi, oj, ok)].
template <bool PAGED>
struct StenAddr;

// Dense grids: the block-major index of the node within its instance's grid,
// formed from per-axis parts with two adds per node (the same value as
// node_index minus I.node_off).
template <>
struct StenAddr<false> {
  int ax[3], ay[3], az[3];
  __device__ __forceinline__ StenAddr(const BatchDev&, const InstDev& I, const int base[3], bool, int) {
    const int sy = I.nb * 64, sx = I.nb * sy;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int i = base[0] + q, j = base[1] + q, k = base[2] + q;
      ax[q] = (i >> 2) * sx + ((i & 3) << 4);
      ay[q] = (j >> 2) * sy + ((j & 3) << 2);
      az[q] = ((k >> 2) << 6) + (k & 3);
    }
  }
  __device__ __forceinline__ int at(int oi, int oj, int ok) const { return ax[oi] + ay[oj] + az[ok]; }
};

// Paged grids: a stencil's 3 nodes per axis span at most 2 blocks per axis
// (base & 3 >= 2 crosses into the next one), so its 27 nodes lie in at most 8
// blocks, whose pool slots are looked up once per particle.  A block without
// a slot (the pool was full when k_alloc claimed it) maps to the spare block
// and flags the instance with STATUS_POOL_FULL.  Lanes without a particle
// (valid = false) load nothing.
template <>
struct StenAddr<true> {
  int s[8];  // slot * 64 of block (X, Y, Z) at 4 X + 2 Y + Z (X = 1: the next block along x)
  int r[3];  // base & 3 per axis
  __device__ __forceinline__ StenAddr(const BatchDev& B, const InstDev& I, const int base[3], bool valid, int inst) {
    bool cross[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      r[a] = base[a] & 3;
      cross[a] = r[a] >= 2;
    }
    const int nb = I.nb;
    const int g0 = (int)(I.node_off >> 6) + ((base[0] >> 2) * nb + (base[1] >> 2)) * nb + (base[2] >> 2);
    bool bad = false;
#pragma unroll
    for (int X = 0; X < 2; ++X)
#pragma unroll
      for (int Y = 0; Y < 2; ++Y)
#pragma unroll
        for (int Z = 0; Z < 2; ++Z) {
          int slot = B.pool_cap;
          if (valid && (X == 0 || cross[0]) && (Y == 0 || cross[1]) && (Z == 0 || cross[2])) {
            const int q = __ldg(B.page + g0 + (X * nb + Y) * nb + Z);
            bad = bad || q < 0;
            slot = q < 0 ? B.pool_cap : q;
          }
          s[4 * X + 2 * Y + Z] = slot << 6;
        }
    if (bad) atomicOr(B.status + inst, STATUS_POOL_FULL);
  }
  __device__ __forceinline__ int at(int oi, int oj, int ok) const {
    const bool X = oi != 0 && r[0] + oi >= 4, Y = oj != 0 && r[1] + oj >= 4, Z = ok != 0 && r[2] + ok >= 4;
    const int z0 = Z ? s[1] : s[0], z1 = Z ? s[3] : s[2], z2 = Z ? s[5] : s[4], z3 = Z ? s[7] : s[6];
    const int y0 = Y ? z1 : z0, y1 = Y ? z3 : z2;
    return (X ? y1 : y0) + (((r[0] + oi) & 3) << 4) + (((r[1] + oj) & 3) << 2) + ((r[2] + ok) & 3);
  }
};

// First node of an instance's grid in a grid array: the instance's offset for
// dense grids, the pool itself for paged ones.
template <bool PAGED, class T>
__device__ __forceinline__ T* grid_base(T* grid, const InstDev& I) {
  return PAGED ? grid : grid + I.node_off;
}

// Quadratic B-spline stencil of one particle (simulation.py:140-142): base node
// = trunc(x/dx - 0.5) per axis, fractional offset fx, 1-D weights and slopes.
// Out-of-domain bases are clamped so every access stays inside the instance's
// grid, and the instance is flagged.  The cell coordinate is formed with
// explicitly rounded operations (no multiply-add contraction), so every kernel
// that builds the stencil of the same particle gets the same base cell.
struct Sten {
  int base[3];
  float fx[3];
  float w[3][3];
  float dw[3][3];
};
__device__ __forceinline__ int base_cell(float p, const InstDev& I, bool& bad) {
  const float t = __fsub_rn(__fmul_rn(p, I.inv_dx), 0.5f);
  int b = (int)t;
  if (!(t >= 0.f) || b > I.G - 3) {
    bad = true;
    b = b < 0 ? 0 : (b > I.G - 3 ? I.G - 3 : b);
    if (!(t == t)) b = 0;
  }
  return b;
}
__device__ __forceinline__ void make_stencil(const float p[3], const InstDev& I, Sten& s, int* status, int inst) {
  bool bad = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int b = base_cell(p[a], I, bad);
    s.base[a] = b;
    s.fx[a] = __fsub_rn(__fmul_rn(p[a], I.inv_dx), (float)b);
    bspline(s.fx[a], s.w[a], s.dw[a]);
  }
  if (bad) atomicOr(status + inst, STATUS_OUT_OF_DOMAIN);
}

// acc + o c for a stencil offset o in {0, 1, 2}.  With o known at compile
// time (unrolled stencil loops) this is nothing, one add or one multiply-add:
// 0 * c cannot be folded away under IEEE rules, so o = 0 must not multiply.
__device__ __forceinline__ float add_off(float acc, int o, float c) {
  return o == 0 ? acc : (o == 1 ? acc + c : fmaf(2.f, c, acc));
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

// ------------------------------------------------------------ warp scatter
// Particle-centric scatter of 27-node stencils, one vector atomic
// (red.global.add.v4.f32, resolved in L2) per issuing lane and node.  The
// particles of a chunk are in Morton order of their base cells, so particles
// sharing a base cell sit in consecutive lanes, and lanes are merged first:
// mode 2 adds aligned lane pairs with the same base cell (one shuffle per
// component), mode 0 reduces each run of equal base cells (as many shuffle
// rounds as the longest run needs), mode 1 merges nothing.  Sums are exact
// float32 additions in a fixed order within the warp.  MARK (P2G) also
// registers the (at most 8) grid blocks an issuing lane's stencil touches as
// active on dense grids (k_alloc claims the blocks of paged ones before the
// substep's P2G).  Every lane of the warp must call it; lanes without a
// particle pass valid = false.  nz = false declares every contribution of the
// lane zero (an adjoint particle whose weights vanish): its atomics are skipped.
template <bool MARK, bool PAGED, class F>
__device__ __forceinline__ void warp_scatter(const BatchDev& B, const InstDev& I, int inst, const int base[3],
                                             bool valid, bool nz, F&& contrib) {
  const unsigned FULL = 0xffffffffu;
  constexpr bool MARKS = MARK && !PAGED;
  float4* grid = grid_base<PAGED>(MARK ? B.grid_pm : B.grid_adj, I);
  const int mode = MARK ? B.scatter_mode : B.adj_scatter_mode;
  if (mode == 2) {
    // pairs: lanes 2i and 2i+1 whose particles share a base cell (neighbours
    // in Morton order often do) add their values with one shuffle per
    // component and issue one atomic per node; other lanes issue their own.
    // A lane whose pair has only zero contributions (nz false on both) issues
    // none; the adjoint grid has no mass component, so w is not exchanged.
    const int lane = threadIdx.x & 31;
    const int key = valid ? ((base[0] << 22) | (base[1] << 11) | base[2]) : -1 - lane;
    const bool pair = __shfl_xor_sync(FULL, key, 1) == key;
    const bool mine = valid && nz;
    const bool theirs = __shfl_xor_sync(FULL, (int)mine, 1) != 0;
    const bool pnz = mine || (pair && theirs);
    const bool issue = valid && (!pair || (lane & 1) == 0);
    if (MARKS && issue) {
#pragma unroll
      for (int bi = 0; bi < 2; ++bi)
#pragma unroll
        for (int bj = 0; bj < 2; ++bj)
#pragma unroll
          for (int bk = 0; bk < 2; ++bk) {
            const int i = base[0] + 2 * bi, j = base[1] + 2 * bj, k = base[2] + 2 * bk;
            if ((bi && (i >> 2) == (base[0] >> 2)) || (bj && (j >> 2) == (base[1] >> 2)) ||
                (bk && (k >> 2) == (base[2] >> 2)))
              continue;
            mark_block(node_index(I, i, j, k), B.flags, B.list_blk, B.list_inst, B.counters, inst);
          }
    }
    if (!__any_sync(FULL, mine)) return;
    const StenAddr<PAGED> no(B, I, base, issue && pnz, inst);
#pragma unroll
    for (int oi = 0; oi < 3; ++oi)
#pragma unroll
      for (int oj = 0; oj < 3; ++oj)
#pragma unroll
        for (int ok = 0; ok < 3; ++ok) {
          float4 v = mine ? contrib(oi, oj, ok) : make_float4(0.f, 0.f, 0.f, 0.f);
          const float x = __shfl_xor_sync(FULL, v.x, 1), y = __shfl_xor_sync(FULL, v.y, 1);
          const float z = __shfl_xor_sync(FULL, v.z, 1);
          const float w = MARK ? __shfl_xor_sync(FULL, v.w, 1) : 0.f;
          if (pair) {
            v.x += x; v.y += y; v.z += z;
            if (MARK) v.w += w;
          }
          if (issue && pnz) atomicAdd(grid + no.at(oi, oj, ok), v);
        }
    return;
  }
  if (mode == 1) {  // per-lane atomics: no shuffles, more L2 traffic
    if (!valid) return;
    if (MARKS) {
#pragma unroll
      for (int bi = 0; bi < 2; ++bi)
#pragma unroll
        for (int bj = 0; bj < 2; ++bj)
#pragma unroll
          for (int bk = 0; bk < 2; ++bk) {
            const int i = base[0] + 2 * bi, j = base[1] + 2 * bj, k = base[2] + 2 * bk;
            if ((bi && (i >> 2) == (base[0] >> 2)) || (bj && (j >> 2) == (base[1] >> 2)) ||
                (bk && (k >> 2) == (base[2] >> 2)))
              continue;
            mark_block(node_index(I, i, j, k), B.flags, B.list_blk, B.list_inst, B.counters, inst);
          }
    }
    if (!nz) return;
    const StenAddr<PAGED> no(B, I, base, valid, inst);
#pragma unroll
    for (int oi = 0; oi < 3; ++oi)
#pragma unroll
      for (int oj = 0; oj < 3; ++oj)
#pragma unroll
        for (int ok = 0; ok < 3; ++ok) atomicAdd(grid + no.at(oi, oj, ok), contrib(oi, oj, ok));
    return;
  }
  const int lane = threadIdx.x & 31;
  const int key = valid ? ((base[0] << 22) | (base[1] << 11) | base[2]) : -1 - lane;
  const int prev = __shfl_up_sync(FULL, key, 1);
  const bool head = lane == 0 || key != prev;
  const unsigned hm = __ballot_sync(FULL, head);
  const int seg = __popc(hm & (0xffffffffu >> (31 - lane)));
  const unsigned after = lane == 31 ? 0u : (hm & (0xffffffffu << (lane + 1)));
  const int run = head ? ((after ? __ffs(after) - 1 : 32) - lane) : 0;
  const int maxrun = __reduce_max_sync(FULL, (unsigned)run);
  const int rounds = maxrun <= 1 ? 0 : 32 - __clz(maxrun - 1);
  bool same[5];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    const int d = 1 << r;
    const int sg = __shfl_down_sync(FULL, seg, d);
    same[r] = lane + d < 32 && sg == seg;
  }
  if (MARKS && head && valid) {
#pragma unroll
    for (int bi = 0; bi < 2; ++bi)
#pragma unroll
      for (int bj = 0; bj < 2; ++bj)
#pragma unroll
        for (int bk = 0; bk < 2; ++bk) {
          const int i = base[0] + 2 * bi, j = base[1] + 2 * bj, k = base[2] + 2 * bk;
          if ((bi && (i >> 2) == (base[0] >> 2)) || (bj && (j >> 2) == (base[1] >> 2)) ||
              (bk && (k >> 2) == (base[2] >> 2)))
            continue;
          mark_block(node_index(I, i, j, k), B.flags, B.list_blk, B.list_inst, B.counters, inst);
        }
  }
  const StenAddr<PAGED> no(B, I, base, head && valid, inst);
#pragma unroll
  for (int oi = 0; oi < 3; ++oi)
#pragma unroll
    for (int oj = 0; oj < 3; ++oj)
#pragma unroll
      for (int ok = 0; ok < 3; ++ok) {
        float4 v = valid ? contrib(oi, oj, ok) : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int r = 0; r < rounds; ++r) {
          const int d = 1 << r;
          const float x = __shfl_down_sync(FULL, v.x, d);
          const float y = __shfl_down_sync(FULL, v.y, d);
          const float z = __shfl_down_sync(FULL, v.z, d);
          const float w = __shfl_down_sync(FULL, v.w, d);
          if (same[r]) {
            v.x += x;
            v.y += y;
            v.z += z;
            v.w += w;
          }
        }
        if (head && valid && (v.x != 0.f || v.y != 0.f || v.z != 0.f || v.w != 0.f))
          atomicAdd(grid + no.at(oi, oj, ok), v);  // (runs check each node: nz unused)
      }
}

// Warp + CTA sum of up to 8 per-thread parameter-gradient contributions, in
// double from the thread on (contributions of both signs cancel over a
// rollout, so float partial sums would set the gradient's error), one atomic
// per value per CTA.
template <int N>
__device__ __forceinline__ void block_sum_atomic(double (&vals)[N], double* dst) {
  __shared__ double red[N][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int a = 0; a < N; ++a) {
    double v = vals[a];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[a][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x][w];
    if (s != 0.0) atomicAdd(dst + threadIdx.x, s);
  }
  __syncthreads();
}

__device__ __forceinline__ float ld(const float* p) { return __ldg(p); }

}  // namespace dcp
