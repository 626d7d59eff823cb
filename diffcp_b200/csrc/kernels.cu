// sm_100a kernels of the batched codimensional-cloth MPM substep, its adjoint
// and the Chamfer loss.  One CTA processes one chunk: a contiguous range of
// one particle species of one cloth instance, in Morton order of the
// particles' stencil base cells (the adjoint substep's P2G launches stride a
// smaller grid over the chunks).
//
// Forward substep (simulation.py:480-488, forward):
//   k_tri_forward    in-plane QR + rotation factor + stress of every triangle
//                    (simulation.py:24-28, 39-42, 214-240), its own-node APIC
//                    scatter and normal force (simulation.py:193-265), and the
//                    per-corner in-plane forces (simulation.py:266-271) summed
//                    per vertex instead of being scattered at the vertices'
//                    stencils (see k_point_p2g)
//   k_point_p2g      vertex / operator / cube APIC scatter (simulation.py:139-191);
//                    a vertex adds the sum of its triangles' corner forces, which
//                    equals the reference's per-triangle scatter with the
//                    vertex's weights (the weights depend only on the vertex)
//   k_grid           grid update and walls (simulation.py:274-302) on active
//                    blocks only
//   k_g2p            G2P for all species + triangle state update
//                    (simulation.py:304-430)
// Reverse substep: k_g2p_adj, k_grid_adj, k_point_adj, k_tri_adj; k_vertex_collect
// after a single substep or after a rollout's last one (inside a rollout the
// next substep's k_g2p_adj takes in the triangles' per-vertex adjoint sums).
// Grid tape (optional): k_tape_reserve and k_grid keep each forward
// substep's particle-to-grid result; the reverse substep's k_grid and
// k_grid_adj read it in place and its P2G launches return at once.
// Replay (forward only, simulation_without_grad.py): k_reset_tri /
// k_reset_vertex re-base the rest frames every few substeps.
#include <cuda_runtime.h>

#include <algorithm>

#include "dcp_internal.cuh"
#include "dcp_launch.h"

namespace dcp {

__device__ __forceinline__ float3 ld3(const float* base, long long stride, long long i) {
  return make_float3(__ldg(base + i), __ldg(base + stride + i), __ldg(base + 2 * stride + i));
}

// ============================================================== init
// initialize_ti_field (simulation.py:447-477): zero displacements, velocities
// and affine matrices; rest positions x0; triangle rest normal n0 = the
// normalised cross product of the eps-normalised edges (norm(1e-6)) and the
// rest-shape inverse D0^-1 of D0 = [e1, e2, n0].
// Rest frame of a triangle with corners pa, pb, pc: D0 = [pb - pa, pc - pa, n]
// with n the normalised cross product of the eps-normalised edges (norm(1e-6)),
// and D0^-1 by the adjugate (simulation.py:462-476, and the same frame in
// reset_quadrature_particles of simulation_without_grad.py:471-485).
__device__ __forceinline__ void rest_frame(const float pa[3], const float pb[3], const float pc[3], float inv[9],
                                           float nrm[3]) {
  const float d1x = pb[0] - pa[0], d1y = pb[1] - pa[1], d1z = pb[2] - pa[2];
  const float d2x = pc[0] - pa[0], d2y = pc[1] - pa[1], d2z = pc[2] - pa[2];
  const float l1 = sqrtf(d1x * d1x + d1y * d1y + d1z * d1z + 1e-6f);
  const float l2 = sqrtf(d2x * d2x + d2y * d2y + d2z * d2z + 1e-6f);
  const float n1x = d1x / l1, n1y = d1y / l1, n1z = d1z / l1;
  const float n2x = d2x / l2, n2y = d2y / l2, n2z = d2z / l2;
  float nx = n1y * n2z - n1z * n2y, ny = n1z * n2x - n1x * n2z, nz = n1x * n2y - n1y * n2x;
  const float l3 = sqrtf(nx * nx + ny * ny + nz * nz + 1e-6f);
  nx /= l3; ny /= l3; nz /= l3;
  const float m00 = d1x, m01 = d2x, m02 = nx, m10 = d1y, m11 = d2y, m12 = ny, m20 = d1z, m21 = d2z, m22 = nz;
  const float c00 = m11 * m22 - m12 * m21, c01 = m02 * m21 - m01 * m22, c02 = m01 * m12 - m02 * m11;
  const float c10 = m12 * m20 - m10 * m22, c11 = m00 * m22 - m02 * m20, c12 = m02 * m10 - m00 * m12;
  const float c20 = m10 * m21 - m11 * m20, c21 = m01 * m20 - m00 * m21, c22 = m00 * m11 - m01 * m10;
  const float det = m00 * c00 + m01 * c10 + m02 * c20;
  const float id = 1.f / det;
  inv[0] = c00 * id; inv[1] = c01 * id; inv[2] = c02 * id;
  inv[3] = c10 * id; inv[4] = c11 * id; inv[5] = c12 * id;
  inv[6] = c20 * id; inv[7] = c21 * id; inv[8] = c22 * id;
  nrm[0] = nx; nrm[1] = ny; nrm[2] = nz;
}

__global__ void k_init(BatchDev B, const float* __restrict__ x0v, const float* __restrict__ x0o,
                       const float* __restrict__ x0c, float* __restrict__ state, float* __restrict__ rest) {
  StateP S = state_ptrs(state, B.nv, B.nt, B.no);
  RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const long long total = (long long)B.nv + B.no + B.nc + B.nt;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    long long i = g;
    if (i < B.nv + B.no + B.nc) {
      float* dst;
      float* rdst;
      const float* src;
      long long n, p;
      if (i < B.nv) { dst = S.v; rdst = const_cast<float*>(R.xv); src = x0v; n = B.nv; p = i; }
      else if (i < B.nv + B.no) { dst = S.o; rdst = const_cast<float*>(R.xo); src = x0o; n = B.no; p = i - B.nv; }
      else { dst = S.c; rdst = const_cast<float*>(R.xc); src = x0c; n = B.nc; p = i - B.nv - B.no; }
      for (int c = 0; c < 3; ++c) rdst[c * n + p] = src[c * n + p];
      for (int c = 0; c < 15; ++c) dst[c * n + p] = 0.f;
      continue;
    }
    const long long t = i - (B.nv + B.no + B.nc);
    const int a = B.tri_v[t], b = B.tri_v[B.nt + t], c = B.tri_v[2 * (long long)B.nt + t];
    const long long nv = B.nv;
    const float pa[3] = {x0v[a], x0v[nv + a], x0v[2 * nv + a]};
    const float pb[3] = {x0v[b], x0v[nv + b], x0v[2 * nv + b]};
    const float pc[3] = {x0v[c], x0v[nv + c], x0v[2 * nv + c]};
    float inv[9], nrm[3];
    rest_frame(pa, pb, pc, inv, nrm);
    const long long nt = B.nt;
    float* Di = const_cast<float*>(R.Di);
    float* n0 = const_cast<float*>(R.n0);
    float* e = const_cast<float*>(R.e);
    float* tc = const_cast<float*>(R.tc);
    for (int q = 0; q < 9; ++q) Di[q * nt + t] = inv[q];
    for (int q = 0; q < TRI_XC; ++q) S.t[q * nt + t] = 0.f;
    const float third = 1.f / 3.f;
    for (int a = 0; a < 3; ++a) {
      n0[a * nt + t] = nrm[a];
      e[a * nt + t] = pb[a] - pa[a];
      e[(3 + a) * nt + t] = pc[a] - pa[a];
      const float c = third * ((pa[a] + pb[a]) + pc[a]);
      tc[a * nt + t] = c;                       // the centroid is the rest centroid at rest
      S.t[(TRI_XC + a) * nt + t] = c;
      S.t[(TRI_VC + a) * nt + t] = 0.f;
    }
  }
}

// Triangle geometry at one state: vertex ids and displacements of the three
// corners (scattered loads), centroid position and velocity (kept in the
// state: coalesced loads).
struct TriGeom {
  int vid[3];
  float U[3][3];  // [corner][axis]
  float xc[3], vc[3];
};
__device__ __forceinline__ void load_tri_ids(const BatchDev& B, long long t, int vid[3]) {
  const long long nt = B.nt;
#pragma unroll
  for (int c = 0; c < 3; ++c) vid[c] = __ldg(B.tri_v + c * nt + t);
}
__device__ __forceinline__ void load_centroid(const BatchDev& B, const StateP& S, long long t, bool need_v, TriGeom& g) {
  const long long nt = B.nt;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g.xc[a] = __ldg(S.t + (TRI_XC + a) * nt + t);
    g.vc[a] = need_v ? __ldg(S.t + (TRI_VC + a) * nt + t) : 0.f;
  }
}
__device__ __forceinline__ void load_corner_u(const BatchDev& B, const StateP& S, long long t, TriGeom& g) {
  const long long nv = B.nv;
  load_tri_ids(B, t, g.vid);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a) g.U[c][a] = __ldg(S.v + a * nv + g.vid[c]);
}
__device__ __forceinline__ void load_rest_edges(const BatchDev& B, const RestP& R, long long t, float e[6]) {
  const long long nt = B.nt;
#pragma unroll
  for (int q = 0; q < 6; ++q) e[q] = __ldg(R.e + q * nt + t);
}

// d = [x2 - x1, x3 - x1, d3] and F = d D0^-1 (simulation.py:395-407), returned
// as the deviation Fe = F - I = (d - D0) D0^-1 with d - D0 formed from
// displacements and delta3 = d3 - n0; e holds D0's first two columns (the
// rest edges).
__device__ __forceinline__ void tri_F(const TriGeom& g, const float e[6], const float dl3[3], const float n0[3],
                                      const float Di[9], M3<float>& d, M3<float>& Fe) {
  float dd[9];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    dd[3 * a + 0] = g.U[1][a] - g.U[0][a];
    dd[3 * a + 1] = g.U[2][a] - g.U[0][a];
    dd[3 * a + 2] = dl3[a];
    d.m[3 * a + 0] = e[a] + dd[3 * a + 0];
    d.m[3 * a + 1] = e[3 + a] + dd[3 * a + 1];
    d.m[3 * a + 2] = n0[a] + dl3[a];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      Fe.m[3 * r + c] = dd[3 * r] * Di[c] + dd[3 * r + 1] * Di[3 + c] + dd[3 * r + 2] * Di[6 + c];
}

__device__ __forceinline__ void load_tri_rest(const BatchDev& B, const RestP& R, const StateP& S, long long t,
                                              float dl3[3], float n0[3], float Di[9]) {
  const long long nt = B.nt;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    dl3[q] = __ldg(S.t + (TRI_D3 + q) * nt + t);
    n0[q] = __ldg(R.n0 + q * nt + t);
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) Di[q] = __ldg(R.Di + q * nt + t);
}

__device__ __forceinline__ void lame(float E, float nu, float& mu, float& la) {
  mu = E / (2.f * (1.f + nu));
  la = E * nu / ((1.f + nu) * (1.f - 2.f * nu));
}

// ============================================================== forward
// One triangle chunk of k_tri_forward.
template <bool PAGED>
__device__ __forceinline__ void tri_forward_chunk(const BatchDev& B, const float* __restrict__ params,
                                                  const float* __restrict__ rest, const float* __restrict__ sin,
                                                  const float* __restrict__ fdev, int c) {
  const Chunk ch = B.chunks[c];
  const InstDev& I = B.inst[ch.inst];
  const int tid = threadIdx.x;
  const bool valid = tid < ch.count;
  const long long t = ch.start + tid;
  const long long nt = B.nt;
  StateP S = state_ptrs(const_cast<float*>(sin), B.nv, B.nt, B.no);
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  Sten st;
  // scatter factors: ed = slope / dx * d3 per axis, so that the normal-force
  // weight grad W . d3 is formed from per-axis products; the APIC payload
  // m (v + C dpos), dpos = (o - fx) dx, is K + Ad o with Ad = m dx C and
  // K = m v - Ad fx (per-axis terms added for the node's offsets o)
  float K[3] = {0.f, 0.f, 0.f}, Ad[9], cP3[3] = {0.f, 0.f, 0.f}, ed[3][3];
  const float m = I.m_q;
  const float dx = I.dx, inv_dx = I.inv_dx;
  if (valid) {
    float A[9];
    // the triangle's own (coalesced) loads first, so that their latency
    // overlaps the dependent vertex gathers of load_tri
    float dl3[3], n0[3], Di[9], e[6];
#pragma unroll
    for (int q = 0; q < 9; ++q) A[q] = __ldg(S.t + q * nt + t) * m;
    load_tri_rest(B, R, S, t, dl3, n0, Di);
    load_rest_edges(B, R, t, e);
    TriGeom g;
    load_centroid(B, S, t, true, g);
    load_corner_u(B, S, t, g);
    make_stencil(g.xc, I, st, B.status, ch.inst);
    const float* prm = params + ch.inst * PRM_STRIDE;
    float mu, la;
    lame(prm[PRM_E], prm[PRM_NU], mu, la);
    const float ks = prm[PRM_KS], kc = prm[PRM_KC];
    M3<float> d, Fe;
    tri_F(g, e, dl3, n0, Di, d, Fe);
    if (fdev) {  // stress from the F kept across a rest-frame reset (replay)
#pragma unroll
      for (int q = 0; q < 9; ++q) Fe.m[q] = __ldg(fdev + q * nt + t);
    }
    Stress<float> sts;
    stress_forward<float>(Fe, mu, la, ks, kc, sts);
    const M3<float>& P = sts.P;
    const float vol = I.vol_q, dt = B.dt;
    // per-corner in-plane forces with r1 = (D0^-1[0,0], d[0,1], d[0,2]),
    // r2 = (D0^-1[1,0], d[1,1], d[1,2]) as in simulation.py:247-248
    const V3<float> r1 = v3(Di[0], d.m[1], d.m[2]);
    const V3<float> r2 = v3(Di[3], d.m[4], d.m[5]);
    const float k = vol * dt;
    const V3<float> f1 = k * matvec(P, r1 + r2);
    const V3<float> f2 = (-k) * matvec(P, r1);
    const V3<float> f3 = (-k) * matvec(P, r2);
    // summed per vertex (one vector reduction per corner); the vertex scatter
    // of k_point_p2g reads the sums
    atomicAdd(B.fvert + g.vid[0], make_float4(f1.x, f1.y, f1.z, 0.f));
    atomicAdd(B.fvert + g.vid[1], make_float4(f2.x, f2.y, f2.z, 0.f));
    atomicAdd(B.fvert + g.vid[2], make_float4(f3.x, f3.y, f3.z, 0.f));
    const float cn = -vol * dt;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      cP3[a] = cn * P.m[3 * a + 2];
      const float ea = inv_dx * d.m[3 * a + 2];
#pragma unroll
      for (int o = 0; o < 3; ++o) ed[a][o] = st.dw[a][o] * ea;
#pragma unroll
      for (int b = 0; b < 3; ++b) Ad[3 * a + b] = dx * A[3 * a + b];
      K[a] = m * g.vc[a] - (Ad[3 * a] * st.fx[0] + Ad[3 * a + 1] * st.fx[1] + Ad[3 * a + 2] * st.fx[2]);
    }
  }
  // own-node APIC momentum, mass and normal force (simulation.py:250-265)
  warp_scatter<true, PAGED>(B, I, ch.inst, st.base, valid, true, [=](int oi, int oj, int ok) -> float4 {
    const float w0 = st.w[0][oi], w1 = st.w[1][oj], w2 = st.w[2][ok];
    const float w01 = w0 * w1;
    const float W = w01 * w2;
    const float nrm = (ed[0][oi] * w1 + w0 * ed[1][oj]) * w2 + w01 * ed[2][ok];
    float4 val;
    val.x = W * add_off(add_off(add_off(K[0], oi, Ad[0]), oj, Ad[1]), ok, Ad[2]) + nrm * cP3[0];
    val.y = W * add_off(add_off(add_off(K[1], oi, Ad[3]), oj, Ad[4]), ok, Ad[5]) + nrm * cP3[1];
    val.z = W * add_off(add_off(add_off(K[2], oi, Ad[6]), oj, Ad[7]), ok, Ad[8]) + nrm * cP3[2];
    val.w = W * m;
    return val;
  });
}

// Triangle P2G.  A full launch has one CTA per chunk; the adjoint substep's
// launch, which returns at once when the tape holds the substep's grid, has a
// few CTAs per SM that stride over the chunks otherwise.
template <int REGS, bool PAGED>
__global__ void __maxnreg__(REGS) k_tri_forward(BatchDev B, const float* __restrict__ params,
                                                     const float* __restrict__ rest, const float* __restrict__ sin,
                                                     const int2* __restrict__ skip, const float* __restrict__ fdev) {
  if (skip && skip->x >= 0) return;  // the grid of this substep is restored from the tape
  for (int c = blockIdx.x; c < B.n_tri_chunks; c += gridDim.x) tri_forward_chunk<PAGED>(B, params, rest, sin, fdev, c);
}

__device__ __forceinline__ void point_arrays(const BatchDev& B, const StateP& S, int kind, float*& base, long long& n) {
  if (kind == CHUNK_VERTEX) { base = S.v; n = B.nv; }
  else if (kind == CHUNK_OPERATOR) { base = S.o; n = B.no; }
  else { base = S.c; n = B.nc; }
}
__device__ __forceinline__ const float* point_rest(const RestP& R, int kind) {
  return kind == CHUNK_VERTEX ? R.xv : (kind == CHUNK_OPERATOR ? R.xo : R.xc);
}

// Operator target velocity of simulation.py:160-165 (keyframe index in float32).
__device__ __forceinline__ bool operator_velocity(const BatchDev& B, const InstDev& I, const float* traj, int step,
                                                  int window, long long p, float v[3], long long& i0, long long& i1) {
  const float tt = (float)step * B.dt;
  const int frame = (int)__fdiv_rn(tt, I.interval) + I.frames_per_window * window;
  const int gid = (int)((p - I.o_off) / I.group_size);
  v[0] = v[1] = v[2] = 0.f;
  if (frame + 1 < I.n_actions && frame >= 0) {
    i0 = I.traj_off + ((long long)frame * I.n_grip + gid) * 3;
    i1 = I.traj_off + ((long long)(frame + 1) * I.n_grip + gid) * 3;
#pragma unroll
    for (int a = 0; a < 3; ++a) v[a] = __fdiv_rn(__ldg(traj + i1 + a) - __ldg(traj + i0 + a), I.interval);
    return true;
  }
  return false;
}

// One point chunk (vertex, operator or cube) of k_point_p2g.
template <bool PAGED>
__device__ __forceinline__ void point_p2g_chunk(const BatchDev& B, const float* __restrict__ traj, int step,
                                                int window, const float* __restrict__ rest,
                                                const float* __restrict__ sin, float* __restrict__ fv_out,
                                                int clear_forces, int c) {
  const Chunk ch = B.chunks[B.n_tri_chunks + c];
  const InstDev& I = B.inst[ch.inst];
  const int tid = threadIdx.x;
  const bool valid = tid < ch.count;
  const long long p = ch.start + tid;
  StateP S = state_ptrs(const_cast<float*>(sin), B.nv, B.nt, B.no);
  float* arr;
  long long n;
  point_arrays(B, S, ch.kind, arr, n);
  const float* x0 = point_rest(rest_ptrs(rest, B.nv, B.nt, B.no), ch.kind);
  const float m = ch.kind == CHUNK_VERTEX ? I.m_v : (ch.kind == CHUNK_OPERATOR ? I.m_o : I.m_c);
  Sten st;
  // payload m (v + C dpos) = K + Ad o per node (as in k_tri_forward)
  float base_v[3] = {0.f, 0.f, 0.f}, A[9], K[3] = {0.f, 0.f, 0.f};
  const float dx = I.dx;
  if (valid) {
    // every load of the particle first (one round of memory latency)
    float X[3], vl[3] = {0.f, 0.f, 0.f};
    float4 fs = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int a = 0; a < 3; ++a) X[a] = __ldg(x0 + a * n + p) + __ldg(arr + a * n + p);
#pragma unroll
    for (int q = 0; q < 9; ++q) A[q] = m * __ldg(arr + (6 + q) * n + p);
    if (ch.kind == CHUNK_VERTEX) {
      fs = B.fvert[p];
#pragma unroll
      for (int a = 0; a < 3; ++a) vl[a] = __ldg(arr + (3 + a) * n + p);
    }
    make_stencil(X, I, st, B.status, ch.inst);
    if (ch.kind == CHUNK_VERTEX) {
      const float f[3] = {fs.x, fs.y, fs.z};
      if (fv_out) {
#pragma unroll
        for (int a = 0; a < 3; ++a) fv_out[a * (long long)B.nv + p] = f[a];
      }
      // temp_v = v + (0, dt*scene_scaling*g, 0) (simulation.py:182)
      base_v[0] = m * vl[0] + f[0];
      base_v[1] = m * (vl[1] + I.gravity_dv) + f[1];
      base_v[2] = m * vl[2] + f[2];
    } else if (ch.kind == CHUNK_OPERATOR) {
      float v[3];
      long long i0, i1;
      operator_velocity(B, I, traj, step, window, p, v, i0, i1);
      base_v[0] = m * v[0]; base_v[1] = m * v[1]; base_v[2] = m * v[2];
    }  // cube: affine momentum only (simulation.py:150-152)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
      for (int b = 0; b < 3; ++b) A[3 * a + b] *= dx;
      K[a] = base_v[a] - (A[3 * a] * st.fx[0] + A[3 * a + 1] * st.fx[1] + A[3 * a + 2] * st.fx[2]);
    }
  }
  warp_scatter<true, PAGED>(B, I, ch.inst, st.base, valid, true, [=](int oi, int oj, int ok) -> float4 {
    const float W = (st.w[0][oi] * st.w[1][oj]) * st.w[2][ok];
    float4 val;
    val.x = W * add_off(add_off(add_off(K[0], oi, A[0]), oj, A[1]), ok, A[2]);
    val.y = W * add_off(add_off(add_off(K[1], oi, A[3]), oj, A[4]), ok, A[5]);
    val.z = W * add_off(add_off(add_off(K[2], oi, A[6]), oj, A[7]), ok, A[8]);
    val.w = W * m;
    return val;
  });
  // cleared after all loads of the kernel, ready for the next substep's sums
  if (clear_forces && valid && ch.kind == CHUNK_VERTEX) B.fvert[p] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Point P2G; launch shapes as for k_tri_forward.  Capped at 56 registers on
// dense grids (no spills; measured faster than the uncapped 62), 80 on paged
// ones (their stencil addressing needs the slots of up to 8 blocks).
template <bool PAGED>
__global__ void __maxnreg__(PAGED ? 80 : 56) k_point_p2g(BatchDev B, const float* __restrict__ traj, int step, int window,
                                                   const float* __restrict__ rest, const float* __restrict__ sin,
                                                   const int2* __restrict__ skip, float* __restrict__ fv_out,
                                                   int clear_forces) {
  if (skip && skip->x >= 0) return;  // the grid of this substep is restored from the tape
  for (int c = blockIdx.x; c < B.n_point_chunks; c += gridDim.x)
    point_p2g_chunk<PAGED>(B, traj, step, window, rest, sin, fv_out, clear_forces, c);
}

// ============================================================== paged grids
// Claims a pool slot for every block that a particle's stencil touches at
// the start of the substep: the blocks that P2G, G2P and their adjoints
// address, found from the same positions by the same base-cell arithmetic.
// The one thread whose compare-and-swap moves a block's page entry from -1 to
// -2 takes the next position of the active-block list and stores it as the
// block's slot; the kernels that read the page table run after this one, so
// no thread waits for another.  Positions past the pool's capacity get the
// spare block and flag the instance (STATUS_POOL_FULL); they stay in the list
// so that k_release clears them.  Lanes whose base cell equals the previous
// lane's (neighbours in Morton order) skip their claims.  Strides over the
// chunks like the P2G launches and returns at once when the tape holds the
// substep (its page entries are restored from the tape by k_grid).
__global__ void __launch_bounds__(256) k_alloc(BatchDev B, const float* __restrict__ rest,
                                               const float* __restrict__ sin, const int2* __restrict__ skip) {
  if (skip && skip->x >= 0) return;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int n_chunks = B.n_tri_chunks + B.n_point_chunks;
  StateP S = state_ptrs(const_cast<float*>(sin), B.nv, B.nt, B.no);
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  for (int c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const Chunk ch = B.chunks[c];
    const InstDev& I = B.inst[ch.inst];
    const bool valid = threadIdx.x < ch.count;
    int base[3] = {0, 0, 0};
    if (valid) {
      float X[3];
      if (ch.kind == CHUNK_TRI) {
        const long long t = ch.start + threadIdx.x, nt = B.nt;
#pragma unroll
        for (int a = 0; a < 3; ++a) X[a] = __ldg(S.t + (TRI_XC + a) * nt + t);
      } else {
        float* arr;
        long long n;
        point_arrays(B, S, ch.kind, arr, n);
        const float* x0 = point_rest(R, ch.kind);
        const long long p = ch.start + threadIdx.x;
#pragma unroll
        for (int a = 0; a < 3; ++a) X[a] = __ldg(x0 + a * n + p) + __ldg(arr + a * n + p);
      }
      bool bad = false;  // flagged by the P2G launches
#pragma unroll
      for (int a = 0; a < 3; ++a) base[a] = base_cell(X[a], I, bad);
    }
    const int key = valid ? ((base[0] << 22) | (base[1] << 11) | base[2]) : -1 - lane;
    const int prev = __shfl_up_sync(FULL, key, 1);
    if (!valid || (lane > 0 && prev == key)) continue;
    const int nb = I.nb;
    const int g0 = (int)(I.node_off >> 6) + ((base[0] >> 2) * nb + (base[1] >> 2)) * nb + (base[2] >> 2);
    const bool cx = (base[0] & 3) >= 2, cy = (base[1] & 3) >= 2, cz = (base[2] & 3) >= 2;
#pragma unroll
    for (int X = 0; X < 2; ++X)
#pragma unroll
      for (int Y = 0; Y < 2; ++Y)
#pragma unroll
        for (int Z = 0; Z < 2; ++Z) {
          if ((X && !cx) || (Y && !cy) || (Z && !cz)) continue;
          const int g = g0 + (X * nb + Y) * nb + Z;
          if (*((volatile int*)(B.page + g)) != -1 || atomicCAS(B.page + g, -1, -2) != -1) continue;
          const int item = atomicAdd(B.counters, 1);
          B.list_blk[item] = g;
          B.list_inst[item] = ch.inst;
          if (item >= B.pool_cap) atomicOr(B.status + ch.inst, STATUS_POOL_FULL);
          B.page[g] = item < B.pool_cap ? item : B.pool_cap;
        }
  }
}

// Returns the substep's blocks to the pool: every page entry that k_alloc or
// the tape restore (k_grid) set is cleared.  GRID_FORWARD: the blocks k_alloc
// listed; GRID_RECOMPUTE: the tape's list when it holds the substep.
__global__ void __launch_bounds__(256) k_release(BatchDev B, TapeP T, int step, int mode) {
  const int2 tm = (mode == GRID_RECOMPUTE && T.meta) ? T.meta[step] : make_int2(-1, 0);
  const bool from_tape = tm.x >= 0;
  const int count = from_tape ? min(tm.y, B.pool_cap) : B.counters[0];
  for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < count; item += gridDim.x * blockDim.x)
    B.page[from_tape ? __ldg(T.blk + (long long)tm.x + item) : B.list_blk[item]] = -1;
}

// Node coordinates of lane l (0..63) of an active block.
__device__ __forceinline__ void block_node(const InstDev& I, int blk, int l, int& i, int& j, int& k) {
  const int lb = blk - (int)(I.node_off >> 6);
  const int nb = I.nb;
  const int bi = lb / (nb * nb), bj = (lb / nb) % nb, bk = lb % nb;
  i = bi * 4 + (l >> 4);
  j = bj * 4 + ((l >> 2) & 3);
  k = bk * 4 + (l & 3);
}

// Kinematic sphere gripper (build extension): returns the index of the last
// gripper whose sphere contains node (i, j, k), or -1.
__device__ __forceinline__ int kinematic_hit(const InstDev& I, const float* traj, int step, int i, int j, int k) {
  if (I.grip_mode != GRIP_KINEMATIC || step >= I.n_traj_steps) return -1;
  const float px = i * I.dx, py = j * I.dx, pz = k * I.dx;
  const float r2 = I.grip_radius * I.grip_radius;
  const long long cbase = I.traj_off + (long long)I.n_traj_steps * I.n_grip * 3;
  int hit = -1;
  for (int q = 0; q < I.n_grip; ++q) {
    const long long o = cbase + ((long long)step * I.n_grip + q) * 3;
    const float dx = px - __ldg(traj + o), dy = py - __ldg(traj + o + 1), dz = pz - __ldg(traj + o + 2);
    if (dx * dx + dy * dy + dz * dz <= r2) hit = q;
  }
  return hit;
}

// GRID_FORWARD: records the (p, m) of this substep into the tape when the tape
// reserved it room.  GRID_RECOMPUTE (adjoint substep): when the tape holds this
// substep's P2G result, reads the active blocks and their (p, m) from the tape
// in place; otherwise from the P2G this substep recomputed.
__global__ void __launch_bounds__(256, 6) k_grid(BatchDev B, const float* __restrict__ params,
                                              const float* __restrict__ traj, int step, int mode, TapeP T) {
  const int2 tm = T.meta ? T.meta[step] : make_int2(-1, 0);
  const bool from_tape = mode == GRID_RECOMPUTE && tm.x >= 0;
  const bool paged = B.pool_cap > 0;
  int count = from_tape ? tm.y : B.counters[0];
  if (paged) count = min(count, B.pool_cap);
  const int record_at = mode == GRID_FORWARD ? tm.x : -1;
  const int per = blockDim.x >> 6, l = threadIdx.x & 63, stride = gridDim.x * per;
  // the block id, instance and (p, m) of a list item; the next item's are
  // loaded before the current one is processed (its loads do not depend on
  // the current item's stores: every item is a different block)
  auto fetch = [&](int it, int& blk, int& inst, float4& pm) {
    const long long slot = (long long)tm.x + it;
    blk = from_tape ? __ldg(T.blk + slot) : B.list_blk[it];
    inst = from_tape ? __ldg(T.inst + slot) : B.list_inst[it];
    pm = from_tape ? __ldg(T.data + slot * 64 + l) : B.grid_pm[(paged ? (long long)it : (long long)blk) * 64 + l];
  };
  int item = blockIdx.x * per + (threadIdx.x >> 6);
  int blk = 0, inst = 0;
  float4 pm = make_float4(0.f, 0.f, 0.f, 0.f);
  if (item < count) fetch(item, blk, inst, pm);
  for (; item < count; item += stride) {
    int blk_n = 0, inst_n = 0;
    float4 pm_n = make_float4(0.f, 0.f, 0.f, 0.f);
    if (item + stride < count) fetch(item + stride, blk_n, inst_n, pm_n);
    const InstDev& I = B.inst[inst];
    int i, j, k;
    block_node(I, blk, l, i, j, k);
    // paged: the pool slot is the list position (the tape's list restores
    // the page entries of its blocks for the adjoint kernels)
    const long long n = (paged ? (long long)item : (long long)blk) * 64 + l;
    if (paged && from_tape && l == 0) B.page[blk] = item;
    // the rounded reciprocal: measured faster here than the approximate one
    // that the build selects for divisions (16.5 against 20.2 ms per sweep step)
    const float inv_m = __frcp_rn(pm.w + 1e-9f);
    const float v[3] = {inv_m * pm.x, inv_m * pm.y, inv_m * pm.z};
    float out[3];
    grid_bc<float>(v, i, j, k, I.G, I.bound, __ldg(params + inst * PRM_STRIDE + PRM_FRICTION), out);
    const int hit = kinematic_hit(I, traj, step, i, j, k);
    if (hit >= 0) {
      const long long o = I.traj_off + ((long long)step * I.n_grip + hit) * 3;
      out[0] = __ldg(traj + o); out[1] = __ldg(traj + o + 1); out[2] = __ldg(traj + o + 2);
    }
    B.grid_v[n] = make_float4(out[0], out[1], out[2], 0.f);
    if (record_at >= 0) {
      const long long rs = (long long)record_at + item;
      T.data[rs * 64 + l] = pm;
      if (l == 0) {
        T.blk[rs] = blk;
        T.inst[rs] = inst;
      }
    }
    if (mode == GRID_FORWARD) {
      B.grid_pm[n] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (!paged && l == 0) B.flags[blk] = 0u;
    } else {
      B.grid_adj[n] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    blk = blk_n;
    inst = inst_n;
    pm = pm_n;
  }
}

template <class A>
__device__ __forceinline__ float3 gv_at(const float4* g, const A& o, int oi, int oj, int ok) {
  const float4 v = __ldg(g + o.at(oi, oj, ok));
  return make_float3(v.x, v.y, v.z);
}

// APIC gather of the grid velocities over a particle's stencil: v = sum W g
// and C = 4/dx sum W g (x) (o - fx), the latter from the moments
// mo[a][b] = sum W g_a o_b as C = 4/dx (mo - v fx^T) (o the node's offset
// 0, 1, 2 per axis).  v may be null.  gnb and nofs address the stencil's
// nodes (gv_at).
template <class A>
__device__ __forceinline__ void gather_affine(const float4* gnb, const A& nofs, const Sten& st, float inv_dx,
                                              float* v_out, float C[9]) {
  float v[3] = {0.f, 0.f, 0.f}, mo[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int oi = 0; oi < 3; ++oi)
#pragma unroll
    for (int oj = 0; oj < 3; ++oj) {
      const float w01 = st.w[0][oi] * st.w[1][oj];
#pragma unroll
      for (int ok = 0; ok < 3; ++ok) {
        const float W = w01 * st.w[2][ok];
        const float3 gn = gv_at(gnb, nofs, oi, oj, ok);
        const float ga[3] = {gn.x, gn.y, gn.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float Wg = W * ga[a];
          v[a] += Wg;
          mo[3 * a] = add_off(mo[3 * a], oi, Wg);
          mo[3 * a + 1] = add_off(mo[3 * a + 1], oj, Wg);
          mo[3 * a + 2] = add_off(mo[3 * a + 2], ok, Wg);
        }
      }
    }
  const float c4 = 4.f * inv_dx;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) C[3 * a + b] = c4 * (mo[3 * a + b] - v[a] * st.fx[b]);
    if (v_out) v_out[a] = v[a];
  }
}

// TRI: launched over the triangle chunks; otherwise over the point chunks
// (vertex, operator, cube), which follow the triangle chunks in the table.
template <bool TRI, bool PAGED>
__global__ void __launch_bounds__(256) k_g2p(BatchDev B, const float* __restrict__ params,
                                             const float* __restrict__ rest, const float* __restrict__ sin,
                                             float* __restrict__ sout) {
  const Chunk ch = B.chunks[(TRI ? 0 : B.n_tri_chunks) + blockIdx.x];
  if (threadIdx.x >= ch.count) return;
  const InstDev& I = B.inst[ch.inst];
  StateP Si = state_ptrs(const_cast<float*>(sin), B.nv, B.nt, B.no);
  StateP So = state_ptrs(sout, B.nv, B.nt, B.no);
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const float dt = B.dt, inv_dx = I.inv_dx;
  if (TRI) {
    const long long t = ch.start + threadIdx.x, nt = B.nt, nv = B.nv;
    TriGeom g;
    load_centroid(B, Si, t, false, g);
    Sten st;
    make_stencil(g.xc, I, st, B.status, ch.inst);
    float Ct[9];
    gather_affine(grid_base<PAGED>(B.grid_v, I), StenAddr<PAGED>(B, I, st.base, true, ch.inst), st, inv_dx,
                  nullptr, Ct);
    // C = skew + (1 - damping) sym (simulation.py:381-383)
    const float keep = 1.f - __ldg(params + ch.inst * PRM_STRIDE + PRM_DAMPING);
    float Cn[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float sk = 0.5f * (Ct[3 * a + b] - Ct[3 * b + a]);
        const float sy = 0.5f * (Ct[3 * a + b] + Ct[3 * b + a]);
        Cn[3 * a + b] = sk + keep * sy;
      }
    float dl3[3], d3[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      dl3[q] = __ldg(Si.t + (TRI_D3 + q) * nt + t);
      d3[q] = __ldg(R.n0 + q * nt + t) + dl3[q];
    }
    // d3 += (dt C + dt^2/2 C C) d3 (simulation.py:397-400), kept as delta3 = d3 - n0
    float Md[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float acc = 0.f;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float cc = 0.f;
#pragma unroll
        for (int q = 0; q < 3; ++q) cc += Cn[3 * a + q] * Cn[3 * q + b];
        acc += (dt * Cn[3 * a + b] + 0.5f * dt * dt * cc) * d3[b];
      }
      Md[a] = acc;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) So.t[(TRI_C + q) * nt + t] = Cn[q];
#pragma unroll
    for (int q = 0; q < 3; ++q) So.t[(TRI_D3 + q) * nt + t] = dl3[q] + Md[q];
    // centroid and its velocity in the next state (simulation.py:390-393),
    // from the vertices' new displacements and velocities, which the point
    // launch of this substep wrote before this launch
    int vid[3];
    load_tri_ids(B, t, vid);
    float su[3], sv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      su[a] = (So.v[a * nv + vid[0]] + So.v[a * nv + vid[1]]) + So.v[a * nv + vid[2]];
      sv[a] = (So.v[(3 + a) * nv + vid[0]] + So.v[(3 + a) * nv + vid[1]]) + So.v[(3 + a) * nv + vid[2]];
    }
    const float third = 1.f / 3.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      So.t[(TRI_XC + a) * nt + t] = __ldg(R.tc + a * nt + t) + third * su[a];
      So.t[(TRI_VC + a) * nt + t] = third * sv[a];
    }
    return;
  }
  float *ai, *ao;
  long long n;
  point_arrays(B, Si, ch.kind, ai, n);
  point_arrays(B, So, ch.kind, ao, n);
  const float* x0 = point_rest(R, ch.kind);
  const long long p = ch.start + threadIdx.x;
  float X[3], U[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    U[a] = __ldg(ai + a * n + p);
    X[a] = __ldg(x0 + a * n + p) + U[a];
  }
  Sten st;
  make_stencil(X, I, st, B.status, ch.inst);
  float v[3], C[9];
  gather_affine(grid_base<PAGED>(B.grid_v, I), StenAddr<PAGED>(B, I, st.base, true, ch.inst), st, inv_dx, v, C);
  bool finite = true;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ao[a * n + p] = U[a] + dt * v[a];
    ao[(3 + a) * n + p] = v[a];
    finite = finite && isfinite(v[a]);
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) ao[(6 + q) * n + p] = C[q];
  if (!finite) atomicOr(B.status + ch.inst, STATUS_NONFINITE);
}

// ============================================================== adjoint
// Reverse of k_g2p: scatter dL/dv_out into the adjoint grid and accumulate
// the position adjoint of the gather; triangle: reverse of the d3 update and of
// the skew/sym damping.
template <int REGS, bool PAGED>
__global__ void __maxnreg__(REGS) k_g2p_adj(BatchDev B, const float* __restrict__ params,
                                                 const float* __restrict__ rest, const float* __restrict__ sin,
                                                 const float* __restrict__ aout, float* __restrict__ ain,
                                                 double* __restrict__ gparams, const float* __restrict__ snext,
                                                 int fold) {
  const Chunk ch = B.chunks[blockIdx.x];
  const InstDev& I = B.inst[ch.inst];
  const int tid = threadIdx.x;
  const bool valid = tid < ch.count;
  StateP Si = state_ptrs(const_cast<float*>(sin), B.nv, B.nt, B.no);
  StateP Ao = state_ptrs(const_cast<float*>(aout), B.nv, B.nt, B.no);
  StateP Ai = state_ptrs(ain, B.nv, B.nt, B.no);
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const float dt = B.dt, inv_dx = I.inv_dx;
  const bool tri = ch.kind == CHUNK_TRI;
  const long long idx = ch.start + tid;
  Sten st;
  double gdamp[1] = {0.0};
  float bV[3] = {0.f, 0.f, 0.f}, Kg[3] = {0.f, 0.f, 0.f};  // dL/dv', node weight base
  float cbC[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // 4/dx dL/dC of the gather
  if (valid) {
    float X[3];
    float *ai = nullptr, *ao = nullptr, *aa = nullptr;
    long long n = 0;
    // triangle: its own loads first, overlapping the vertex gathers
    float Cn[9], d3[3], bd3o[3], bCo[9];
    if (tri) {
      const long long nt = B.nt;
      if (snext) {
        const float* cn = snext + (long long)kPointState * B.nv;
#pragma unroll
        for (int q = 0; q < 9; ++q) Cn[q] = __ldg(cn + q * nt + idx);
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        d3[q] = __ldg(R.n0 + q * nt + idx) + __ldg(Si.t + (TRI_D3 + q) * nt + idx);
        bd3o[q] = __ldg(Ao.t + (TRI_D3 + q) * nt + idx);
      }
#pragma unroll
      for (int q = 0; q < 9; ++q) bCo[q] = __ldg(Ao.t + q * nt + idx);
#pragma unroll
      for (int a = 0; a < 3; ++a) X[a] = __ldg(Si.t + (TRI_XC + a) * nt + idx);
    } else {
      point_arrays(B, Si, ch.kind, ai, n);
      point_arrays(B, Ao, ch.kind, ao, n);
      point_arrays(B, Ai, ch.kind, aa, n);
      const float* x0 = point_rest(R, ch.kind);
#pragma unroll
      for (int a = 0; a < 3; ++a) X[a] = __ldg(x0 + a * n + idx) + __ldg(ai + a * n + idx);
    }
    make_stencil(X, I, st, B.status, ch.inst);
    float bC[9];  // adjoint of the gathered C (4 inv_dx sum W g (x) dpos)
    float bx[3] = {0.f, 0.f, 0.f};
    if (tri) {
      const long long nt = B.nt;
      const float damping = __ldg(params + ch.inst * PRM_STRIDE + PRM_DAMPING);
      const float keep = 1.f - damping;
      float sym[9];
      if (snext && keep > 0.f) {
        // the damped C of the forward is the next state's C (loaded above); its
        // symmetric part is keep times that of the gathered C (uniform per chunk)
        const float ik = 1.f / keep;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) sym[3 * a + b] = 0.5f * (Cn[3 * a + b] + Cn[3 * b + a]) * ik;
      } else {
        float Ct[9];
        gather_affine(grid_base<PAGED>(B.grid_v, I), StenAddr<PAGED>(B, I, st.base, true, ch.inst), st, inv_dx,
                      nullptr, Ct);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            sym[3 * a + b] = 0.5f * (Ct[3 * a + b] + Ct[3 * b + a]);
            Cn[3 * a + b] = 0.5f * (Ct[3 * a + b] - Ct[3 * b + a]) + keep * sym[3 * a + b];
          }
      }
      // M = dt C + dt^2/2 C C ; d3' = d3 + M d3
      float Mm[9];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          float cc = 0.f;
#pragma unroll
          for (int q = 0; q < 3; ++q) cc += Cn[3 * a + q] * Cn[3 * q + b];
          Mm[3 * a + b] = dt * Cn[3 * a + b] + 0.5f * dt * dt * cc;
        }
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float acc = bd3o[b];
#pragma unroll
        for (int a = 0; a < 3; ++a) acc += Mm[3 * a + b] * bd3o[a];
        Ai.t[(TRI_D3 + b) * nt + idx] = acc;  // partial; k_tri_adj adds the P2G part
      }
      // dL/dC' = bCo + dt G + dt^2/2 (G C'^T + C'^T G), G = bd3' d3^T
      float G[9];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) G[3 * a + b] = bd3o[a] * d3[b];
      float bCn[9];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          float gc = 0.f, cg = 0.f;
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            gc += G[3 * a + q] * Cn[3 * b + q];
            cg += Cn[3 * q + a] * G[3 * q + b];
          }
          bCn[3 * a + b] = bCo[3 * a + b] + dt * G[3 * a + b] + 0.5f * dt * dt * (gc + cg);
        }
      float gd = 0.f;
#pragma unroll
      for (int q = 0; q < 9; ++q) gd -= bCn[q] * sym[q];
      gdamp[0] = (double)gd;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
          bC[3 * a + b] = 0.5f * (bCn[3 * a + b] - bCn[3 * b + a]) + keep * 0.5f * (bCn[3 * a + b] + bCn[3 * b + a]);
    } else {
      float sum_x[3] = {0.f, 0.f, 0.f}, sum_v[3] = {0.f, 0.f, 0.f};
      if (fold && ch.kind == CHUNK_VERTEX) {
        // the triangles' per-vertex sums of the previous adjoint substep,
        // still to be added to this vertex's position / velocity adjoint
        const float4 sx = B.vadj[idx], sv = B.vadj[B.nv + idx];
        sum_x[0] = sx.x; sum_x[1] = sx.y; sum_x[2] = sx.z;
        sum_v[0] = sv.x; sum_v[1] = sv.y; sum_v[2] = sv.z;
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        bx[a] = __ldg(ao + a * n + idx) + sum_x[a];
        bV[a] = (__ldg(ao + (3 + a) * n + idx) + sum_v[a]) + dt * bx[a];
      }
#pragma unroll
      for (int q = 0; q < 9; ++q) bC[q] = __ldg(ao + (6 + q) * n + idx);
    }
    // position adjoint of the gather (second pass over the stencil).  The
    // node's weight dL/dv' + 4/dx dL/dC (o - fx) is Kg + cbC o with
    // cbC = 4/dx dL/dC and Kg = dL/dv' - cbC fx (per-axis terms added for the
    // node's offsets o); the scatter below uses the same weights.
    float px[3] = {0.f, 0.f, 0.f}, vs[3] = {0.f, 0.f, 0.f};
    const float c4 = 4.f * inv_dx;
#pragma unroll
    for (int q = 0; q < 9; ++q) cbC[q] = c4 * bC[q];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      Kg[a] = bV[a] - (cbC[3 * a] * st.fx[0] + cbC[3 * a + 1] * st.fx[1] + cbC[3 * a + 2] * st.fx[2]);
    float ed[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int o = 0; o < 3; ++o) ed[a][o] = st.dw[a][o] * inv_dx;
    const float4* gnb = grid_base<PAGED>(B.grid_v, I);
    const StenAddr<PAGED> nofs(B, I, st.base, true, ch.inst);
#pragma unroll
    for (int oi = 0; oi < 3; ++oi)
#pragma unroll
      for (int oj = 0; oj < 3; ++oj) {
        const float w0 = st.w[0][oi], w1 = st.w[1][oj];
        const float w01 = w0 * w1, e0w1 = ed[0][oi] * w1, w0e1 = w0 * ed[1][oj];
        float kij[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) kij[a] = add_off(add_off(Kg[a], oi, cbC[3 * a]), oj, cbC[3 * a + 1]);
        // sum factorisation over the column's z nodes, as in k_tri_adj
        float Rw[3] = {0.f, 0.f, 0.f}, Sw = 0.f, Se = 0.f;
#pragma unroll
        for (int ok = 0; ok < 3; ++ok) {
          const float w2 = st.w[2][ok];
          const float3 gn = gv_at(gnb, nofs, oi, oj, ok);
          const float ga[3] = {gn.x, gn.y, gn.z};
          float s1 = 0.f;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            s1 += ga[a] * add_off(kij[a], ok, cbC[3 * a + 2]);
            Rw[a] += w2 * ga[a];
          }
          Sw += w2 * s1;
          Se += ed[2][ok] * s1;
        }
        px[0] += e0w1 * Sw;
        px[1] += w0e1 * Sw;
        px[2] += w01 * Se;
#pragma unroll
        for (int b = 0; b < 3; ++b) vs[b] += w01 * Rw[b];
      }
    // - c4 inv_dx sum_nodes W bC^T g = - inv_dx cbC^T (sum_nodes W g)
#pragma unroll
    for (int b = 0; b < 3; ++b) px[b] -= inv_dx * (cbC[b] * vs[0] + cbC[3 + b] * vs[1] + cbC[6 + b] * vs[2]);
    if (tri) {
      const long long nt = B.nt;
#pragma unroll
      for (int a = 0; a < 3; ++a) B.tri_tmp[a * nt + idx] = px[a];
    } else {
#pragma unroll
      for (int a = 0; a < 3; ++a) aa[a * n + idx] = bx[a] + px[a];
    }
  }
  // dL/dv_out at a node: W (dL/dv' + 4 inv_dx dL/dC dpos) = W (Kg + cbC o),
  // zero at every node when Kg and cbC are
  bool nz = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) nz = nz || Kg[a] != 0.f;
#pragma unroll
  for (int q = 0; q < 9; ++q) nz = nz || cbC[q] != 0.f;
  warp_scatter<false, PAGED>(B, I, ch.inst, st.base, valid, nz, [=](int oi, int oj, int ok) -> float4 {
    const float W = (st.w[0][oi] * st.w[1][oj]) * st.w[2][ok];
    float4 val;
    val.x = W * add_off(add_off(add_off(Kg[0], oi, cbC[0]), oj, cbC[1]), ok, cbC[2]);
    val.y = W * add_off(add_off(add_off(Kg[1], oi, cbC[3]), oj, cbC[4]), ok, cbC[5]);
    val.z = W * add_off(add_off(add_off(Kg[2], oi, cbC[6]), oj, cbC[7]), ok, cbC[8]);
    val.w = 0.f;
    return val;
  });
  if (tri) block_sum_atomic<1>(gdamp, gparams + ch.inst * PRM_STRIDE + PRM_DAMPING);
  // folded sums cleared after all of the kernel's loads (a store before them
  // makes them wait), ready for this substep's k_tri_adj
  if (fold && valid && ch.kind == CHUNK_VERTEX) {
    B.vadj[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
    B.vadj[B.nv + idx] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// Reverse of k_grid: dL/dp, dL/dm of every active node from dL/dv_out.  The
// active blocks and their (p, m) come from the tape when it holds this
// substep (as in k_grid), otherwise from this substep's recomputed P2G, whose
// grid and block flags are cleared here for the next substep.
__global__ void __launch_bounds__(256, 6) k_grid_adj(BatchDev B, const float* __restrict__ params,
                                                  const float* __restrict__ traj, int step, double* __restrict__ gparams,
                                                  double* __restrict__ gtraj, TapeP T) {
  const int2 tm = T.meta ? T.meta[step] : make_int2(-1, 0);
  const bool from_tape = tm.x >= 0;
  const bool paged = B.pool_cap > 0;
  int count = from_tape ? tm.y : B.counters[0];
  if (paged) count = min(count, B.pool_cap);
  const int per = blockDim.x >> 6, l = threadIdx.x & 63, stride = gridDim.x * per;
  // the next item's loads are issued before the current item is processed
  // (every item is a different block, so they do not depend on its stores)
  auto fetch = [&](int it, int& blk, int& inst, float4& pm, float4& ga) {
    const long long slot = (long long)tm.x + it;
    blk = from_tape ? __ldg(T.blk + slot) : B.list_blk[it];
    inst = from_tape ? __ldg(T.inst + slot) : B.list_inst[it];
    const long long n = (paged ? (long long)it : (long long)blk) * 64 + l;
    pm = from_tape ? __ldg(T.data + slot * 64 + l) : B.grid_pm[n];
    ga = B.grid_adj[n];
  };
  int item = blockIdx.x * per + (threadIdx.x >> 6);
  int blk = 0, inst = 0;
  float4 pm = make_float4(0.f, 0.f, 0.f, 0.f), ga = pm;
  if (item < count) fetch(item, blk, inst, pm, ga);
  for (; item < count; item += stride) {
    int blk_n = 0, inst_n = 0;
    float4 pm_n = make_float4(0.f, 0.f, 0.f, 0.f), ga_n = pm_n;
    if (item + stride < count) fetch(item + stride, blk_n, inst_n, pm_n, ga_n);
    const InstDev& I = B.inst[inst];
    int i, j, k;
    block_node(I, blk, l, i, j, k);
    const long long n = (paged ? (long long)item : (long long)blk) * 64 + l;
    const float inv_m = 1.f / (pm.w + 1e-9f);
    const float v[3] = {inv_m * pm.x, inv_m * pm.y, inv_m * pm.z};
    const float mu_g = __ldg(params + inst * PRM_STRIDE + PRM_FRICTION);
    float out[3];
    const NodeBC<float> r = grid_bc<float>(v, i, j, k, I.G, I.bound, mu_g, out);
    float bv[3] = {0.f, 0.f, 0.f};
    float gmu = 0.f;
    const float gout[3] = {ga.x, ga.y, ga.z};
    const int hit = kinematic_hit(I, traj, step, i, j, k);
    if (hit >= 0) {
      const long long o = I.traj_off + ((long long)step * I.n_grip + hit) * 3;
      if (ga.x != 0.f) atomicAdd(gtraj + o, (double)ga.x);
      if (ga.y != 0.f) atomicAdd(gtraj + o + 1, (double)ga.y);
      if (ga.z != 0.f) atomicAdd(gtraj + o + 2, (double)ga.z);
    } else {
      grid_bc_backward<float>(v, r, mu_g, gout, bv, gmu);
    }
    const float bp[3] = {inv_m * bv[0], inv_m * bv[1], inv_m * bv[2]};
    const float bm = -inv_m * (bv[0] * v[0] + bv[1] * v[1] + bv[2] * v[2]);
    B.grid_adj[n] = make_float4(bp[0], bp[1], bp[2], bm);
    if (!from_tape) {
      B.grid_pm[n] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (!paged && l == 0) B.flags[blk] = 0u;
    }
    double gmud = (double)gmu;
    for (int o = 16; o > 0; o >>= 1) gmud += __shfl_xor_sync(0xffffffffu, gmud, o);
    if ((threadIdx.x & 31) == 0 && gmud != 0.0) atomicAdd(gparams + inst * PRM_STRIDE + PRM_FRICTION, gmud);
    blk = blk_n;
    inst = inst_n;
    pm = pm_n;
    ga = ga_n;
  }
}

// Reverse of k_point_p2g: gather dL/dp, dL/dm over the stencil.
template <bool PAGED>
__global__ void __launch_bounds__(256, 4) k_point_adj(BatchDev B, const float* __restrict__ traj, int step, int window,
                                                   const float* __restrict__ rest, const float* __restrict__ sin,
                                                   float* __restrict__ ain, double* __restrict__ gtraj,
                                                   const int2* __restrict__ tmeta, const float* __restrict__ fv_in) {
  const Chunk ch = B.chunks[B.n_tri_chunks + blockIdx.x];
  if (threadIdx.x >= ch.count) return;
  const InstDev& I = B.inst[ch.inst];
  StateP Si = state_ptrs(const_cast<float*>(sin), B.nv, B.nt, B.no);
  StateP Ai = state_ptrs(ain, B.nv, B.nt, B.no);
  float *ai, *aa;
  long long n;
  point_arrays(B, Si, ch.kind, ai, n);
  point_arrays(B, Ai, ch.kind, aa, n);
  const float* x0 = point_rest(rest_ptrs(rest, B.nv, B.nt, B.no), ch.kind);
  const long long p = ch.start + threadIdx.x;
  float X[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) X[a] = __ldg(x0 + a * n + p) + __ldg(ai + a * n + p);
  Sten st;
  make_stencil(X, I, st, B.status, ch.inst);
  float m, base_v[3] = {0.f, 0.f, 0.f};
  long long i0 = -1, i1 = -1;
  bool op_active = false;
  if (ch.kind == CHUNK_VERTEX) {
    m = I.m_v;
    float f[3] = {0.f, 0.f, 0.f};
    if (fv_in && tmeta->x >= 0) {  // summed corner forces kept by the forward substep
#pragma unroll
      for (int a = 0; a < 3; ++a) f[a] = __ldg(fv_in + a * (long long)B.nv + p);
    } else {  // recomputed by this substep's k_tri_forward; cleared at the end of this kernel
      const float4 fs = B.fvert[p];
      f[0] = fs.x; f[1] = fs.y; f[2] = fs.z;
    }
    base_v[0] = m * __ldg(ai + 3 * n + p) + f[0];
    base_v[1] = m * (__ldg(ai + 4 * n + p) + I.gravity_dv) + f[1];
    base_v[2] = m * __ldg(ai + 5 * n + p) + f[2];
  } else if (ch.kind == CHUNK_OPERATOR) {
    m = I.m_o;
    float v[3];
    op_active = operator_velocity(B, I, traj, step, window, p, v, i0, i1);
    base_v[0] = m * v[0]; base_v[1] = m * v[1]; base_v[2] = m * v[2];
  } else {
    m = I.m_c;
  }
  // the APIC payload m (v + C dpos) of a node is K + Cd o with Cd = m dx C and
  // K = m v - Cd fx; sum W bp dpos comes from the moments mo = sum W bp o
  // (both as in k_tri_adj)
  const float dx = I.dx, inv_dx = I.inv_dx;
  float Cd[9], K[3];
#pragma unroll
  for (int q = 0; q < 9; ++q) Cd[q] = (m * dx) * __ldg(ai + (6 + q) * n + p);
#pragma unroll
  for (int a = 0; a < 3; ++a)
    K[a] = base_v[a] - (Cd[3 * a] * st.fx[0] + Cd[3 * a + 1] * st.fx[1] + Cd[3 * a + 2] * st.fx[2]);
  float ed[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int o = 0; o < 3; ++o) ed[a][o] = st.dw[a][o] * inv_dx;
  float sp[3] = {0.f, 0.f, 0.f};     // sum W bp
  float mo[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // sum W bp (x) o
  float px[3] = {0.f, 0.f, 0.f};
  const float4* gnb = grid_base<PAGED>(B.grid_adj, I);
  const StenAddr<PAGED> nofs(B, I, st.base, true, ch.inst);
  // sum factorisation over each (oi, oj) column's z nodes, as in k_tri_adj
#pragma unroll
  for (int oi = 0; oi < 3; ++oi)
#pragma unroll
    for (int oj = 0; oj < 3; ++oj) {
      const float w0 = st.w[0][oi], w1 = st.w[1][oj];
      const float w01 = w0 * w1, e0w1 = ed[0][oi] * w1, w0e1 = w0 * ed[1][oj];
      float kij[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) kij[a] = add_off(add_off(K[a], oi, Cd[3 * a]), oj, Cd[3 * a + 1]);
      float Rw[3] = {0.f, 0.f, 0.f}, Rk[3] = {0.f, 0.f, 0.f}, Sw = 0.f, Se = 0.f;
#pragma unroll
      for (int ok = 0; ok < 3; ++ok) {
        const float w2 = st.w[2][ok];
        const float4 g = __ldg(gnb + nofs.at(oi, oj, ok));
        const float bp[3] = {g.x, g.y, g.z};
        float s = g.w * m;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          s += bp[a] * add_off(kij[a], ok, Cd[3 * a + 2]);
          const float wb = w2 * bp[a];
          Rw[a] += wb;
          Rk[a] = add_off(Rk[a], ok, wb);
        }
        Sw += w2 * s;
        Se += ed[2][ok] * s;
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float Wb = w01 * Rw[a];
        sp[a] += Wb;
        mo[3 * a] = add_off(mo[3 * a], oi, Wb);
        mo[3 * a + 1] = add_off(mo[3 * a + 1], oj, Wb);
        mo[3 * a + 2] += w01 * Rk[a];
      }
      px[0] += e0w1 * Sw;
      px[1] += w0e1 * Sw;
      px[2] += w01 * Se;
    }
  float spd[9];  // sum W bp (x) dpos
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) spd[3 * a + b] = dx * (mo[3 * a + b] - st.fx[b] * sp[a]);
  // - sum_nodes W m C^T bp = - m C^T sp = - Cd^T sp / dx
#pragma unroll
  for (int b = 0; b < 3; ++b) px[b] -= inv_dx * (Cd[b] * sp[0] + Cd[3 + b] * sp[1] + Cd[6 + b] * sp[2]);
#pragma unroll
  for (int a = 0; a < 3; ++a) aa[a * n + p] += px[a];
#pragma unroll
  for (int q = 0; q < 9; ++q) aa[(6 + q) * n + p] = m * spd[q];
  if (ch.kind == CHUNK_VERTEX) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      aa[(3 + a) * n + p] = m * sp[a];
      B.barf[a * (long long)B.nv + p] = sp[a];
    }
    if (!(fv_in && tmeta->x >= 0)) B.fvert[p] = make_float4(0.f, 0.f, 0.f, 0.f);  // for the next sums
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) aa[(3 + a) * n + p] = 0.f;
    if (ch.kind == CHUNK_OPERATOR && op_active) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double gvt = (double)(m * sp[a]) / (double)I.interval;
        if (gvt != 0.0) {
          atomicAdd(gtraj + i1 + a, gvt);
          atomicAdd(gtraj + i0 + a, -gvt);
        }
      }
    }
  }
}

// Reverse of k_tri_forward for one triangle: own-stencil gather, per-corner
// force adjoints from dL/df of the three vertices, stress adjoint, and the
// contributions to the three vertices (summed per vertex, added to the vertex
// adjoint by k_vertex_collect or, inside a rollout, by the next adjoint
// substep's k_g2p_adj).
template <int REGS, bool PAGED>
__global__ void __maxnreg__(REGS) k_tri_adj(BatchDev B, const float* __restrict__ params,
                                                 const float* __restrict__ rest, const float* __restrict__ sin,
                                                 float* __restrict__ ain, double* __restrict__ gparams) {
  const Chunk ch = B.chunks[blockIdx.x];
  const InstDev& I = B.inst[ch.inst];
  const bool valid = threadIdx.x < ch.count;
  const long long t = ch.start + threadIdx.x, nt = B.nt;
  StateP Si = state_ptrs(const_cast<float*>(sin), B.nv, B.nt, B.no);
  StateP Ai = state_ptrs(ain, B.nv, B.nt, B.no);
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const float* prm = params + ch.inst * PRM_STRIDE;
  float E = prm[PRM_E], nu = prm[PRM_NU];
  float mu, la;
  lame(E, nu, mu, la);
  const float ks = prm[PRM_KS], kc = prm[PRM_KC];
  double gsum[4] = {0.0, 0.0, 0.0, 0.0};
  if (valid) {
    float C[9], dl3[3], n0[3], Di[9], e[6];   // own loads first, overlapping the vertex gathers
#pragma unroll
    for (int q = 0; q < 9; ++q) C[q] = __ldg(Si.t + q * nt + t);
    load_tri_rest(B, R, Si, t, dl3, n0, Di);
    load_rest_edges(B, R, t, e);
    TriGeom g;
    load_centroid(B, Si, t, true, g);
    load_corner_u(B, Si, t, g);
    Sten st;
    make_stencil(g.xc, I, st, B.status, ch.inst);
    M3<float> d, Fe;
    tri_F(g, e, dl3, n0, Di, d, Fe);
    const float d3[3] = {d.m[2], d.m[5], d.m[8]};
    // The stencil loop needs only P's third column, which depends on the QR
    // alone: P[:,2] = Q (A R^-T)[:,2] = k_s (r02 q1 + r12 q2) + A22 / n3 q3
    // (R^-1 is upper triangular).  The full stress is formed after the loop,
    // so that it is not held in registers across it.
    float P3[3];
    {
      QR<float> q;
      qr_forward(Fe, q);
      const float a22 = q.a3 <= 0.f ? (-kc) * (q.a3 * q.a3) : 0.f;
      P3[0] = ks * (q.r02 * q.q1.x + q.r12 * q.q2.x) + a22 * q.q3.x;
      P3[1] = ks * (q.r02 * q.q1.y + q.r12 * q.q2.y) + a22 * q.q3.y;
      P3[2] = ks * (q.r02 * q.q1.z + q.r12 * q.q2.z) + a22 * q.q3.z;
    }
    const float vol = I.vol_q, dt = B.dt, m = I.m_q, dx = I.dx, inv_dx = I.inv_dx;
    const float cn = -vol * dt;
    const float i2 = inv_dx * inv_dx;
    // Per-node factors are products of per-axis ones: slopes pre-scaled by
    // 1/dx, curvatures (1, -2, 1) by 1/dx^2.  The APIC payload
    // m (v + C dpos), dpos = (o - fx) dx, is K + Cm o with Cm = m dx C and
    // K = m v - Cm fx, so each node adds the per-axis terms of its offsets o
    // (0, 1 or 2) instead of forming C dpos.  Sums that are linear in the
    // node's own data are accumulated as moments and finished after the loop:
    //   mo[a][b] = sum W g_a o_b          -> sum W g_a dpos_b = dx (mo - fx_b sp_a)
    //   hs[bc]   = sum (g . P3) H_bc      -> sum (g . P3) (H d3)_b = sum_c hs[bc] d3_c
    float ed[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int o = 0; o < 3; ++o) ed[a][o] = st.dw[a][o] * inv_dx;
    const float ddc[3] = {i2, -2.f * i2, i2};
    float Cm[9], K[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
      for (int b = 0; b < 3; ++b) Cm[3 * a + b] = (m * dx) * C[3 * a + b];
      K[a] = m * g.vc[a] - (Cm[3 * a] * st.fx[0] + Cm[3 * a + 1] * st.fx[1] + Cm[3 * a + 2] * st.fx[2]);
    }
    float sp[3] = {0.f, 0.f, 0.f}, mo[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float g3[3] = {0.f, 0.f, 0.f}, sg[3] = {0.f, 0.f, 0.f}, bx[3] = {0.f, 0.f, 0.f};
    float hs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // (00, 01, 02, 11, 12, 22)
    const float4* gnb = grid_base<PAGED>(B.grid_adj, I);
    const StenAddr<PAGED> nofs(B, I, st.base, true, ch.inst);
    // Sum factorisation: every node weight is a product of per-axis factors,
    // so the sums over the stencil's z column (ok) are formed first, per
    // (oi, oj), and scaled by the (x, y) factors once per column:
    //   Rw[a] = sum_k w2 bp_a, Rk[a] = sum_k o_k w2 bp_a, Re[a] = sum_k e2 bp_a
    //   Tw, Te, Td = sum_k (w2, e2, dd2) (bp . P3), Sw, Se = sum_k (w2, e2) s
#pragma unroll
    for (int oi = 0; oi < 3; ++oi)
#pragma unroll
      for (int oj = 0; oj < 3; ++oj) {
        const float w0 = st.w[0][oi], w1 = st.w[1][oj], e0 = ed[0][oi], e1 = ed[1][oj];
        const float w01 = w0 * w1, e0w1 = e0 * w1, w0e1 = w0 * e1, e0e1 = e0 * e1;
        const float d0w1 = ddc[oi] * w1, w0d1 = w0 * ddc[oj];
        float kij[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) kij[a] = add_off(add_off(K[a], oi, Cm[3 * a]), oj, Cm[3 * a + 1]);
        float Rw[3] = {0.f, 0.f, 0.f}, Rk[3] = {0.f, 0.f, 0.f}, Re[3] = {0.f, 0.f, 0.f};
        float Tw = 0.f, Te = 0.f, Td = 0.f, Sw = 0.f, Se = 0.f;
#pragma unroll
        for (int ok = 0; ok < 3; ++ok) {
          const float w2 = st.w[2][ok], e2 = ed[2][ok];
          const float4 ga = __ldg(gnb + nofs.at(oi, oj, ok));
          const float bp[3] = {ga.x, ga.y, ga.z};
          const float sP = bp[0] * P3[0] + bp[1] * P3[1] + bp[2] * P3[2];
          float sn = ga.w * m;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            sn += bp[a] * add_off(kij[a], ok, Cm[3 * a + 2]);
            const float wb = w2 * bp[a];
            Rw[a] += wb;
            Rk[a] = add_off(Rk[a], ok, wb);
            Re[a] += e2 * bp[a];
          }
          Tw += w2 * sP;
          Te += e2 * sP;
          Td += ddc[ok] * sP;
          Sw += w2 * sn;
          Se += e2 * sn;
        }
        const float c1 = d3[0] * e0w1 + d3[1] * w0e1, c2 = d3[2] * w01;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float Wb = w01 * Rw[a];
          sp[a] += Wb;
          mo[3 * a] = add_off(mo[3 * a], oi, Wb);
          mo[3 * a + 1] = add_off(mo[3 * a + 1], oj, Wb);
          mo[3 * a + 2] += w01 * Rk[a];
          g3[a] += c1 * Rw[a] + c2 * Re[a];
        }
        sg[0] += e0w1 * Tw;
        sg[1] += w0e1 * Tw;
        sg[2] += w01 * Te;
        hs[0] += d0w1 * Tw;
        hs[1] += e0e1 * Tw;
        hs[2] += e0w1 * Te;
        hs[3] += w0d1 * Tw;
        hs[4] += w0e1 * Te;
        hs[5] += w01 * Td;
        bx[0] += e0w1 * Sw;
        bx[1] += w0e1 * Sw;
        bx[2] += w01 * Se;
      }
    float spd[9], bP3[3], bd3[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      bP3[a] = cn * g3[a];
      bd3[a] = cn * sg[a];
#pragma unroll
      for (int b = 0; b < 3; ++b) spd[3 * a + b] = dx * (mo[3 * a + b] - st.fx[b] * sp[a]);
    }
    {
      const float hd[3] = {hs[0] * d3[0] + hs[1] * d3[1] + hs[2] * d3[2],
                           hs[1] * d3[0] + hs[3] * d3[1] + hs[4] * d3[2],
                           hs[2] * d3[0] + hs[4] * d3[1] + hs[5] * d3[2]};
      // - sum_nodes W m C^T bp = - m C^T sp = - Cm^T sp / dx
#pragma unroll
      for (int b = 0; b < 3; ++b)
        bx[b] += cn * hd[b] - inv_dx * (Cm[b] * sp[0] + Cm[3 + b] * sp[1] + Cm[6 + b] * sp[2]);
    }
    Stress<float> sts;
    stress_forward<float>(Fe, mu, la, ks, kc, sts);
    // in-plane corner forces: f1 = k P (r1 + r2), f2 = -k P r1, f3 = -k P r2
    const float kf = vol * dt;
    float bf[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 3; ++a) bf[c][a] = B.barf[a * (long long)B.nv + g.vid[c]];
    // D0^-1 read again rather than held in registers across the stencil loop
#pragma unroll
    for (int q = 0; q < 9; ++q) Di[q] = __ldg(R.Di + q * nt + t);
    const float r1[3] = {Di[0], d.m[1], d.m[2]};
    const float r2[3] = {Di[3], d.m[4], d.m[5]};
    M3<float> bP;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        bP.m[3 * a + b] = kf * (bf[0][a] * (r1[b] + r2[b]) - bf[1][a] * r1[b] - bf[2][a] * r2[b]);
    bP.m[2] += bP3[0]; bP.m[5] += bP3[1]; bP.m[8] += bP3[2];
    float br1[3], br2[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      br1[b] = kf * (sts.P.m[b] * (bf[0][0] - bf[1][0]) + sts.P.m[3 + b] * (bf[0][1] - bf[1][1]) +
                     sts.P.m[6 + b] * (bf[0][2] - bf[1][2]));
      br2[b] = kf * (sts.P.m[b] * (bf[0][0] - bf[2][0]) + sts.P.m[3 + b] * (bf[0][1] - bf[2][1]) +
                     sts.P.m[6 + b] * (bf[0][2] - bf[2][2]));
    }
    M3<float> bF;
    float gmu = 0.f, gla = 0.f, gks = 0.f, gkc = 0.f;
    stress_backward<float>(sts, mu, la, ks, kc, bP, B.svd_grad, bF, gmu, gla, gks, gkc);
    // dL/dd = dL/dF D0^-T plus the direct uses of d in r1, r2 and the normal force
    float bd[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k)
        bd[3 * r + k] = bF.m[3 * r] * Di[3 * k] + bF.m[3 * r + 1] * Di[3 * k + 1] + bF.m[3 * r + 2] * Di[3 * k + 2];
    bd[1] += br1[1];  // d[0,1]
    bd[2] += br1[2];  // d[0,2]
    bd[4] += br2[1];  // d[1,1]
    bd[5] += br2[2];  // d[1,2]
    const float be1[3] = {bd[0], bd[3], bd[6]};
    const float be2[3] = {bd[1], bd[4], bd[7]};
#pragma unroll
    for (int a = 0; a < 3; ++a) bd3[a] += bd[3 * a + 2];
    const float third = 1.f / 3.f;
    float bxt[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) bxt[a] = third * (bx[a] + B.tri_tmp[a * nt + t]);
    // per-vertex sums of the corners' position and velocity adjoints
    const float4 bvc = make_float4(third * m * sp[0], third * m * sp[1], third * m * sp[2], 0.f);
    const long long nv = B.nv;
    atomicAdd(B.vadj + g.vid[0], make_float4(bxt[0] - be1[0] - be2[0], bxt[1] - be1[1] - be2[1],
                                             bxt[2] - be1[2] - be2[2], 0.f));
    atomicAdd(B.vadj + g.vid[1], make_float4(bxt[0] + be1[0], bxt[1] + be1[1], bxt[2] + be1[2], 0.f));
    atomicAdd(B.vadj + g.vid[2], make_float4(bxt[0] + be2[0], bxt[1] + be2[1], bxt[2] + be2[2], 0.f));
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(B.vadj + nv + g.vid[c], bvc);
#pragma unroll
    for (int q = 0; q < 9; ++q) Ai.t[q * nt + t] = m * spd[q];
#pragma unroll
    for (int a = 0; a < 3; ++a) Ai.t[(TRI_D3 + a) * nt + t] += bd3[a];
    // (mu, la) -> (E, nu)
    const float dmu_dE = 1.f / (2.f * (1.f + nu)), dmu_dnu = -E / (2.f * (1.f + nu) * (1.f + nu));
    const float D = (1.f + nu) * (1.f - 2.f * nu);
    const float dla_dE = nu / D, dla_dnu = E * (1.f + 2.f * nu * nu) / (D * D);
    // the (mu, lambda) -> (E, nu) chain in double: the two terms cancel in part
    gsum[0] = (double)gmu * (double)dmu_dE + (double)gla * (double)dla_dE;
    gsum[1] = (double)gmu * (double)dmu_dnu + (double)gla * (double)dla_dnu;
    gsum[2] = (double)gks;
    gsum[3] = (double)gkc;
  }
  block_sum_atomic<4>(gsum, gparams + ch.inst * PRM_STRIDE);
}

__global__ void k_vertex_collect(BatchDev B, float* __restrict__ ain) {
  StateP Ai = state_ptrs(ain, B.nv, B.nt, B.no);
  const long long nv = B.nv;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x) {
    const float4 bx = B.vadj[v], bv = B.vadj[nv + v];
    Ai.v[v] += bx.x;
    Ai.v[nv + v] += bx.y;
    Ai.v[2 * nv + v] += bx.z;
    Ai.v[3 * nv + v] += bv.x;
    Ai.v[4 * nv + v] += bv.y;
    Ai.v[5 * nv + v] += bv.z;
    B.vadj[v] = make_float4(0.f, 0.f, 0.f, 0.f);       // ready for the next substep's sums
    B.vadj[nv + v] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// ============================================================== Chamfer
// compute_loss (parameter_fitting_functions.py:3-15): for every target point
// the minimum over vertices of |x - t|^2 / 3; ties go to the vertex of lowest
// rank.  x - t is formed rest-relative, (x0 - t) + u, with explicitly rounded
// float32 operations (the reference subtracts the target from a stored
// absolute position, which rounds differently).  NaN distances are skipped
// and flag the instance non-finite; a target with no distance below +inf gets
// a NaN minimum (the instance's loss becomes NaN) and argmin -1.
__global__ void __launch_bounds__(128) k_chamfer_fwd(BatchDev B, const float* __restrict__ rest,
                                                     const float* __restrict__ state, const float* __restrict__ targets,
                                                     int* __restrict__ qarg) {
  __shared__ float sx[256], sy[256], sz[256], ux[256], uy[256], uz[256];
  __shared__ int sr[256];
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const int inst = blockIdx.y;
  const InstDev& I = B.inst[inst];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x * blockDim.x >= I.nq) return;
  const bool valid = q < I.nq;
  const long long nq = B.nq, nv = B.nv;
  const long long gq = (long long)I.q_off + q;
  float tx = 0.f, ty = 0.f, tz = 0.f;
  if (valid) {
    tx = __ldg(targets + gq);
    ty = __ldg(targets + nq + gq);
    tz = __ldg(targets + 2 * nq + gq);
  }
  float best = __int_as_float(0x7f800000);
  int brank = 0x7fffffff, bv = -1;
  bool nan_seen = false;
  for (int base = 0; base < I.nv; base += 256) {
    for (int j = threadIdx.x; j < 256; j += blockDim.x) {
      const int v = base + j;
      if (v < I.nv) {
        const long long gv = I.v_off + v;
        sx[j] = __ldg(R.xv + gv);
        sy[j] = __ldg(R.xv + nv + gv);
        sz[j] = __ldg(R.xv + 2 * nv + gv);
        ux[j] = __ldg(state + gv);
        uy[j] = __ldg(state + nv + gv);
        uz[j] = __ldg(state + 2 * nv + gv);
        sr[j] = __ldg(B.vertex_rank + gv);
      }
    }
    __syncthreads();
    const int cnt = min(256, I.nv - base);
    if (valid) {
      for (int j = 0; j < cnt; ++j) {
        // x - t = (x0 - t) + u
        const float dx = __fadd_rn(__fsub_rn(sx[j], tx), ux[j]);
        const float dy = __fadd_rn(__fsub_rn(sy[j], ty), uy[j]);
        const float dz = __fadd_rn(__fsub_rn(sz[j], tz), uz[j]);
        const float dd = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)), 3.f);
        nan_seen |= dd != dd;
        if (dd < best || (dd == best && sr[j] < brank)) {
          best = dd;
          brank = sr[j];
          bv = base + j;
        }
      }
    }
    __syncthreads();
  }
  if (valid) {
    B.qmin[gq] = bv >= 0 ? best : __int_as_float(0x7fc00000);
    qarg[gq] = bv >= 0 ? I.v_off + bv : -1;
    if (nan_seen || bv < 0) atomicOr(B.status + inst, STATUS_NONFINITE);
  }
}

__global__ void k_chamfer_loss(BatchDev B, float* __restrict__ loss) {
  __shared__ double red[32];
  const InstDev& I = B.inst[blockIdx.x];
  double s = 0.0;
  for (int q = threadIdx.x; q < I.nq; q += blockDim.x) s += (double)__fdiv_rn(B.qmin[I.q_off + q], (float)I.nq);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    loss[blockIdx.x] = (float)t;
  }
}

__global__ void k_chamfer_bwd(BatchDev B, const float* __restrict__ rest, const float* __restrict__ state,
                              const float* __restrict__ targets, const int* __restrict__ qarg,
                              const float* __restrict__ gloss, float* __restrict__ adj) {
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const int inst = blockIdx.y;
  const InstDev& I = B.inst[inst];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= I.nq) return;
  const long long nq = B.nq, nv = B.nv;
  const long long gq = (long long)I.q_off + q;
  const int v = qarg[gq];
  if (v < 0) return;
  const float s = __fdiv_rn(__ldg(gloss + inst), (float)I.nq) * (2.f / 3.f);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float d = (__ldg(R.xv + a * nv + v) - __ldg(targets + a * nq + gq)) + __ldg(state + a * nv + v);
    atomicAdd(adj + a * nv + v, s * d);
  }
}

// ============================================================== replay reset
// reset_quadrature_particles (simulation_without_grad.py:471-485), triangle
// part: the rest frame becomes [e1, e2, n] of the current vertices, d3 becomes
// n (delta3 = 0), and the stored F is kept: F - I of the old frame goes to
// fdev for the next substep's stress.  Runs before k_reset_vertex, which
// moves the vertex rest positions to the current ones.
__global__ void __launch_bounds__(256) k_reset_tri(BatchDev B, float* __restrict__ rest, float* __restrict__ state,
                                                   float* __restrict__ fdev) {
  StateP S = state_ptrs(state, B.nv, B.nt, B.no);
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const long long nt = B.nt, nv = B.nv;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nt; t += (long long)gridDim.x * blockDim.x) {
    TriGeom g;
    load_corner_u(B, S, t, g);
    float dl3[3], n0[3], Di[9], e[6];
    load_tri_rest(B, R, S, t, dl3, n0, Di);
    load_rest_edges(B, R, t, e);
    M3<float> d, Fe;
    tri_F(g, e, dl3, n0, Di, d, Fe);
    for (int q = 0; q < 9; ++q) fdev[q * nt + t] = Fe.m[q];
    float p[3][3];
    for (int c = 0; c < 3; ++c)
      for (int a = 0; a < 3; ++a) p[c][a] = R.xv[a * nv + g.vid[c]] + g.U[c][a];
    float inv[9], nrm[3];
    rest_frame(p[0], p[1], p[2], inv, nrm);
    float* DiW = const_cast<float*>(R.Di);
    float* n0W = const_cast<float*>(R.n0);
    float* eW = const_cast<float*>(R.e);
    float* tcW = const_cast<float*>(R.tc);
    for (int q = 0; q < 9; ++q) DiW[q * nt + t] = inv[q];
    for (int q = 0; q < 3; ++q) {
      n0W[q * nt + t] = nrm[q];
      eW[q * nt + t] = p[1][q] - p[0][q];
      eW[(3 + q) * nt + t] = p[2][q] - p[0][q];
      // the kept centroid becomes the rest centroid: the vertices' rest
      // positions move to their current ones (k_reset_vertex) and their
      // displacements become 0
      tcW[q * nt + t] = S.t[(TRI_XC + q) * nt + t];
      S.t[(TRI_D3 + q) * nt + t] = 0.f;
    }
  }
}

// Vertex part of the reset: rest position := current position, displacement 0.
__global__ void __launch_bounds__(256) k_reset_vertex(BatchDev B, float* __restrict__ rest, float* __restrict__ state) {
  StateP S = state_ptrs(state, B.nv, B.nt, B.no);
  const RestP R = rest_ptrs(rest, B.nv, B.nt, B.no);
  const long long nv = B.nv;
  float* xv = const_cast<float*>(R.xv);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < nv; p += (long long)gridDim.x * blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      xv[a * nv + p] = xv[a * nv + p] + S.v[a * nv + p];
      S.v[a * nv + p] = 0.f;
    }
  }
}

// ============================================================== grid tape
// Reserve tape slots for the active blocks of substep `step` (one thread).
__global__ void k_tape_reserve(BatchDev B, TapeP T, int step) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int count = B.pool_cap > 0 ? min(B.counters[0], B.pool_cap) : B.counters[0];
  const int top = *T.top;
  if ((long long)top + count <= T.cap) {
    T.meta[step] = make_int2(top, count);
    *T.top = top + count;
  } else {
    T.meta[step] = make_int2(-1, count);
  }
}

// ============================================================== launchers
const char* const kKernelNames[KID_COUNT] = {
    "k_tri_forward", "k_point_p2g", "k_grid", "k_g2p", "k_g2p_adj", "k_grid_adj", "k_point_adj", "k_tri_adj",
    "k_vertex_collect", "k_chamfer_fwd", "k_chamfer_loss", "k_chamfer_bwd", "k_init", "k_tape", "k_reset",
    "k_alloc", "k_release"};

static inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
// Register-cap variants of the three register-heavy kernels, by level:
// 1 = no cap (255 registers), 2 = 128, 3 = 96, 4 = 80, 5 = 72, 6 = 64; for
// dense or paged grids.  A cap trades spills for resident warps.
#define DCP_MINB_P(kernel, L, i, P)                                                                     \
  (L.min_blocks[i] >= 6   ? kernel<64, P>                                                               \
   : L.min_blocks[i] == 5 ? kernel<72, P>                                                               \
   : L.min_blocks[i] == 4 ? kernel<80, P>                                                               \
   : L.min_blocks[i] == 3 ? kernel<96, P>                                                               \
   : L.min_blocks[i] == 2 ? kernel<128, P>                                                              \
                          : kernel<255, P>)
#define DCP_MINB(kernel, L, i) (B.pool_cap > 0 ? DCP_MINB_P(kernel, L, i, true) : DCP_MINB_P(kernel, L, i, false))
// Dense or paged variant of a kernel template whose last parameter selects it.
#define DCP_PAGED(kernel, ...) (B.pool_cap > 0 ? kernel<__VA_ARGS__, true> : kernel<__VA_ARGS__, false>)
#define DCP_PAGED1(kernel) (B.pool_cap > 0 ? kernel<true> : kernel<false>)
#define DCP_LAUNCH(id, ...)                   \
  do {                                        \
    ProfScope _scope(L.prof, (id), s);        \
    __VA_ARGS__;                              \
  } while (0)

cudaError_t launch_init(const BatchDev& B, const LaunchCfg& L, const float* x0v, const float* x0o, const float* x0c,
                        float* state, float* rest, cudaStream_t s) {
  const long long total = (long long)B.nv + B.no + B.nc + B.nt;
  const int grid = total > 0 ? std::min(ceil_div(total, 256), L.sm_count * 16) : 1;
  DCP_LAUNCH(KID_INIT, (k_init<<<grid, 256, 0, s>>>(B, x0v, x0o, x0c, state, rest)));
  return cudaGetLastError();
}



cudaError_t launch_reset(const BatchDev& B, const LaunchCfg& L, float* rest, float* state, float* fdev,
                         cudaStream_t s) {
  if (B.nt) {
    const int grid = std::min(ceil_div(B.nt, 256), L.sm_count * 16);
    DCP_LAUNCH(KID_RESET, (k_reset_tri<<<grid, 256, 0, s>>>(B, rest, state, fdev)));
  }
  if (B.nv) {
    const int grid = std::min(ceil_div(B.nv, 256), L.sm_count * 16);
    DCP_LAUNCH(KID_RESET, (k_reset_vertex<<<grid, 256, 0, s>>>(B, rest, state)));
  }
  return cudaGetLastError();
}

static TapeP no_tape() {
  TapeP t;
  t.top = nullptr; t.meta = nullptr; t.blk = nullptr; t.inst = nullptr; t.data = nullptr; t.fv = nullptr; t.cap = 0;
  return t;
}

cudaError_t launch_forward(const BatchDev& B, const LaunchCfg& L, const float* params, const float* traj, const float* rest,
                           int step, int window, const float* sin, float* sout, cudaStream_t s, const TapeP* T,
                           const float* fdev) {
  const TapeP tp = T ? *T : no_tape();
  const bool paged = B.pool_cap > 0;
  const int n_chunks = B.n_tri_chunks + B.n_point_chunks;
  cudaMemsetAsync(B.counters, 0, sizeof(int), s);
  if (paged && n_chunks)
    DCP_LAUNCH(KID_ALLOC, (k_alloc<<<n_chunks, L.block, 0, s>>>(B, rest, sin, nullptr)));
  if (B.n_tri_chunks)
    DCP_LAUNCH(KID_TRI_FORWARD, (DCP_MINB(k_tri_forward, L, 0)<<<B.n_tri_chunks, L.block, 0, s>>>(
                                    B, params, rest, sin, nullptr, fdev)));
  if (B.n_point_chunks)
    DCP_LAUNCH(KID_POINT_P2G, (DCP_PAGED1(k_point_p2g)<<<B.n_point_chunks, L.block, 0, s>>>(
                                  B, traj, step, window, rest, sin, nullptr,
                                  T ? tp.fv + (long long)step * 3 * B.nv : nullptr, 1)));
  if (T) DCP_LAUNCH(KID_TAPE, (k_tape_reserve<<<1, 32, 0, s>>>(B, tp, step)));
  DCP_LAUNCH(KID_GRID, (k_grid<<<L.grid_ctas, 256, 0, s>>>(B, params, traj, step, GRID_FORWARD, tp)));
  // points first: the triangle launch forms the next centroids from the vertices' new state
  if (B.n_point_chunks)
    DCP_LAUNCH(KID_G2P, (DCP_PAGED(k_g2p, false)<<<B.n_point_chunks, L.block, 0, s>>>(B, params, rest, sin, sout)));
  if (B.n_tri_chunks)
    DCP_LAUNCH(KID_G2P, (DCP_PAGED(k_g2p, true)<<<B.n_tri_chunks, L.block, 0, s>>>(B, params, rest, sin, sout)));
  if (paged) DCP_LAUNCH(KID_RELEASE, (k_release<<<L.sm_count * 4, 256, 0, s>>>(B, tp, step, GRID_FORWARD)));
  return cudaGetLastError();
}

cudaError_t launch_backward(const BatchDev& B, const LaunchCfg& L, const float* params, const float* traj,
                            const float* rest, int step, int window, const float* sin, const float* aout, float* ain,
                            double* gparams, double* gtraj, cudaStream_t s, const TapeP* T, const float* snext,
                            bool fold, bool collect) {
  const TapeP tp = T ? *T : no_tape();
  const int2* meta = T ? T->meta + step : nullptr;
  cudaMemsetAsync(B.counters, 0, sizeof(int), s);
  // with a tape the P2G recompute usually returns at once: launch a few CTAs
  // per SM that stride over the chunks instead of one CTA per chunk
  const int stride_ctas = 2 * L.grid_ctas;
  const int tri_ctas = T && B.n_tri_chunks > stride_ctas ? stride_ctas : B.n_tri_chunks;
  const int point_ctas = T && B.n_point_chunks > stride_ctas ? stride_ctas : B.n_point_chunks;
  const bool paged = B.pool_cap > 0;
  const int n_chunks = B.n_tri_chunks + B.n_point_chunks;
  if (paged && n_chunks)
    DCP_LAUNCH(KID_ALLOC, (k_alloc<<<T && n_chunks > stride_ctas ? stride_ctas : n_chunks, L.block, 0, s>>>(
                              B, rest, sin, meta)));
  if (B.n_tri_chunks)
    DCP_LAUNCH(KID_TRI_FORWARD, (DCP_MINB(k_tri_forward, L, 0)<<<tri_ctas, L.block, 0, s>>>(
                                    B, params, rest, sin, meta, nullptr)));
  if (B.n_point_chunks)
    DCP_LAUNCH(KID_POINT_P2G, (DCP_PAGED1(k_point_p2g)<<<point_ctas, L.block, 0, s>>>(B, traj, step, window, rest,
                                                                                    sin, meta, nullptr, 0)));
  DCP_LAUNCH(KID_GRID, (k_grid<<<L.grid_ctas, 256, 0, s>>>(B, params, traj, step, GRID_RECOMPUTE, tp)));
  DCP_LAUNCH(KID_G2P_ADJ, (DCP_MINB(k_g2p_adj, L, 1)<<<B.n_tri_chunks + B.n_point_chunks, L.block, 0, s>>>(
                              B, params, rest, sin, aout, ain, gparams, snext, fold ? 1 : 0)));
  DCP_LAUNCH(KID_GRID_ADJ, (k_grid_adj<<<L.grid_ctas, 256, 0, s>>>(B, params, traj, step, gparams, gtraj, tp)));
  if (B.n_point_chunks)
    DCP_LAUNCH(KID_POINT_ADJ, (DCP_PAGED1(k_point_adj)<<<B.n_point_chunks, L.block, 0, s>>>(
                                  B, traj, step, window, rest, sin, ain, gtraj, meta,
                                  T ? T->fv + (long long)step * 3 * B.nv : nullptr)));
  if (B.n_tri_chunks)
    DCP_LAUNCH(KID_TRI_ADJ, (DCP_MINB(k_tri_adj, L, 2)<<<B.n_tri_chunks, L.block, 0, s>>>(B, params, rest, sin, ain,
                                                                                        gparams)));
  if (B.nv && collect)
    DCP_LAUNCH(KID_VERTEX_COLLECT, (k_vertex_collect<<<ceil_div(B.nv, 256), 256, 0, s>>>(B, ain)));
  if (paged) DCP_LAUNCH(KID_RELEASE, (k_release<<<L.sm_count * 4, 256, 0, s>>>(B, tp, step, GRID_RECOMPUTE)));
  return cudaGetLastError();
}

cudaError_t launch_chamfer_forward(const BatchDev& B, const LaunchCfg& L, int max_nq, const float* rest,
                                   const float* state, const float* targets, int* qarg, float* loss, cudaStream_t s) {
  if (max_nq > 0) {
    dim3 grid(ceil_div(max_nq, 128), B.n_inst);
    DCP_LAUNCH(KID_CHAMFER_FWD, (k_chamfer_fwd<<<grid, 128, 0, s>>>(B, rest, state, targets, qarg)));
  }
  DCP_LAUNCH(KID_CHAMFER_LOSS, (k_chamfer_loss<<<B.n_inst, 256, 0, s>>>(B, loss)));
  return cudaGetLastError();
}

cudaError_t launch_chamfer_backward(const BatchDev& B, const LaunchCfg& L, int max_nq, const float* rest,
                                    const float* state, const float* targets, const int* qarg, const float* gloss,
                                    float* adj, cudaStream_t s) {
  if (max_nq > 0) {
    dim3 grid(ceil_div(max_nq, 128), B.n_inst);
    DCP_LAUNCH(KID_CHAMFER_BWD, (k_chamfer_bwd<<<grid, 128, 0, s>>>(B, rest, state, targets, qarg, gloss, adj)));
  }
  return cudaGetLastError();
}

cudaError_t configure_kernels(const BatchDev& B, const LaunchCfg& L) { return cudaSuccess; }

}  // namespace dcp
