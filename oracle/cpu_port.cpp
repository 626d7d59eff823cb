// Compiled CPU restatement of the differentiable cloth substep and its adjoint
// for the benchmark's cloths (kinematic-gripper sheets: vertices and triangles,
// no operator or cube particles).  TEST INFRASTRUCTURE and the timed CPU
// baseline of bench.py (its reference arm and cpu_baseline): nothing in the
// product calls it.
//
// It restates the reference's substep (src/simulation.py: p2g 176-271,
// grid_op 274-302, g2p 304-383, update_particle_state 386-430) with the
// build's two extensions that the benchmark uses (Coulomb floor friction and
// kinematic sphere grippers, as in oracle/sim64.py), the Chamfer loss
// (src/parameter_fitting_functions.py:3-15), and a hand-written reverse pass
// over a stored history of every substep, as the reference's Taichi Tape keeps
// one.  Positions are absolute, as in the reference.  Node-by-node stencil
// loops in the oracle's order; the per-particle stress, QR and grid-condition
// math comes from diffcp_b200/csrc/cloth_math.cuh.  Templated on the float
// type: the float64 build is checked against oracle/sim64.py, the float32
// build (the reference's precision) is the one timed.  Rollouts of different
// cloths run on different OpenMP threads.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../diffcp_b200/csrc/cloth_math.cuh"

using namespace dcp;

extern "C" {
struct CpuScene {
  int32_t nv, nt, nq, n_grid, bound, n_grip, n_steps;
  double dt, m_v, m_q, vol_q, gravity_dv, grip_radius;
  double E, nu, ks, kc, friction, damping;
  const double* x0;       // [nv][3] rest (initial) vertex positions
  const int32_t* tris;    // [nt][3]
  const double* vel;      // [n_steps][n_grip][3] gripper velocities
  const double* centers;  // [n_steps][n_grip][3] gripper centres
  const double* targets;  // [nq][3]
};
}

namespace {

template <class T>
struct Sten {
  int base[3];
  T fx[3], w[3][3], dw[3][3], ddw[3][3];
};

template <class T>
inline void stencil(const T* x, T inv_dx, int G, Sten<T>& s) {
  for (int a = 0; a < 3; ++a) {
    const T t = x[a] * inv_dx - T(0.5);
    int b = (int)t;
    b = std::max(0, std::min(b, G - 3));
    s.base[a] = b;
    s.fx[a] = x[a] * inv_dx - (T)b;
    bspline(s.fx[a], s.w[a], s.dw[a]);
    for (int o = 0; o < 3; ++o) {
      s.dw[a][o] *= inv_dx;                                  // d w / d x (physical units)
      s.ddw[a][o] = bspline_dd<T>(o) * inv_dx * inv_dx;      // d2 w / d x2
    }
  }
}

template <class T>
struct Rollout {
  const CpuScene& sc;
  int nv, nt, G, bound;
  T dx, inv_dx, dt, mv, mq, vol, gdv, mu, la, ks, kc, fr, keep;
  std::vector<T> X, V, Cv, Ct, D3;  // history, [n_steps + 1][...]
  std::vector<T> D0i;               // [nt][9]
  // grid of the current substep
  std::vector<T> gp, gm, gv;        // [G^3][3], [G^3], [G^3][3]
  std::vector<NodeBC<T>> bc;
  std::vector<int> hit;             // kinematic gripper overriding each node, or -1
  std::vector<T> ga;                // adjoint grid [G^3][4]: dL/dv_out xyz, then dL/dp xyz, dL/dm
  std::vector<T> ap, am;
  int lo[3], hi[3];                 // node box touched this substep
  // per-substep triangle intermediates
  std::vector<Stress<T>> st;
  std::vector<T> fvert;             // [nv][3] summed corner forces
  double g_E = 0, g_nu = 0, g_ks = 0, g_kc = 0, g_fr = 0, g_damp = 0;
  std::vector<double> g_vel;        // [n_steps][n_grip][3]

  explicit Rollout(const CpuScene& s) : sc(s) {
    nv = s.nv; nt = s.nt; G = s.n_grid; bound = s.bound;
    dx = T(1) / T(G); inv_dx = T(G); dt = (T)s.dt;
    mv = (T)s.m_v; mq = (T)s.m_q; vol = (T)s.vol_q; gdv = (T)s.gravity_dv;
    const T E = (T)s.E, nu = (T)s.nu;
    mu = E / (T(2) * (T(1) + nu));
    la = E * nu / ((T(1) + nu) * (T(1) - T(2) * nu));
    ks = (T)s.ks; kc = (T)s.kc; fr = (T)s.friction; keep = T(1) - (T)s.damping;
    const size_t n1 = (size_t)s.n_steps + 1;
    X.assign(n1 * nv * 3, T(0)); V.assign(n1 * nv * 3, T(0)); Cv.assign(n1 * nv * 9, T(0));
    Ct.assign(n1 * nt * 9, T(0)); D3.assign(n1 * nt * 3, T(0)); D0i.assign((size_t)nt * 9, T(0));
    const size_t nn = (size_t)G * G * G;
    gp.assign(nn * 3, T(0)); gm.assign(nn, T(0)); gv.assign(nn * 3, T(0)); bc.resize(nn); hit.assign(nn, -1);
    ga.assign(nn * 3, T(0)); ap.assign(nn * 3, T(0)); am.assign(nn, T(0));
    st.resize(nt); fvert.assign((size_t)nv * 3, T(0));
    g_vel.assign((size_t)s.n_steps * s.n_grip * 3, 0.0);
    // initialize_ti_field (simulation.py:447-477): D0 = [e1, e2, n], n from the
    // eps-normalised edges (norm(1e-6))
    for (int p = 0; p < nv * 3; ++p) X[p] = (T)s.x0[p];
    for (int t = 0; t < nt; ++t) {
      const int* v = s.tris + 3 * t;
      T e1[3], e2[3], n1[3], n2[3], n[3];
      for (int a = 0; a < 3; ++a) { e1[a] = X[3 * v[1] + a] - X[3 * v[0] + a]; e2[a] = X[3 * v[2] + a] - X[3 * v[0] + a]; }
      const T l1 = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2] + T(1e-6));
      const T l2 = std::sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2] + T(1e-6));
      for (int a = 0; a < 3; ++a) { n1[a] = e1[a] / l1; n2[a] = e2[a] / l2; }
      n[0] = n1[1] * n2[2] - n1[2] * n2[1]; n[1] = n1[2] * n2[0] - n1[0] * n2[2]; n[2] = n1[0] * n2[1] - n1[1] * n2[0];
      const T l3 = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + T(1e-6));
      for (int a = 0; a < 3; ++a) n[a] /= l3;
      const T m[9] = {e1[0], e2[0], n[0], e1[1], e2[1], n[1], e1[2], e2[2], n[2]};
      const T c00 = m[4] * m[8] - m[5] * m[7], c01 = m[2] * m[7] - m[1] * m[8], c02 = m[1] * m[5] - m[2] * m[4];
      const T c10 = m[5] * m[6] - m[3] * m[8], c11 = m[0] * m[8] - m[2] * m[6], c12 = m[2] * m[3] - m[0] * m[5];
      const T c20 = m[3] * m[7] - m[4] * m[6], c21 = m[1] * m[6] - m[0] * m[7], c22 = m[0] * m[4] - m[1] * m[3];
      const T det = m[0] * c00 + m[1] * c10 + m[2] * c20;
      const T inv[9] = {c00 / det, c01 / det, c02 / det, c10 / det, c11 / det, c12 / det, c20 / det, c21 / det, c22 / det};
      for (int q = 0; q < 9; ++q) D0i[9 * t + q] = inv[q];
      for (int a = 0; a < 3; ++a) D3[3 * t + a] = n[a];
    }
  }

  size_t node(int i, int j, int k) const { return ((size_t)i * G + j) * G + k; }
  T* Xf(int f) { return X.data() + (size_t)f * nv * 3; }
  T* Vf(int f) { return V.data() + (size_t)f * nv * 3; }
  T* Cvf(int f) { return Cv.data() + (size_t)f * nv * 9; }
  T* Ctf(int f) { return Ct.data() + (size_t)f * nt * 9; }
  T* D3f(int f) { return D3.data() + (size_t)f * nt * 3; }

  void centroid(int f, int t, T xc[3], T vc[3]) {
    const int* v = sc.tris + 3 * t;
    const T* x = Xf(f);
    const T* vv = Vf(f);
    for (int a = 0; a < 3; ++a) {
      xc[a] = (x[3 * v[0] + a] + x[3 * v[1] + a] + x[3 * v[2] + a]) / T(3);
      vc[a] = (vv[3 * v[0] + a] + vv[3 * v[1] + a] + vv[3 * v[2] + a]) / T(3);
    }
  }
  // d = [x_b - x_a, x_c - x_a, d3] and F - I = d D0^-1 - I
  void tri_d(int f, int t, M3<T>& d, M3<T>& Fe) {
    const int* v = sc.tris + 3 * t;
    const T* x = Xf(f);
    const T* d3 = D3f(f) + 3 * t;
    for (int a = 0; a < 3; ++a) {
      d.m[3 * a] = x[3 * v[1] + a] - x[3 * v[0] + a];
      d.m[3 * a + 1] = x[3 * v[2] + a] - x[3 * v[0] + a];
      d.m[3 * a + 2] = d3[a];
    }
    const T* Di = D0i.data() + 9 * t;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        Fe.m[3 * r + c] = d.m[3 * r] * Di[c] + d.m[3 * r + 1] * Di[3 + c] + d.m[3 * r + 2] * Di[6 + c] -
                          (r == c ? T(1) : T(0));
  }

  void touch(const Sten<T>& s) {
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], s.base[a]); hi[a] = std::max(hi[a], s.base[a] + 2); }
  }
  template <class Fn>
  void each_box_node(Fn&& fn) {
    for (int i = lo[0]; i <= hi[0]; ++i)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int k = lo[2]; k <= hi[2]; ++k) fn(i, j, k, node(i, j, k));
  }

  // P2G and grid update of substep f (state f): fills gp, gm, gv, bc, hit, st, fvert
  void grid_of(int f) {
    const T* x = Xf(f); const T* v = Vf(f); const T* C = Cvf(f); const T* tC = Ctf(f); const T* d3s = D3f(f);
    lo[0] = lo[1] = lo[2] = G; hi[0] = hi[1] = hi[2] = -1;
    std::vector<Sten<T>> vs(nv), ts(nt);
    for (int p = 0; p < nv; ++p) { stencil(x + 3 * p, inv_dx, G, vs[p]); touch(vs[p]); }
    T xc[3], vc[3];
    for (int t = 0; t < nt; ++t) { centroid(f, t, xc, vc); stencil(xc, inv_dx, G, ts[t]); touch(ts[t]); }
    each_box_node([&](int, int, int, size_t n) { gp[3 * n] = gp[3 * n + 1] = gp[3 * n + 2] = gm[n] = T(0); });
    std::fill(fvert.begin(), fvert.end(), T(0));
    // triangle stress (simulation.py:214-240) and corner forces (266-271)
    const T k = vol * dt;
    for (int t = 0; t < nt; ++t) {
      M3<T> d, Fe;
      tri_d(f, t, d, Fe);
      stress_forward(Fe, mu, la, ks, kc, st[t]);
      const M3<T>& P = st[t].P;
      const T* Di = D0i.data() + 9 * t;
      const T r1[3] = {Di[0], d.m[1], d.m[2]}, r2[3] = {Di[3], d.m[4], d.m[5]};
      const int* vi = sc.tris + 3 * t;
      for (int a = 0; a < 3; ++a) {
        const T p1 = P.m[3 * a] * r1[0] + P.m[3 * a + 1] * r1[1] + P.m[3 * a + 2] * r1[2];
        const T p2 = P.m[3 * a] * r2[0] + P.m[3 * a + 1] * r2[1] + P.m[3 * a + 2] * r2[2];
        fvert[3 * vi[0] + a] += k * (p1 + p2);
        fvert[3 * vi[1] + a] -= k * p1;
        fvert[3 * vi[2] + a] -= k * p2;
      }
    }
    // vertices (simulation.py:176-191) with their corner-force sums
    for (int p = 0; p < nv; ++p) {
      const Sten<T>& s = vs[p];
      const T vt[3] = {v[3 * p], v[3 * p + 1] + gdv, v[3 * p + 2]};
      for (int oi = 0; oi < 3; ++oi)
        for (int oj = 0; oj < 3; ++oj)
          for (int ok = 0; ok < 3; ++ok) {
            const T W = s.w[0][oi] * s.w[1][oj] * s.w[2][ok];
            const T dp[3] = {((T)oi - s.fx[0]) * dx, ((T)oj - s.fx[1]) * dx, ((T)ok - s.fx[2]) * dx};
            const size_t n = node(s.base[0] + oi, s.base[1] + oj, s.base[2] + ok);
            for (int a = 0; a < 3; ++a) {
              const T cd = C[9 * p + 3 * a] * dp[0] + C[9 * p + 3 * a + 1] * dp[1] + C[9 * p + 3 * a + 2] * dp[2];
              gp[3 * n + a] += W * (mv * vt[a] + mv * cd + fvert[3 * p + a]);
            }
            gm[n] += W * mv;
          }
    }
    // triangles (simulation.py:193-265): own-node momentum, mass and normal force
    for (int t = 0; t < nt; ++t) {
      const Sten<T>& s = ts[t];
      centroid(f, t, xc, vc);
      const T* Ca = tC + 9 * t;
      const T* d3 = d3s + 3 * t;
      const M3<T>& P = st[t].P;
      for (int oi = 0; oi < 3; ++oi)
        for (int oj = 0; oj < 3; ++oj)
          for (int ok = 0; ok < 3; ++ok) {
            const T W = s.w[0][oi] * s.w[1][oj] * s.w[2][ok];
            const T gW[3] = {s.dw[0][oi] * s.w[1][oj] * s.w[2][ok], s.w[0][oi] * s.dw[1][oj] * s.w[2][ok],
                             s.w[0][oi] * s.w[1][oj] * s.dw[2][ok]};
            const T gd = gW[0] * d3[0] + gW[1] * d3[1] + gW[2] * d3[2];
            const T dp[3] = {((T)oi - s.fx[0]) * dx, ((T)oj - s.fx[1]) * dx, ((T)ok - s.fx[2]) * dx};
            const size_t n = node(s.base[0] + oi, s.base[1] + oj, s.base[2] + ok);
            for (int a = 0; a < 3; ++a) {
              const T cd = Ca[3 * a] * dp[0] + Ca[3 * a + 1] * dp[1] + Ca[3 * a + 2] * dp[2];
              gp[3 * n + a] += W * (mq * vc[a] + mq * cd) - vol * P.m[3 * a + 2] * gd * dt;
            }
            gm[n] += W * mq;
          }
    }
    // grid update (simulation.py:274-302) and kinematic grippers
    const T r2g = (T)(sc.grip_radius * sc.grip_radius);
    each_box_node([&](int i, int j, int kk, size_t n) {
      const T im = T(1) / (gm[n] + T(1e-9));
      const T vv[3] = {im * gp[3 * n], im * gp[3 * n + 1], im * gp[3 * n + 2]};
      T out[3];
      bc[n] = grid_bc<T>(vv, i, j, kk, G, bound, fr, out);
      int h = -1;
      if (f < sc.n_steps)
        for (int q = 0; q < sc.n_grip; ++q) {
          const double* c = sc.centers + ((size_t)f * sc.n_grip + q) * 3;
          const T ddx = (T)i * dx - (T)c[0], ddy = (T)j * dx - (T)c[1], ddz = (T)kk * dx - (T)c[2];
          if (ddx * ddx + ddy * ddy + ddz * ddz <= r2g) h = q;
        }
      hit[n] = h;
      if (h >= 0) {
        const double* gvel = sc.vel + ((size_t)f * sc.n_grip + h) * 3;
        out[0] = (T)gvel[0]; out[1] = (T)gvel[1]; out[2] = (T)gvel[2];
      }
      gv[3 * n] = out[0]; gv[3 * n + 1] = out[1]; gv[3 * n + 2] = out[2];
    });
  }

  void forward(int f) {
    grid_of(f);
    const T* x = Xf(f); const T* d3s = D3f(f);
    T* xn = Xf(f + 1); T* vn = Vf(f + 1); T* Cn = Cvf(f + 1); T* tCn = Ctf(f + 1); T* d3n = D3f(f + 1);
    for (int p = 0; p < nv; ++p) {  // g2p, simulation.py:346-365
      Sten<T> s;
      stencil(x + 3 * p, inv_dx, G, s);
      T vv[3] = {0, 0, 0}, CC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int oi = 0; oi < 3; ++oi)
        for (int oj = 0; oj < 3; ++oj)
          for (int ok = 0; ok < 3; ++ok) {
            const T W = s.w[0][oi] * s.w[1][oj] * s.w[2][ok];
            const T dp[3] = {(T)oi - s.fx[0], (T)oj - s.fx[1], (T)ok - s.fx[2]};
            const T* g = gv.data() + 3 * node(s.base[0] + oi, s.base[1] + oj, s.base[2] + ok);
            for (int a = 0; a < 3; ++a) {
              vv[a] += W * g[a];
              for (int b = 0; b < 3; ++b) CC[3 * a + b] += T(4) * inv_dx * W * g[a] * dp[b];
            }
          }
      for (int a = 0; a < 3; ++a) { vn[3 * p + a] = vv[a]; xn[3 * p + a] = x[3 * p + a] + dt * vv[a]; }
      for (int q = 0; q < 9; ++q) Cn[9 * p + q] = CC[q];
    }
    for (int t = 0; t < nt; ++t) {  // triangles: C (367-383), d3 (397-400)
      T xc[3], vc[3];
      centroid(f, t, xc, vc);
      Sten<T> s;
      stencil(xc, inv_dx, G, s);
      T CC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int oi = 0; oi < 3; ++oi)
        for (int oj = 0; oj < 3; ++oj)
          for (int ok = 0; ok < 3; ++ok) {
            const T W = s.w[0][oi] * s.w[1][oj] * s.w[2][ok];
            const T dp[3] = {(T)oi - s.fx[0], (T)oj - s.fx[1], (T)ok - s.fx[2]};
            const T* g = gv.data() + 3 * node(s.base[0] + oi, s.base[1] + oj, s.base[2] + ok);
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) CC[3 * a + b] += T(4) * inv_dx * W * g[a] * dp[b];
          }
      T Cd[9];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          Cd[3 * a + b] = T(0.5) * (CC[3 * a + b] - CC[3 * b + a]) + keep * T(0.5) * (CC[3 * a + b] + CC[3 * b + a]);
      const T* d3 = d3s + 3 * t;
      for (int a = 0; a < 3; ++a) {
        T acc = d3[a];
        for (int b = 0; b < 3; ++b) {
          T cc = 0;
          for (int q = 0; q < 3; ++q) cc += Cd[3 * a + q] * Cd[3 * q + b];
          acc += (dt * Cd[3 * a + b] + T(0.5) * dt * dt * cc) * d3[b];
        }
        d3n[3 * t + a] = acc;
      }
      for (int q = 0; q < 9; ++q) tCn[9 * t + q] = Cd[q];
    }
  }

  // Chamfer loss of vertex state f and its adjoint into aX
  double chamfer(int f, std::vector<T>& aX) {
    const T* x = Xf(f);
    double loss = 0;
    for (int q = 0; q < sc.nq; ++q) {
      const double* tq = sc.targets + 3 * q;
      T best = T(0); int bp = -1;
      for (int p = 0; p < nv; ++p) {
        const T dx0 = x[3 * p] - (T)tq[0], dy = x[3 * p + 1] - (T)tq[1], dz = x[3 * p + 2] - (T)tq[2];
        const T dd = (dx0 * dx0 + dy * dy + dz * dz) / T(3);
        if (bp < 0 || dd < best) { best = dd; bp = p; }
      }
      loss += (double)(best / (T)sc.nq);
      for (int a = 0; a < 3; ++a) aX[3 * bp + a] += T(2) / T(3) * (x[3 * bp + a] - (T)tq[a]) / (T)sc.nq;
    }
    return loss;
  }

  // reverse of substep f: (aX, aV, aC, atC, ad3) hold dL/d state f+1 on entry
  // and dL/d state f on return
  void backward(int f, std::vector<T>& aX, std::vector<T>& aV, std::vector<T>& aC, std::vector<T>& atC,
                std::vector<T>& ad3) {
    grid_of(f);
    const T* x = Xf(f); const T* C = Cvf(f); const T* tC = Ctf(f); const T* d3s = D3f(f);
    const T* tCn = Ctf(f + 1);
    std::vector<T> nX(aX.size(), T(0)), nV(aV.size(), T(0)), nC(aC.size(), T(0)), ntC(atC.size(), T(0)),
        nd3(ad3.size(), T(0));
    each_box_node([&](int, int, int, size_t n) { ga[3 * n] = ga[3 * n + 1] = ga[3 * n + 2] = T(0); });
    std::vector<T> axc((size_t)nt * 3, T(0)), avc((size_t)nt * 3, T(0));
    // ---- g2p adjoint, vertices: x' = x + dt v', v' = sum W g, C' = 4/dx sum W g (o - fx)^T
    for (int p = 0; p < nv; ++p) {
      Sten<T> s;
      stencil(x + 3 * p, inv_dx, G, s);
      T bv[3], bC[9];
      for (int a = 0; a < 3; ++a) { nX[3 * p + a] += aX[3 * p + a]; bv[a] = aV[3 * p + a] + dt * aX[3 * p + a]; }
      for (int q = 0; q < 9; ++q) bC[q] = aC[9 * p + q];
      gather_adj(s, bv, bC, nX.data() + 3 * p);
    }
    // ---- triangles: d3' = (I + M) d3, M = dt Cd + dt^2/2 Cd Cd; Cd = skew Ct + keep sym Ct
    for (int t = 0; t < nt; ++t) {
      const T* Cd = tCn + 9 * t;
      const T* d3 = d3s + 3 * t;
      const T* b3 = ad3.data() + 3 * t;
      T Mm[9];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          T cc = 0;
          for (int q = 0; q < 3; ++q) cc += Cd[3 * a + q] * Cd[3 * q + b];
          Mm[3 * a + b] = dt * Cd[3 * a + b] + T(0.5) * dt * dt * cc;
        }
      for (int b = 0; b < 3; ++b) {
        T acc = b3[b];
        for (int a = 0; a < 3; ++a) acc += Mm[3 * a + b] * b3[a];
        nd3[3 * t + b] += acc;
      }
      T Gm[9], bCd[9];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Gm[3 * a + b] = b3[a] * d3[b];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          T gc = 0, cg = 0;
          for (int q = 0; q < 3; ++q) { gc += Gm[3 * a + q] * Cd[3 * b + q]; cg += Cd[3 * q + a] * Gm[3 * q + b]; }
          bCd[3 * a + b] = atC[9 * t + 3 * a + b] + dt * Gm[3 * a + b] + T(0.5) * dt * dt * (gc + cg);
        }
      // Cd = skew(Ct) + keep sym(Ct); sym(Ct) = sym(Cd) / keep, from the stored Cd
      T bC[9];
      double gd = 0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const T sy = T(0.5) * (Cd[3 * a + b] + Cd[3 * b + a]) / keep;
          gd -= (double)(bCd[3 * a + b] * sy);
          bC[3 * a + b] = T(0.5) * (bCd[3 * a + b] - bCd[3 * b + a]) + keep * T(0.5) * (bCd[3 * a + b] + bCd[3 * b + a]);
        }
      g_damp += gd;
      T xc[3], vc[3];
      centroid(f, t, xc, vc);
      Sten<T> s;
      stencil(xc, inv_dx, G, s);
      const T zero3[3] = {0, 0, 0};
      gather_adj(s, zero3, bC, axc.data() + 3 * t);
    }
    // ---- grid adjoint
    const T r2g = (T)(sc.grip_radius * sc.grip_radius);
    (void)r2g;
    each_box_node([&](int, int, int, size_t n) {
      const T gout[3] = {ga[3 * n], ga[3 * n + 1], ga[3 * n + 2]};
      const T im = T(1) / (gm[n] + T(1e-9));
      const T vv[3] = {im * gp[3 * n], im * gp[3 * n + 1], im * gp[3 * n + 2]};
      T bvv[3] = {0, 0, 0};
      if (hit[n] >= 0) {
        double* gvel = g_vel.data() + ((size_t)f * sc.n_grip + hit[n]) * 3;
        for (int a = 0; a < 3; ++a) gvel[a] += (double)gout[a];
      } else {
        T gmu = 0;
        grid_bc_backward<T>(vv, bc[n], fr, gout, bvv, gmu);
        g_fr += (double)gmu;
      }
      for (int a = 0; a < 3; ++a) ap[3 * n + a] = im * bvv[a];
      am[n] = -im * (bvv[0] * vv[0] + bvv[1] * vv[1] + bvv[2] * vv[2]);
    });
    // ---- p2g adjoint, vertices
    const T* v = Vf(f);
    std::vector<T> afv((size_t)nv * 3, T(0));
    for (int p = 0; p < nv; ++p) {
      Sten<T> s;
      stencil(x + 3 * p, inv_dx, G, s);
      const T vt[3] = {v[3 * p], v[3 * p + 1] + gdv, v[3 * p + 2]};
      const T* Cp = C + 9 * p;
      const T* fp = fvert.data() + 3 * p;
      for (int oi = 0; oi < 3; ++oi)
        for (int oj = 0; oj < 3; ++oj)
          for (int ok = 0; ok < 3; ++ok) {
            const T W = s.w[0][oi] * s.w[1][oj] * s.w[2][ok];
            const T gW[3] = {s.dw[0][oi] * s.w[1][oj] * s.w[2][ok], s.w[0][oi] * s.dw[1][oj] * s.w[2][ok],
                             s.w[0][oi] * s.w[1][oj] * s.dw[2][ok]};
            const T dp[3] = {((T)oi - s.fx[0]) * dx, ((T)oj - s.fx[1]) * dx, ((T)ok - s.fx[2]) * dx};
            const size_t n = node(s.base[0] + oi, s.base[1] + oj, s.base[2] + ok);
            const T* bp = ap.data() + 3 * n;
            T pay = am[n] * mv;
            for (int a = 0; a < 3; ++a) {
              const T cd = Cp[3 * a] * dp[0] + Cp[3 * a + 1] * dp[1] + Cp[3 * a + 2] * dp[2];
              pay += bp[a] * (mv * vt[a] + mv * cd + fp[a]);
              nV[3 * p + a] += W * mv * bp[a];
              afv[3 * p + a] += W * bp[a];
              for (int b = 0; b < 3; ++b) nC[9 * p + 3 * a + b] += W * mv * bp[a] * dp[b];
            }
            for (int b = 0; b < 3; ++b) {
              T ct = 0;  // d(C dpos)/dx_b = -C[:, b]
              for (int a = 0; a < 3; ++a) ct += bp[a] * Cp[3 * a + b];
              nX[3 * p + b] += gW[b] * pay - W * mv * ct;
            }
          }
    }
    // ---- p2g adjoint, triangles: own-node momentum, mass, normal force; stress; corner forces
    const T kf = vol * dt;
    for (int t = 0; t < nt; ++t) {
      T xc[3], vc[3];
      centroid(f, t, xc, vc);
      Sten<T> s;
      stencil(xc, inv_dx, G, s);
      const T* Ca = tC + 9 * t;
      const T* d3 = d3s + 3 * t;
      const Stress<T>& sts = st[t];
      const M3<T>& P = sts.P;
      M3<T> bP;
      for (int q = 0; q < 9; ++q) bP.m[q] = T(0);
      T bxc[3] = {0, 0, 0}, bd3[3] = {0, 0, 0};
      for (int oi = 0; oi < 3; ++oi)
        for (int oj = 0; oj < 3; ++oj)
          for (int ok = 0; ok < 3; ++ok) {
            const T w0 = s.w[0][oi], w1 = s.w[1][oj], w2 = s.w[2][ok];
            const T e0 = s.dw[0][oi], e1 = s.dw[1][oj], e2 = s.dw[2][ok];
            const T W = w0 * w1 * w2;
            const T gW[3] = {e0 * w1 * w2, w0 * e1 * w2, w0 * w1 * e2};
            // Hessian of W (symmetric)
            const T H[9] = {s.ddw[0][oi] * w1 * w2, e0 * e1 * w2, e0 * w1 * e2,
                            e0 * e1 * w2, w0 * s.ddw[1][oj] * w2, w0 * e1 * e2,
                            e0 * w1 * e2, w0 * e1 * e2, w0 * w1 * s.ddw[2][ok]};
            const T gd = gW[0] * d3[0] + gW[1] * d3[1] + gW[2] * d3[2];
            const T dp[3] = {((T)oi - s.fx[0]) * dx, ((T)oj - s.fx[1]) * dx, ((T)ok - s.fx[2]) * dx};
            const size_t n = node(s.base[0] + oi, s.base[1] + oj, s.base[2] + ok);
            const T* bp = ap.data() + 3 * n;
            T pay = am[n] * mq, sP = 0;
            for (int a = 0; a < 3; ++a) {
              const T cd = Ca[3 * a] * dp[0] + Ca[3 * a + 1] * dp[1] + Ca[3 * a + 2] * dp[2];
              pay += bp[a] * (mq * vc[a] + mq * cd);
              avc[3 * t + a] += W * mq * bp[a];
              for (int b = 0; b < 3; ++b) ntC[9 * t + 3 * a + b] += W * mq * bp[a] * dp[b];
              bP.m[3 * a + 2] += -vol * dt * bp[a] * gd;
              sP += bp[a] * P.m[3 * a + 2];
            }
            for (int b = 0; b < 3; ++b) {
              T ct = 0, hd = 0;
              for (int a = 0; a < 3; ++a) { ct += bp[a] * Ca[3 * a + b]; hd += H[3 * b + a] * d3[a]; }
              bxc[b] += gW[b] * pay - W * mq * ct - vol * dt * sP * hd;
              bd3[b] += -vol * dt * sP * gW[b];
            }
          }
      // corner forces f1 = k P (r1 + r2), f2 = -k P r1, f3 = -k P r2
      M3<T> d, Fe;
      tri_d(f, t, d, Fe);
      const T* Di = D0i.data() + 9 * t;
      const T r1[3] = {Di[0], d.m[1], d.m[2]}, r2[3] = {Di[3], d.m[4], d.m[5]};
      const int* vi = sc.tris + 3 * t;
      const T* b1 = afv.data() + 3 * vi[0];
      const T* b2 = afv.data() + 3 * vi[1];
      const T* b3 = afv.data() + 3 * vi[2];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) bP.m[3 * a + b] += kf * (b1[a] * (r1[b] + r2[b]) - b2[a] * r1[b] - b3[a] * r2[b]);
      T br1[3], br2[3];
      for (int b = 0; b < 3; ++b) {
        br1[b] = kf * (P.m[b] * (b1[0] - b2[0]) + P.m[3 + b] * (b1[1] - b2[1]) + P.m[6 + b] * (b1[2] - b2[2]));
        br2[b] = kf * (P.m[b] * (b1[0] - b3[0]) + P.m[3 + b] * (b1[1] - b3[1]) + P.m[6 + b] * (b1[2] - b3[2]));
      }
      M3<T> bF;
      for (int q = 0; q < 9; ++q) bF.m[q] = T(0);
      T gmu = 0, gla = 0, gks = 0, gkc = 0;
      stress_backward<T>(sts, mu, la, ks, kc, bP, SVD_GRAD_EXACT, bF, gmu, gla, gks, gkc);
      const T E = (T)sc.E, nu = (T)sc.nu;
      const double dmu_dE = 1.0 / (2.0 * (1.0 + (double)nu)), dmu_dnu = -(double)E / (2.0 * (1.0 + nu) * (1.0 + nu));
      const double D = (1.0 + (double)nu) * (1.0 - 2.0 * (double)nu);
      const double dla_dE = nu / D, dla_dnu = (double)E * (1.0 + 2.0 * nu * nu) / (D * D);
      g_E += gmu * dmu_dE + gla * dla_dE;
      g_nu += gmu * dmu_dnu + gla * dla_dnu;
      g_ks += gks;
      g_kc += gkc;
      // dL/dd = dL/dF D0^-T + the uses of d in r1, r2
      T bd[9];
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k)
          bd[3 * r + k] = bF.m[3 * r] * Di[3 * k] + bF.m[3 * r + 1] * Di[3 * k + 1] + bF.m[3 * r + 2] * Di[3 * k + 2];
      bd[1] += br1[1]; bd[2] += br1[2]; bd[4] += br2[1]; bd[5] += br2[2];
      for (int a = 0; a < 3; ++a) {
        nX[3 * vi[1] + a] += bd[3 * a];
        nX[3 * vi[0] + a] -= bd[3 * a] + bd[3 * a + 1];
        nX[3 * vi[2] + a] += bd[3 * a + 1];
        nd3[3 * t + a] += bd[3 * a + 2] + bd3[a];
        const T bx = (bxc[a] + axc[3 * t + a]) / T(3), bvc = avc[3 * t + a] / T(3);
        for (int c = 0; c < 3; ++c) { nX[3 * vi[c] + a] += bx; nV[3 * vi[c] + a] += bvc; }
      }
    }
    aX.swap(nX); aV.swap(nV); aC.swap(nC); atC.swap(ntC); ad3.swap(nd3);
  }

  // adjoint of the APIC gather v = sum W g, C = 4/dx sum W g (o - fx)^T at a
  // stencil: scatters into ga and accumulates the position adjoint into bx
  void gather_adj(const Sten<T>& s, const T bv[3], const T bC[9], T* bx) {
    for (int oi = 0; oi < 3; ++oi)
      for (int oj = 0; oj < 3; ++oj)
        for (int ok = 0; ok < 3; ++ok) {
          const T W = s.w[0][oi] * s.w[1][oj] * s.w[2][ok];
          const T gW[3] = {s.dw[0][oi] * s.w[1][oj] * s.w[2][ok], s.w[0][oi] * s.dw[1][oj] * s.w[2][ok],
                           s.w[0][oi] * s.w[1][oj] * s.dw[2][ok]};
          const T dp[3] = {(T)oi - s.fx[0], (T)oj - s.fx[1], (T)ok - s.fx[2]};
          const size_t n = node(s.base[0] + oi, s.base[1] + oj, s.base[2] + ok);
          const T* g = gv.data() + 3 * n;
          T s1 = 0, wc[3] = {0, 0, 0};
          for (int a = 0; a < 3; ++a) {
            T cb = 0;
            for (int b = 0; b < 3; ++b) cb += bC[3 * a + b] * dp[b];
            const T wa = bv[a] + T(4) * inv_dx * cb;   // dL/dv_out(node) per unit weight
            ga[3 * n + a] += W * wa;
            s1 += g[a] * wa;
            for (int b = 0; b < 3; ++b) wc[b] += bC[3 * a + b] * g[a];
          }
          // d(o - fx)/dx = -inv_dx
          for (int b = 0; b < 3; ++b) bx[b] += gW[b] * s1 - T(4) * inv_dx * inv_dx * W * wc[b];
        }
  }
};

template <class T>
int run(const CpuScene* sc, int n_steps, double* loss, double* grads, double* gvel) {
  Rollout<T> r(*sc);
  if (n_steps > sc->n_steps) return 1;
  for (int f = 0; f < n_steps; ++f) r.forward(f);
  const size_t nv = sc->nv, nt = sc->nt;
  std::vector<T> aX(nv * 3, T(0)), aV(nv * 3, T(0)), aC(nv * 9, T(0)), atC(nt * 9, T(0)), ad3(nt * 3, T(0));
  *loss = r.chamfer(n_steps, aX);
  for (int f = n_steps - 1; f >= 0; --f) r.backward(f, aX, aV, aC, atC, ad3);
  grads[0] = r.g_E; grads[1] = r.g_nu; grads[2] = r.g_ks; grads[3] = r.g_kc; grads[4] = r.g_fr; grads[5] = r.g_damp;
  if (gvel) std::memcpy(gvel, r.g_vel.data(), sizeof(double) * r.g_vel.size());
  return 0;
}

}  // namespace

extern "C" {

// One cloth: forward rollout of n_steps substeps, Chamfer loss of the final
// vertex state, and the reverse pass; grads[6] = dL/d(E, nu, k_s, k_c,
// friction, damping); gvel (may be NULL): dL/d gripper velocities.
// double_precision != 0 runs the float64 build.
int cpu_rollout_grad(const CpuScene* sc, int32_t n_steps, int32_t double_precision, double* loss, double* grads,
                     double* gvel) {
  return double_precision ? run<double>(sc, n_steps, loss, grads, gvel) : run<float>(sc, n_steps, loss, grads, gvel);
}

// n cloths, one OpenMP thread each (n_threads threads), float32: the timed
// CPU baseline.  Returns 0 when every rollout ran.
int cpu_rollouts(const CpuScene* scenes, int32_t n, int32_t n_steps, int32_t n_threads, double* losses,
                 double* grads) {
  int bad = 0;
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 1) reduction(+ : bad)
  for (int i = 0; i < n; ++i) bad += run<float>(scenes + i, n_steps, losses + i, grads + 6 * (size_t)i, nullptr);
  return bad;
}

}
