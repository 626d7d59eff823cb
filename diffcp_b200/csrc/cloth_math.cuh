// Per-particle math of the codimensional-cloth MPM substep and its hand-written
// adjoints.  Header-only and __host__ __device__: the CUDA kernels use it, and
// the CPU test harness compiles the same code with g++ to check every adjoint
// against torch.autograd of the oracle.
//
// Reference (denzelzheng/diffcp): src/simulation.py.
//   quadratic B-spline stencil          simulation.py:140-142, 197
//   Gram-Schmidt QR                      simulation.py:123-135
//   in-plane 2x2 SVD / rotation factor   simulation.py:39-42, 235
//   clamped 2x2 SVD backward             simulation.py:44-50, 71-94
//   triangle stress quadrature_P         simulation.py:214-240
//   grid boundary conditions             simulation.py:274-302
#pragma once

#ifdef __CUDACC__
#define DCP_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#define DCP_HD inline
#endif

namespace dcp {

#ifndef __CUDACC__
using std::sqrt;
using std::fabs;
#endif

// ------------------------------------------------------------------ vectors
template <class T> struct V3 {
  T x, y, z;
};
template <class T> DCP_HD V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> DCP_HD V3<T> operator+(V3<T> a, V3<T> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> DCP_HD V3<T> operator-(V3<T> a, V3<T> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> DCP_HD V3<T> operator*(T s, V3<T> a) { return v3(s * a.x, s * a.y, s * a.z); }
template <class T> DCP_HD V3<T> operator/(V3<T> a, T s) { return v3(a.x / s, a.y / s, a.z / s); }
template <class T> DCP_HD T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> DCP_HD void addto(V3<T>& a, V3<T> b) { a.x += b.x; a.y += b.y; a.z += b.z; }

// Row-major 3x3: m[3*r + c].
template <class T> struct M3 {
  T m[9];
};
template <class T> DCP_HD V3<T> col(const M3<T>& A, int c) { return v3(A.m[c], A.m[3 + c], A.m[6 + c]); }
template <class T> DCP_HD M3<T> matmul(const M3<T>& A, const M3<T>& B) {
  M3<T> C;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      C.m[3 * r + c] = A.m[3 * r] * B.m[c] + A.m[3 * r + 1] * B.m[3 + c] + A.m[3 * r + 2] * B.m[6 + c];
  return C;
}
template <class T> DCP_HD M3<T> transpose(const M3<T>& A) {
  M3<T> B;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) B.m[3 * r + c] = A.m[3 * c + r];
  return B;
}
template <class T> DCP_HD V3<T> matvec(const M3<T>& A, V3<T> v) {
  return v3(A.m[0] * v.x + A.m[1] * v.y + A.m[2] * v.z, A.m[3] * v.x + A.m[4] * v.y + A.m[5] * v.z,
            A.m[6] * v.x + A.m[7] * v.y + A.m[8] * v.z);
}
template <class T> DCP_HD V3<T> matTvec(const M3<T>& A, V3<T> v) {
  return v3(A.m[0] * v.x + A.m[3] * v.y + A.m[6] * v.z, A.m[1] * v.x + A.m[4] * v.y + A.m[7] * v.z,
            A.m[2] * v.x + A.m[5] * v.y + A.m[8] * v.z);
}

// ------------------------------------------------------------ B-spline
// 1-D quadratic B-spline weights at offsets 0,1,2 from the base node for the
// fractional coordinate fx in cell units, and their derivatives d/dfx.
template <class T> DCP_HD void bspline(T fx, T w[3], T dw[3]) {
  const T a = T(1.5) - fx, b = fx - T(1.0), c = fx - T(0.5);
  w[0] = T(0.5) * a * a;
  w[1] = T(0.75) - b * b;
  w[2] = T(0.5) * c * c;
  dw[0] = fx - T(1.5);
  dw[1] = T(2) * (T(1.0) - fx);
  dw[2] = fx - T(0.5);
}
// Second derivative d^2 w / d fx^2 at offsets 0,1,2.
template <class T> DCP_HD T bspline_dd(int o) { return o == 1 ? T(-2) : T(1); }

// ------------------------------------------------------- Gram-Schmidt QR
// Classical Gram-Schmidt with norm(eps) = sqrt(|v|^2 + 1e-9) as in
// simulation.py:123-135.  R = Q^-1 F is the upper-triangular coefficient
// matrix [[n1, r01, r02], [0, n2, r12], [0, 0, n3]] (exactly, as a function of F).
//
// The input is the deviation Ed = F - I.  Cloth strains are small, so the
// quantities that drive the stress (n_i - 1, J - 1, 1 - R22) would lose most
// of their float32 digits if formed as differences of O(1) numbers; here they
// are evaluated from Ed through exact identities instead:
//   |f1|^2 - 1 = 2 e1.x + |e1|^2,  f2.f1 = e2.x + e1.y + e1.e2, ...
//   |h2|^2 - 1 = (|f2|^2 - 1) - r01^2 (2 - |q1|^2), and likewise for h3.
// Under strong compression a column's squared norm falls towards 0, where
// 1 + (identity) loses its relative precision and rounding can even make it
// negative (a NaN under the square root); below 1/4 the squared norm is
// therefore summed from the column's components, which is never negative.
// The backward pass differentiates n = sqrt(|h|^2 + eps) through h and does
// not depend on which form gave the value.
template <class T> struct QR {
  V3<T> f1, f2, f3, q1, q2, q3, h2, h3;
  T n1, n2, n3, r01, r02, r12;
  T a1, a2, a3;  // n_i - 1
};
// n = sqrt(|h|^2 + eps) and a = n - 1 from t = |h|^2 - 1 (small-strain
// identity) or, when |h|^2 < 1/4, from |h|^2 summed over h's components.
template <class T> DCP_HD void column_norm(T t, const V3<T>& h, T eps, T& n, T& a) {
  if (T(1) + t < T(0.25)) {
    n = sqrt(dot(h, h) + eps);
    a = n - T(1);
  } else {
    n = sqrt(T(1) + (t + eps));
    a = (t + eps) / (n + T(1));
  }
}
template <class T> DCP_HD void qr_forward(const M3<T>& Ed, QR<T>& s) {
  const T eps = T(1e-9);
  const V3<T> e1 = col(Ed, 0), e2 = col(Ed, 1), e3 = col(Ed, 2);
  s.f1 = v3(T(1) + e1.x, e1.y, e1.z);
  s.f2 = v3(e2.x, T(1) + e2.y, e2.z);
  s.f3 = v3(e3.x, e3.y, T(1) + e3.z);
  column_norm(T(2) * e1.x + dot(e1, e1), s.f1, eps, s.n1, s.a1);      // |f1|^2 - 1
  s.q1 = s.f1 / s.n1;
  const T q11 = T(1) - eps / (s.n1 * s.n1);           // |q1|^2
  s.r01 = (e2.x + e1.y + dot(e1, e2)) / s.n1;         // f2 . q1
  s.h2 = s.f2 - s.r01 * s.q1;
  column_norm((T(2) * e2.y + dot(e2, e2)) - s.r01 * s.r01 * (T(2) - q11), s.h2, eps, s.n2, s.a2);  // |h2|^2 - 1
  s.q2 = s.h2 / s.n2;
  const T q22 = T(1) - eps / (s.n2 * s.n2);           // |q2|^2
  const T q12 = s.r01 * (T(1) - q11) / s.n2;          // q1 . q2
  s.r02 = (e3.x + e1.z + dot(e1, e3)) / s.n1;         // f3 . q1
  s.r12 = ((e3.y + e2.z + dot(e2, e3)) - s.r01 * s.r02) / s.n2;   // f3 . q2
  s.h3 = s.f3 - s.r02 * s.q1 - s.r12 * s.q2;
  column_norm((T(2) * e3.z + dot(e3, e3)) - s.r02 * s.r02 * (T(2) - q11) - s.r12 * s.r12 * (T(2) - q22) +
                  T(2) * s.r02 * s.r12 * q12, s.h3, eps, s.n3, s.a3);                     // |h3|^2 - 1
  s.q3 = s.h3 / s.n3;
}
// Adjoint of y = h / n with n = sqrt(|h|^2 + eps): returns dL/dh.
template <class T> DCP_HD V3<T> normalize_adj(V3<T> h, T n, V3<T> gy, T gn) {
  const T n3 = n * n * n;
  const T k = dot(gy, h) / n3;
  return v3(gy.x / n - k * h.x + gn * h.x / n, gy.y / n - k * h.y + gn * h.y / n, gy.z / n - k * h.z + gn * h.z / n);
}
// Reverse of qr_forward given dL/dq1..3 and dL/d(upper-triangular R entries).
template <class T>
DCP_HD void qr_backward(const QR<T>& s, V3<T> gq1, V3<T> gq2, V3<T> gq3, T gn1, T gr01, T gr02, T gn2, T gr12, T gn3,
                        M3<T>& gF) {
  V3<T> gf1 = v3(T(0), T(0), T(0)), gf2 = gf1, gf3 = gf1;
  const V3<T> gh3 = normalize_adj(s.h3, s.n3, gq3, gn3);
  addto(gf3, gh3);
  gr02 -= dot(gh3, s.q1);
  gq1 = gq1 - s.r02 * gh3;
  gr12 -= dot(gh3, s.q2);
  gq2 = gq2 - s.r12 * gh3;
  addto(gf3, gr12 * s.q2);
  addto(gq2, gr12 * s.f3);
  addto(gf3, gr02 * s.q1);
  addto(gq1, gr02 * s.f3);
  const V3<T> gh2 = normalize_adj(s.h2, s.n2, gq2, gn2);
  addto(gf2, gh2);
  gr01 -= dot(gh2, s.q1);
  gq1 = gq1 - s.r01 * gh2;
  addto(gf2, gr01 * s.q1);
  addto(gq1, gr01 * s.f2);
  addto(gf1, normalize_adj(s.f1, s.n1, gq1, gn1));
  gF.m[0] = gf1.x; gF.m[3] = gf1.y; gF.m[6] = gf1.z;
  gF.m[1] = gf2.x; gF.m[4] = gf2.y; gF.m[7] = gf2.z;
  gF.m[2] = gf3.x; gF.m[5] = gf3.y; gF.m[8] = gf3.z;
}

// ------------------------------------------------------ 2x2 SVD (Taichi)
// U, Sigma, V of a 2x2 matrix A (row-major a[4]) in the convention of the
// reference's ti.svd: rotation polar factor from (A00 + A11, A10 - A01), one
// Jacobi rotation of the symmetric remainder (skipped when |S01| < 1e-5),
// singular values sorted descending, V kept a rotation; U = Rpolar V.
template <class T> DCP_HD void svd2(const T a[4], T U[4], T sig[2], T V[4]) {
  const T x = a[0] + a[3], y = a[2] - a[1];
  const T sc = T(1) / sqrt(x * x + y * y);
  const T c0 = x * sc, s0 = y * sc;
  // S = Rp^T A, Rp = [[c0, -s0], [s0, c0]]
  const T S00 = c0 * a[0] + s0 * a[2], S01 = c0 * a[1] + s0 * a[3];
  const T S11 = -s0 * a[1] + c0 * a[3];
  T c, s, s1, s2;
  if (fabs(S01) < T(1e-5)) {
    c = T(1); s = T(0); s1 = S00; s2 = S11;
  } else {
    const T tau = T(0.5) * (S00 - S11);
    const T w = sqrt(tau * tau + S01 * S01);
    const T t = tau > T(0) ? S01 / (tau + w) : S01 / (tau - w);
    c = T(1) / sqrt(t * t + T(1));
    s = -t * c;
    s1 = c * c * S00 - T(2) * c * s * S01 + s * s * S11;
    s2 = s * s * S00 + T(2) * c * s * S01 + c * c * S11;
  }
  if (s1 < s2) {
    const T tmp = s1; s1 = s2; s2 = tmp;
    V[0] = -s; V[1] = c; V[2] = -c; V[3] = -s;
  } else {
    V[0] = c; V[1] = s; V[2] = -s; V[3] = c;
  }
  sig[0] = s1; sig[1] = s2;
  U[0] = c0 * V[0] - s0 * V[2]; U[1] = c0 * V[1] - s0 * V[3];
  U[2] = s0 * V[0] + c0 * V[2]; U[3] = s0 * V[1] + c0 * V[3];
}

template <class T> DCP_HD T clamp_ref(T a) {  // simulation.py:44-50
  if (a >= T(0)) return a > T(1e-6) ? a : T(1e-6);
  return a < T(-1e-6) ? a : T(-1e-6);
}

template <class T> DCP_HD void mm2(const T A[4], const T B[4], T C[4]) {
  C[0] = A[0] * B[0] + A[1] * B[2]; C[1] = A[0] * B[1] + A[1] * B[3];
  C[2] = A[2] * B[0] + A[3] * B[2]; C[3] = A[2] * B[1] + A[3] * B[3];
}
template <class T> DCP_HD void mtm2(const T A[4], const T B[4], T C[4]) {  // A^T B
  C[0] = A[0] * B[0] + A[2] * B[2]; C[1] = A[0] * B[1] + A[2] * B[3];
  C[2] = A[1] * B[0] + A[3] * B[2]; C[3] = A[1] * B[1] + A[3] * B[3];
}
template <class T> DCP_HD void mmt2(const T A[4], const T B[4], T C[4]) {  // A B^T
  C[0] = A[0] * B[0] + A[1] * B[1]; C[1] = A[0] * B[2] + A[1] * B[3];
  C[2] = A[2] * B[0] + A[3] * B[1]; C[3] = A[2] * B[2] + A[3] * B[3];
}

// backward_inplane_svd (simulation.py:71-88) with gSigma = 0: returns dL/dA.
template <class T>
DCP_HD void svd2_backward_clamped(const T gU[4], const T gV[4], const T U[4], const T sig[2], const T V[4], T gA[4]) {
  const T sa = sig[0] * sig[0], sb = sig[1] * sig[1];
  const T F01 = T(1) / clamp_ref(sb - sa), F10 = T(1) / clamp_ref(sa - sb);
  T t1[4], t2[4], XU[4], XV[4];
  mtm2(U, gU, t1);  // U^T gU
  mtm2(gU, U, t2);  // gU^T U
  XU[0] = T(0); XU[1] = F01 * (t1[1] - t2[1]); XU[2] = F10 * (t1[2] - t2[2]); XU[3] = T(0);
  mtm2(V, gV, t1);
  mtm2(gV, V, t2);
  XV[0] = T(0); XV[1] = F01 * (t1[1] - t2[1]); XV[2] = F10 * (t1[2] - t2[2]); XV[3] = T(0);
  // u_term = U ((F o XU) S) V^T ; v_term = U (S ((F o XV) V^T))
  T a[4], b[4];
  a[0] = XU[0] * sig[0]; a[1] = XU[1] * sig[1]; a[2] = XU[2] * sig[0]; a[3] = XU[3] * sig[1];
  mmt2(XV, V, b);
  // u_term = U a V^T ; v_term = U (S b)
  T uaV[4], Ua[4];
  mm2(U, a, Ua);
  mmt2(Ua, V, uaV);
  T Sb[4] = {sig[0] * b[0], sig[0] * b[1], sig[1] * b[2], sig[1] * b[3]};
  T USb[4];
  mm2(U, Sb, USb);
  gA[0] = uaV[0] + USb[0]; gA[1] = uaV[1] + USb[1]; gA[2] = uaV[2] + USb[2]; gA[3] = uaV[3] + USb[3];
}

// ----------------------------------------------------- triangle stress
// quadrature_P = Q pad(P_fc) + Q A R^-T (simulation.py:214-240) with the
// in-plane block Fh = R[0:2, 0:2] = [[n1, r01], [0, n2]] (compute_inplane_F_tmp,
// simulation.py:24-28), fixed-corotated P_fc = 2mu(Fh - Rp) + la (J-1) J Fh^-T
// and J Fh^-T = cof(Fh).
enum SvdGrad { SVD_GRAD_EXACT = 0, SVD_GRAD_REFERENCE = 1 };

template <class T> struct Stress {
  QR<T> qr;
  T c, s, rr;        // rotation factor Rp = [[c, -s], [s, c]], rr = |(x, y)|
  T cm1;             // c - 1
  T J, Jm1;          // det Fh and det Fh - 1
  T Ri[6];           // R^-1 upper triangle: i00 i01 i02 i11 i12 i22
  T A[6];            // symmetric A: a00 a01 a02 a11 a12 a22
  bool contact;      // R22 <= 1
  M3<T> M;           // pad(P_fc) + A R^-T
  M3<T> P;
};

// ``Ed`` is F - I (see qr_forward).
template <class T> DCP_HD void stress_forward(const M3<T>& Ed, T mu, T la, T ks, T kc, Stress<T>& st) {
  QR<T>& q = st.qr;
  qr_forward(Ed, q);
  const T n1 = q.n1, n2 = q.n2, n3 = q.n3, r01 = q.r01, r02 = q.r02, r12 = q.r12;
  const T a1 = q.a1, a2 = q.a2, a3 = q.a3;
  // A (simulation.py:215-229); the first write of A[0,0] (line 216) is dead.
  st.contact = a3 <= T(0);
  st.A[0] = ks * r02 * r02;
  st.A[1] = ks * r02 * r12;
  st.A[2] = ks * r02 * n3;
  st.A[3] = ks * r12 * r12;
  st.A[4] = ks * r12 * n3;
  st.A[5] = st.contact ? (-kc) * (a3 * a3) * n3 : T(0);
  // R^-1 of the upper-triangular R
  const T i00 = T(1) / n1, i11 = T(1) / n2, i22 = T(1) / n3;
  st.Ri[0] = i00;
  st.Ri[1] = -r01 * i00 * i11;
  st.Ri[2] = (r01 * r12 - r02 * n2) * i00 * i11 * i22;
  st.Ri[3] = i11;
  st.Ri[4] = -r12 * i11 * i22;
  st.Ri[5] = i22;
  // rotation factor of Fh = [[n1, r01], [0, n2]]: (c, s) = (x, y) / |(x, y)|,
  // x = n1 + n2 > 0, y = -r01; c - 1 = -tau^2 / (w (1 + w)), tau = y / x.
  const T x = T(2) + (a1 + a2), y = -r01;
  const T tau = y / x;
  const T w = sqrt(T(1) + tau * tau);
  st.rr = x * w;
  st.c = T(1) / w;
  st.s = tau / w;
  st.cm1 = -(tau * tau) / (w * (T(1) + w));
  st.J = n1 * n2;
  st.Jm1 = a1 + a2 + a1 * a2;
  const T lj = la * st.Jm1;
  const T p00 = T(2) * mu * (a1 - st.cm1) + lj * n2;
  const T p01 = T(2) * mu * (r01 + st.s);
  const T p10 = T(2) * mu * (-st.s) + lj * (-r01);
  const T p11 = T(2) * mu * (a2 - st.cm1) + lj * n1;
  // M = pad(P_fc) + A R^-T, (A R^-T)[r][c] = sum_{k>=c} A[r][k] Rinv[c][k]
  const T* a = st.A;
  const T Ar[3][3] = {{a[0], a[1], a[2]}, {a[1], a[3], a[4]}, {a[2], a[4], a[5]}};
  const T Rinv[3][3] = {{st.Ri[0], st.Ri[1], st.Ri[2]}, {T(0), st.Ri[3], st.Ri[4]}, {T(0), T(0), st.Ri[5]}};
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T acc = T(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) acc += Ar[r][k] * Rinv[c][k];
      st.M.m[3 * r + c] = acc;
    }
  st.M.m[0] += p00; st.M.m[1] += p01; st.M.m[3] += p10; st.M.m[4] += p11;
  // P = Q M, Q = [q1 q2 q3]
  M3<T> Q;
  Q.m[0] = q.q1.x; Q.m[1] = q.q2.x; Q.m[2] = q.q3.x;
  Q.m[3] = q.q1.y; Q.m[4] = q.q2.y; Q.m[5] = q.q3.y;
  Q.m[6] = q.q1.z; Q.m[7] = q.q2.z; Q.m[8] = q.q3.z;
  st.P = matmul(Q, st.M);
}

// Reverse of stress_forward: given dL/dP, accumulate dL/dF and the parameter
// adjoints (dL/dmu, dL/dla, dL/dks, dL/dkc).  ``svd_grad`` selects the
// derivative of the rotation factor: the closed-form derivative of the polar
// rotation (exact), or the reference's clamped SVD backward evaluated in
// double precision near degenerate singular values.
template <class T>
DCP_HD void stress_backward(const Stress<T>& st, T mu, T la, T ks, T kc, const M3<T>& gP, int svd_grad, M3<T>& gF,
                            T& gmu, T& gla, T& gks, T& gkc) {
  const QR<T>& q = st.qr;
  const T n1 = q.n1, n2 = q.n2, n3 = q.n3, r01 = q.r01, r02 = q.r02, r12 = q.r12;
  M3<T> Q;
  Q.m[0] = q.q1.x; Q.m[1] = q.q2.x; Q.m[2] = q.q3.x;
  Q.m[3] = q.q1.y; Q.m[4] = q.q2.y; Q.m[5] = q.q3.y;
  Q.m[6] = q.q1.z; Q.m[7] = q.q2.z; Q.m[8] = q.q3.z;
  const M3<T> gM = matmul(transpose(Q), gP);
  const M3<T> gQ = matmul(gP, transpose(st.M));
  V3<T> gq1 = col(gQ, 0), gq2 = col(gQ, 1), gq3 = col(gQ, 2);
  const T g00 = gM.m[0], g01 = gM.m[1], g10 = gM.m[3], g11 = gM.m[4];
  // --- A R^-T part
  const T* a = st.A;
  const T Ar[3][3] = {{a[0], a[1], a[2]}, {a[1], a[3], a[4]}, {a[2], a[4], a[5]}};
  const T Rinv[3][3] = {{st.Ri[0], st.Ri[1], st.Ri[2]}, {T(0), st.Ri[3], st.Ri[4]}, {T(0), T(0), st.Ri[5]}};
  T gA[3][3];   // gM Rinv
  T AgM[3][3];  // A gM  (= gradient w.r.t. R^-T)
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T acc = T(0), acc2 = T(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        acc += gM.m[3 * r + k] * Rinv[k][c];
        acc2 += Ar[r][k] * gM.m[3 * k + c];
      }
      gA[r][c] = acc;
      AgM[r][c] = acc2;
    }
  // gR = -R^-T (A gM)^T R^-T  ;  (R^-T)[i][j] = Rinv[j][i]
  T tmp[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      T acc = T(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) acc += Rinv[k][i] * AgM[j][k];
      tmp[i][j] = acc;
    }
  T gR[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      T acc = T(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) acc += tmp[i][k] * Rinv[j][k];
      gR[i][j] = -acc;
    }
  T gn1 = gR[0][0], gr01 = gR[0][1], gr02 = gR[0][2], gn2 = gR[1][1], gr12 = gR[1][2], gn3 = gR[2][2];
  // A entries
  const T s01 = gA[0][1] + gA[1][0], s02 = gA[0][2] + gA[2][0], s12 = gA[1][2] + gA[2][1];
  gks += gA[0][0] * r02 * r02 + s01 * r02 * r12 + s02 * r02 * n3 + gA[1][1] * r12 * r12 + s12 * r12 * n3;
  gr02 += ks * (T(2) * r02 * gA[0][0] + r12 * s01 + n3 * s02);
  gr12 += ks * (r02 * s01 + T(2) * r12 * gA[1][1] + n3 * s12);
  gn3 += ks * (r02 * s02 + r12 * s12);
  if (st.contact) {
    const T om = -st.qr.a3;  // 1 - n3
    gn3 += gA[2][2] * (-kc) * (om * om - T(2) * om * n3);
    gkc += gA[2][2] * (-(om * om) * n3);
  }
  // --- fixed-corotated in-plane part
  const T c = st.c, s = st.s;
  gmu += T(2) * (g00 * (st.qr.a1 - st.cm1) + g01 * (r01 + s) + g10 * (-s) + g11 * (st.qr.a2 - st.cm1));
  gla += st.Jm1 * (g00 * n2 + g10 * (-r01) + g11 * n1);
  // direct Fh term
  gn1 += T(2) * mu * g00;
  gr01 += T(2) * mu * g01;
  gn2 += T(2) * mu * g11;
  // la (J-1) cof(Fh): J = n1 n2, cof = [[n2, 0], [-r01, n1]]
  const T gJ = la * (g00 * n2 + g10 * (-r01) + g11 * n1);
  gn1 += gJ * n2;
  gn2 += gJ * n1;
  const T lj = la * st.Jm1;
  gn2 += lj * g00;
  gr01 -= lj * g10;
  gn1 += lj * g11;
  // rotation factor, dL/dRp = -2 mu gPfc
  const T gRp[4] = {T(-2) * mu * g00, T(-2) * mu * g01, T(-2) * mu * g10, T(-2) * mu * g11};
  if (svd_grad == SVD_GRAD_EXACT) {
    const T gc = gRp[0] + gRp[3], gs = gRp[2] - gRp[1];
    const T gth = -s * gc + c * gs;
    const T x = n1 + n2, y = -r01;
    const T r2 = st.rr * st.rr;
    const T gx = -y * gth / r2, gy = x * gth / r2;
    gn1 += gx;
    gn2 += gx;
    gr01 -= gy;  // y = Fh10 - Fh01 with Fh01 = r01
  } else {
    // The reference's clamped SVD backward, in double precision: its
    // 1/(s_j - s_i) factors cancel catastrophically in float32 when the
    // in-plane singular values are close, which is the common case for cloth.
    const double fh[4] = {double(n1), double(r01), 0.0, double(n2)};
    double U[4], sig[2], V[4];
    svd2<double>(fh, U, sig, V);
    const double gr[4] = {double(gRp[0]), double(gRp[1]), double(gRp[2]), double(gRp[3])};
    double gU[4], gV[4];
    mm2<double>(gr, V, gU);   // gU = gRp V
    mtm2<double>(gr, U, gV);  // gV = gRp^T U
    double gfh[4];
    svd2_backward_clamped<double>(gU, gV, U, sig, V, gfh);
    gn1 += T(gfh[0]);
    gr01 += T(gfh[1]);
    gn2 += T(gfh[3]);
  }
  qr_backward(q, gq1, gq2, gq3, gn1, gr01, gr02, gn2, gr12, gn3, gF);
}

// ---------------------------------------------------------- grid update
// simulation.py:276-302 on one node: v = p / (m + 1e-9) then sticky walls on
// x, z and the y-top, a slip floor (y < bound, vy < 0 -> vy = 0) with optional
// Coulomb friction mu_g on the tangential velocity (mu_g = 0 is the reference).
// Returns 0 = free, 1 = stuck (all zero), 2 = floor.
template <class T> struct NodeBC {
  int kind;
  T scale;   // friction factor on (vx, vz) when kind == 2
  T vt;      // |(vx, vz)| before friction
};
template <class T>
DCP_HD NodeBC<T> grid_bc(const T v[3], int i, int j, int k, int G, int bound, T mu_g, T out[3]) {
  NodeBC<T> r;
  r.kind = 0;
  r.scale = T(1);
  r.vt = T(0);
  bool zero = (i < bound && v[0] < T(0)) || (i > G - bound && v[0] > T(0)) || (k < bound && v[2] < T(0)) ||
              (k > G - bound && v[2] > T(0));
  if (zero) {
    r.kind = 1;
    out[0] = out[1] = out[2] = T(0);
    return r;
  }
  out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
  if (j < bound && v[1] < T(0)) {
    r.kind = 2;
    const T vt2 = v[0] * v[0] + v[2] * v[2];
    if (vt2 > T(0)) {
      r.vt = sqrt(vt2);
      T sc = T(1) - mu_g * (-v[1]) / r.vt;
      r.scale = sc > T(0) ? sc : T(0);
      out[0] = v[0] * r.scale;
      out[2] = v[2] * r.scale;
    }
    out[1] = T(0);
    return r;
  }
  if (j > G - bound && v[1] > T(0)) {
    r.kind = 1;
    out[0] = out[1] = out[2] = T(0);
  }
  return r;
}
// Adjoint of grid_bc: dL/dv (pre-BC) from dL/dout; accumulates dL/dmu_g.
template <class T>
DCP_HD void grid_bc_backward(const T v[3], const NodeBC<T>& r, T mu_g, const T gout[3], T gv[3], T& gmu) {
  if (r.kind == 1) {
    gv[0] = gv[1] = gv[2] = T(0);
    return;
  }
  if (r.kind == 0) {
    gv[0] = gout[0]; gv[1] = gout[1]; gv[2] = gout[2];
    return;
  }
  gv[1] = T(0);
  if (r.vt > T(0)) {
    if (r.scale > T(0)) {
      // written with the unit tangent t and 1 - scale = mu |vn| / |vt|, both
      // bounded, so that tiny tangential speeds cannot overflow
      const T tx = v[0] / r.vt, tz = v[2] / r.vt;
      const T gh = gout[0] * tx + gout[2] * tz;
      const T one_m = T(1) - r.scale;
      gv[0] = r.scale * gout[0] + one_m * gh * tx;
      gv[2] = r.scale * gout[2] + one_m * gh * tz;
      gv[1] = mu_g * gh;
      gmu += v[1] * gh;
    } else {
      gv[0] = gv[2] = T(0);
    }
  } else {
    gv[0] = gout[0];
    gv[2] = gout[2];
  }
}

}  // namespace dcp
