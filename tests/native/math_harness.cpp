// Host build of diffcp_b200/csrc/cloth_math.cuh for the CPU tests: exposes the
// per-particle forward/adjoint math through plain C entry points so that the
// tests can compare it with torch.autograd of the oracle.  Not product code.
#include "../../diffcp_b200/csrc/cloth_math.cuh"

using namespace dcp;

// The kernels pass F - I; form it in double so the float build sees the exact deviation.
template <class T>
static M3<T> deviation(const double* F) {
  M3<T> e;
  for (int i = 0; i < 9; ++i) e.m[i] = T(F[i] - ((i % 4 == 0) ? 1.0 : 0.0));
  return e;
}

template <class T>
static void stress_fwd_T(const double* F, const double* prm, double* P) {
  M3<T> f = deviation<T>(F);
  Stress<T> st;
  stress_forward<T>(f, T(prm[0]), T(prm[1]), T(prm[2]), T(prm[3]), st);
  for (int i = 0; i < 9; ++i) P[i] = double(st.P.m[i]);
}

template <class T>
static void stress_bwd_T(const double* F, const double* prm, const double* gP, int mode, double* gF, double* gprm) {
  M3<T> f = deviation<T>(F), gp, gf;
  for (int i = 0; i < 9; ++i) gp.m[i] = T(gP[i]);
  Stress<T> st;
  stress_forward<T>(f, T(prm[0]), T(prm[1]), T(prm[2]), T(prm[3]), st);
  T gmu = 0, gla = 0, gks = 0, gkc = 0;
  stress_backward<T>(st, T(prm[0]), T(prm[1]), T(prm[2]), T(prm[3]), gp, mode, gf, gmu, gla, gks, gkc);
  for (int i = 0; i < 9; ++i) gF[i] = double(gf.m[i]);
  gprm[0] = double(gmu); gprm[1] = double(gla); gprm[2] = double(gks); gprm[3] = double(gkc);
}

extern "C" {
void h_stress_fwd(int n, int dbl, const double* F, const double* prm, double* P) {
  for (int i = 0; i < n; ++i) {
    if (dbl) stress_fwd_T<double>(F + 9 * i, prm + 4 * i, P + 9 * i);
    else stress_fwd_T<float>(F + 9 * i, prm + 4 * i, P + 9 * i);
  }
}
void h_stress_bwd(int n, int dbl, const double* F, const double* prm, const double* gP, int mode, double* gF,
                  double* gprm) {
  for (int i = 0; i < n; ++i) {
    if (dbl) stress_bwd_T<double>(F + 9 * i, prm + 4 * i, gP + 9 * i, mode, gF + 9 * i, gprm + 4 * i);
    else stress_bwd_T<float>(F + 9 * i, prm + 4 * i, gP + 9 * i, mode, gF + 9 * i, gprm + 4 * i);
  }
}
void h_svd2(int n, const double* A, double* U, double* S, double* V) {
  for (int i = 0; i < n; ++i) svd2<double>(A + 4 * i, U + 4 * i, S + 2 * i, V + 4 * i);
}
void h_svd2_bwd(int n, const double* gU, const double* gV, const double* U, const double* S, const double* V,
                double* gA) {
  for (int i = 0; i < n; ++i)
    svd2_backward_clamped<double>(gU + 4 * i, gV + 4 * i, U + 4 * i, S + 2 * i, V + 4 * i, gA + 4 * i);
}
void h_grid_bc(int n, const double* v, const int* ijk, int G, int bound, double mu, double* out) {
  for (int i = 0; i < n; ++i) grid_bc<double>(v + 3 * i, ijk[3 * i], ijk[3 * i + 1], ijk[3 * i + 2], G, bound, mu, out + 3 * i);
}
void h_grid_bc_bwd(int n, const double* v, const int* ijk, int G, int bound, double mu, const double* gout,
                   double* gv, double* gmu) {
  for (int i = 0; i < n; ++i) {
    double o[3];
    NodeBC<double> r = grid_bc<double>(v + 3 * i, ijk[3 * i], ijk[3 * i + 1], ijk[3 * i + 2], G, bound, mu, o);
    double g = 0;
    grid_bc_backward<double>(v + 3 * i, r, mu, gout + 3 * i, gv + 3 * i, g);
    gmu[i] = g;
  }
}
}
