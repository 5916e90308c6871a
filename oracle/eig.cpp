// Hermitian eigensolver for the oracle (test infrastructure only).
//
// The reference diagonalises the dynamical matrix with Eigen 3.4.0's
// SelfAdjointEigenSolver (src/harmonic/phonon_h0.cpp:863, pinned at
// lib/CMakeLists.txt:48), i.e. Householder reduction to a real tridiagonal
// matrix followed by implicit symmetric QL/QR iterations.  This file restates
// that published algorithm (Householder + implicit-shift QL with Wilkinson
// shifts, as in EISPACK tql2) in plain C++; it deliberately differs from the
// product's Jacobi solver so that the two are independent.
#include "oracle_common.h"
#include <algorithm>
#include <numeric>

namespace orc {

int hermitian_eig(int n, cd* A, double* w, cd* Z) {
  std::vector<cd> Q(n * n, cd(0, 0));
  for (int i = 0; i < n; ++i) Q[i * n + i] = 1.0;
  std::vector<cd> v(n), p(n), wv(n);
  // --- Householder tridiagonalisation: A <- H A H, Q <- Q H
  for (int k = 0; k + 2 < n; ++k) {
    double xnorm2 = 0.0;
    for (int i = k + 1; i < n; ++i) xnorm2 += std::norm(A[i * n + k]);
    double xnorm = std::sqrt(xnorm2);
    if (xnorm == 0.0) continue;
    cd x0 = A[(k + 1) * n + k];
    double ax0 = std::abs(x0);
    cd phase = ax0 > 0.0 ? x0 / ax0 : cd(1.0, 0.0);
    cd alpha = -phase * xnorm;
    std::fill(v.begin(), v.end(), cd(0, 0));
    for (int i = k + 1; i < n; ++i) v[i] = A[i * n + k];
    v[k + 1] -= alpha;
    double vn = 0.0;
    for (int i = k + 1; i < n; ++i) vn += std::norm(v[i]);
    vn = std::sqrt(vn);
    if (vn == 0.0) continue;
    for (int i = k + 1; i < n; ++i) v[i] /= vn;
    // p = A v, beta = v^H p, w = p - beta v, A -= 2 v w^H + 2 w v^H
    for (int i = 0; i < n; ++i) {
      cd s = 0.0;
      for (int j = k + 1; j < n; ++j) s += A[i * n + j] * v[j];
      p[i] = s;
    }
    cd beta = 0.0;
    for (int i = k + 1; i < n; ++i) beta += std::conj(v[i]) * p[i];
    for (int i = 0; i < n; ++i) wv[i] = p[i] - beta.real() * v[i];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        A[i * n + j] -= 2.0 * (v[i] * std::conj(wv[j]) + wv[i] * std::conj(v[j]));
    for (int i = 0; i < n; ++i) {
      cd s = 0.0;
      for (int j = k + 1; j < n; ++j) s += Q[i * n + j] * v[j];
      for (int j = k + 1; j < n; ++j) Q[i * n + j] -= 2.0 * s * std::conj(v[j]);
    }
  }
  // --- phase normalisation: T = D^H A D real tridiagonal
  std::vector<double> d(n), e(n, 0.0);
  std::vector<cd> ph(n, cd(1.0, 0.0));
  for (int k = 0; k + 1 < n; ++k) {
    cd ek = A[(k + 1) * n + k];
    double a = std::abs(ek);
    ph[k + 1] = a > 0.0 ? ek * ph[k] / a : ph[k];
    e[k] = a;
  }
  for (int k = 0; k < n; ++k) d[k] = A[k * n + k].real();
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) Q[i * n + k] *= ph[k];
  // --- implicit QL on (d, e); e[i] couples d[i], d[i+1]
  std::vector<double> zr(n * n, 0.0);
  for (int i = 0; i < n; ++i) zr[i * n + i] = 1.0;
  const double eps = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int m;
    do {
      for (m = l; m < n - 1; ++m) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= eps * dd) break;
      }
      if (m != l) {
        if (++iter > 200) return 1;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
        double s = 1.0, c = 1.0, pp = 0.0;
        int i;
        bool underflow = false;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i];
          double b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= pp;
            e[m] = 0.0;
            underflow = true;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - pp;
          r = (d[i] - g) * s + 2.0 * c * b;
          pp = s * r;
          d[i + 1] = g + pp;
          g = c * r - b;
          for (int k = 0; k < n; ++k) {
            double fz = zr[k * n + i + 1];
            zr[k * n + i + 1] = s * zr[k * n + i] + c * fz;
            zr[k * n + i] = c * zr[k * n + i] - s * fz;
          }
        }
        if (underflow) continue;
        d[l] -= pp;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  // --- sort ascending and back-transform Z = Q * zr
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
  for (int j = 0; j < n; ++j) {
    int src = order[j];
    w[j] = d[src];
    for (int i = 0; i < n; ++i) {
      cd s = 0.0;
      for (int k = 0; k < n; ++k) s += Q[i * n + k] * zr[k * n + src];
      Z[i * n + j] = s;
    }
  }
  return 0;
}

}  // namespace orc
