// Device helpers shared by the FP64 and split-precision pair kernels.
#pragma once
#include <cmath>

#include "cplx.cuh"
#include "phx_consts.h"
#include "phx_internal.h"

namespace pairc {

constexpr int kMaxT = 4;     // temperatures handled per launch

struct MeshArgs {
  int nq, nb, nT, n0, n1, n2;
  const double* E;      // (nq,nb)
  const double2* U;     // (nq,nb,nb)
  const double* vg;     // (nq,nb,3) or null
  const double* bose;   // (nT,nq,nb)
  const double* qcart;  // (nq,3)
  int smearing;
  double sigma;
  double qT[9];         // adaptive: reciprocal cell rows / mesh
  double norm;          // 1/Nq
};

__device__ __forceinline__ int mesh_add(int i, int j, int n0, int n1, int n2) {
  const int ix = i % n0, iy = (i / n0) % n1, iz = i / (n0 * n1);
  const int jx = j % n0, jy = (j / n0) % n1, jz = j / (n0 * n1);
  return ((iz + jz) % n2) * n0 * n1 + ((iy + jy) % n1) * n0 + (ix + jx) % n0;
}

__device__ __forceinline__ int mesh_neg(int i, int n0, int n1, int n2) {
  const int ix = i % n0, iy = (i / n0) % n1, iz = i / (n0 * n1);
  return ((n2 - iz) % n2) * n0 * n1 + ((n1 - iy) % n1) * n0 + (n0 - ix) % n0;
}

// AdaptiveGaussianDeltaFunction sigma (delta_function.cpp:71-83) before the floor.
__device__ __forceinline__ double adaptive_sigma(const double* qT, double v0, double v1, double v2) {
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double d = qT[3 * i] * v0 + qT[3 * i + 1] * v1 + qT[3 * i + 2] * v2;
    s += d * d;
  }
  return sqrt(s / 6.0);
}

__device__ __forceinline__ double floor_sigma(double s) {
  return (s != 0.0 && s < phxc::adaptiveCutoff) ? phxc::adaptiveCutoff : s;
}

// delta(E) with the reference's cut-offs; vzero: velocity difference is 0.
__device__ __forceinline__ double delta_fn(int smearing, double sigma, double e, bool vzero) {
  if (smearing == PHX_SMEAR_GAUSSIAN) {
    const double x = e / sigma;
    if (x > 6.0) return 0.0;
    return 1.0 / sigma / phxc::sqrtPi * exp(-x * x);
  }
  if (vzero && e == 0.0) return 1.0;
  if (sigma == 0.0) return 0.0;
  if (fabs(e) > 2.0 * sigma) return 0.0;
  const double x = e / sigma;
  if (x > 6.0) return 0.0;
  return exp(-x * x) / phxc::sqrtPi / sigma / phxc::erf2;
}

// Forward-scan degeneracy blocks (scattering.cpp:1218-1230): gs[b] = first
// band of b's block, gn[b] = its size.
template <int NB>
__device__ __forceinline__ void deg_blocks(const double* e, int* gs, int* gn) {
  int start = 0;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    if (b > start) {
      // b continues the block iff |e[start] - e[b]| < thr and all between did
      if (!(fabs(e[start] - e[b]) < phxc::degThreshold)) start = b;
    }
    gs[b] = start;
  }
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    int n = 0;
#pragma unroll
    for (int k = 0; k < NB; ++k) n += (gs[k] == gs[b]);
    gn[b] = n;
  }
}


}  // namespace pairc
