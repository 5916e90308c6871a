// Fused 3-phonon linewidth builder (PhScatteringMatrix::builder, linewidth
// mode) on a full Gamma-centred mesh -- plain FP64 path.
//
// Reference: src/bte/ph_scattering.cpp:60-613 (q2 outer loop, q1 batches,
// HOT LOOP 3), src/bte/scattering.cpp:1209-1318 (symmetrizeCoupling),
// :1168-1207 (degeneracyAveragingLinewidths), src/delta_function.cpp:34-96,
// src/particle.cpp:64-96, src/bte/helper_3rd_state.cpp:128-170 (q3 lookup).
//
// Restructuring (same arithmetic, different order):
//  * q3 = q1 + q2 is found by integer mesh arithmetic, which is what the
//    reference's Cartesian round trip + rounding computes on a Gamma-centred
//    mesh (src/points.cpp:404-423).
//  * The e2 contraction and every q2-only phase are folded into the cached
//    vertex once per q2:  Dp(q2)[r3][a][b2][c] = e^{-i q2.R3} sum_b e2(b,b2)
//    sum_r2 D3w(r3,r2,a,b,c) e^{+i q2.R2}, so each (q1,q2) pair costs one
//    [r3] x [a,b2,c] complex contraction plus two 6x6x6 contractions.
//  * Only the "+" vertex is evaluated.  By time reversal (D(-q) = conj D(q)
//    for real force constants, so e(-q) = conj e(q) up to a gauge) the
//    symmetrised |V-(q1,-q2)|^2 equals the symmetrised |V+(q1,q2)|^2 with the
//    same q3 = q1+q2; each evaluated pair therefore feeds the "+" rate of
//    (q1,q2) and the "-" rates of (q1,-q2).  Energies, velocities and Bose
//    factors of -q2 are read from the mesh tables at the index of -q2.
//  * Accumulation is owner-computes per q1 tile: a CTA owns 32 q1 points and a
//    slice of q2, keeps its partial linewidths in registers and adds them to
//    its own slot of a partial buffer; a final kernel sums the slots in a
//    fixed order (deterministic, no atomics), then applies degeneracy
//    averaging and the exclusion of acoustic Gamma modes.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include <cuda.h>

#include "cplx.cuh"
#include "phx_consts.h"
#include "phx_internal.h"

#include "pair_common.cuh"
#include "wide.cuh"

using namespace pairc;

namespace {

constexpr int kTile = 32;    // q1 points per CTA

__global__ void bose_kernel(int nq, int nb, int nT, const double* __restrict__ E,
                            const double* __restrict__ temps, double* __restrict__ bose) {
  const int ns = nq * nb;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns * nT; i += gridDim.x * blockDim.x) {
    const int c = i / ns, s = i % ns;
    const double t = temps[c], e = E[s];
    double n;
    if (t <= 0.0) n = e <= 0.0 ? 1.0 : 0.0;
    else {
      n = 1.0 / (exp(e / t) - 1.0);
      if (n < 0.0) n = 0.0;
    }
    bose[i] = n;
  }
}

// Dp[j][r3][a][b2][c] for q2 = q2_first + j (one block per (r3, group of q2)).
__global__ void fold_q2_kernel(int nb, int nr2, int nr3, const double* __restrict__ D3w,
                               const double* __restrict__ R2, const double* __restrict__ R3,
                               const double* __restrict__ qcart, const double2* __restrict__ U,
                               int q2_first, int q2_count, int q2_per_block,
                               double2* __restrict__ Dp) {
  extern __shared__ __align__(16) char sraw[];
  double2* ph2 = reinterpret_cast<double2*>(sraw);   // nr2
  double2* Y = ph2 + nr2;                            // nb*nb
  double2* e2 = Y + nb * nb;                         // nb*nb
  const int r3 = blockIdx.x;
  const int nbb = nb * nb, nb3 = nbb * nb;
  const int j0 = blockIdx.y * q2_per_block, j1 = min(q2_count, j0 + q2_per_block);
  for (int j = j0; j < j1; ++j) {
    const int iq2 = q2_first + j;
    const double* q = qcart + 3 * iq2;
    for (int r = threadIdx.x; r < nr2; r += blockDim.x) {
      double sn, cs;
      sincos(q[0] * R2[3 * r] + q[1] * R2[3 * r + 1] + q[2] * R2[3 * r + 2], &sn, &cs);
      ph2[r] = cmk(cs, sn);
    }
    for (int e = threadIdx.x; e < nbb; e += blockDim.x) e2[e] = U[(size_t)iq2 * nbb + e];
    double sn3, cs3;
    sincos(-(q[0] * R3[3 * r3] + q[1] * R3[3 * r3 + 1] + q[2] * R3[3 * r3 + 2]), &sn3, &cs3);
    const double2 p3 = cmk(cs3, sn3);
    __syncthreads();
    for (int a = 0; a < nb; ++a) {
      for (int bc = threadIdx.x; bc < nbb; bc += blockDim.x) {
        double2 acc = cmk(0.0, 0.0);
        const double* d = D3w + (size_t)r3 * nr2 * nb3 + (size_t)a * nbb + bc;
        for (int r = 0; r < nr2; ++r) {
          const double x = d[(size_t)r * nb3];
          acc.x = fma(x, ph2[r].x, acc.x);
          acc.y = fma(x, ph2[r].y, acc.y);
        }
        Y[bc] = acc;
      }
      __syncthreads();
      for (int e = threadIdx.x; e < nbb; e += blockDim.x) {
        const int b2 = e / nb, c = e % nb;
        double2 z = cmk(0.0, 0.0);
        for (int b = 0; b < nb; ++b) cfma(z, e2[b * nb + b2], Y[b * nb + c]);
        Dp[(((size_t)j * nr3 + r3) * nb + a) * nbb + b2 * nb + c] = cmul(z, p3);
      }
      __syncthreads();
    }
  }
}

// Same Dp, one block per (r3, 8 consecutive q2): every thread accumulates one
// (a,b,c) of the R2 transform for the 8 q2 at once (the D3w element is read
// once for 8 phases), then the e2 contraction runs from shared memory.  The
// sums run in the same order as fold_q2_kernel (r2 ascending, then b), so the
// results are identical.  nb <= 8.
constexpr int kFoldQ = 8;
__global__ void __launch_bounds__(256) fold_q2_tiled_kernel(int nb, int nr2, int nr3, const double* __restrict__ D3w,
                                                            const double* __restrict__ R2, const double* __restrict__ R3,
                                                            const double* __restrict__ qcart, const double2* __restrict__ U,
                                                            int q2_first, int q2_count, double2* __restrict__ Dp,
                                                            unsigned* __restrict__ dmax) {
  extern __shared__ __align__(16) char sraw[];
  const int nbb = nb * nb, nb3 = nbb * nb;
  double2* ph2 = reinterpret_cast<double2*>(sraw);   // [kFoldQ][nr2]
  double2* e2 = ph2 + kFoldQ * nr2;                  // [kFoldQ][nbb]
  double2* Y = e2 + kFoldQ * nbb;                    // [kFoldQ][nb3]
  double2* p3 = Y + kFoldQ * nb3;                    // [kFoldQ]
  const int r3 = blockIdx.x;
  const int j0 = blockIdx.y * kFoldQ;
  const int nj = min(kFoldQ, q2_count - j0);
  for (int e = threadIdx.x; e < kFoldQ * nr2; e += blockDim.x) {
    const int jl = e / nr2, r = e % nr2;
    double2 v = cmk(0.0, 0.0);
    if (jl < nj) {
      const double* q = qcart + 3 * (q2_first + j0 + jl);
      double sn, cs;
      sincos(q[0] * R2[3 * r] + q[1] * R2[3 * r + 1] + q[2] * R2[3 * r + 2], &sn, &cs);
      v = cmk(cs, sn);
    }
    ph2[e] = v;
  }
  for (int e = threadIdx.x; e < kFoldQ * nbb; e += blockDim.x) {
    const int jl = e / nbb;
    e2[e] = jl < nj ? U[(size_t)(q2_first + j0 + jl) * nbb + e % nbb] : cmk(0.0, 0.0);
  }
  if (threadIdx.x < kFoldQ) {
    double2 v = cmk(0.0, 0.0);
    if ((int)threadIdx.x < nj) {
      const double* q = qcart + 3 * (q2_first + j0 + threadIdx.x);
      double sn3, cs3;
      sincos(-(q[0] * R3[3 * r3] + q[1] * R3[3 * r3 + 1] + q[2] * R3[3 * r3 + 2]), &sn3, &cs3);
      v = cmk(cs3, sn3);
    }
    p3[threadIdx.x] = v;
  }
  __syncthreads();
  const double* d0 = D3w + (size_t)r3 * nr2 * nb3;
  for (int abc = threadIdx.x; abc < nb3; abc += blockDim.x) {
    double2 acc[kFoldQ];
#pragma unroll
    for (int jl = 0; jl < kFoldQ; ++jl) acc[jl] = cmk(0.0, 0.0);
    for (int r = 0; r < nr2; ++r) {
      const double x = __ldg(d0 + (size_t)r * nb3 + abc);
#pragma unroll
      for (int jl = 0; jl < kFoldQ; ++jl) {
        const double2 p = ph2[jl * nr2 + r];
        acc[jl].x = fma(x, p.x, acc[jl].x);
        acc[jl].y = fma(x, p.y, acc[jl].y);
      }
    }
#pragma unroll
    for (int jl = 0; jl < kFoldQ; ++jl) Y[jl * nb3 + abc] = acc[jl];
  }
  __syncthreads();
  // Dp[j][r3][a][b2][c] = p3 * sum_b e2(b,b2) Y(a,b,c)
  float m = 0.f;   // largest |component| written (FP16 operand scale of the split path)
  for (int e = threadIdx.x; e < nj * nb3; e += blockDim.x) {
    const int jl = e / nb3, rest = e % nb3;
    const int a = rest / nbb, b2 = (rest / nb) % nb, c = rest % nb;
    const double2* y = Y + jl * nb3 + a * nbb + c;
    const double2* u = e2 + jl * nbb + b2;
    double2 z = cmk(0.0, 0.0);
    for (int b = 0; b < nb; ++b) cfma(z, u[b * nb], y[b * nb]);
    const double2 d = cmul(z, p3[jl]);
    Dp[(((size_t)(j0 + jl) * nr3 + r3) * nb + a) * nbb + b2 * nb + c] = d;
    m = fmaxf(m, (float)fmax(fabs(d.x), fabs(d.y)));
  }
  if (dmax) {
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative floats order like their bit patterns
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(dmax, __float_as_uint(m));
  }
}

size_t fold_tiled_smem(int nb, int nr2) {
  return sizeof(double2) * ((size_t)kFoldQ * (nr2 + nb * nb + nb * nb * nb) + kFoldQ);
}
void fold_tiled_launch(int nb, int nr2, int nr3, const phx_v3* v, const phx_bands* b, int c0, int cnt,
                       double2* Dp, cudaStream_t st, unsigned* dmax = nullptr) {
  dim3 gf(nr3, (cnt + kFoldQ - 1) / kFoldQ);
  fold_q2_tiled_kernel<<<gf, 256, fold_tiled_smem(nb, nr2), st>>>(nb, nr2, nr3, v->d_D3w, v->d_R2, v->d_R3, b->d_q,
                                                                  reinterpret_cast<const double2*>(b->d_U), c0, cnt, Dp,
                                                                  dmax);
}

struct PairArgs {
  MeshArgs m;
  int nr3;
  const double* R3;
  const double2* Dp;
  int q2_first, q2_count, q2_per_slot;
  double* partial;   // (S, nq, nb, nT)
  // matrix modes (pair_fp64_kernel<NB, true>): column-major blocks of the
  // scattering matrix, element (row, col) at col * ld + row, row = q1 nb + b1.
  //   mat_full = 1: matP is the whole matrix (one temperature); the "+" rates
  //     of (q1 b1, q2 b2) and minus the "-" rates of (q1 b1, -q2 b2) are added
  //     atomically (each element receives one of each).
  //   mat_full = 0: slabs of the chunk, column j nb + b2 (j = q2 - q2_first):
  //     matP the "+" rates of (q1 b1, q2 b2), matM the "-" rates of
  //     (q1 b1, -q2 b2), each temperature mat_tstride elements further on;
  //     every element of the slabs is stored.
  double* matP;
  double* matM;
  long long ld;
  size_t mat_tstride;
  int mat_full;
};

template <int NB, bool MAT = false>
__global__ void __launch_bounds__(kTile * NB, 1) pair_fp64_kernel(PairArgs P) {
  const MeshArgs& M = P.m;
  extern __shared__ __align__(16) char sraw[];
  const int nr3 = P.nr3, nT = M.nT;
  double2* ph = reinterpret_cast<double2*>(sraw);      // [nr3][32]
  double2* e1s = ph + (size_t)nr3 * kTile;             // [NB*NB][32]
  double2* e3s = e1s + NB * NB * kTile;                // [NB*NB][32]
  double* Wx = reinterpret_cast<double*>(e3s + NB * NB * kTile);  // [NB][NB*NB][32]
  double* b1s = Wx + NB * NB * NB * kTile;              // [nT][NB][32]
  const int tid = threadIdx.x, ql = tid & 31, b2 = tid >> 5;
  const int q1 = blockIdx.x * kTile + ql;
  const bool valid = q1 < M.nq;
  const int q1c = valid ? q1 : M.nq - 1;
  const int n0 = M.n0, n1 = M.n1, n2 = M.n2, nq = M.nq;
  // --- per-CTA setup: phases e^{-i q1.R3}, e1, Bose(q1)
  for (int i = tid; i < nr3 * kTile; i += blockDim.x) {
    const int r = i / kTile, l = i % kTile;
    const int qq = min(blockIdx.x * kTile + l, nq - 1);
    const double* q = M.qcart + 3 * qq;
    double sn, cs;
    sincos(-(q[0] * P.R3[3 * r] + q[1] * P.R3[3 * r + 1] + q[2] * P.R3[3 * r + 2]), &sn, &cs);
    ph[i] = cmk(cs, sn);
  }
  for (int i = tid; i < NB * NB * kTile; i += blockDim.x) {
    const int e = i / kTile, l = i % kTile;
    const int qq = min(blockIdx.x * kTile + l, nq - 1);
    e1s[i] = M.U[(size_t)qq * NB * NB + e];
  }
  for (int i = tid; i < nT * NB * kTile; i += blockDim.x) {
    const int l = i % kTile, cb = i / kTile, b = cb % NB, c = cb / NB;
    const int qq = min(blockIdx.x * kTile + l, nq - 1);
    b1s[i] = M.bose[((size_t)c * nq + qq) * NB + b];
  }
  double E1[NB];
  int g1s[NB], g1n[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) E1[b] = M.E[(size_t)q1c * NB + b];
  deg_blocks<NB>(E1, g1s, g1n);
  double acc[NB][kMaxT];
#pragma unroll
  for (int b = 0; b < NB; ++b)
#pragma unroll
    for (int c = 0; c < kMaxT; ++c) acc[b][c] = 0.0;
  __syncthreads();

  const int jbeg = blockIdx.y * P.q2_per_slot;
  const int jend = min(P.q2_count, jbeg + P.q2_per_slot);
  for (int j = jbeg; j < jend; ++j) {
    const int iq2 = P.q2_first + j;
    const int iq2m = mesh_neg(iq2, n0, n1, n2);
    const int iq3 = mesh_add(q1c, iq2, n0, n1, n2);
    // stage e3 of the 32 q3 points
    for (int i = tid; i < NB * NB * kTile; i += blockDim.x) {
      const int e = i / kTile, l = i % kTile;
      const int qq = min(blockIdx.x * kTile + l, nq - 1);
      const int q3 = mesh_add(qq, iq2, n0, n1, n2);
      e3s[i] = M.U[(size_t)q3 * NB * NB + e];
    }
    __syncthreads();
    // T(a,c) = sum_r3 e^{-i q1.R3} Dp(q2)[r3][a][b2][c]
    double2 T[NB][NB];
#pragma unroll
    for (int a = 0; a < NB; ++a)
#pragma unroll
      for (int c = 0; c < NB; ++c) T[a][c] = cmk(0.0, 0.0);
    const double2* D = P.Dp + (size_t)j * nr3 * NB * NB * NB + b2 * NB;
    for (int r = 0; r < nr3; ++r) {
      const double2 p = ph[r * kTile + ql];
      const double2* Dr = D + (size_t)r * NB * NB * NB;
#pragma unroll
      for (int a = 0; a < NB; ++a)
#pragma unroll
        for (int c = 0; c < NB; ++c) cfma(T[a][c], p, __ldg(Dr + a * NB * NB + c));
    }
    // X(b1,c) = sum_a e1(a,b1) T(a,c), in place column by column
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      double2 col[NB];
#pragma unroll
      for (int a = 0; a < NB; ++a) col[a] = T[a][c];
#pragma unroll
      for (int b1 = 0; b1 < NB; ++b1) {
        double2 x = cmk(0.0, 0.0);
#pragma unroll
        for (int a = 0; a < NB; ++a) cfma(x, e1s[(a * NB + b1) * kTile + ql], col[a]);
        T[b1][c] = x;
      }
    }
    // V(b1,b3) = sum_c X(b1,c) conj(e3(c,b3)); W = |V|^2
    double W[NB][NB];
#pragma unroll
    for (int b1 = 0; b1 < NB; ++b1) {
#pragma unroll
      for (int b3 = 0; b3 < NB; ++b3) {
        double2 v = cmk(0.0, 0.0);
#pragma unroll
        for (int c = 0; c < NB; ++c) cfmac(v, T[b1][c], e3s[(c * NB + b3) * kTile + ql]);
        W[b1][b3] = v.x * v.x + v.y * v.y;
      }
    }
    // symmetrise over degenerate blocks of b1 (E1) and b3 (E3)
    double E3[NB];
    int g3s[NB], g3n[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) E3[b] = M.E[(size_t)iq3 * NB + b];
    deg_blocks<NB>(E3, g3s, g3n);
#pragma unroll
    for (int b1 = 0; b1 < NB; ++b1) {
      double row[NB];
#pragma unroll
      for (int b3 = 0; b3 < NB; ++b3) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NB; ++k) s += (g3s[k] == g3s[b3]) ? W[b1][k] : 0.0;
        row[b3] = s / (double)g3n[b3];
      }
#pragma unroll
      for (int b3 = 0; b3 < NB; ++b3) W[b1][b3] = row[b3];
    }
#pragma unroll
    for (int b3 = 0; b3 < NB; ++b3) {
      double colv[NB];
#pragma unroll
      for (int b1 = 0; b1 < NB; ++b1) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NB; ++k) s += (g1s[k] == g1s[b1]) ? W[k][b3] : 0.0;
        colv[b1] = s / (double)g1n[b1];
      }
#pragma unroll
      for (int b1 = 0; b1 < NB; ++b1) W[b1][b3] = colv[b1];
    }
    // exchange across b2 (one warp per b2) and average over E2 blocks
#pragma unroll
    for (int b1 = 0; b1 < NB; ++b1)
#pragma unroll
      for (int b3 = 0; b3 < NB; ++b3) Wx[((b2 * NB + b1) * NB + b3) * kTile + ql] = W[b1][b3];
    __syncthreads();
    double E2v[NB];
    int g2s[NB], g2n[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) E2v[b] = M.E[(size_t)iq2 * NB + b];
    deg_blocks<NB>(E2v, g2s, g2n);
    int mys = 0, myn = 1;
#pragma unroll
    for (int b = 0; b < NB; ++b)
      if (b == b2) { mys = g2s[b]; myn = g2n[b]; }
    if (myn > 1) {
#pragma unroll
      for (int b1 = 0; b1 < NB; ++b1)
#pragma unroll
        for (int b3 = 0; b3 < NB; ++b3) {
          double s = 0.0;
          for (int k = mys; k < mys + myn; ++k) s += Wx[((k * NB + b1) * NB + b3) * kTile + ql];
          W[b1][b3] = s / (double)myn;
        }
    }
    // epilogue: "+" rates of (q1,q2) and "-" rates of (q1,-q2)
    const double en2 = M.E[(size_t)iq2 * NB + b2];
    const double en2m = M.E[(size_t)iq2m * NB + b2];
    const bool ok2 = en2 >= phxc::phExcludeCutoff && en2 >= phxc::phEnergyCutoff;
    const bool ok2m = en2m >= phxc::phExcludeCutoff && en2m >= phxc::phEnergyCutoff;
    double v2[3] = {0, 0, 0}, v2m[3] = {0, 0, 0};
    if (M.smearing == PHX_SMEAR_ADAPTIVE) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        v2[i] = M.vg[((size_t)iq2 * NB + b2) * 3 + i];
        v2m[i] = M.vg[((size_t)iq2m * NB + b2) * 3 + i];
      }
    }
    if constexpr (MAT) {
      // one temperature at a time: the sums over b3 of the "+" rates (sp) and
      // of the two "-" rates (sm) of each b1, which also make the linewidths
#pragma unroll 1
      for (int c = 0; c < nT; ++c) {
        double sp[NB], sm[NB];
#pragma unroll
        for (int b1 = 0; b1 < NB; ++b1) sp[b1] = sm[b1] = 0.0;
        if (valid && (ok2 || ok2m)) {
          const double n2c = M.bose[((size_t)c * nq + iq2) * NB + b2];
          const double n2mc = M.bose[((size_t)c * nq + iq2m) * NB + b2];
#pragma unroll
          for (int b3 = 0; b3 < NB; ++b3) {
            const double en3 = E3[b3];
            if (en3 < phxc::phEnergyCutoff) continue;
            double sgp = M.sigma, sgm = M.sigma;
            bool vzp = false, vzm = false;
            if (M.smearing == PHX_SMEAR_ADAPTIVE) {
              const double* v3 = M.vg + ((size_t)iq3 * NB + b3) * 3;
              const double dp0 = v2[0] - v3[0], dp1 = v2[1] - v3[1], dp2 = v2[2] - v3[2];
              const double dm0 = v2m[0] - v3[0], dm1 = v2m[1] - v3[1], dm2 = v2m[2] - v3[2];
              vzp = (dp0 * dp0 + dp1 * dp1 + dp2 * dp2) == 0.0;
              vzm = (dm0 * dm0 + dm1 * dm1 + dm2 * dm2) == 0.0;
              sgp = floor_sigma(adaptive_sigma(M.qT, dp0, dp1, dp2));
              sgm = floor_sigma(adaptive_sigma(M.qT, dm0, dm1, dm2));
            }
            const double n3c = M.bose[((size_t)c * nq + iq3) * NB + b3];
#pragma unroll
            for (int b1 = 0; b1 < NB; ++b1) {
              const double en1 = E1[b1];
              if (en1 < phxc::phExcludeCutoff || en1 < phxc::phEnergyCutoff) continue;
              const double w = W[b1][b3];
              const double n1 = b1s[(c * NB + b1) * kTile + ql];
              if (ok2) {
                const double dlt = delta_fn(M.smearing, sgp, en1 + en2 - en3, vzp);
                if (dlt > 0.0) sp[b1] += phxc::pi * 0.25 * w * dlt * M.norm / (en1 * en2 * en3) * n1 * n2c * (n3c + 1.0);
              }
              if (ok2m) {
                double d1 = delta_fn(M.smearing, sgm, en1 + en3 - en2m, vzm);
                double d2 = delta_fn(M.smearing, sgm, en2m + en3 - en1, vzm);
                if (d1 > 0.0 || d2 > 0.0) {
                  d1 = fmax(d1, 0.0);
                  d2 = fmax(d2, 0.0);
                  const double f = phxc::pi * 0.25 * w * M.norm / (en1 * en2m * en3);
                  sm[b1] += f * n3c * n1 * (n2mc + 1.0) * d1 + f * n2mc * n3c * (n1 + 1.0) * d2;
                }
              }
            }
          }
        }
#pragma unroll
        for (int b1 = 0; b1 < NB; ++b1)
#pragma unroll
          for (int cc = 0; cc < kMaxT; ++cc)
            if (cc == c) acc[b1][cc] += 0.5 * (sp[b1] + sm[b1]);
        if (valid) {
          const size_t row = (size_t)q1 * NB;
          if (P.mat_full) {
            double* colp = P.matP + (size_t)(iq2 * NB + b2) * P.ld + row;
            double* colm = P.matP + (size_t)(iq2m * NB + b2) * P.ld + row;
#pragma unroll
            for (int b1 = 0; b1 < NB; ++b1) {
              if (sp[b1] != 0.0) atomicAdd(colp + b1, sp[b1]);
              if (sm[b1] != 0.0) atomicAdd(colm + b1, -sm[b1]);
            }
          } else {
            const size_t o = c * P.mat_tstride + (size_t)(j * NB + b2) * P.ld + row;
#pragma unroll
            for (int b1 = 0; b1 < NB; ++b1) {
              P.matP[o + b1] = sp[b1];
              P.matM[o + b1] = sm[b1];
            }
          }
        }
      }
    } else if (valid && (ok2 || ok2m)) {
#pragma unroll
      for (int b3 = 0; b3 < NB; ++b3) {
        const double en3 = E3[b3];
        if (en3 < phxc::phEnergyCutoff) continue;
        double sp = M.sigma, sm = M.sigma;
        bool vzp = false, vzm = false;
        if (M.smearing == PHX_SMEAR_ADAPTIVE) {
          const double* v3 = M.vg + ((size_t)iq3 * NB + b3) * 3;
          const double dp0 = v2[0] - v3[0], dp1 = v2[1] - v3[1], dp2 = v2[2] - v3[2];
          const double dm0 = v2m[0] - v3[0], dm1 = v2m[1] - v3[1], dm2 = v2m[2] - v3[2];
          vzp = (dp0 * dp0 + dp1 * dp1 + dp2 * dp2) == 0.0;
          vzm = (dm0 * dm0 + dm1 * dm1 + dm2 * dm2) == 0.0;
          sp = floor_sigma(adaptive_sigma(M.qT, dp0, dp1, dp2));
          sm = floor_sigma(adaptive_sigma(M.qT, dm0, dm1, dm2));
        }
        double n3[kMaxT];
#pragma unroll
        for (int c = 0; c < kMaxT; ++c)
          n3[c] = c < nT ? M.bose[((size_t)c * nq + iq3) * NB + b3] : 0.0;
        double n2[kMaxT], n2m[kMaxT];
#pragma unroll
        for (int c = 0; c < kMaxT; ++c) {
          n2[c] = c < nT ? M.bose[((size_t)c * nq + iq2) * NB + b2] : 0.0;
          n2m[c] = c < nT ? M.bose[((size_t)c * nq + iq2m) * NB + b2] : 0.0;
        }
#pragma unroll
        for (int b1 = 0; b1 < NB; ++b1) {
          const double en1 = E1[b1];
          if (en1 < phxc::phExcludeCutoff || en1 < phxc::phEnergyCutoff) continue;
          const double w = W[b1][b3];
          if (ok2) {
            const double dlt = delta_fn(M.smearing, sp, en1 + en2 - en3, vzp);
            if (dlt > 0.0) {
              const double f = phxc::pi * 0.25 * w * dlt * M.norm / (en1 * en2 * en3);
#pragma unroll
              for (int c = 0; c < kMaxT; ++c)
                if (c < nT) {
                  const double n1 = b1s[(c * NB + b1) * kTile + ql];
                  acc[b1][c] += 0.5 * (f * n1 * n2[c] * (n3[c] + 1.0));
                }
            }
          }
          if (ok2m) {
            double d1 = delta_fn(M.smearing, sm, en1 + en3 - en2m, vzm);
            double d2 = delta_fn(M.smearing, sm, en2m + en3 - en1, vzm);
            if (d1 > 0.0 || d2 > 0.0) {
              d1 = fmax(d1, 0.0);
              d2 = fmax(d2, 0.0);
              const double f = phxc::pi * 0.25 * w * M.norm / (en1 * en2m * en3);
#pragma unroll
              for (int c = 0; c < kMaxT; ++c)
                if (c < nT) {
                  const double n1 = b1s[(c * NB + b1) * kTile + ql];
                  const double r1 = f * n3[c] * n1 * (n2m[c] + 1.0) * d1;
                  const double r2 = f * n2m[c] * n3[c] * (n1 + 1.0) * d2;
                  acc[b1][c] += 0.5 * (r1 + r2);
                }
            }
          }
        }
      }
    }
    __syncthreads();
  }
  // reduce over the b2 warps and add to this CTA's partial slot
#pragma unroll
  for (int b1 = 0; b1 < NB; ++b1)
#pragma unroll
    for (int c = 0; c < kMaxT; ++c) Wx[((b2 * NB + b1) * kMaxT + c) * kTile + ql] = acc[b1][c];
  __syncthreads();
  if (b2 == 0 && valid) {
    double* out = P.partial + ((size_t)blockIdx.y * nq + q1) * NB * nT;
    for (int b1 = 0; b1 < NB; ++b1)
      for (int c = 0; c < nT; ++c) {
        double s = 0.0;
        for (int k = 0; k < NB; ++k) s += Wx[((k * NB + b1) * kMaxT + c) * kTile + ql];
        out[b1 * nT + c] += s;
      }
  }
}

// ---------------------------------------------------------------------------
// Any nb up to kMaxNbGeneric (the 15-branch cells), with an optional per-q1
// window on q2: one block per (q1, q2 slot), the R3 transform, the e1 and e3
// contractions, |V|^2, the three symmetrisation passes and the rates of each
// q2 run through shared memory (two nb^3 complex buffers).  Same algebra,
// cutoffs and time-reversal pairing as pair_fp64_kernel: the "+" vertex of
// (q1, q2) gives the "+" process of (q1, q2) and the "-" process of
// (q1, -q2); with a window, each of the two is counted only when its q2 is
// inside the window of q1.
// ---------------------------------------------------------------------------
constexpr int kMaxNbGeneric = 16;
constexpr int kGenThreads = 512;
constexpr int kGenRSplit = 2;   // R3 halves of the T phase (threads per T element)

struct Q2Window {
  const double* energy;   // (nq) or null: no window
  const double* cut;      // (nq): q2 is paired with q1 iff energy[q2] <= cut[q1]
};

// Shared memory of pair_generic_kernel<Q1>: per q1 of the tile its phases,
// e1, e3, the b2 slices of T and X, and the coupling W of all (b1, b2, b3).
__host__ __device__ inline size_t generic_smem_bytes(int nb, int nr3, int q1s) {
  const size_t nbb = (size_t)nb * nb, nb3 = nbb * nb;
  return (size_t)q1s * (sizeof(double2) * ((size_t)nr3 + (3 + kGenRSplit) * nbb) +
                        sizeof(double) * (nb3 + (size_t)nb * kMaxT + 2 * nb) +
                        sizeof(int) * (2 * nb + 4)) +
         sizeof(double) * 2 * nb + sizeof(int) * nb;
}

// forward-scan degenerate blocks (scattering.cpp:1223,1257,1291): gs[b] = start of b's block
__device__ inline void scan_blocks(const double* e, int nb, int* gs) {
  int start = 0;
  for (int b = 0; b < nb; ++b) {
    if (b > start && !(fabs(e[start] - e[b]) < phxc::degThreshold)) start = b;
    gs[b] = start;
  }
}

// Q1 q1 points per block (q1_order[blockIdx.x * Q1 + i]): each element of
// the q2 slab of the cached vertex is read once per block and used for all Q1
// (Q1 independent accumulators per thread), one b2 slice at a time:
//   T(a,c) = sum_r3 e^{-i q1.R3} Dp(q2)[r3][a][b2][c]
//   X(b1,c) = sum_a e1(a,b1) T(a,c)
//   W(b1,b2,b3) = |sum_c X(b1,c) conj(e3(c,b3))|^2
// then the three symmetrisation passes and the rates of each q1 of the tile.
// With a window, a q2 outside the windows of every q1 of the tile is skipped
// (the host orders q1 by window so that tiles hold similar windows).
template <int Q1>
__global__ void __launch_bounds__(kGenThreads) pair_generic_kernel(PairArgs P, Q2Window win, const int* q1_order) {
  const MeshArgs& M = P.m;
  extern __shared__ __align__(16) char sraw[];
  const int nb = M.nb, nbb = nb * nb, nb3 = nbb * nb, nr3 = P.nr3, nT = M.nT, nq = M.nq;
  double2* ph = reinterpret_cast<double2*>(sraw);   // [Q1][nr3]
  double2* e1 = ph + Q1 * nr3;                      // [Q1][nb][nb]
  double2* e3 = e1 + Q1 * nbb;                      // [Q1][nb][nb]
  double2* Tb = e3 + Q1 * nbb;                      // [kGenRSplit][Q1][a][c] partial T of the current b2
  double2* Xb = Tb + kGenRSplit * Q1 * nbb;         // [Q1][b1][c] of the current b2
  double* W = reinterpret_cast<double*>(Xb + Q1 * nbb);   // [Q1][b1][b2][b3]
  double* acc = W + Q1 * nb3;                       // [Q1][nb][kMaxT]
  double* E1 = acc + Q1 * nb * kMaxT;               // [Q1][nb]
  double* E3 = E1 + Q1 * nb;                        // [Q1][nb]
  double* E2 = E3 + Q1 * nb;                        // [nb]
  double* E2m = E2 + nb;                            // [nb]
  int* g1s = reinterpret_cast<int*>(E2m + nb);      // [Q1][nb]
  int* g3s = g1s + Q1 * nb;                         // [Q1][nb]
  int* g2s = g3s + Q1 * nb;                         // [nb]
  int* q1s = g2s + nb;                              // [Q1] q1 of each slot of the tile, -1: none
  int* q3s = q1s + Q1;                              // [Q1]
  int* inw = q3s + Q1;                              // [Q1] bit 0: q2 in the window, bit 1: -q2
  const int tid = threadIdx.x, NT = blockDim.x;
  const int n0 = M.n0, n1 = M.n1, n2 = M.n2;
  if (tid < Q1) {
    const int i = blockIdx.x * Q1 + tid;
    q1s[tid] = i < nq ? (q1_order ? q1_order[i] : i) : -1;
  }
  __syncthreads();
  for (int e = tid; e < Q1 * nr3; e += NT) {
    const int t = e / nr3, r = e % nr3;
    const int q1 = max(q1s[t], 0);
    const double* q = M.qcart + 3 * q1;
    double sn, cs;
    sincos(-(q[0] * P.R3[3 * r] + q[1] * P.R3[3 * r + 1] + q[2] * P.R3[3 * r + 2]), &sn, &cs);
    ph[e] = cmk(cs, sn);
  }
  for (int e = tid; e < Q1 * nbb; e += NT) e1[e] = M.U[(size_t)max(q1s[e / nbb], 0) * nbb + e % nbb];
  for (int i = tid; i < Q1 * nb * kMaxT; i += NT) acc[i] = 0.0;
  for (int e = tid; e < Q1 * nb; e += NT) E1[e] = M.E[(size_t)max(q1s[e / nb], 0) * nb + e % nb];
  __syncthreads();
  if (tid < Q1) scan_blocks(E1 + tid * nb, nb, g1s + tid * nb);
  const int jbeg = blockIdx.y * P.q2_per_slot;
  const int jend = min(P.q2_count, jbeg + P.q2_per_slot);
  for (int j = jbeg; j < jend; ++j) {
    const int iq2 = P.q2_first + j;
    const int iq2m = mesh_neg(iq2, n0, n1, n2);
    __syncthreads();   // the previous q2's rates are done with this q2's shared buffers
    if (tid < Q1) {
      const int q1 = q1s[tid];
      int f = 0;
      if (q1 >= 0) {
        f |= (!win.energy || win.energy[iq2] <= win.cut[q1]) ? 1 : 0;
        f |= (!win.energy || win.energy[iq2m] <= win.cut[q1]) ? 2 : 0;
      }
      inw[tid] = f;
      q3s[tid] = mesh_add(max(q1, 0), iq2, n0, n1, n2);
    }
    __syncthreads();
    int any = 0;
#pragma unroll
    for (int t = 0; t < Q1; ++t) any |= inw[t];
    if (!any) continue;   // uniform over the block
    for (int e = tid; e < Q1 * nbb; e += NT) e3[e] = M.U[(size_t)q3s[e / nbb] * nbb + e % nbb];
    for (int e = tid; e < Q1 * nb; e += NT) E3[e] = M.E[(size_t)q3s[e / nb] * nb + e % nb];
    for (int b = tid; b < nb; b += NT) {
      E2[b] = M.E[(size_t)iq2 * nb + b];
      E2m[b] = M.E[(size_t)iq2m * nb + b];
    }
    __syncthreads();
    if (tid < Q1) scan_blocks(E3 + tid * nb, nb, g3s + tid * nb);
    if (tid == Q1) scan_blocks(E2, nb, g2s);
    const double2* D = P.Dp + (size_t)j * nr3 * nb3;
    for (int b2 = 0; b2 < nb; ++b2) {
      // T(a,c) of every q1 of the tile: one read of Dp per element, the R3
      // sum split in kGenRSplit parts (more loads in flight)
      for (int y = tid; y < kGenRSplit * nbb; y += NT) {
        const int h = y / nbb, x = y % nbb, a = x / nb, c = x % nb;
        const int rb = h * nr3 / kGenRSplit, re = (h + 1) * nr3 / kGenRSplit;
        const double2* Dx = D + ((size_t)a * nb + b2) * nb + c;
        double2 t[Q1];
#pragma unroll
        for (int q = 0; q < Q1; ++q) t[q] = cmk(0.0, 0.0);
#pragma unroll 4
        for (int r = rb; r < re; ++r) {
          const double2 d = __ldg(Dx + (size_t)r * nb3);
#pragma unroll
          for (int q = 0; q < Q1; ++q) cfma(t[q], ph[q * nr3 + r], d);
        }
#pragma unroll
        for (int q = 0; q < Q1; ++q) Tb[(h * Q1 + q) * nbb + x] = t[q];
      }
      __syncthreads();
      for (int y = tid; y < Q1 * nbb; y += NT) {
        const int q = y / nbb, x = y % nbb, b1 = x / nb, c = x % nb;
        const double2* eq = e1 + q * nbb;
        const double2* tq = Tb + q * nbb;
        double2 v = cmk(0.0, 0.0);
        for (int a = 0; a < nb; ++a) {
          double2 tt = tq[a * nb + c];
#pragma unroll
          for (int h = 1; h < kGenRSplit; ++h) {
            const double2 u = tq[h * Q1 * nbb + a * nb + c];
            tt.x += u.x;
            tt.y += u.y;
          }
          cfma(v, eq[a * nb + b1], tt);
        }
        Xb[y] = v;
      }
      __syncthreads();
      for (int y = tid; y < Q1 * nbb; y += NT) {
        const int q = y / nbb, x = y % nbb, b1 = x / nb, b3 = x % nb;
        const double2* xq = Xb + q * nbb + b1 * nb;
        const double2* eq = e3 + q * nbb;
        double2 v = cmk(0.0, 0.0);
        for (int c = 0; c < nb; ++c) cfmac(v, xq[c], eq[c * nb + b3]);
        W[(size_t)q * nb3 + ((size_t)b1 * nb + b2) * nb + b3] = v.x * v.x + v.y * v.y;
      }
      // the next b2 writes Tb, which nothing reads now; Xb is rewritten after its T barrier
    }
    __syncthreads();
    // symmetrizeCoupling (scattering.cpp:1209-1318): average over the blocks of
    // b3, then b1, then b2 (projections on different indices commute)
    for (int y = tid; y < Q1 * nbb; y += NT) {
      const int q = y / nbb, x = y % nbb;
      double* w = W + (size_t)q * nb3 + (size_t)x * nb;   // (b1,b2) row over b3
      const int* g = g3s + q * nb;
      for (int s0 = 0; s0 < nb;) {
        int s1 = s0 + 1;
        while (s1 < nb && g[s1] == s0) ++s1;
        if (s1 - s0 > 1) {
          double t = 0.0;
          for (int k = s0; k < s1; ++k) t += w[k];
          for (int k = s0; k < s1; ++k) w[k] = t / (double)(s1 - s0);
        }
        s0 = s1;
      }
    }
    __syncthreads();
    for (int y = tid; y < Q1 * nbb; y += NT) {
      const int q = y / nbb, x = y % nbb, b2 = x / nb, b3 = x % nb;   // column over b1
      double* w = W + (size_t)q * nb3;
      const int* g = g1s + q * nb;
      for (int s0 = 0; s0 < nb;) {
        int s1 = s0 + 1;
        while (s1 < nb && g[s1] == s0) ++s1;
        if (s1 - s0 > 1) {
          double t = 0.0;
          for (int k = s0; k < s1; ++k) t += w[((size_t)k * nb + b2) * nb + b3];
          for (int k = s0; k < s1; ++k) w[((size_t)k * nb + b2) * nb + b3] = t / (double)(s1 - s0);
        }
        s0 = s1;
      }
    }
    __syncthreads();
    for (int y = tid; y < Q1 * nbb; y += NT) {
      const int q = y / nbb, x = y % nbb, b1 = x / nb, b3 = x % nb;   // over b2
      double* w = W + (size_t)q * nb3;
      for (int s0 = 0; s0 < nb;) {
        int s1 = s0 + 1;
        while (s1 < nb && g2s[s1] == s0) ++s1;
        if (s1 - s0 > 1) {
          double t = 0.0;
          for (int k = s0; k < s1; ++k) t += w[((size_t)b1 * nb + k) * nb + b3];
          for (int k = s0; k < s1; ++k) w[((size_t)b1 * nb + k) * nb + b3] = t / (double)(s1 - s0);
        }
        s0 = s1;
      }
    }
    __syncthreads();
    // rates: "+" of (q1,q2), "-" of (q1,-q2) (ph_scattering.cpp:338-380, 466-518)
    for (int y = tid; y < Q1 * nb3; y += NT) {
      const int q = y / nb3, x = y % nb3;
      const int q1 = q1s[q];
      if (q1 < 0 || !inw[q]) continue;
      const int iq3 = q3s[q];
      const int b1 = x / nbb, b2 = (x / nb) % nb, b3 = x % nb;
      const double en1 = E1[q * nb + b1], en3 = E3[q * nb + b3];
      if (en1 < phxc::phExcludeCutoff || en1 < phxc::phEnergyCutoff || en3 < phxc::phEnergyCutoff) continue;
      const double en2 = E2[b2];
      const double en2m = E2m[b2];
      const bool ok2 = (inw[q] & 1) && en2 >= phxc::phExcludeCutoff && en2 >= phxc::phEnergyCutoff;
      const bool ok2m = (inw[q] & 2) && en2m >= phxc::phExcludeCutoff && en2m >= phxc::phEnergyCutoff;
      if (!ok2 && !ok2m) continue;
      double sp = M.sigma, sm = M.sigma;
      bool vzp = false, vzm = false;
      if (M.smearing == PHX_SMEAR_ADAPTIVE) {
        const double* v3 = M.vg + ((size_t)iq3 * nb + b3) * 3;
        const double* v2 = M.vg + ((size_t)iq2 * nb + b2) * 3;
        const double* v2m = M.vg + ((size_t)iq2m * nb + b2) * 3;
        const double dp0 = v2[0] - v3[0], dp1 = v2[1] - v3[1], dp2 = v2[2] - v3[2];
        const double dm0 = v2m[0] - v3[0], dm1 = v2m[1] - v3[1], dm2 = v2m[2] - v3[2];
        vzp = (dp0 * dp0 + dp1 * dp1 + dp2 * dp2) == 0.0;
        vzm = (dm0 * dm0 + dm1 * dm1 + dm2 * dm2) == 0.0;
        sp = floor_sigma(adaptive_sigma(M.qT, dp0, dp1, dp2));
        sm = floor_sigma(adaptive_sigma(M.qT, dm0, dm1, dm2));
      }
      const double w = W[y];
      double r[kMaxT];
#pragma unroll
      for (int c = 0; c < kMaxT; ++c) r[c] = 0.0;
      if (ok2) {
        const double dlt = delta_fn(M.smearing, sp, en1 + en2 - en3, vzp);
        if (dlt > 0.0) {
          const double f = phxc::pi * 0.25 * w * dlt * M.norm / (en1 * en2 * en3);
#pragma unroll
          for (int c = 0; c < kMaxT; ++c)
            if (c < nT) {
              const double n1 = M.bose[((size_t)c * nq + q1) * nb + b1];
              const double n2 = M.bose[((size_t)c * nq + iq2) * nb + b2];
              const double n3 = M.bose[((size_t)c * nq + iq3) * nb + b3];
              r[c] += 0.5 * (f * n1 * n2 * (n3 + 1.0));
            }
        }
      }
      if (ok2m) {
        double d1 = delta_fn(M.smearing, sm, en1 + en3 - en2m, vzm);
        double d2 = delta_fn(M.smearing, sm, en2m + en3 - en1, vzm);
        if (d1 > 0.0 || d2 > 0.0) {
          d1 = fmax(d1, 0.0);
          d2 = fmax(d2, 0.0);
          const double f = phxc::pi * 0.25 * w * M.norm / (en1 * en2m * en3);
#pragma unroll
          for (int c = 0; c < kMaxT; ++c)
            if (c < nT) {
              const double n1 = M.bose[((size_t)c * nq + q1) * nb + b1];
              const double n2m = M.bose[((size_t)c * nq + iq2m) * nb + b2];
              const double n3 = M.bose[((size_t)c * nq + iq3) * nb + b3];
              r[c] += 0.5 * (f * n3 * n1 * (n2m + 1.0) * d1 + f * n2m * n3 * (n1 + 1.0) * d2);
            }
        }
      }
#pragma unroll
      for (int c = 0; c < kMaxT; ++c)
        if (c < nT && r[c] != 0.0) atomicAdd(&acc[(q * nb + b1) * kMaxT + c], r[c]);
    }
  }
  __syncthreads();
  for (int i = tid; i < Q1 * nb * nT; i += NT) {
    const int q = i / (nb * nT), rest = i % (nb * nT), b1 = rest / nT, c = rest % nT;
    const int q1 = q1s[q];
    if (q1 >= 0) P.partial[((size_t)blockIdx.y * nq + q1) * nb * nT + rest] += acc[(q * nb + b1) * kMaxT + c];
  }
}

// Isotope scattering (ph_scattering.cpp:616-793), linewidth mode: one thread
// per (q1, b1) of a tile of kTile q1, looping over the q2 of its slot;
//   rate = pi/2 norm w1 w2 delta(w1 - w2) sum_atoms g_a |sum_k conj(U1(3a+k,b1)) U2(3a+k,b2)|^2
//          (n1 n2 + (n1 + n2)/2),
// with U mass-scaled and g_a the reference's massVariance (variance x mass^2).
// Adaptive smearing takes its width from v1 and halves the delta, as the
// reference does (:684-687).  Rates go to the partial sums of the slot and,
// in the matrix modes, are subtracted from the element (q1 b1, q2 b2) of the
// matrix or of the "+" slab (same layouts as PairArgs; this kernel runs after
// the pair kernels, and each element has one writer).
struct IsoArgs {
  MeshArgs m;
  int nat;
  const double* g;      // (nat)
  int q2_first, q2_count, q2_per_slot;
  double* partial;      // (S, nq, nb, nT)
  double* mat = nullptr;
  long long ld = 0;
  size_t mat_tstride = 0;
  int mat_full = 0;
};

inline size_t iso_smem(int nb) { return sizeof(double2) * nb * nb + sizeof(double) * nb; }

__global__ void __launch_bounds__(kTile * kMaxNbGeneric) isotope_kernel(IsoArgs A) {
  const MeshArgs& M = A.m;
  extern __shared__ __align__(16) char sraw[];
  const int nb = M.nb, nbb = nb * nb, nT = M.nT, nq = M.nq;
  double2* U2 = reinterpret_cast<double2*>(sraw);           // [nb][nb]
  double* E2 = reinterpret_cast<double*>(U2 + nbb);         // [nb]
  const int tid = threadIdx.x, ql = tid % kTile, b1 = tid / kTile;
  const int q1 = blockIdx.x * kTile + ql;
  const bool active = b1 < nb && q1 < nq;
  const int q1c = active ? q1 : 0, b1c = active ? b1 : 0;
  const double en1 = M.E[(size_t)q1c * nb + b1c];
  const bool ok1 = active && en1 >= phxc::phExcludeCutoff && en1 >= phxc::phEnergyCutoff;
  double2 u1[kMaxNbGeneric];
#pragma unroll
  for (int a = 0; a < kMaxNbGeneric; ++a)
    u1[a] = a < nb ? M.U[(size_t)q1c * nbb + a * nb + b1c] : cmk(0.0, 0.0);
  double sg1 = M.sigma;
  bool vz1 = false;
  if (M.smearing == PHX_SMEAR_ADAPTIVE && M.vg) {
    const double* v = M.vg + ((size_t)q1c * nb + b1c) * 3;
    vz1 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) == 0.0;
    sg1 = floor_sigma(adaptive_sigma(M.qT, v[0], v[1], v[2]));
  }
  double n1[kMaxT], acc[kMaxT];
#pragma unroll
  for (int c = 0; c < kMaxT; ++c) {
    n1[c] = c < nT ? M.bose[((size_t)c * nq + q1c) * nb + b1c] : 0.0;
    acc[c] = 0.0;
  }
  const int jbeg = blockIdx.y * A.q2_per_slot;
  const int jend = min(A.q2_count, jbeg + A.q2_per_slot);
  for (int j = jbeg; j < jend; ++j) {
    const int iq2 = A.q2_first + j;
    __syncthreads();
    for (int e = tid; e < nbb; e += blockDim.x) U2[e] = M.U[(size_t)iq2 * nbb + e];
    for (int b = tid; b < nb; b += blockDim.x) E2[b] = M.E[(size_t)iq2 * nb + b];
    __syncthreads();
    if (!ok1) continue;
    for (int b2 = 0; b2 < nb; ++b2) {
      const double en2 = E2[b2];
      if (en2 < phxc::phExcludeCutoff || en2 < phxc::phEnergyCutoff) continue;
      double dl;
      if (M.smearing == PHX_SMEAR_GAUSSIAN) dl = delta_fn(PHX_SMEAR_GAUSSIAN, M.sigma, en1 - en2, false);
      else dl = 0.5 * delta_fn(PHX_SMEAR_ADAPTIVE, sg1, en1 - en2, vz1);
      if (dl == 0.0) continue;
      // z_atom = sum_k conj(U1(3 atom + k, b1)) U2(3 atom + k, b2)
      constexpr int kAt = (kMaxNbGeneric + 2) / 3;
      double2 z[kAt];
#pragma unroll
      for (int at = 0; at < kAt; ++at) z[at] = cmk(0.0, 0.0);
#pragma unroll
      for (int a = 0; a < kMaxNbGeneric; ++a)
        if (a < nb) cfmac(z[a / 3], U2[a * nb + b2], u1[a]);
      double term = 0.0;
#pragma unroll
      for (int at = 0; at < kAt; ++at)
        if (at < A.nat) term += (z[at].x * z[at].x + z[at].y * z[at].y) * A.g[at];
      term *= phxc::pi * 0.5 * M.norm * en1 * en2 * dl;
#pragma unroll
      for (int c = 0; c < kMaxT; ++c)
        if (c < nT) {
          const double n2 = M.bose[((size_t)c * nq + iq2) * nb + b2];
          const double r = term * (n1[c] * n2 + 0.5 * (n1[c] + n2));
          acc[c] += r;
          if (A.mat) {
            const size_t row = (size_t)q1 * nb + b1;
            double* dst = A.mat_full ? A.mat + (size_t)(iq2 * nb + b2) * A.ld + row
                                     : A.mat + c * A.mat_tstride + (size_t)(j * nb + b2) * A.ld + row;
            *dst -= r;
          }
        }
    }
  }
  if (active) {
    double* out = A.partial + (((size_t)blockIdx.y * nq + q1) * nb + b1) * nT;
    for (int c = 0; c < nT; ++c) out[c] += acc[c];
  }
}

// Sums the partial slots into A_out; with finalize: degeneracy averaging of
// row 0, then boundary scattering |v|/L n(n+1) on every row (added after the
// averaging, ph_scattering.cpp:819-860), then zero for excluded states.
// The matrix modes pass average = 0: their diagonal is not averaged
// (ph_scattering.cpp:809-817).
__global__ void finalize_kernel(int nq, int nb, int nT, int nslots, const double* __restrict__ partial,
                                const double* __restrict__ E, int finalize, const double* __restrict__ vg,
                                const double* __restrict__ temps, double boundary_length,
                                double* __restrict__ Aout, int average = 1) {
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= nq) return;
  const size_t ns = (size_t)nq * nb;
  double lw[64];
  for (int c = 0; c < nT; ++c) {
    for (int b = 0; b < nb; ++b) {
      double s = 0.0;
      for (int k = 0; k < nslots; ++k) s += partial[(((size_t)k * nq + iq) * nb + b) * nT + c];
      lw[b] = s;
    }
    if (finalize && average && c == 0) {
      // degeneracyAveragingLinewidths (scattering.cpp:1168-1207), row 0 only
      double tmp[64];
      for (int b1 = 0; b1 < nb; ++b1) {
        int n = 0;
        double t = 0.0;
        for (int b2 = 0; b2 < nb; ++b2)
          if (fabs(E[(size_t)iq * nb + b2] - E[(size_t)iq * nb + b1]) < phxc::degThreshold) {
            ++n;
            t += lw[b2];
          }
        tmp[b1] = t / (double)(float)n;
      }
      for (int b = 0; b < nb; ++b) lw[b] = tmp[b];
    }
    if (finalize && boundary_length > 0.0 && vg) {
      for (int b = 0; b < nb; ++b) {
        const double e = E[(size_t)iq * nb + b];
        if (e < phxc::phExcludeCutoff) continue;
        const double* v = vg + ((size_t)iq * nb + b) * 3;
        const double x = sinh(e / 2.0 / temps[c]);
        lw[b] += sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / boundary_length * (0.25 / x / x);
      }
    }
    for (int b = 0; b < nb; ++b) {
      double v = lw[b];
      if (finalize && E[(size_t)iq * nb + b] < phxc::phExcludeCutoff) v = 0.0;
      Aout[(size_t)c * ns + (size_t)iq * nb + b] = v;
    }
  }
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

// split-precision path (split.cu)
int phx_split_kp(int nr3);
size_t phx_split_bimg_bytes(int chunk, int nr3);
size_t phx_split_smem_bytes(int nr3, int nT);
int phx_split_set_attributes(phx_ctx* ctx, int nr3, int nT);
int phx_split_prepare_bands(phx_ctx* ctx, phx_bands* b);
size_t phx_split_rec_bytes(int nq);
int phx_split_pack_records(phx_ctx* ctx, const pairc::MeshArgs& M, void* rec, int* launches);
int phx_split_pair_chunk(phx_ctx* ctx, const pairc::MeshArgs& M, const phx_v3* v, const phx_bands* b,
                         const double2* Dp, uint8_t* Bimg, const void* rec, double emax, int q2_first,
                         int q2_count, int slots, double* partial, int* launches, cudaEvent_t ev_begin,
                         cudaEvent_t ev_end, int fp16, const unsigned* dmax, void* edges, unsigned* edge_count,
                         unsigned edge_cap, unsigned* edge_peak, unsigned* edge_overflow, int edge_only,
                         const phx_split_matrix* mat = nullptr);
unsigned phx_split_edge_cap();
size_t phx_split_edge_bytes();

int phx_scratch_reserve(phx_v3* v, size_t bytes) {
  return phx_ctx_reserve(v->ctx, &v->ctx->d_scratch, &v->ctx->scratch_bytes, bytes);
}

// ---------------------------------------------------------------------------
// band structures on a mesh
// ---------------------------------------------------------------------------
void phx_mesh_cartesian(const int* mesh, const double* recip, std::vector<double>& q) {
  const int nq = mesh[0] * mesh[1] * mesh[2];
  q.resize(3 * (size_t)nq);
  for (int i = 0; i < nq; ++i) {
    const int iz = i / (mesh[0] * mesh[1]);
    const int r = i - iz * mesh[0] * mesh[1];
    const int iy = r / mesh[0], ix = r % mesh[0];
    const double c[3] = {double(ix) / double(mesh[0]), double(iy) / double(mesh[1]),
                         double(iz) / double(mesh[2])};
    for (int k = 0; k < 3; ++k)
      q[3 * i + k] = recip[k * 3 + 0] * c[0] + recip[k * 3 + 1] * c[1] + recip[k * 3 + 2] * c[2];
  }
}

extern "C" int phx_bands_create_mesh(phx_ph_h0* h0, const int* mesh, int with_velocities,
                                     phx_bands** out) {
  PHX_ARG(nullptr, h0 && mesh && out, "phx_bands_create_mesh: bad arguments");
  phx_ctx* ctx = h0->ctx;
  PHX_ARG(ctx, mesh[0] > 0 && mesh[1] > 0 && mesh[2] > 0, "bad mesh");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  phx_bands* b = new phx_bands;
  b->ctx = ctx;
  b->nb = h0->nb;
  b->nq = mesh[0] * mesh[1] * mesh[2];
  for (int i = 0; i < 3; ++i) b->mesh[i] = mesh[i];
  for (int i = 0; i < 9; ++i) b->recip[i] = h0->recip[i];
  std::vector<double> q;
  phx_mesh_cartesian(mesh, h0->recip, q);
  const size_t nq = b->nq, nb = b->nb;
  cudaError_t e = phx_dev_alloc(ctx, (void**)&b->d_E, sizeof(double) * nq * nb);
  if (e == cudaSuccess) e = phx_dev_alloc(ctx, (void**)&b->d_U, sizeof(double) * 2 * nq * nb * nb);
  if (e == cudaSuccess && with_velocities) e = phx_dev_alloc(ctx, (void**)&b->d_vg, sizeof(double) * 3 * nq * nb);
  if (e == cudaSuccess) e = phx_dev_alloc(ctx, (void**)&b->d_q, sizeof(double) * 3 * nq);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_q, q.data(), sizeof(double) * 3 * nq, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
    phx_bands_destroy(b);
    return PHX_ERR_CUDA;
  }
  int rc = phx_launch_ph_bands(h0, b->nq, b->d_q, b->d_E, b->d_U, b->d_vg, 1);
  if (rc != PHX_OK) {
    phx_bands_destroy(b);
    return rc;
  }
  *out = b;
  return PHX_OK;
}

extern "C" int phx_bands_create_from_host(phx_ctx* ctx, const int* mesh,
                                          const double* reciprocal_cell, int nb, const double* E,
                                          const double* U, const double* vg, phx_bands** out) {
  PHX_ARG(ctx, ctx && mesh && reciprocal_cell && E && U && out && nb > 0 && nb <= 63,
          "phx_bands_create_from_host: bad arguments");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  phx_bands* b = new phx_bands;
  b->ctx = ctx;
  b->nb = nb;
  b->nq = mesh[0] * mesh[1] * mesh[2];
  for (int i = 0; i < 3; ++i) b->mesh[i] = mesh[i];
  for (int i = 0; i < 9; ++i) b->recip[i] = reciprocal_cell[i];
  std::vector<double> q;
  phx_mesh_cartesian(mesh, reciprocal_cell, q);
  const size_t nq = b->nq;
  cudaError_t e = phx_dev_alloc(ctx, (void**)&b->d_E, sizeof(double) * nq * nb);
  if (e == cudaSuccess) e = phx_dev_alloc(ctx, (void**)&b->d_U, sizeof(double) * 2 * nq * nb * nb);
  if (e == cudaSuccess && vg) e = phx_dev_alloc(ctx, (void**)&b->d_vg, sizeof(double) * 3 * nq * nb);
  if (e == cudaSuccess) e = phx_dev_alloc(ctx, (void**)&b->d_q, sizeof(double) * 3 * nq);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_E, E, sizeof(double) * nq * nb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_U, U, sizeof(double) * 2 * nq * nb * nb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && vg)
    e = cudaMemcpyAsync(b->d_vg, vg, sizeof(double) * 3 * nq * nb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_q, q.data(), sizeof(double) * 3 * nq, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
    phx_bands_destroy(b);
    return PHX_ERR_CUDA;
  }
  *out = b;
  return PHX_OK;
}

extern "C" int phx_bands_destroy(phx_bands* b) {
  if (!b) return PHX_OK;
  if (b->ctx) {
    cudaSetDevice(b->ctx->device);
    phx_dev_free(b->ctx, b->d_E);
    phx_dev_free(b->ctx, b->d_U);
    phx_dev_free(b->ctx, b->d_vg);
    phx_dev_free(b->ctx, b->d_q);
    phx_dev_free(b->ctx, b->d_U32);
    phx_dev_free(b->ctx, b->d_q1_order);
  }
  delete b;
  return PHX_OK;
}

extern "C" int phx_bands_num_points(const phx_bands* b) { return b ? b->nq : 0; }

extern "C" int phx_bands_get(phx_bands* b, double* E, double* U, double* vg) {
  PHX_ARG(nullptr, b, "null bands handle");
  phx_ctx* ctx = b->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t nq = b->nq, nb = b->nb;
  if (E) PHX_CUDA(ctx, cudaMemcpyAsync(E, b->d_E, sizeof(double) * nq * nb, cudaMemcpyDeviceToHost, ctx->stream));
  if (U)
    PHX_CUDA(ctx, cudaMemcpyAsync(U, b->d_U, sizeof(double) * 2 * nq * nb * nb, cudaMemcpyDeviceToHost, ctx->stream));
  if (vg) {
    PHX_ARG(ctx, b->d_vg != nullptr, "band structure has no velocities");
    PHX_CUDA(ctx, cudaMemcpyAsync(vg, b->d_vg, sizeof(double) * 3 * nq * nb, cudaMemcpyDeviceToHost, ctx->stream));
  }
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

// ---------------------------------------------------------------------------
// builder
// ---------------------------------------------------------------------------
namespace {

struct BuilderPlan {
  int chunk = 512;      // q2 per fold/pair launch
  int slots = 8;        // partial-sum slots (q2 slices per chunk)
};

// ---------------------------------------------------------------------------
// Launch plans and CUDA graphs of the builder
//
// Autotuner: the first call for a problem shape (path, nb, nq, nr3, nr2, nT,
// device) times each candidate (chunk, slots) on one chunk of q2 with CUDA
// events and keeps the fastest per q2 for the rest of the process
// (PHX_TUNE=0: fixed defaults).  Graphs: the device work of a call -- the
// memsets, Bose factors, records, every fold / conversion / pair launch of
// the q2 loop and the finalisation -- is captured into a CUDA graph owned by
// the v3 object and replayed when a later call touches the same buffers with
// the same parameters (PHX_GRAPHS=0: eager launches).  Temperatures and
// windows are copied to the device outside the graph, so their values may
// change between replays.
// ---------------------------------------------------------------------------
bool env_off(const char* name) {
  const char* e = std::getenv(name);
  return e && e[0] == '0';
}
bool env_on(const char* name) {
  const char* e = std::getenv(name);
  return e && e[0] == '1';
}

struct PlanKey {
  int kind, nb, nq, nr3, nr2, nT, device;
  bool operator<(const PlanKey& o) const {
    return std::tie(kind, nb, nq, nr3, nr2, nT, device) < std::tie(o.kind, o.nb, o.nq, o.nr3, o.nr2, o.nT, o.device);
  }
};
std::mutex g_plan_mutex;
std::map<PlanKey, BuilderPlan> g_plans;

bool find_plan(const PlanKey& k, BuilderPlan* out) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = g_plans.find(k);
  if (it == g_plans.end()) return false;
  *out = it->second;
  return true;
}
void store_plan(const PlanKey& k, const BuilderPlan& p) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  g_plans[k] = p;
}

}  // namespace

struct phx_builder_graph {
  std::vector<uint64_t> key;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t vertex_begin = nullptr, vertex_end = nullptr;
  std::vector<cudaEvent_t> pair_events;
  int launches = 0;
};
struct phx_builder_graphs {
  std::vector<phx_builder_graph> entries;   // most recent last, at most 4
};

void phx_builder_graph_free(phx_builder_graph& g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.vertex_begin) cudaEventDestroy(g.vertex_begin);
  if (g.vertex_end) cudaEventDestroy(g.vertex_end);
  for (cudaEvent_t e : g.pair_events) cudaEventDestroy(e);
  g = phx_builder_graph();
}

void phx_builder_release(phx_v3* v) {
  if (!v->graphs) return;
  for (auto& g : v->graphs->entries) phx_builder_graph_free(g);
  delete v->graphs;
  v->graphs = nullptr;
}

namespace {

uint64_t bits(double x) {
  uint64_t u;
  std::memcpy(&u, &x, sizeof(u));
  return u;
}
uint64_t bits(const void* p) { return (uint64_t)(uintptr_t)p; }

// Runs `work` (the device work of one call, which records the vertex-loop
// events and appends its pair events) eagerly the first time a key is seen,
// captured into a graph the second time, and as a replay of that graph after
// that (objects used for a single call never build one).  On return, *g
// points at the entry whose events carry this call's timings (`tmp` when
// eager).
template <class Work>
int run_device_work(phx_v3* v, const std::vector<uint64_t>& key, Work&& work, phx_builder_graph* tmp,
                    phx_builder_graph** g, int* graph_state) {
  phx_ctx* ctx = v->ctx;
  cudaStream_t st = ctx->stream;
  auto make_events = [&](phx_builder_graph& e) -> int {
    PHX_CUDA(ctx, cudaEventCreate(&e.vertex_begin));
    PHX_CUDA(ctx, cudaEventCreate(&e.vertex_end));
    return PHX_OK;
  };
  if (env_off("PHX_GRAPHS")) {
    PHX_TRY(make_events(*tmp));
    PHX_TRY(work(*tmp));
    *g = tmp;
    *graph_state = 0;
    return PHX_OK;
  }
  if (!v->graphs) v->graphs = new phx_builder_graphs;
  auto& es = v->graphs->entries;
  bool seen = false;
  for (size_t i = 0; i < es.size(); ++i)
    if (es[i].key == key) {
      std::rotate(es.begin() + i, es.begin() + i + 1, es.end());
      if (es.back().exec) {
        PHX_CUDA(ctx, cudaGraphLaunch(es.back().exec, st));
        *g = &es.back();
        *graph_state = 2;
        return PHX_OK;
      }
      phx_builder_graph_free(es.back());
      es.pop_back();
      seen = true;
      break;
    }
  if (!seen) {
    // first call with this key: eager, remembered for the next one
    PHX_TRY(make_events(*tmp));
    PHX_TRY(work(*tmp));
    if (es.size() >= 4) {
      phx_builder_graph_free(es.front());
      es.erase(es.begin());
    }
    phx_builder_graph mark;
    mark.key = key;
    es.push_back(std::move(mark));
    *g = tmp;
    *graph_state = 0;
    return PHX_OK;
  }
  phx_builder_graph e;
  e.key = key;
  int rc = make_events(e);
  cudaGraph_t graph = nullptr;
  if (rc == PHX_OK) {
    cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      rc = PHX_ERR_CUDA;
    } else {
      rc = work(e);
      ce = cudaStreamEndCapture(st, &graph);
      if (rc == PHX_OK && ce != cudaSuccess) {
        phx_set_error(ctx, PHX_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        rc = PHX_ERR_CUDA;
      }
    }
  }
  if (rc == PHX_OK) {
    cudaError_t ce = cudaGraphInstantiate(&e.exec, graph, 0);
    if (ce != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
      rc = PHX_ERR_CUDA;
    }
  }
  if (graph) cudaGraphDestroy(graph);
  if (rc != PHX_OK) {
    phx_builder_graph_free(e);
    return rc;
  }
  PHX_CUDA(ctx, cudaGraphLaunch(e.exec, st));
  if (es.size() >= 4) {
    phx_builder_graph_free(es.front());
    es.erase(es.begin());
  }
  es.push_back(std::move(e));
  *g = &es.back();
  *graph_state = 1;
  return PHX_OK;
}

template <int NB>
int run_builder(phx_v3* v, phx_bands* b, const phx_lw_params* p, double* Aout_d,
                phx_lw_stats* stats) {
  phx_ctx* ctx = v->ctx;
  cudaStream_t st = ctx->stream;
  const int nq = b->nq, nT = p->num_temperatures, nr3 = v->nr3, nr2 = v->nr2;
  const int q2b = p->q2_begin, q2e = p->q2_end;
  const bool split = v->precision != PHX_PREC_FP64;
  // candidate plans; the first is the default
  std::vector<BuilderPlan> cands;
  if (split)
    cands = {{448, 7}, {448, 14}, {896, 14}, {896, 28}, {1792, 14}, {1792, 28}};
  else
    cands = {{512, 8}, {512, 4}, {512, 16}, {1024, 16}};
  int max_chunk = 0;
  for (auto& c : cands) max_chunk = std::max(max_chunk, c.chunk);
  max_chunk = std::min(max_chunk, std::max(1, q2e - q2b));
  int max_slots = 0;
  for (auto& c : cands) max_slots = std::max(max_slots, c.slots);
  const size_t nb3 = (size_t)NB * NB * NB;
  const size_t sz_dp = align_up(sizeof(double2) * max_chunk * nr3 * nb3);
  const size_t sz_part = align_up(sizeof(double) * max_slots * nq * NB * nT);
  const size_t sz_bose = align_up(sizeof(double) * nT * nq * NB);
  const size_t sz_T = align_up(sizeof(double) * 8);
  const size_t sz_img = split ? align_up(phx_split_bimg_bytes(max_chunk, nr3)) : 0;
  const size_t sz_rec = split ? align_up(phx_split_rec_bytes(nq)) : 0;
  const size_t sz_iso = p->isotope_coupling ? align_up(sizeof(double) * v->nat) : 0;
  // per chunk: flag of a near-cut-off event list that overflowed (the smallest candidate chunk is 448 q2)
  const int max_chunks = (q2e - q2b + 447) / 448 + 1;
  const size_t sz_max = align_up(sizeof(unsigned) * (4 + max_chunks + 1));
  const size_t sz_edge = split ? align_up(phx_split_edge_bytes()) : 0;
  PHX_TRY(phx_scratch_reserve(v, sz_dp + sz_part + sz_bose + sz_T + sz_img + sz_rec + sz_iso + sz_max + sz_edge));
  char* base = static_cast<char*>(v->ctx->d_scratch);
  double2* Dp = reinterpret_cast<double2*>(base);
  double* partial = reinterpret_cast<double*>(base + sz_dp);
  double* bose = reinterpret_cast<double*>(base + sz_dp + sz_part);
  double* temps = reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose);
  uint8_t* Bimg = reinterpret_cast<uint8_t*>(base + sz_dp + sz_part + sz_bose + sz_T);
  void* rec = base + sz_dp + sz_part + sz_bose + sz_T + sz_img;
  double* giso = p->isotope_coupling ? reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose + sz_T + sz_img +
                                                                 sz_rec)
                                     : nullptr;
  // FP16 operands of the split path: max |Dp| of the current chunk
  const int fp16 = v->precision == PHX_PREC_SPLIT_FP16 ? 1 : 0;
  unsigned* dmax = reinterpret_cast<unsigned*>(base + sz_dp + sz_part + sz_bose + sz_T + sz_img + sz_rec + sz_iso);
  unsigned* edge_count = dmax + 1;
  unsigned* edge_peak = dmax + 2;   // largest near-cut-off event count of the call's pair launches
  unsigned* edge_flags = dmax + 4;  // [max_chunks] overflow flag of each chunk, then one for re-runs
  const unsigned edge_cap = phx_split_edge_cap();
  void* edges = base + sz_dp + sz_part + sz_bose + sz_T + sz_img + sz_rec + sz_iso + sz_max;
  if (split) {
    PHX_ARG(ctx, NB == 6, "split-precision path supports nb = 6");
    PHX_ARG(ctx, phx_split_smem_bytes(nr3, nT) <= 227 * 1024, "too many R3 vectors for the split path");
    PHX_TRY(phx_split_prepare_bands(ctx, b));
    if (b->emax < 0.0) {
      // largest energy of the mesh (margin of the split path's FP32 windows), once per band structure
      std::vector<double> Eh((size_t)nq * NB);
      PHX_CUDA(ctx, cudaMemcpy(Eh.data(), b->d_E, sizeof(double) * Eh.size(), cudaMemcpyDeviceToHost));
      double m = 0.0;
      for (double e : Eh) m = std::max(m, std::fabs(e));
      b->emax = m;
    }
  }
  const double emax = split ? b->emax : 0.0;
  PairArgs P{};
  P.m.nq = nq;
  P.m.nb = NB;
  P.m.nT = nT;
  P.m.n0 = b->mesh[0];
  P.m.n1 = b->mesh[1];
  P.m.n2 = b->mesh[2];
  P.m.E = b->d_E;
  P.m.U = reinterpret_cast<const double2*>(b->d_U);
  P.m.vg = b->d_vg;
  P.m.bose = bose;
  P.m.qcart = b->d_q;
  P.m.smearing = p->smearing;
  P.m.sigma = p->sigma;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P.m.qT[i * 3 + j] = b->recip[i * 3 + j] / b->mesh[i];
  P.m.norm = 1.0 / (double)nq;
  P.nr3 = nr3;
  P.R3 = v->d_R3;
  P.Dp = Dp;
  P.partial = partial;
  const size_t smem_pair = sizeof(double2) * ((size_t)nr3 * kTile + 2 * NB * NB * kTile) +
                           sizeof(double) * ((size_t)NB * NB * NB * kTile + (size_t)kMaxT * NB * kTile);
  if (!split) {
    PHX_ARG(ctx, smem_pair <= 227 * 1024, "phx_ph_linewidths: too many R3 vectors for the FP64 path");
    PHX_CUDA(ctx, cudaFuncSetAttribute(pair_fp64_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_pair));
  }
  const size_t smem_fold = fold_tiled_smem(NB, nr2);
  PHX_ARG(ctx, smem_fold <= 227 * 1024, "phx_ph_linewidths: too many R2 vectors");
  if (smem_fold > 48 * 1024)
    PHX_CUDA(ctx, cudaFuncSetAttribute(fold_q2_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_fold));
  if (split) PHX_TRY(phx_split_set_attributes(ctx, nr3, nT));
  const int tiles = (nq + kTile - 1) / kTile;
  // one chunk of the q2 loop; pe0/pe1 (may be null) bracket its pair kernel
  auto chunk_work = [&](const BuilderPlan& pl, int c0, int cnt, cudaEvent_t pe0, cudaEvent_t pe1,
                        int* launches, unsigned* overflow = nullptr, int edge_only = 0) -> int {
    if (fp16) PHX_CUDA(ctx, cudaMemsetAsync(dmax, 0, sizeof(unsigned), st));
    fold_tiled_launch(NB, nr2, nr3, v, b, c0, cnt, Dp, st, fp16 ? dmax : nullptr);
    ++*launches;
    if (split)
      return phx_split_pair_chunk(ctx, P.m, v, b, Dp, Bimg, rec, emax, c0, cnt, pl.slots, partial, launches,
                                  pe0, pe1, fp16, dmax, edges, edge_count, edge_cap, edge_peak, overflow,
                                  edge_only);
    PairArgs Q = P;
    Q.q2_first = c0;
    Q.q2_count = cnt;
    Q.q2_per_slot = (cnt + pl.slots - 1) / pl.slots;
    if (pe0) PHX_CUDA(ctx, phx_record_event(pe0, st));
    pair_fp64_kernel<NB><<<dim3(tiles, pl.slots), kTile * NB, smem_pair, st>>>(Q);
    if (pe1) PHX_CUDA(ctx, phx_record_event(pe1, st));
    ++*launches;
    PHX_CUDA(ctx, cudaGetLastError());
    return PHX_OK;
  };
  PHX_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
  PHX_CUDA(ctx, cudaMemcpyAsync(temps, p->temperatures, sizeof(double) * nT, cudaMemcpyHostToDevice, st));
  if (giso)
    PHX_CUDA(ctx, cudaMemcpyAsync(giso, p->isotope_coupling, sizeof(double) * v->nat, cudaMemcpyHostToDevice, st));
  // launch plan: tuned once per problem shape
  int dev = 0;
  cudaGetDevice(&dev);
  const PlanKey pk{split ? 1 + fp16 : 0, NB, nq, nr3, nr2, nT, dev};
  BuilderPlan plan = cands[0];
  if (!env_off("PHX_TUNE") && q2e - q2b >= 2 * cands[0].chunk && !find_plan(pk, &plan)) {
    int dummy = 0;
    if (split) PHX_TRY(phx_split_pack_records(ctx, P.m, rec, &dummy));
    bose_kernel<<<std::min(1024, (nq * NB * nT + 255) / 256), 256, 0, st>>>(nq, NB, nT, b->d_E, temps, bose);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    PHX_CUDA(ctx, cudaEventCreate(&t0));
    PHX_CUDA(ctx, cudaEventCreate(&t1));
    double best = 1e300;
    int rc = PHX_OK;
    for (const auto& c : cands) {
      const int cnt = std::min(c.chunk, q2e - q2b);
      const BuilderPlan cc{cnt, std::min(c.slots, cnt)};
      cudaEventRecord(t0, st);
      rc = chunk_work(cc, q2b, cnt, nullptr, nullptr, &dummy);
      cudaEventRecord(t1, st);
      if (rc == PHX_OK && cudaEventSynchronize(t1) != cudaSuccess) rc = PHX_ERR_CUDA;
      if (rc != PHX_OK) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, t0, t1);
      if (ms / cnt < best) {
        best = ms / cnt;
        plan = c;
      }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != PHX_OK) {
      if (rc == PHX_ERR_CUDA) phx_set_error(ctx, PHX_ERR_CUDA, "builder autotuner: a timed candidate failed");
      return rc;
    }
    store_plan(pk, plan);
  }
  plan.chunk = std::min(plan.chunk, std::max(1, q2e - q2b));
  plan.slots = std::min(plan.slots, plan.chunk);
  const int nslots = plan.slots;
  // the device work of the call
  auto work = [&](phx_builder_graph& g) -> int {
    int launches = 0;
    PHX_CUDA(ctx, cudaMemsetAsync(partial, 0, sizeof(double) * nslots * nq * NB * nT, st));
    if (split) PHX_CUDA(ctx, cudaMemsetAsync(edge_peak, 0, sizeof(unsigned) * (3 + max_chunks), st));
    bose_kernel<<<std::min(1024, (nq * NB * nT + 255) / 256), 256, 0, st>>>(nq, NB, nT, b->d_E, temps, bose);
    ++launches;
    if (split) PHX_TRY(phx_split_pack_records(ctx, P.m, rec, &launches));
    PHX_CUDA(ctx, phx_record_event(g.vertex_begin, st));
    for (int c0 = q2b; c0 < q2e; c0 += plan.chunk) {
      const int cnt = std::min(plan.chunk, q2e - c0);
      cudaEvent_t pe0 = nullptr, pe1 = nullptr;
      PHX_CUDA(ctx, cudaEventCreate(&pe0));
      g.pair_events.push_back(pe0);
      PHX_CUDA(ctx, cudaEventCreate(&pe1));
      g.pair_events.push_back(pe1);
      PHX_TRY(chunk_work(plan, c0, cnt, pe0, pe1, &launches, split ? edge_flags + (c0 - q2b) / plan.chunk : nullptr));
    }
    PHX_CUDA(ctx, phx_record_event(g.vertex_end, st));
    if (giso) {
      IsoArgs I{P.m, v->nat, giso, q2b, q2e - q2b, (q2e - q2b + nslots - 1) / nslots, partial};
      isotope_kernel<<<dim3(tiles, nslots), kTile * NB, iso_smem(NB), st>>>(I);
      ++launches;
      PHX_CUDA(ctx, cudaGetLastError());
    }
    finalize_kernel<<<(nq + 127) / 128, 128, 0, st>>>(nq, NB, nT, nslots, partial, b->d_E, p->finalize, b->d_vg,
                                                      temps, p->boundary_length, Aout_d);
    ++launches;
    PHX_CUDA(ctx, cudaGetLastError());
    g.launches = launches;
    return PHX_OK;
  };
  const std::vector<uint64_t> key = {
      (uint64_t)(split ? 1 + fp16 : 0), (uint64_t)NB, (uint64_t)nq, (uint64_t)nT, (uint64_t)q2b, (uint64_t)q2e,
      (uint64_t)p->smearing, bits(p->sigma), (uint64_t)p->finalize, (uint64_t)plan.chunk, (uint64_t)plan.slots,
      bits(emax), bits(base), bits(Aout_d), bits(b->d_E), bits(b->d_U), bits(b->d_vg), bits(b->d_q),
      bits(b->d_U32), bits(b->d_q1_order), bits(v->d_D3w), bits(v->d_R2), bits(v->d_R3), bits(ctx->d_status),
      bits(giso), bits(p->boundary_length), (uint64_t)edge_cap};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  PHX_CUDA(ctx, cudaEventCreate(&ev0));
  PHX_CUDA(ctx, cudaEventCreate(&ev1));
  PHX_CUDA(ctx, cudaEventRecord(ev0, st));
  phx_builder_graph eager;
  phx_builder_graph* g = nullptr;
  int graph_state = 0;
  int rc = run_device_work(v, key, work, &eager, &g, &graph_state);
  int kst = 0;
  unsigned epeak = 0;
  if (rc == PHX_OK) {
    cudaError_t ce = cudaEventRecord(ev1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev1);
    if (ce == cudaSuccess) ce = cudaMemcpy(&kst, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess && split) ce = cudaMemcpy(&epeak, edge_peak, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(ce));
      rc = PHX_ERR_CUDA;
    }
  }
  if (rc == PHX_OK && kst) {
    cudaMemset(ctx->d_status, 0, sizeof(int));
    phx_set_error(ctx, PHX_ERR_CUDA,
                  "pair kernel gave up waiting on a pipeline barrier (status " + std::to_string(kst) + ")");
    rc = PHX_ERR_CUDA;
  }
  // Chunks whose near-cut-off events overflowed the list applied none of
  // them: re-run their q2 with the rates off, in pieces whose events fit,
  // then finalise again.  Eager launches, outside any graph.
  int overflowed = 0;
  if (rc == PHX_OK && split) {
    const int nchunks = (q2e - q2b + plan.chunk - 1) / plan.chunk;
    std::vector<unsigned> fl(nchunks, 0u);
    if (cudaMemcpy(fl.data(), edge_flags, sizeof(unsigned) * nchunks, cudaMemcpyDeviceToHost) != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, "reading the near-cut-off overflow flags failed");
      rc = PHX_ERR_CUDA;
    }
    unsigned* piece_flag = edge_flags + max_chunks;
    int dummy = 0;
    for (int ci = 0; ci < nchunks && rc == PHX_OK; ++ci) {
      if (!fl[ci]) continue;
      ++overflowed;
      std::vector<std::pair<int, int>> todo = {{q2b + ci * plan.chunk, std::min(plan.chunk, q2e - (q2b + ci * plan.chunk))}};
      while (!todo.empty() && rc == PHX_OK) {
        const std::pair<int, int> pc = todo.back();
        todo.pop_back();
        const BuilderPlan pp{pc.second, std::min(plan.slots, pc.second)};
        unsigned f = 0;
        rc = [&]() -> int {
          PHX_CUDA(ctx, cudaMemsetAsync(piece_flag, 0, sizeof(unsigned), st));
          PHX_TRY(chunk_work(pp, pc.first, pc.second, nullptr, nullptr, &dummy, piece_flag, 1));
          PHX_CUDA(ctx, cudaMemcpyAsync(&f, piece_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
          PHX_CUDA(ctx, cudaStreamSynchronize(st));
          return PHX_OK;
        }();
        if (rc == PHX_OK && f) {
          if (pc.second == 1) {
            phx_set_error(ctx, PHX_ERR_ARG, "split path: the near-cut-off events of one q2 exceed the event list");
            rc = PHX_ERR_ARG;
          } else {
            const int h = pc.second / 2;
            todo.push_back({pc.first, h});
            todo.push_back({pc.first + h, pc.second - h});
          }
        }
      }
    }
    if (rc == PHX_OK && overflowed) {
      finalize_kernel<<<(nq + 127) / 128, 128, 0, st>>>(nq, NB, nT, nslots, partial, b->d_E, p->finalize, b->d_vg,
                                                        temps, p->boundary_length, Aout_d);
      cudaError_t ce = cudaGetLastError();
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
      if (ce == cudaSuccess) ce = cudaMemcpy(&kst, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
      if (ce != cudaSuccess || kst) {
        cudaMemset(ctx->d_status, 0, sizeof(int));
        phx_set_error(ctx, PHX_ERR_CUDA, ce != cudaSuccess ? std::string(cudaGetErrorString(ce))
                                                           : "re-run of an overflowed chunk: kernel status " +
                                                                 std::to_string(kst));
        rc = PHX_ERR_CUDA;
      }
    }
  }
  if (rc == PHX_OK && stats) {
    float ms = 0, msv = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventElapsedTime(&msv, g->vertex_begin, g->vertex_end);
    stats->ms_total = ms;
    stats->ms_vertex = msv;
    stats->pairs = (long long)nq * (q2e - q2b);
    stats->kernel_launches = g->launches;
    stats->pair_launches = (int)(g->pair_events.size() / 2);
    double msp = 0.0;
    for (size_t i = 0; i + 1 < g->pair_events.size(); i += 2) {
      float x = 0.f;
      cudaEventElapsedTime(&x, g->pair_events[i], g->pair_events[i + 1]);
      msp += x;
    }
    stats->ms_pair = msp;
    stats->plan_chunk = plan.chunk;
    stats->plan_slots = plan.slots;
    stats->graph = graph_state;
    stats->edge_events_peak = (long long)epeak;
    stats->edge_events_cap = split ? (long long)edge_cap : 0;
    stats->edge_overflow_chunks = overflowed;
    cudaGetLastError();   // an elapsed-time query that failed must not leak into the next call
  }
  phx_builder_graph_free(eager);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  return rc;
}

// Builder for any nb <= kMaxNbGeneric, or with a per-q1 q2 window, FP64:
// fold_q2_kernel (one q2 slab of the cached vertex) + pair_generic_kernel.
int run_builder_generic(phx_v3* v, phx_bands* b, const phx_lw_params* p, double* Aout_d, phx_lw_stats* stats) {
  phx_ctx* ctx = v->ctx;
  cudaStream_t st = ctx->stream;
  const int nq = b->nq, nb = b->nb, nT = p->num_temperatures, nr3 = v->nr3, nr2 = v->nr2;
  const int q2b = p->q2_begin, q2e = p->q2_end;
  PHX_ARG(ctx, nb <= kMaxNbGeneric, "phx_ph_linewidths: at most 16 branches");
  const bool windowed = p->window_energy != nullptr;
  PHX_ARG(ctx, !windowed || p->window_cut, "phx_ph_linewidths: window_energy without window_cut");
  // q1 per block: the most that fits in shared memory (each q2 slab element is read once per block)
  int q1t = 4;
  while (q1t > 1 && generic_smem_bytes(nb, nr3, q1t) > 227 * 1024) q1t /= 2;
  const size_t smem_pair = generic_smem_bytes(nb, nr3, q1t);
  PHX_ARG(ctx, smem_pair <= 227 * 1024, "phx_ph_linewidths: too many R3 vectors for this band count");
  const int tiles = (nq + q1t - 1) / q1t;
  const size_t smem_fold = sizeof(double2) * ((size_t)nr2 + 2 * (size_t)nb * nb);
  PHX_ARG(ctx, smem_fold <= 227 * 1024, "phx_ph_linewidths: too many R2 vectors");
  const size_t nb3 = (size_t)nb * nb * nb, per_q2 = sizeof(double2) * nr3 * nb3;
  // q2 per cached-vertex slab: at most 512 MB of it, at most 512 q2
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>({(size_t)512, (size_t)(q2e - q2b),
                                                                (size_t(512) << 20) / std::max<size_t>(per_q2, 1)}));
  // (q1 tile, slot) blocks: the candidates fill the GPU 4, 8 or 16 times over
  const int fill = std::max(1, (4 * ctx->num_sms + tiles - 1) / tiles);
  const int max_slots = std::min(chunk, 4 * fill);
  const size_t sz_dp = align_up(per_q2 * chunk);
  const size_t sz_part = align_up(sizeof(double) * max_slots * nq * nb * nT);
  const size_t sz_bose = align_up(sizeof(double) * nT * nq * nb);
  const size_t sz_T = align_up(sizeof(double) * 8);
  const size_t sz_win = windowed ? align_up(sizeof(double) * 2 * nq + sizeof(int) * nq) : 0;
  const size_t sz_iso = p->isotope_coupling ? align_up(sizeof(double) * v->nat) : 0;
  PHX_TRY(phx_scratch_reserve(v, sz_dp + sz_part + sz_bose + sz_T + sz_win + sz_iso));
  char* base = static_cast<char*>(v->ctx->d_scratch);
  double2* Dp = reinterpret_cast<double2*>(base);
  double* partial = reinterpret_cast<double*>(base + sz_dp);
  double* bose = reinterpret_cast<double*>(base + sz_dp + sz_part);
  double* temps = reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose);
  double* wdev = reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose + sz_T);
  double* giso = p->isotope_coupling ? reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose + sz_T + sz_win)
                                     : nullptr;
  PHX_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
  if (giso)
    PHX_CUDA(ctx, cudaMemcpyAsync(giso, p->isotope_coupling, sizeof(double) * v->nat, cudaMemcpyHostToDevice, st));
  PHX_CUDA(ctx, cudaMemcpyAsync(temps, p->temperatures, sizeof(double) * nT, cudaMemcpyHostToDevice, st));
  // with a window, q1 in order of their cut: the q1 of a tile keep similar q2 sets
  int* order = windowed ? reinterpret_cast<int*>(wdev + 2 * nq) : nullptr;
  std::vector<int> order_h;
  if (windowed) {
    PHX_CUDA(ctx, cudaMemcpyAsync(wdev, p->window_energy, sizeof(double) * nq, cudaMemcpyHostToDevice, st));
    PHX_CUDA(ctx, cudaMemcpyAsync(wdev + nq, p->window_cut, sizeof(double) * nq, cudaMemcpyHostToDevice, st));
    order_h.resize(nq);
    for (int i = 0; i < nq; ++i) order_h[i] = i;
    std::stable_sort(order_h.begin(), order_h.end(),
                     [&](int a, int c) { return p->window_cut[a] < p->window_cut[c]; });
    PHX_CUDA(ctx, cudaMemcpyAsync(order, order_h.data(), sizeof(int) * nq, cudaMemcpyHostToDevice, st));
  }
  PairArgs P{};
  P.m.nq = nq;
  P.m.nb = nb;
  P.m.nT = nT;
  P.m.n0 = b->mesh[0];
  P.m.n1 = b->mesh[1];
  P.m.n2 = b->mesh[2];
  P.m.E = b->d_E;
  P.m.U = reinterpret_cast<const double2*>(b->d_U);
  P.m.vg = b->d_vg;
  P.m.bose = bose;
  P.m.qcart = b->d_q;
  P.m.smearing = p->smearing;
  P.m.sigma = p->sigma;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P.m.qT[i * 3 + j] = b->recip[i * 3 + j] / b->mesh[i];
  P.m.norm = 1.0 / (double)nq;
  P.nr3 = nr3;
  P.R3 = v->d_R3;
  P.Dp = Dp;
  P.partial = partial;
  Q2Window W{windowed ? wdev : nullptr, windowed ? wdev + nq : nullptr};
  auto generic_fn = q1t == 4 ? pair_generic_kernel<4> : q1t == 2 ? pair_generic_kernel<2> : pair_generic_kernel<1>;
  if (smem_pair > 48 * 1024)
    PHX_CUDA(ctx, cudaFuncSetAttribute(generic_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_pair));
  if (smem_fold > 48 * 1024)
    PHX_CUDA(ctx, cudaFuncSetAttribute(fold_q2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fold));
  auto chunk_work = [&](int c0, int cnt, int slots, int* launches) -> int {
    const int per_block = 8;
    fold_q2_kernel<<<dim3(nr3, (cnt + per_block - 1) / per_block), 128, smem_fold, st>>>(
        nb, nr2, nr3, v->d_D3w, v->d_R2, v->d_R3, b->d_q, reinterpret_cast<const double2*>(b->d_U), c0, cnt,
        per_block, Dp);
    ++*launches;
    PHX_CUDA(ctx, cudaGetLastError());
    PairArgs Q = P;
    Q.q2_first = c0;
    Q.q2_count = cnt;
    Q.q2_per_slot = (cnt + slots - 1) / slots;
    generic_fn<<<dim3(tiles, slots), kGenThreads, smem_pair, st>>>(Q, W, order);
    ++*launches;
    PHX_CUDA(ctx, cudaGetLastError());
    return PHX_OK;
  };
  // slot count tuned once per problem shape (a window makes the work per block uneven)
  int dev = 0;
  cudaGetDevice(&dev);
  const PlanKey pk{windowed ? 3 : 2, nb, nq, nr3, nr2, nT, dev};
  BuilderPlan plan{chunk, std::min(chunk, fill)};
  if (!env_off("PHX_TUNE") && q2e - q2b >= 2 * chunk && !find_plan(pk, &plan)) {
    bose_kernel<<<std::min(1024, (nq * nb * nT + 255) / 256), 256, 0, st>>>(nq, nb, nT, b->d_E, temps, bose);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    PHX_CUDA(ctx, cudaEventCreate(&t0));
    PHX_CUDA(ctx, cudaEventCreate(&t1));
    double best = 1e300;
    int rc = PHX_OK, dummy = 0;
    for (int f : {fill, 2 * fill, 4 * fill}) {
      const int sl = std::min(chunk, f);
      cudaEventRecord(t0, st);
      rc = chunk_work(q2b, chunk, sl, &dummy);
      cudaEventRecord(t1, st);
      if (rc == PHX_OK && cudaEventSynchronize(t1) != cudaSuccess) rc = PHX_ERR_CUDA;
      if (rc != PHX_OK) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, t0, t1);
      if (ms < best) {
        best = ms;
        plan.slots = sl;
      }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != PHX_OK) {
      if (rc == PHX_ERR_CUDA) phx_set_error(ctx, PHX_ERR_CUDA, "builder autotuner: a timed candidate failed");
      return rc;
    }
    store_plan(pk, plan);
  }
  const int slots = plan.slots;
  long long pairs = 0;
  for (int c0 = q2b; c0 < q2e; c0 += chunk) pairs += (long long)nq * std::min(chunk, q2e - c0);
  auto work = [&](phx_builder_graph& g) -> int {
    int launches = 0;
    PHX_CUDA(ctx, cudaMemsetAsync(partial, 0, sizeof(double) * slots * nq * nb * nT, st));
    bose_kernel<<<std::min(1024, (nq * nb * nT + 255) / 256), 256, 0, st>>>(nq, nb, nT, b->d_E, temps, bose);
    ++launches;
    PHX_CUDA(ctx, phx_record_event(g.vertex_begin, st));
    for (int c0 = q2b; c0 < q2e; c0 += chunk) PHX_TRY(chunk_work(c0, std::min(chunk, q2e - c0), slots, &launches));
    PHX_CUDA(ctx, phx_record_event(g.vertex_end, st));
    if (giso) {
      IsoArgs I{P.m, v->nat, giso, q2b, q2e - q2b, (q2e - q2b + slots - 1) / slots, partial};
      isotope_kernel<<<dim3((nq + kTile - 1) / kTile, slots), kTile * nb, iso_smem(nb), st>>>(I);
      ++launches;
      PHX_CUDA(ctx, cudaGetLastError());
    }
    finalize_kernel<<<(nq + 127) / 128, 128, 0, st>>>(nq, nb, nT, slots, partial, b->d_E, p->finalize, b->d_vg,
                                                      temps, p->boundary_length, Aout_d);
    ++launches;
    PHX_CUDA(ctx, cudaGetLastError());
    g.launches = launches;
    return PHX_OK;
  };
  const std::vector<uint64_t> key = {
      (uint64_t)(windowed ? 3 : 2), (uint64_t)nb, (uint64_t)nq, (uint64_t)nT, (uint64_t)q2b, (uint64_t)q2e,
      (uint64_t)p->smearing, bits(p->sigma), (uint64_t)p->finalize, (uint64_t)chunk, (uint64_t)slots, bits(base),
      bits(Aout_d), bits(b->d_E), bits(b->d_U), bits(b->d_vg), bits(b->d_q), bits(v->d_D3w), bits(v->d_R2),
      bits(v->d_R3), bits(ctx->d_status), bits(giso), bits(p->boundary_length)};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  PHX_CUDA(ctx, cudaEventCreate(&ev0));
  PHX_CUDA(ctx, cudaEventCreate(&ev1));
  PHX_CUDA(ctx, cudaEventRecord(ev0, st));
  phx_builder_graph eager;
  phx_builder_graph* g = nullptr;
  int graph_state = 0;
  int rc = run_device_work(v, key, work, &eager, &g, &graph_state);
  if (rc == PHX_OK) {
    cudaError_t ce = cudaEventRecord(ev1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev1);
    if (ce != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(ce));
      rc = PHX_ERR_CUDA;
    }
  }
  if (rc == PHX_OK && stats) {
    float ms = 0, msv = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventElapsedTime(&msv, g->vertex_begin, g->vertex_end);
    stats->ms_total = ms;
    stats->ms_vertex = msv;
    stats->pairs = pairs;
    stats->kernel_launches = g->launches;
    stats->pair_launches = 0;
    stats->ms_pair = 0.0;
    stats->plan_chunk = chunk;
    stats->plan_slots = slots;
    stats->graph = graph_state;
    cudaGetLastError();
  }
  phx_builder_graph_free(eager);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  return rc;
}

// ---------------------------------------------------------------------------
// Matrix modes of the builder (ph_scattering.cpp, switchCase 0 and 1, without
// symmetries), FP64, nb = 6.  The q2 loop is the linewidth builder's: the R2
// fold of a chunk, then pair_fp64_kernel<6, true>, whose epilogue also keeps,
// per (q1 b1, q2 b2), the sums over b3 of the "+" and of the "-" rates.
//   mode 0 (A_full): they go straight into the stored matrix (ns x ns,
//     column-major; nT = 1), isotope rates after the last chunk, then the
//     un-averaged linewidths with boundary scattering on the diagonal;
//   mode 1 (x_d, y_d): they go into two slabs of the chunk's columns, which
//     are multiplied with x at once (smatrix_dot_kernel) and dropped, so A x
//     costs one builder pass and slab memory only; then the diagonal term.
// ---------------------------------------------------------------------------
template <int NB>
int run_matrix_builder(phx_v3* v, phx_bands* b, const phx_lw_params* p, double* A_full, double* lw_d, int nvec,
                       const double* x_d, double* y_d, phx_lw_stats* stats) {
  phx_ctx* ctx = v->ctx;
  cudaStream_t st = ctx->stream;
  const int nq = b->nq, nT = p->num_temperatures, nr3 = v->nr3, nr2 = v->nr2;
  const int q2b = p->q2_begin, q2e = p->q2_end;
  const int ns = nq * NB;
  const bool full = A_full != nullptr;
  const bool split = v->precision != PHX_PREC_FP64;
  const int fp16 = v->precision == PHX_PREC_SPLIT_FP16 ? 1 : 0;
  // plan: the FP64 kernel's default, or the split kernel's large plan (the
  // matrix-free mode takes its small one: the slabs are zeroed per chunk);
  // slab memory of mode 1: at most 4 GiB for the two slabs of all temperatures
  int chunk = std::min(split ? (full ? 1792 : 448) : 512, q2e - q2b);
  if (!full) {
    const size_t per_q2 = 2 * sizeof(double) * (size_t)nT * ns * NB;
    chunk = (int)std::max<size_t>(1, std::min<size_t>(chunk, (size_t(4) << 30) / per_q2));
  }
  const int slots = std::min(split ? (full ? 28 : 7) : 8, chunk);
  const size_t nb3 = (size_t)NB * NB * NB;
  const size_t sz_dp = align_up(sizeof(double2) * chunk * nr3 * nb3);
  const size_t sz_part = align_up(sizeof(double) * slots * nq * NB * nT);
  const size_t sz_bose = align_up(sizeof(double) * nT * nq * NB);
  const size_t sz_T = align_up(sizeof(double) * 8);
  const size_t sz_iso = p->isotope_coupling ? align_up(sizeof(double) * v->nat) : 0;
  const size_t slab_elems = (size_t)ns * chunk * NB;
  const size_t sz_slab = full ? 0 : align_up(sizeof(double) * 2 * nT * slab_elems);
  const size_t sz_img = split ? align_up(phx_split_bimg_bytes(chunk, nr3)) : 0;
  const size_t sz_rec = split ? align_up(phx_split_rec_bytes(nq)) : 0;
  const size_t sz_max = split ? align_up(sizeof(unsigned) * 4) : 0;
  const size_t sz_edge = split ? align_up(phx_split_edge_bytes()) : 0;
  PHX_TRY(phx_scratch_reserve(v, sz_dp + sz_part + sz_bose + sz_T + sz_iso + sz_slab + sz_img + sz_rec + sz_max +
                                     sz_edge));
  char* base = static_cast<char*>(v->ctx->d_scratch);
  double2* Dp = reinterpret_cast<double2*>(base);
  double* partial = reinterpret_cast<double*>(base + sz_dp);
  double* bose = reinterpret_cast<double*>(base + sz_dp + sz_part);
  double* temps = reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose);
  double* giso =
      p->isotope_coupling ? reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose + sz_T) : nullptr;
  double* slabP = full ? nullptr : reinterpret_cast<double*>(base + sz_dp + sz_part + sz_bose + sz_T + sz_iso);
  double* slabM = full ? nullptr : slabP + nT * slab_elems;
  char* sbase = base + sz_dp + sz_part + sz_bose + sz_T + sz_iso + sz_slab;
  uint8_t* Bimg = reinterpret_cast<uint8_t*>(sbase);
  void* rec = sbase + sz_img;
  unsigned* dmax = reinterpret_cast<unsigned*>(sbase + sz_img + sz_rec);
  unsigned* edge_count = dmax + 1;
  unsigned* edge_peak = dmax + 2;
  unsigned* edge_over = dmax + 3;   // the matrix modes fail on an overflow
  void* edges = sbase + sz_img + sz_rec + sz_max;
  if (split) {
    PHX_ARG(ctx, phx_split_smem_bytes(nr3, nT) <= 227 * 1024, "too many R3 vectors for the split path");
    PHX_TRY(phx_split_prepare_bands(ctx, b));
    if (b->emax < 0.0) {
      std::vector<double> Eh((size_t)nq * NB);
      PHX_CUDA(ctx, cudaMemcpy(Eh.data(), b->d_E, sizeof(double) * Eh.size(), cudaMemcpyDeviceToHost));
      double m = 0.0;
      for (double e : Eh) m = std::max(m, std::fabs(e));
      b->emax = m;
    }
    PHX_TRY(phx_split_set_attributes(ctx, nr3, nT));
  }
  PairArgs P{};
  P.m.nq = nq;
  P.m.nb = NB;
  P.m.nT = nT;
  P.m.n0 = b->mesh[0];
  P.m.n1 = b->mesh[1];
  P.m.n2 = b->mesh[2];
  P.m.E = b->d_E;
  P.m.U = reinterpret_cast<const double2*>(b->d_U);
  P.m.vg = b->d_vg;
  P.m.bose = bose;
  P.m.qcart = b->d_q;
  P.m.smearing = p->smearing;
  P.m.sigma = p->sigma;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P.m.qT[i * 3 + j] = b->recip[i * 3 + j] / b->mesh[i];
  P.m.norm = 1.0 / (double)nq;
  P.nr3 = nr3;
  P.R3 = v->d_R3;
  P.Dp = Dp;
  P.partial = partial;
  P.matP = full ? A_full : slabP;
  P.matM = slabM;
  P.ld = ns;
  P.mat_tstride = slab_elems;
  P.mat_full = full ? 1 : 0;
  const size_t smem_pair = sizeof(double2) * ((size_t)nr3 * kTile + 2 * NB * NB * kTile) +
                           sizeof(double) * ((size_t)NB * NB * NB * kTile + (size_t)kMaxT * NB * kTile);
  PHX_ARG(ctx, smem_pair <= 227 * 1024, "scattering matrix: too many R3 vectors for the FP64 path");
  PHX_CUDA(ctx, cudaFuncSetAttribute(pair_fp64_kernel<NB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_pair));
  const size_t smem_fold = fold_tiled_smem(NB, nr2);
  PHX_ARG(ctx, smem_fold <= 227 * 1024, "scattering matrix: too many R2 vectors");
  if (smem_fold > 48 * 1024)
    PHX_CUDA(ctx, cudaFuncSetAttribute(fold_q2_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_fold));
  const int tiles = (nq + kTile - 1) / kTile;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evv0 = nullptr, evv1 = nullptr;
  PHX_CUDA(ctx, cudaEventCreate(&ev0));
  PHX_CUDA(ctx, cudaEventCreate(&ev1));
  PHX_CUDA(ctx, cudaEventCreate(&evv0));
  PHX_CUDA(ctx, cudaEventCreate(&evv1));
  int launches = 0;
  auto work = [&]() -> int {
    PHX_CUDA(ctx, cudaEventRecord(ev0, st));
    PHX_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
    PHX_CUDA(ctx, cudaMemcpyAsync(temps, p->temperatures, sizeof(double) * nT, cudaMemcpyHostToDevice, st));
    if (giso)
      PHX_CUDA(ctx, cudaMemcpyAsync(giso, p->isotope_coupling, sizeof(double) * v->nat, cudaMemcpyHostToDevice, st));
    PHX_CUDA(ctx, cudaMemsetAsync(partial, 0, sizeof(double) * slots * nq * NB * nT, st));
    if (full) PHX_CUDA(ctx, cudaMemsetAsync(A_full, 0, sizeof(double) * ns * (size_t)ns, st));
    else PHX_CUDA(ctx, cudaMemsetAsync(y_d, 0, sizeof(double) * nvec * nT * 3 * (size_t)ns, st));
    bose_kernel<<<std::min(1024, (nq * NB * nT + 255) / 256), 256, 0, st>>>(nq, NB, nT, b->d_E, temps, bose);
    ++launches;
    if (split) PHX_TRY(phx_split_pack_records(ctx, P.m, rec, &launches));
    if (split) PHX_CUDA(ctx, cudaMemsetAsync(edge_peak, 0, sizeof(unsigned) * 2, st));
    PHX_CUDA(ctx, cudaEventRecord(evv0, st));
    for (int c0 = q2b; c0 < q2e; c0 += chunk) {
      const int cnt = std::min(chunk, q2e - c0);
      if (split) {
        // tensor-core pair kernel: its matrix sums go in by atomics, onto zeroed slabs
        if (!full) PHX_CUDA(ctx, cudaMemsetAsync(slabP, 0, sizeof(double) * 2 * nT * slab_elems, st));
        if (fp16) PHX_CUDA(ctx, cudaMemsetAsync(dmax, 0, sizeof(unsigned), st));
        fold_tiled_launch(NB, nr2, nr3, v, b, c0, cnt, Dp, st, fp16 ? dmax : nullptr);
        ++launches;
        const phx_split_matrix mo{full ? A_full : slabP, slabM, (long long)ns, slab_elems, full ? 1 : 0};
        PHX_TRY(phx_split_pair_chunk(ctx, P.m, v, b, Dp, Bimg, rec, b->emax, c0, cnt, slots, partial, &launches,
                                     nullptr, nullptr, fp16, dmax, edges, edge_count, phx_split_edge_cap(),
                                     edge_peak, edge_over, 0, &mo));
      } else {
        fold_tiled_launch(NB, nr2, nr3, v, b, c0, cnt, Dp, st);
        ++launches;
        PairArgs Q = P;
        Q.q2_first = c0;
        Q.q2_count = cnt;
        Q.q2_per_slot = (cnt + slots - 1) / slots;
        pair_fp64_kernel<NB, true><<<dim3(tiles, slots), kTile * NB, smem_pair, st>>>(Q);
        ++launches;
        PHX_CUDA(ctx, cudaGetLastError());
      }
      if (!full) {
        if (giso) {
          IsoArgs I{P.m, v->nat, giso, c0, cnt, (cnt + slots - 1) / slots, partial, slabP, ns, slab_elems, 0};
          isotope_kernel<<<dim3(tiles, slots), kTile * NB, iso_smem(NB), st>>>(I);
          ++launches;
          PHX_CUDA(ctx, cudaGetLastError());
        }
        phx_dot_args a{};
        a.ns = ns;
        a.ncols = cnt * NB;
        a.ld = ns;
        a.Sp = slabP;
        a.Sm = slabM;
        a.tstride = slab_elems;
        a.slab = 1;
        a.q2_first = c0;
        a.nb = NB;
        a.n0 = b->mesh[0];
        a.n1 = b->mesh[1];
        a.n2 = b->mesh[2];
        a.nT = nT;
        a.nvec = nvec;
        a.x = x_d;
        a.y = y_d;
        a.skip = 0;
        a.E = b->d_E;
        if (phx_smatrix_dot_launch(a, st, &launches) != PHX_OK) {
          phx_set_error(ctx, PHX_ERR_CUDA, "scattering matrix: slab product launch failed");
          return PHX_ERR_CUDA;
        }
      }
    }
    if (full && giso) {
      IsoArgs I{P.m, v->nat, giso, q2b, q2e - q2b, (q2e - q2b + slots - 1) / slots, partial, A_full, ns, 0, 1};
      isotope_kernel<<<dim3(tiles, slots), kTile * NB, iso_smem(NB), st>>>(I);
      ++launches;
      PHX_CUDA(ctx, cudaGetLastError());
    }
    PHX_CUDA(ctx, cudaEventRecord(evv1, st));
    finalize_kernel<<<(nq + 127) / 128, 128, 0, st>>>(nq, NB, nT, slots, partial, b->d_E, p->finalize, b->d_vg, temps,
                                                      p->boundary_length, lw_d, 0);
    ++launches;
    PHX_CUDA(ctx, cudaGetLastError());
    if (full) {
      if (p->finalize) {
        PHX_TRY(phx_smatrix_set_diag_launch(ns, ns, lw_d, A_full, st));
        ++launches;
      }
    } else {
      PHX_TRY(phx_smatrix_diag_term_launch(ns, nT, nvec, lw_d, x_d, y_d, b->d_E, p->finalize, st));
      ++launches;
    }
    PHX_CUDA(ctx, cudaEventRecord(ev1, st));
    return PHX_OK;
  };
  int rc = work();
  if (rc == PHX_OK) {
    cudaError_t ce = cudaEventSynchronize(ev1);
    int kst = 0;
    unsigned over = 0;
    if (ce == cudaSuccess) ce = cudaMemcpy(&kst, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess && split) ce = cudaMemcpy(&over, edge_over, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(ce));
      rc = PHX_ERR_CUDA;
    } else if (kst) {
      cudaMemset(ctx->d_status, 0, sizeof(int));
      phx_set_error(ctx, PHX_ERR_CUDA, "scattering matrix: kernel status " + std::to_string(kst));
      rc = PHX_ERR_CUDA;
    } else if (over) {
      phx_set_error(ctx, PHX_ERR_ARG,
                    "scattering matrix (split path): a pair launch had more near-cut-off events than the event "
                    "list holds; use PHX_PREC_FP64 or a smaller mesh");
      rc = PHX_ERR_ARG;
    }
  }
  if (rc == PHX_OK && stats) {
    float ms = 0.f, msv = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventElapsedTime(&msv, evv0, evv1);
    *stats = phx_lw_stats{};
    stats->ms_total = ms;
    stats->ms_vertex = msv;
    stats->pairs = (long long)nq * (q2e - q2b);
    stats->kernel_launches = launches;
    stats->plan_chunk = chunk;
    stats->plan_slots = slots;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  cudaEventDestroy(evv0);
  cudaEventDestroy(evv1);
  return rc;
}

// argument checks shared by the three builder modes
int check_builder_args(phx_v3* v, phx_bands* b, const phx_lw_params* p) {
  PHX_ARG(nullptr, v && b && p, "builder: bad arguments");
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, b->ctx == ctx, "v3 and bands belong to different contexts");
  PHX_ARG(ctx, b->nb == v->nb, "band count of bands and v3 differ");
  PHX_ARG(ctx, p->num_temperatures >= 1 && p->num_temperatures <= kMaxT && p->temperatures,
          "1..4 temperatures per call");
  PHX_ARG(ctx, p->smearing == PHX_SMEAR_GAUSSIAN || p->smearing == PHX_SMEAR_ADAPTIVE, "bad smearing");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_GAUSSIAN || p->sigma > 0.0, "Gaussian smearing needs sigma > 0");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_ADAPTIVE || b->d_vg, "adaptive smearing needs velocities");
  PHX_ARG(ctx, 0 <= p->q2_begin && p->q2_begin <= p->q2_end && p->q2_end <= b->nq, "bad q2 range");
  PHX_ARG(ctx, !(p->boundary_length > 0.0) || b->d_vg, "boundary scattering needs velocities");
  return PHX_OK;
}

int check_matrix_args(phx_v3* v, phx_bands* b, const phx_lw_params* p) {
  PHX_TRY(check_builder_args(v, b, p));
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, v->nb == 6, "scattering matrix modes: nb = 6 (the fused kernels)");
  PHX_ARG(ctx, !p->window_energy && !p->window_cut, "scattering matrix modes take no q2 window");
  return PHX_OK;
}

}  // namespace

extern "C" int phx_ph_smatrix_create(phx_v3* v, phx_bands* b, const phx_lw_params* p, phx_smatrix** out,
                                     phx_lw_stats* stats) {
  PHX_TRY(check_matrix_args(v, b, p));
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, out, "phx_ph_smatrix_create: null output handle");
  PHX_ARG(ctx, p->num_temperatures == 1,
          "a stored scattering matrix holds one temperature (scatteringMatrixInMemory)");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t ns = (size_t)b->nq * b->nb;
  size_t fr = 0, tot = 0;
  PHX_CUDA(ctx, cudaMemGetInfo(&fr, &tot));
  PHX_ARG(ctx, sizeof(double) * ns * ns < fr,
          "scattering matrix of " + std::to_string(ns) + " states does not fit in free device memory");
  phx_smatrix* m = new phx_smatrix;
  m->ctx = ctx;
  m->nq = b->nq;
  m->nb = b->nb;
  m->ns = (int)ns;
  for (int i = 0; i < 3; ++i) m->mesh[i] = b->mesh[i];
  m->temperature = p->temperatures[0];
  cudaError_t e = cudaMalloc(&m->d_A, sizeof(double) * ns * ns);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_E, sizeof(double) * ns);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_diag, sizeof(double) * ns);
  if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_E, b->d_E, sizeof(double) * ns, cudaMemcpyDeviceToDevice, ctx->stream);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_ph_smatrix_create: ") + cudaGetErrorString(e));
    phx_smatrix_destroy(m);
    return PHX_ERR_CUDA;
  }
  int rc = PHX_OK;
  if (p->q2_begin == p->q2_end) {
    if (cudaMemsetAsync(m->d_A, 0, sizeof(double) * ns * ns, ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_diag, 0, sizeof(double) * ns, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, "phx_ph_smatrix_create: memset failed");
      rc = PHX_ERR_CUDA;
    }
  } else {
    rc = run_matrix_builder<6>(v, b, p, m->d_A, m->d_diag, 0, nullptr, nullptr, stats);
  }
  if (rc != PHX_OK) {
    phx_smatrix_destroy(m);
    return rc;
  }
  *out = m;
  return PHX_OK;
}

namespace {

// switchCase 1 with device vectors; lw_d: (nT, ns) device scratch of the diagonal term
int matrix_dot(phx_v3* v, phx_bands* b, const phx_lw_params* p, int nvec, const double* x_d, double* y_d,
               double* lw_d, phx_lw_stats* stats) {
  phx_ctx* ctx = v->ctx;
  const size_t ns = (size_t)b->nq * b->nb, nT = p->num_temperatures;
  if (p->q2_begin == p->q2_end) {
    PHX_CUDA(ctx, cudaMemsetAsync(y_d, 0, sizeof(double) * nvec * nT * 3 * ns, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PHX_OK;
  }
  return run_matrix_builder<6>(v, b, p, nullptr, lw_d, nvec, x_d, y_d, stats);
}

}  // namespace

extern "C" int phx_ph_smatrix_dot_d(phx_v3* v, phx_bands* b, const phx_lw_params* p, int nvec, const double* x_d,
                                    double* y_d, phx_lw_stats* stats) {
  PHX_TRY(check_matrix_args(v, b, p));
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, nvec >= 1 && x_d && y_d, "phx_ph_smatrix_dot: bad vectors");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t ns = (size_t)b->nq * b->nb;
  PHX_TRY(phx_ctx_reserve(ctx, &ctx->d_out, &ctx->out_bytes, sizeof(double) * p->num_temperatures * ns));
  return matrix_dot(v, b, p, nvec, x_d, y_d, static_cast<double*>(ctx->d_out), stats);
}

extern "C" int phx_ph_smatrix_dot(phx_v3* v, phx_bands* b, const phx_lw_params* p, int nvec, const double* x,
                                  double* y, phx_lw_stats* stats) {
  PHX_TRY(check_matrix_args(v, b, p));
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, nvec >= 1 && x && y, "phx_ph_smatrix_dot: bad vectors");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t ns = (size_t)b->nq * b->nb, nT = p->num_temperatures;
  const size_t n = (size_t)nvec * nT * 3 * ns;
  // output staging: the diagonal term's linewidths, x, y
  PHX_TRY(phx_ctx_reserve(ctx, &ctx->d_out, &ctx->out_bytes, sizeof(double) * (nT * ns + 2 * n)));
  double* lw = static_cast<double*>(ctx->d_out);
  double* xd = lw + nT * ns;
  double* yd = xd + n;
  PHX_CUDA(ctx, cudaMemcpyAsync(xd, x, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  PHX_TRY(matrix_dot(v, b, p, nvec, xd, yd, lw, stats));
  PHX_CUDA(ctx, cudaMemcpyAsync(y, yd, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

namespace {

}  // namespace

namespace {

// Non-zero (r3, r2) blocks of the folded vertex, once per coupling object:
// the many-branch fold sums over them only.
int wide_prepare_blocks(phx_v3* v) {
  if (v->d_r2_ofs) return PHX_OK;
  phx_ctx* ctx = v->ctx;
  cudaStream_t st = ctx->stream;
  const int nr3 = v->nr3, nr2 = v->nr2;
  int* d_flags = nullptr;
  PHX_CUDA(ctx, phx_dev_alloc(ctx, (void**)&d_flags, sizeof(int) * (size_t)nr3 * nr2));
  std::vector<int> flags((size_t)nr3 * nr2);
  cudaError_t e = wide::launch_nonzero_blocks(v->nb, nr3, nr2, v->d_D3w, d_flags, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(flags.data(), d_flags, sizeof(int) * flags.size(), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  phx_dev_free(ctx, d_flags);
  PHX_CUDA(ctx, e);
  std::vector<int> ofs(nr3 + 1, 0), list;
  int maxl = 1;
  for (int r3 = 0; r3 < nr3; ++r3) {
    for (int r2 = 0; r2 < nr2; ++r2)
      if (flags[(size_t)r3 * nr2 + r2]) list.push_back(r2);
    ofs[r3 + 1] = (int)list.size();
    maxl = std::max(maxl, ofs[r3 + 1] - ofs[r3]);
  }
  if (list.empty()) list.push_back(0);
  PHX_CUDA(ctx, phx_dev_alloc(ctx, (void**)&v->d_r2_ofs, sizeof(int) * ofs.size()));
  PHX_CUDA(ctx, phx_dev_alloc(ctx, (void**)&v->d_r2_list, sizeof(int) * list.size()));
  PHX_CUDA(ctx, cudaMemcpyAsync(v->d_r2_ofs, ofs.data(), sizeof(int) * ofs.size(), cudaMemcpyHostToDevice, st));
  PHX_CUDA(ctx, cudaMemcpyAsync(v->d_r2_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, st));
  PHX_CUDA(ctx, cudaStreamSynchronize(st));
  v->r2_max_list = maxl;
  return PHX_OK;
}

// Builder for cells with many branches (wide.cu), both precisions, with an
// optional per-q1 q2 window: per chunk of q2 the sparse R2 fold, for the
// split path the FP16/BF16 hi/lo image of the folded vertex, then one
// persistent pair kernel over (q2, q1 tile) items from a work queue.
int run_builder_wide(phx_v3* v, phx_bands* b, const phx_lw_params* p, double* Aout_d, phx_lw_stats* stats,
                     const uint8_t* skip = nullptr) {
  phx_ctx* ctx = v->ctx;
  cudaStream_t st = ctx->stream;
  const int nq = b->nq, nT = p->num_temperatures, nr3 = v->nr3, nr2 = v->nr2, nb = v->nb;
  const int q2b = p->q2_begin, q2e = p->q2_end;
  const bool split = v->precision != PHX_PREC_FP64;
  const int fp16 = v->precision == PHX_PREC_SPLIT_FP16 ? 1 : 0;
  const bool windowed = p->window_energy != nullptr;
  PHX_ARG(ctx, nb <= wide::kMaxNb, "phx_ph_linewidths: at most 48 branches (16 atoms)");
  PHX_ARG(ctx, !p->isotope_coupling || nb <= 32, "phx_ph_linewidths: isotope scattering supports nb <= 32");
  const int Kp = wide::split_kp(nr3);
  int nq1 = wide::kQ1;
  if (split) {
    PHX_ARG(ctx, wide::split_smem(nb, Kp, 2) > 0,
            "phx_ph_linewidths: too many branches or R3 vectors for the split path");
  } else {
    nq1 = wide::fp64_q1(nb, nr3);
    PHX_ARG(ctx, nq1 > 0, "phx_ph_linewidths: too many branches or R3 vectors for the FP64 path");
  }
  PHX_TRY(wide_prepare_blocks(v));
  PHX_ARG(ctx, wide::fold_smem(nb, v->r2_max_list) <= 227 * 1024, "phx_ph_linewidths: too many R2 vectors");
  const size_t nb3 = (size_t)nb * nb * nb;
  const size_t per_q2 = sizeof(double2) * nr3 * nb3 + (split ? wide::split_img_bytes(nb, Kp) : 0);
  // q2 per chunk: at most 2 GiB of folded vertex (and its image), at most 512 q2
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>({(size_t)512, (size_t)(q2e - q2b),
                                                                (size_t(2) << 30) / per_q2}));
  const int nchunks = (q2e - q2b + chunk - 1) / chunk;
  const size_t sz_dp = align_up(sizeof(double2) * nr3 * nb3 * chunk);
  const size_t sz_img = split ? align_up(wide::split_img_bytes(nb, Kp) * chunk) : 0;
  const size_t sz_lw = align_up(sizeof(double) * (size_t)nq * nb * nT);
  const size_t sz_bose = align_up(sizeof(double) * (size_t)nT * nq * nb);
  const size_t sz_T = align_up(sizeof(double) * 8);
  const size_t sz_win = align_up(sizeof(double) * 2 * nq);
  const size_t sz_ord = align_up(sizeof(int) * nq);
  const size_t sz_iso = p->isotope_coupling ? align_up(sizeof(double) * v->nat) : 0;
  const size_t sz_cnt = align_up(sizeof(unsigned) * (nchunks + 1));
  const size_t sz_u32 = split && !b->d_U32 ? 0 : 0;
  (void)sz_u32;
  PHX_TRY(phx_scratch_reserve(v, sz_dp + sz_img + sz_lw + sz_bose + sz_T + sz_win + sz_ord + sz_iso + sz_cnt));
  char* base = static_cast<char*>(v->ctx->d_scratch);
  size_t o = 0;
  double2* Dp = reinterpret_cast<double2*>(base + o); o += sz_dp;
  uint8_t* img = reinterpret_cast<uint8_t*>(base + o); o += sz_img;
  double* lw = reinterpret_cast<double*>(base + o); o += sz_lw;
  double* bose = reinterpret_cast<double*>(base + o); o += sz_bose;
  double* temps = reinterpret_cast<double*>(base + o); o += sz_T;
  double* wdev = reinterpret_cast<double*>(base + o); o += sz_win;
  int* order = reinterpret_cast<int*>(base + o); o += sz_ord;
  double* giso = p->isotope_coupling ? reinterpret_cast<double*>(base + o) : nullptr; o += sz_iso;
  unsigned* counters = reinterpret_cast<unsigned*>(base + o);   // [nchunks] work queues, then dmax
  unsigned* dmax = counters + nchunks;
  if (split && !b->d_U32) {
    const size_t n = (size_t)nq * nb * nb;
    PHX_CUDA(ctx, phx_dev_alloc(ctx, (void**)&b->d_U32, sizeof(float2) * n));
    PHX_CUDA(ctx, wide::launch_u32(reinterpret_cast<const double2*>(b->d_U), reinterpret_cast<float2*>(b->d_U32), n,
                                   st));
  }
  PHX_CUDA(ctx, wide::set_attributes(nb, nr3, split));
  // q1 order: by window cut with a window (tiles of similar q2 sets), else the mesh order
  std::vector<int> order_h(nq);
  for (int i = 0; i < nq; ++i) order_h[i] = i;
  if (windowed)
    std::stable_sort(order_h.begin(), order_h.end(), [&](int a, int c) { return p->window_cut[a] < p->window_cut[c]; });
  PHX_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
  PHX_CUDA(ctx, cudaMemcpyAsync(temps, p->temperatures, sizeof(double) * nT, cudaMemcpyHostToDevice, st));
  PHX_CUDA(ctx, cudaMemcpyAsync(order, order_h.data(), sizeof(int) * nq, cudaMemcpyHostToDevice, st));
  if (windowed) {
    PHX_CUDA(ctx, cudaMemcpyAsync(wdev, p->window_energy, sizeof(double) * nq, cudaMemcpyHostToDevice, st));
    PHX_CUDA(ctx, cudaMemcpyAsync(wdev + nq, p->window_cut, sizeof(double) * nq, cudaMemcpyHostToDevice, st));
  }
  if (giso)
    PHX_CUDA(ctx, cudaMemcpyAsync(giso, p->isotope_coupling, sizeof(double) * v->nat, cudaMemcpyHostToDevice, st));
  wide::Args A{};
  A.m.nq = nq;
  A.m.nb = nb;
  A.m.nT = nT;
  A.m.n0 = b->mesh[0];
  A.m.n1 = b->mesh[1];
  A.m.n2 = b->mesh[2];
  A.m.E = b->d_E;
  A.m.U = reinterpret_cast<const double2*>(b->d_U);
  A.m.vg = b->d_vg;
  A.m.bose = bose;
  A.m.qcart = b->d_q;
  A.m.smearing = p->smearing;
  A.m.sigma = p->sigma;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A.m.qT[i * 3 + j] = b->recip[i * 3 + j] / b->mesh[i];
  A.m.norm = 1.0 / (double)nq;
  A.nr3 = nr3;
  A.R3 = v->d_R3;
  A.Dp = Dp;
  A.q1_order = order;
  A.nq1 = nq1;
  A.ntiles = (nq + nq1 - 1) / nq1;
  A.win_energy = windowed ? wdev : nullptr;
  A.win_cut = windowed ? wdev + nq : nullptr;
  A.lw = lw;
  A.status = ctx->d_status;
  A.img = img;
  A.U32 = reinterpret_cast<const float2*>(b->d_U32);
  A.Kp = Kp;
  A.mtiles = wide::split_mtiles(nb);
  A.fp16 = fp16;
  A.dmax = dmax;
  A.skip = skip;
  A.skip_base = q2b;
  A.rt = nb > 24 ? 4 : 2;
  A.qp = wide::split_default_qp(nb, Kp);
  const int grid = ctx->num_sms * wide::blocks_per_sm(nb, nr3, split);
  // split path: the tile shape (register tile, q1 planes per contraction pass)
  // tuned once per problem shape on one chunk (PHX_TUNE=0: the defaults)
  int dev = 0;
  cudaGetDevice(&dev);
  const PlanKey pk{20 + fp16, nb, nq, nr3, nr2, nT, dev};
  BuilderPlan shape{A.rt, A.qp};   // (chunk, slots) fields hold (rt, qp) here
  const int tune_q2 = std::min(chunk, 64);   // q2 of the timed chunk (every q1)
  if (split && !skip && !env_off("PHX_TUNE") && q2e - q2b >= 2 * tune_q2 && !find_plan(pk, &shape)) {
    bose_kernel<<<std::min(1024, (nq * nb * nT + 255) / 256), 256, 0, st>>>(nq, nb, nT, b->d_E, temps, bose);
    if (fp16) PHX_CUDA(ctx, cudaMemsetAsync(dmax, 0, sizeof(unsigned), st));
    PHX_CUDA(ctx, wide::launch_fold(nb, nr2, nr3, v->d_D3w, v->d_r2_ofs, v->d_r2_list, v->r2_max_list, v->d_R2,
                                    v->d_R3, b->d_q, reinterpret_cast<const double2*>(b->d_U), q2b, tune_q2, Dp,
                                    fp16 ? dmax : nullptr, st));
    PHX_CUDA(ctx, wide::launch_convert(nb, nr3, Kp, tune_q2, Dp, img, fp16, dmax, st));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    PHX_CUDA(ctx, cudaEventCreate(&t0));
    PHX_CUDA(ctx, cudaEventCreate(&t1));
    double best = 1e300;
    int rc = PHX_OK;
    for (int rt : {2, 4})
      for (int qp : {8, 4, 2}) {
        if (!wide::split_smem(nb, Kp, qp)) continue;
        wide::Args Ac = A;
        Ac.rt = rt;
        Ac.qp = qp;
        Ac.q2_first = q2b;
        Ac.q2_count = tune_q2;
        Ac.counter = counters;
        cudaMemsetAsync(counters, 0, sizeof(unsigned), st);
        cudaEventRecord(t0, st);
        cudaError_t e = wide::launch_split(Ac, grid, st);
        cudaEventRecord(t1, st);
        if (e == cudaSuccess) e = cudaEventSynchronize(t1);
        if (e != cudaSuccess) {
          phx_set_error(ctx, PHX_ERR_CUDA, std::string("builder autotuner: ") + cudaGetErrorString(e));
          rc = PHX_ERR_CUDA;
          break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        if (ms < best) {
          best = ms;
          shape = BuilderPlan{rt, qp};
        }
      }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != PHX_OK) return rc;
    store_plan(pk, shape);
  }
  if (split) {
    A.rt = shape.chunk;
    A.qp = shape.slots;
  }
  long long pairs = 0;
  for (int c0 = q2b; c0 < q2e; c0 += chunk) pairs += (long long)nq * std::min(chunk, q2e - c0);
  auto work = [&](phx_builder_graph& g) -> int {
    int launches = 0;
    PHX_CUDA(ctx, cudaMemsetAsync(lw, 0, sizeof(double) * (size_t)nq * nb * nT, st));
    PHX_CUDA(ctx, cudaMemsetAsync(counters, 0, sizeof(unsigned) * (nchunks + 1), st));
    bose_kernel<<<std::min(1024, (nq * nb * nT + 255) / 256), 256, 0, st>>>(nq, nb, nT, b->d_E, temps, bose);
    ++launches;
    PHX_CUDA(ctx, phx_record_event(g.vertex_begin, st));
    for (int ci = 0; ci < nchunks; ++ci) {
      const int c0 = q2b + ci * chunk, cnt = std::min(chunk, q2e - c0);
      if (fp16) PHX_CUDA(ctx, cudaMemsetAsync(dmax, 0, sizeof(unsigned), st));
      PHX_CUDA(ctx, wide::launch_fold(nb, nr2, nr3, v->d_D3w, v->d_r2_ofs, v->d_r2_list, v->r2_max_list, v->d_R2,
                                      v->d_R3, b->d_q, reinterpret_cast<const double2*>(b->d_U), c0, cnt, Dp,
                                      fp16 ? dmax : nullptr, st));
      ++launches;
      if (split) {
        PHX_CUDA(ctx, wide::launch_convert(nb, nr3, Kp, cnt, Dp, img, fp16, dmax, st));
        ++launches;
      }
      wide::Args Ac = A;
      Ac.q2_first = c0;
      Ac.q2_count = cnt;
      Ac.counter = counters + ci;
      cudaEvent_t pe0 = nullptr, pe1 = nullptr;
      PHX_CUDA(ctx, cudaEventCreate(&pe0));
      g.pair_events.push_back(pe0);
      PHX_CUDA(ctx, cudaEventCreate(&pe1));
      g.pair_events.push_back(pe1);
      PHX_CUDA(ctx, phx_record_event(pe0, st));
      PHX_CUDA(ctx, split ? wide::launch_split(Ac, grid, st) : wide::launch_fp64(Ac, grid, st));
      PHX_CUDA(ctx, phx_record_event(pe1, st));
      ++launches;
    }
    PHX_CUDA(ctx, phx_record_event(g.vertex_end, st));
    if (giso) {
      IsoArgs I{A.m, v->nat, giso, q2b, q2e - q2b, q2e - q2b, lw};
      isotope_kernel<<<dim3((nq + kTile - 1) / kTile, 1), kTile * nb, iso_smem(nb), st>>>(I);
      ++launches;
      PHX_CUDA(ctx, cudaGetLastError());
    }
    finalize_kernel<<<(nq + 127) / 128, 128, 0, st>>>(nq, nb, nT, 1, lw, b->d_E, p->finalize, b->d_vg, temps,
                                                      p->boundary_length, Aout_d);
    ++launches;
    PHX_CUDA(ctx, cudaGetLastError());
    g.launches = launches;
    return PHX_OK;
  };
  const std::vector<uint64_t> key = {
      (uint64_t)(split ? 10 + fp16 : 9), (uint64_t)nb, (uint64_t)nq, (uint64_t)nT, (uint64_t)q2b, (uint64_t)q2e,
      (uint64_t)p->smearing, bits(p->sigma), (uint64_t)p->finalize, (uint64_t)chunk, (uint64_t)windowed, bits(base),
      bits(Aout_d), bits(b->d_E), bits(b->d_U), bits(b->d_vg), bits(b->d_q), bits(b->d_U32), bits(v->d_D3w),
      bits(v->d_R2), bits(v->d_R3), bits(ctx->d_status), bits(giso), bits(p->boundary_length), (uint64_t)grid,
      bits(skip), (uint64_t)A.rt, (uint64_t)A.qp};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  PHX_CUDA(ctx, cudaEventCreate(&ev0));
  PHX_CUDA(ctx, cudaEventCreate(&ev1));
  PHX_CUDA(ctx, cudaEventRecord(ev0, st));
  phx_builder_graph eager;
  phx_builder_graph* g = nullptr;
  int graph_state = 0;
  int rc = run_device_work(v, key, work, &eager, &g, &graph_state);
  int kst = 0;
  if (rc == PHX_OK) {
    cudaError_t ce = cudaEventRecord(ev1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev1);
    if (ce == cudaSuccess) ce = cudaMemcpy(&kst, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(ce));
      rc = PHX_ERR_CUDA;
    }
  }
  if (rc == PHX_OK && kst) {
    cudaMemset(ctx->d_status, 0, sizeof(int));
    phx_set_error(ctx, PHX_ERR_CUDA,
                  "many-branch pair kernel gave up waiting on a pipeline barrier (status " + std::to_string(kst) + ")");
    rc = PHX_ERR_CUDA;
  }
  if (rc == PHX_OK && stats) {
    float ms = 0, msv = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventElapsedTime(&msv, g->vertex_begin, g->vertex_end);
    *stats = phx_lw_stats{};
    stats->ms_total = ms;
    stats->ms_vertex = msv;
    stats->pairs = pairs;
    stats->kernel_launches = g->launches;
    stats->pair_launches = (int)(g->pair_events.size() / 2);
    double msp = 0.0;
    for (size_t i = 0; i + 1 < g->pair_events.size(); i += 2) {
      float x = 0.f;
      cudaEventElapsedTime(&x, g->pair_events[i], g->pair_events[i + 1]);
      msp += x;
    }
    stats->ms_pair = msp;
    stats->plan_chunk = chunk;
    stats->plan_slots = grid;
    stats->graph = graph_state;
    stats->tile_rt = split ? A.rt : 0;
    stats->tile_qp = split ? A.qp : 0;
    cudaGetLastError();
  }
  phx_builder_graph_free(eager);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  return rc;
}

}  // namespace

extern "C" int phx_ph_linewidths_d(phx_v3* v, phx_bands* b, const phx_lw_params* p,
                                   double* Aout_d, phx_lw_stats* stats) {
  PHX_ARG(nullptr, v && b && p && Aout_d, "phx_ph_linewidths: bad arguments");
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, b->ctx == ctx, "v3 and bands belong to different contexts");
  PHX_ARG(ctx, b->nb == v->nb, "band count of bands and v3 differ");
  PHX_ARG(ctx, p->num_temperatures >= 1 && p->num_temperatures <= kMaxT && p->temperatures,
          "1..4 temperatures per call");
  PHX_ARG(ctx, p->smearing == PHX_SMEAR_GAUSSIAN || p->smearing == PHX_SMEAR_ADAPTIVE, "bad smearing");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_GAUSSIAN || p->sigma > 0.0, "Gaussian smearing needs sigma > 0");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_ADAPTIVE || b->d_vg, "adaptive smearing needs velocities");
  PHX_ARG(ctx, 0 <= p->q2_begin && p->q2_begin <= p->q2_end && p->q2_end <= b->nq, "bad q2 range");
  PHX_ARG(ctx, !(p->boundary_length > 0.0) || b->d_vg, "boundary scattering needs velocities");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  if (p->q2_begin == p->q2_end) {
    PHX_CUDA(ctx, cudaMemsetAsync(Aout_d, 0, sizeof(double) * p->num_temperatures * b->nq * b->nb, ctx->stream));
    return PHX_OK;
  }
  // PHX_WIDE=1: every problem on the many-branch builder (its cross-check
  // against the nb = 6 kernels)
  if (env_on("PHX_WIDE")) return run_builder_wide(v, b, p, Aout_d, stats);
  if (v->nb == 6 && !p->window_energy) return run_builder<6>(v, b, p, Aout_d, stats);
  // the split precisions and cells beyond 16 branches run on the many-branch
  // builder; FP64 up to 16 branches (or with a window) on the shared-memory one
  if (v->precision != PHX_PREC_FP64 || v->nb > kMaxNbGeneric) return run_builder_wide(v, b, p, Aout_d, stats);
  return run_builder_generic(v, b, p, Aout_d, stats);
}

// Shared argument checks of the linewidth entry points.
int check_lw_args(phx_v3* v, phx_bands* b, const phx_lw_params* p) {
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, b->ctx == ctx, "v3 and bands belong to different contexts");
  PHX_ARG(ctx, b->nb == v->nb, "band count of bands and v3 differ");
  PHX_ARG(ctx, p->num_temperatures >= 1 && p->num_temperatures <= kMaxT && p->temperatures,
          "1..4 temperatures per call");
  PHX_ARG(ctx, p->smearing == PHX_SMEAR_GAUSSIAN || p->smearing == PHX_SMEAR_ADAPTIVE, "bad smearing");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_GAUSSIAN || p->sigma > 0.0, "Gaussian smearing needs sigma > 0");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_ADAPTIVE || b->d_vg, "adaptive smearing needs velocities");
  PHX_ARG(ctx, 0 <= p->q2_begin && p->q2_begin <= p->q2_end && p->q2_end <= b->nq, "bad q2 range");
  PHX_ARG(ctx, !(p->boundary_length > 0.0) || b->d_vg, "boundary scattering needs velocities");
  return PHX_OK;
}

extern "C" int phx_ph_linewidths_screened(phx_v3* v, phx_bands* b, const phx_lw_params* p, phx_mlp* net,
                                          double log10_threshold, double* Aout, phx_lw_stats* stats) {
  PHX_ARG(nullptr, v && b && p && Aout && net, "phx_ph_linewidths_screened: bad arguments");
  phx_ctx* ctx = v->ctx;
  PHX_TRY(check_lw_args(v, b, p));
  PHX_ARG(ctx, phx_mlp_context(net) == ctx, "screening network and v3 belong to different contexts");
  PHX_ARG(ctx, phx_mlp_num_inputs(net) == wide::kPairFeatures, "screening network: 12 inputs expected");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int nq = b->nq, nb = b->nb, q2b = p->q2_begin, q2e = p->q2_end;
  const size_t n_out = (size_t)p->num_temperatures * nq * nb;
  PHX_TRY(phx_ctx_reserve(ctx, &ctx->d_out, &ctx->out_bytes, sizeof(double) * std::max<size_t>(n_out, 1)));
  double* Aout_d = static_cast<double*>(ctx->d_out);
  if (q2b == q2e) {
    std::fill(Aout, Aout + n_out, 0.0);
    if (stats) *stats = phx_lw_stats{};
    return PHX_OK;
  }
  if (b->emax < 0.0) {
    std::vector<double> Eh((size_t)nq * nb);
    PHX_CUDA(ctx, cudaMemcpy(Eh.data(), b->d_E, sizeof(double) * Eh.size(), cudaMemcpyDeviceToHost));
    double m = 0.0;
    for (double e : Eh) m = std::max(m, std::fabs(e));
    b->emax = m;
  }
  // the network's verdict on every vertex (q1, q2) of the range, in chunks of q2
  const size_t npairs = (size_t)(q2e - q2b) * nq;
  const int qc = std::max(1, std::min(q2e - q2b, (int)(((size_t)1 << 20) / std::max(nq, 1)) + 1));
  uint8_t* skip = nullptr;
  float *X = nullptr, *y = nullptr;
  unsigned long long* nskip = nullptr;
  int rc = PHX_OK;
  auto dev = [&](void** ptr, size_t bytes) {
    if (rc == PHX_OK && phx_dev_alloc(ctx, ptr, bytes) != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, "phx_ph_linewidths_screened: device allocation failed");
      rc = PHX_ERR_CUDA;
    }
  };
  dev((void**)&skip, npairs);
  dev((void**)&X, sizeof(float) * wide::kPairFeatures * (size_t)qc * nq);
  dev((void**)&y, sizeof(float) * (size_t)qc * nq);
  dev((void**)&nskip, sizeof(unsigned long long));
  if (rc == PHX_OK && cudaMemsetAsync(nskip, 0, sizeof(unsigned long long), st) != cudaSuccess) rc = PHX_ERR_CUDA;
  for (int c0 = q2b; c0 < q2e && rc == PHX_OK; c0 += qc) {
    const int cnt = std::min(qc, q2e - c0);
    const size_t n = (size_t)cnt * nq;
    cudaError_t e = wide::launch_pair_features(nq, nb, b->mesh[0], b->mesh[1], b->mesh[2], b->d_E, b->emax, c0, cnt,
                                               X, st);
    if (e != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
      rc = PHX_ERR_CUDA;
      break;
    }
    rc = phx_mlp_forward_device(net, (long long)n, X, y);
    if (rc != PHX_OK) break;
    e = wide::launch_screen_mask(n, y, (float)log10_threshold, skip + (size_t)(c0 - q2b) * nq, nskip, st);
    if (e != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
      rc = PHX_ERR_CUDA;
    }
  }
  unsigned long long skipped = 0;
  if (rc == PHX_OK && (cudaMemcpyAsync(&skipped, nskip, sizeof(skipped), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                       cudaStreamSynchronize(st) != cudaSuccess)) {
    phx_set_error(ctx, PHX_ERR_CUDA, "phx_ph_linewidths_screened: screening pass failed");
    rc = PHX_ERR_CUDA;
  }
  phx_lw_stats st_local{};
  if (rc == PHX_OK) rc = run_builder_wide(v, b, p, Aout_d, &st_local, skip);
  if (rc == PHX_OK) {
    cudaError_t e = cudaMemcpyAsync(Aout, Aout_d, sizeof(double) * n_out, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
      rc = PHX_ERR_CUDA;
    }
  }
  phx_dev_free(ctx, skip);
  phx_dev_free(ctx, X);
  phx_dev_free(ctx, y);
  phx_dev_free(ctx, nskip);
  if (rc == PHX_OK && stats) {
    *stats = st_local;
    stats->pairs_screened_out = (long long)skipped;
  }
  return rc;
}

extern "C" int phx_ph_linewidths(phx_v3* v, phx_bands* b, const phx_lw_params* p, double* Aout,
                                 phx_lw_stats* stats) {
  PHX_ARG(nullptr, v && b && p && Aout, "phx_ph_linewidths: bad arguments");
  phx_ctx* ctx = v->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t n = (size_t)p->num_temperatures * b->nq * b->nb;
  PHX_TRY(phx_ctx_reserve(ctx, &ctx->d_out, &ctx->out_bytes, sizeof(double) * std::max<size_t>(n, 1)));
  double* d = static_cast<double*>(ctx->d_out);
  int rc = phx_ph_linewidths_d(v, b, p, d, stats);
  if (rc == PHX_OK) {
    cudaError_t e = cudaMemcpyAsync(Aout, d, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
      rc = PHX_ERR_CUDA;
    }
  }
  return rc;
}

extern "C" int phx_ph_rta_kappa(phx_bands* b, int nT, const double* temps, const double* Aout,
                                double volume, double* kappa) {
  PHX_ARG(nullptr, b && temps && Aout && kappa && nT > 0 && volume > 0, "phx_ph_rta_kappa: bad arguments");
  PHX_ARG(b->ctx, b->d_vg, "phx_ph_rta_kappa needs velocities");
  const size_t ns = (size_t)b->nq * b->nb;
  std::vector<double> E(ns), vg(3 * ns);
  PHX_TRY(phx_bands_get(b, E.data(), nullptr, vg.data()));
  for (int c = 0; c < nT; ++c) {
    double k[9] = {0};
    const double T = temps[c];
    for (size_t s = 0; s < ns; ++s) {
      const double en = E[s];
      if (en < phxc::phExcludeCutoff) continue;
      const double x = std::sinh(en / 2.0 / T);
      const double pp = 0.25 / x / x;
      const double tau = pp / Aout[c * ns + s];
      const double dndt = pp * en / T / T;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          k[i * 3 + j] += dndt * vg[3 * s + i] * tau * vg[3 * s + j] * en / (double)b->nq / volume;
    }
    for (int i = 0; i < 9; ++i) kappa[c * 9 + i] = k[i];
  }
  return PHX_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the fused builder (plain FP64 path).
//
// For callers that cannot allocate device memory when they call the builder:
// for example a host application that has handed all free device memory to
// its own pool allocator before calling into this library, or one that must
// not pay the implicit device-wide synchronisation of cudaMalloc/cudaFree
// inside a latency-critical loop.  All intermediate buffers of this variant
// live in one array of fixed size that the library reserves statically on
// every GPU where it is loaded; it is held until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB per GPU

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mutex;
// device address of g_static_scratch, per device, with the CUDA context it was
// looked up in: a new context on the device (after cudaDeviceReset, say) is
// looked up again
struct StaticAddr {
  CUcontext cu = nullptr;
  void* addr = nullptr;
};
StaticAddr g_static_addr[64];

// The current CUDA context, through the driver entry point the runtime hands
// out (no link-time dependency on the driver library); null if unavailable.
CUcontext current_cu_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<Fn>(p);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) c = nullptr;
  return c;
}

// Looks the array up once per device and context (the device must be current).
// This lookup is one reason the entry point is never called inside a stream
// capture.
int static_scratch_address(phx_ctx* ctx, void** out) {
  std::lock_guard<std::mutex> lk(g_static_mutex);
  PHX_ARG(ctx, ctx->device >= 0 && ctx->device < 64, "device index out of range");
  CUcontext cur = current_cu_context();
  StaticAddr& s = g_static_addr[ctx->device];
  if (!s.addr || s.cu != cur) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_static_scratch);
    if (e != cudaSuccess || !addr) {
      phx_set_error(ctx, PHX_ERR_CUDA,
                    std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
      return PHX_ERR_CUDA;
    }
    // the runtime call makes the primary context current when none was
    cur = current_cu_context();
    s.cu = cur;
    s.addr = addr;
  }
  *out = s.addr;
  return PHX_OK;
}

template <int NB>
int run_builder_static(phx_v3* v, phx_bands* b, const phx_lw_params* p, double* Aout_d) {
  phx_ctx* ctx = v->ctx;
  cudaStream_t st = ctx->stream;
  const int nq = b->nq, nT = p->num_temperatures, nr3 = v->nr3, nr2 = v->nr2;
  const int q2b = p->q2_begin, q2e = p->q2_end;
  const size_t nb3 = (size_t)NB * NB * NB;
  const size_t sz_part = align_up(sizeof(double) * (size_t)nq * NB * nT);  // one slot
  const size_t sz_bose = align_up(sizeof(double) * (size_t)nT * nq * NB);
  const size_t sz_T = align_up(sizeof(double) * 8);
  const size_t per_q2 = sizeof(double2) * (size_t)nr3 * nb3;
  const size_t fixed = sz_part + sz_bose + sz_T;
  // every argument-only check comes before the first call that touches the device
  if (fixed + align_up(per_q2) > kStaticScratchBytes) {
    phx_set_error(ctx, PHX_ERR_ARG,
                  "phx_ph_linewidths_static: this problem needs " + std::to_string(fixed + align_up(per_q2)) +
                      " bytes of scratch at least; the static scratch holds " +
                      std::to_string(kStaticScratchBytes) + " bytes (reduce mesh points or temperatures)");
    return PHX_ERR_ARG;
  }
  const size_t smem_pair = sizeof(double2) * ((size_t)nr3 * kTile + 2 * NB * NB * kTile) +
                           sizeof(double) * ((size_t)NB * NB * NB * kTile + (size_t)kMaxT * NB * kTile);
  PHX_ARG(ctx, smem_pair <= 227 * 1024, "phx_ph_linewidths_static: too many R3 vectors");
  const size_t smem_fold = sizeof(double2) * ((size_t)nr2 + 2 * NB * NB);
  PHX_ARG(ctx, smem_fold <= 227 * 1024, "phx_ph_linewidths_static: too many R2 vectors");
  const int chunk = (int)std::min<size_t>({(kStaticScratchBytes - fixed) / per_q2, (size_t)512,
                                           (size_t)(q2e - q2b)});
  PHX_CUDA(ctx, cudaFuncSetAttribute(pair_fp64_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_pair));
  if (smem_fold > 48 * 1024)
    PHX_CUDA(ctx, cudaFuncSetAttribute(fold_q2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_fold));
  void* base_v = nullptr;
  PHX_TRY(static_scratch_address(ctx, &base_v));
  char* base = static_cast<char*>(base_v);
  double* partial = reinterpret_cast<double*>(base);
  double* bose = reinterpret_cast<double*>(base + sz_part);
  double* temps = reinterpret_cast<double*>(base + sz_part + sz_bose);
  double2* Dp = reinterpret_cast<double2*>(base + fixed);
  // the array keeps the previous call's contents: clear what accumulates
  PHX_CUDA(ctx, cudaMemcpyAsync(temps, p->temperatures, sizeof(double) * nT, cudaMemcpyHostToDevice, st));
  PHX_CUDA(ctx, cudaMemsetAsync(partial, 0, sizeof(double) * (size_t)nq * NB * nT, st));
  bose_kernel<<<std::min(1024, (nq * NB * nT + 255) / 256), 256, 0, st>>>(nq, NB, nT, b->d_E, temps, bose);
  PairArgs P{};
  P.m.nq = nq;
  P.m.nb = NB;
  P.m.nT = nT;
  P.m.n0 = b->mesh[0];
  P.m.n1 = b->mesh[1];
  P.m.n2 = b->mesh[2];
  P.m.E = b->d_E;
  P.m.U = reinterpret_cast<const double2*>(b->d_U);
  P.m.vg = b->d_vg;
  P.m.bose = bose;
  P.m.qcart = b->d_q;
  P.m.smearing = p->smearing;
  P.m.sigma = p->sigma;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P.m.qT[i * 3 + j] = b->recip[i * 3 + j] / b->mesh[i];
  P.m.norm = 1.0 / (double)nq;
  P.nr3 = nr3;
  P.R3 = v->d_R3;
  P.Dp = Dp;
  P.partial = partial;
  const int tiles = (nq + kTile - 1) / kTile;
  for (int c0 = q2b; c0 < q2e; c0 += chunk) {
    const int cnt = std::min(chunk, q2e - c0);
    const int per_block = 8;
    fold_q2_kernel<<<dim3(nr3, (cnt + per_block - 1) / per_block), 128, smem_fold, st>>>(
        NB, nr2, nr3, v->d_D3w, v->d_R2, v->d_R3, b->d_q, reinterpret_cast<const double2*>(b->d_U), c0,
        cnt, per_block, Dp);
    P.q2_first = c0;
    P.q2_count = cnt;
    P.q2_per_slot = cnt;
    pair_fp64_kernel<NB><<<dim3(tiles, 1), kTile * NB, smem_pair, st>>>(P);
    PHX_CUDA(ctx, cudaGetLastError());
  }
  finalize_kernel<<<(nq + 127) / 128, 128, 0, st>>>(nq, NB, nT, 1, partial, b->d_E, p->finalize, nullptr, nullptr,
                                                    0.0, Aout_d);
  PHX_CUDA(ctx, cudaGetLastError());
  PHX_CUDA(ctx, cudaStreamSynchronize(st));
  return PHX_OK;
}

}  // namespace

extern "C" int phx_ph_linewidths_static(phx_v3* v, phx_bands* b, const phx_lw_params* p,
                                        double* Aout_d) {
  PHX_ARG(nullptr, v && b && p && Aout_d, "phx_ph_linewidths_static: bad arguments");
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, b->ctx == ctx, "v3 and bands belong to different contexts");
  PHX_ARG(ctx, b->nb == v->nb, "band count of bands and v3 differ");
  PHX_ARG(ctx, p->num_temperatures >= 1 && p->num_temperatures <= kMaxT && p->temperatures,
          "1..4 temperatures per call");
  PHX_ARG(ctx, p->smearing == PHX_SMEAR_GAUSSIAN || p->smearing == PHX_SMEAR_ADAPTIVE, "bad smearing");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_GAUSSIAN || p->sigma > 0.0, "Gaussian smearing needs sigma > 0");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_ADAPTIVE || b->d_vg, "adaptive smearing needs velocities");
  PHX_ARG(ctx, 0 <= p->q2_begin && p->q2_begin <= p->q2_end && p->q2_end <= b->nq, "bad q2 range");
  PHX_ARG(ctx, v->nb == 6, "phx_ph_linewidths_static: this build supports nb = 6");
  PHX_ARG(ctx, !p->window_energy && !p->window_cut, "phx_ph_linewidths_static: no q2 window");
  PHX_ARG(ctx, !p->isotope_coupling && !(p->boundary_length > 0.0),
          "phx_ph_linewidths_static: no isotope or boundary scattering");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  if (p->q2_begin == p->q2_end) {
    PHX_CUDA(ctx, cudaMemsetAsync(Aout_d, 0, sizeof(double) * p->num_temperatures * b->nq * b->nb, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PHX_OK;
  }
  return run_builder_static<6>(v, b, p, Aout_d);
}
