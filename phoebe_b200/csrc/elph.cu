// Electron-phonon Wannier path on the GPU, plain FP64:
//   * cacheElPh (interaction_elph.cpp:492-701): g1 = sum_Re e^{+i k1.Re}/deg g(Re, Rp, nu, w1, w2)
//     and cached(Rp, nu, b1, w2) = sum_w1 U1[w1][b1] g1.  The coupling tensor is
//     read from HBM once per 16 k1 (a batched GEMV), FP32 elements, FP64 sums.
//   * calcCouplingSquared (:229-448, no polar term): g3 = sum_Rp e^{+i q3.Rp}/deg cached,
//     g4 = sum_nu g3 ev3[nu][nu2], g = sum_w2 conj(U2[w2][b2]) g4, |g|^2.
//   * ElScatteringMatrix::builder, linewidth mode (el_scattering.cpp:38-405) with
//     symmetrizeCoupling (scattering.cpp:1209-1318) and degeneracyAveragingLinewidths
//     (:1168-1207): one thread block per 4 final states k2 = k1 + q computes their
//     couplings, symmetrises them and accumulates the rates of the k1 states.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cplx.cuh"
#include "pair_common.cuh"
#include "phx_consts.h"
#include "phx_internal.h"

// split-precision Rp transform (el_split.cu)
void phx_el_split_dims(int nRp, int nq, int* nKC, int* nMT);
size_t phx_el_split_phase_bytes(int nRp, int nq);
size_t phx_el_split_coupling_bytes(int nRp, int xmax);
int phx_el_split_max_batch();
int phx_el_split_phases(phx_ctx* ctx, int nq, const double* qcart, int nRp, const double* Rp, const double* degP,
                        uint8_t* img);
int phx_el_split_g3_batch(phx_ctx* ctx, const uint8_t* Aimg, uint8_t* Bimg, const double2* cached, size_t per,
                          int nRp, int nph, int nw, int nq, int nb, const int* nb1, float2* g3T, int* ldq_out,
                          int* xoff_out);
size_t phx_el_split_g_image_bytes(int nRe, long long N);
size_t phx_el_split_k1_image_bytes();
int phx_el_split_g_image(phx_ctx* ctx, const float* g, int nRe, long long N, uint8_t* img);
int phx_el_split_g1(phx_ctx* ctx, const uint8_t* gimg, int nRe, long long N, const double* Re, const double* degE,
                    int nb, const double* k1s, uint8_t* kimg, double2* g1);

namespace {

constexpr int kB1 = 16;       // k1 points per pass over the coupling tensor
constexpr int kQT = 1;        // final states per pair block
constexpr int kMaxW = 8;      // Wannier orbitals
constexpr int kMaxPh = 12;    // phonon branches
constexpr int kPairThreads = 64;

// g1[b][e] = sum_Re ph[b][Re] g[Re][e] for the kB1 k1 of the batch (e over nRp*nph*nw*nw)
__global__ void __launch_bounds__(256) elph_g1_kernel(const float2* __restrict__ g, int nRe, size_t N,
                                                      const double* __restrict__ Re,
                                                      const double* __restrict__ degE,
                                                      const double* __restrict__ k1s, int nb,
                                                      double2* __restrict__ g1) {
  extern __shared__ __align__(16) char sraw[];
  double2* ph = reinterpret_cast<double2*>(sraw);  // [kB1][nRe]
  for (int i = threadIdx.x; i < kB1 * nRe; i += blockDim.x) {
    const int b = i / nRe, r = i % nRe;
    double2 v = cmk(0.0, 0.0);
    if (b < nb) {
      const double* k = k1s + 3 * b;
      double sn, cs;
      sincos(k[0] * Re[3 * r] + k[1] * Re[3 * r + 1] + k[2] * Re[3 * r + 2], &sn, &cs);
      v = cmk(cs / degE[r], sn / degE[r]);
    }
    ph[i] = v;
  }
  __syncthreads();
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x) {
    double2 acc[kB1];
#pragma unroll
    for (int b = 0; b < kB1; ++b) acc[b] = cmk(0.0, 0.0);
    for (int r = 0; r < nRe; ++r) {
      const float2 x = __ldg(g + (size_t)r * N + e);
      const double2 xd = cmk((double)x.x, (double)x.y);
#pragma unroll
      for (int b = 0; b < kB1; ++b) acc[b] = cadd(acc[b], cmul(xd, ph[b * nRe + r]));
    }
#pragma unroll
    for (int b = 0; b < kB1; ++b)
      if (b < nb) g1[(size_t)b * N + e] = acc[b];
  }
}

// cached[b](Rp, nu, b1, w2) = sum_w1 g1[b](Rp, nu, w1, w2) U1[b][w1][b1]   (b1 < nb1[b], else 0)
__global__ void elph_rot_kernel(const double2* __restrict__ g1, int nRpPh, int nw, int nb,
                                const double2* __restrict__ U1s, const int* __restrict__ nb1s,
                                double2* __restrict__ cached) {
  const size_t per = (size_t)nRpPh * nw * nw;
  const size_t total = per * nb;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / per);
    const size_t rest = i % per;
    const int w2 = (int)(rest % nw), b1 = (int)((rest / nw) % nw);
    const size_t rp = rest / (nw * nw);
    double2 acc = cmk(0.0, 0.0);
    if (b1 < nb1s[b]) {
      const double2* G = g1 + (size_t)b * per + rp * nw * nw;
      const double2* U = U1s + (size_t)b * nw * nw;
      for (int w1 = 0; w1 < nw; ++w1) acc = cadd(acc, cmul(G[w1 * nw + w2], U[w1 * nw + b1]));
    }
    cached[i] = acc;
  }
}

// ---------------------------------------------------------------------------
// pair block: couplings of kQT final states of one k1
// ---------------------------------------------------------------------------
struct PairSmem {
  double2* ph;    // [kQT][nRp]
  double2* g3;    // [kQT][nph][kMaxW(b1)][nw]
  double2* g4;    // same
  double2* U2;    // [kQT][nw][kMaxW(b2)]
  double2* ev3;   // [kQT][nph][nph]
  double* cs;     // [kQT][kMaxW][kMaxW][nph] |g|^2
  double* E2;     // [kQT][kMaxW]
  double* E3;     // [kQT][nph]
  double* acc;    // [kMaxW][kMaxT] block sums of the rates
  int* info;      // [kQT][4]: valid, nb2, k2 index, q index
  double* f2;     // [kQT][kMaxW][kMaxT] Fermi occupation of the final electron states
  double* n3;     // [kQT][kMaxPh][kMaxT] Bose occupation of the phonons
  double2* wd;    // [kQT][kMaxW(b1)][kMaxW(b2)] adaptive width: (sigma, |v1 - v2| == 0)
};

__host__ __device__ inline size_t pair_smem_layout(int nRp, int nph, int nw, size_t* off) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o += (bytes + 15) & ~size_t(15);
    return r;
  };
  off[0] = take(sizeof(double2) * kQT * nRp);
  // |g|^2 (cs) is written after g4 is complete, when g3 is dead: it shares g3's space
  const size_t g3b = sizeof(double2) * kQT * nph * kMaxW * nw, csb = sizeof(double) * kQT * kMaxW * kMaxW * nph;
  off[1] = take(g3b > csb ? g3b : csb);
  off[2] = take(sizeof(double2) * kQT * nph * kMaxW * nw);
  off[3] = take(sizeof(double2) * kQT * nw * kMaxW);
  off[4] = take(sizeof(double2) * kQT * nph * nph);
  off[5] = off[1];
  off[6] = take(sizeof(double) * kQT * kMaxW);
  off[7] = take(sizeof(double) * kQT * nph);
  off[8] = take(sizeof(double) * kMaxW * pairc::kMaxT);
  off[9] = take(sizeof(int) * kQT * 4);
  off[10] = take(sizeof(double) * kQT * kMaxW * pairc::kMaxT);
  off[11] = take(sizeof(double) * kQT * kMaxPh * pairc::kMaxT);
  off[12] = take(sizeof(double2) * kQT * kMaxW * kMaxW);
  return o;
}

__device__ inline PairSmem pair_carve(char* base, int nRp, int nph, int nw) {
  size_t off[13];
  pair_smem_layout(nRp, nph, nw, off);
  PairSmem s;
  s.ph = reinterpret_cast<double2*>(base + off[0]);
  s.g3 = reinterpret_cast<double2*>(base + off[1]);
  s.g4 = reinterpret_cast<double2*>(base + off[2]);
  s.U2 = reinterpret_cast<double2*>(base + off[3]);
  s.ev3 = reinterpret_cast<double2*>(base + off[4]);
  s.cs = reinterpret_cast<double*>(base + off[5]);
  s.E2 = reinterpret_cast<double*>(base + off[6]);
  s.E3 = reinterpret_cast<double*>(base + off[7]);
  s.acc = reinterpret_cast<double*>(base + off[8]);
  s.info = reinterpret_cast<int*>(base + off[9]);
  s.f2 = reinterpret_cast<double*>(base + off[10]);
  s.n3 = reinterpret_cast<double*>(base + off[11]);
  s.wd = reinterpret_cast<double2*>(base + off[12]);
  return s;
}

// |g|^2 of the kQT final states whose phases, U2 (nb2 columns) and ev3 are staged;
// cached is (nRp, nph, nw(b1), nw) of one k1 with nb1 active bands.  G3IN:
// g3 comes from the tensor-core GEMM (split path) instead of the FP64 Rp
// transform; each path is its own instantiation, so that each kernel holds
// only its code (the pair kernel is bound by instruction fetch otherwise).
template <bool G3IN>
__device__ void pair_couplings(const double2* __restrict__ cached, int nRp, int nph, int nw, int nb1,
                               const PairSmem& s, const float2* __restrict__ g3in = nullptr, int g3ld = 0) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nx = nph * nb1 * nw;
  if constexpr (G3IN) {
    // g3 from the tensor-core GEMM, stored g3in[x * g3ld + q] (q = phonon mesh index)
    for (int i = tid; i < kQT * nx; i += NT) {
      const int q = i % kQT, x = i / kQT;
      const int w2 = x % nw, b1 = (x / nw) % nb1, nu = x / (nw * nb1);
      double2 v = cmk(0.0, 0.0);
      if (s.info[4 * q]) {
        const float2 f = g3in[(size_t)x * g3ld + s.info[4 * q + 3]];
        v = cmk((double)f.x, (double)f.y);
      }
      s.g3[((q * nph + nu) * kMaxW + b1) * nw + w2] = v;
    }
  }
  // g3[q][nu][b1][w2] = sum_Rp ph[q][Rp] cached[Rp][nu][b1][w2]
  for (int x = tid; x < (G3IN ? 0 : nx); x += NT) {
    const int w2 = x % nw, b1 = (x / nw) % nb1, nu = x / (nw * nb1);
    const size_t cx = ((size_t)nu * nw + b1) * nw + w2;
    double2 acc[kQT];
#pragma unroll
    for (int q = 0; q < kQT; ++q) acc[q] = cmk(0.0, 0.0);
    for (int r = 0; r < nRp; ++r) {
      const double2 c = cached[(size_t)r * nph * nw * nw + cx];
#pragma unroll
      for (int q = 0; q < kQT; ++q) acc[q] = cadd(acc[q], cmul(s.ph[q * nRp + r], c));
    }
#pragma unroll
    for (int q = 0; q < kQT; ++q) s.g3[((q * nph + nu) * kMaxW + b1) * nw + w2] = acc[q];
  }
  __syncthreads();
  // g4[q][nu2][b1][w2] = sum_nu g3[q][nu][b1][w2] ev3[q][nu][nu2]
  for (int x = tid; x < kQT * nx; x += NT) {
    const int q = x / nx, r = x % nx;
    const int w2 = r % nw, b1 = (r / nw) % nb1, nu2 = r / (nw * nb1);
    double2 acc = cmk(0.0, 0.0);
    for (int nu = 0; nu < nph; ++nu)
      acc = cadd(acc, cmul(s.g3[((q * nph + nu) * kMaxW + b1) * nw + w2], s.ev3[(q * nph + nu) * nph + nu2]));
    s.g4[((q * nph + nu2) * kMaxW + b1) * nw + w2] = acc;
  }
  __syncthreads();
  // |g[q][b1][b2][nu]|^2 with g = sum_w2 conj(U2[q][w2][b2]) g4[q][nu][b1][w2]
  for (int x = tid; x < kQT * nb1 * kMaxW * nph; x += NT) {
    const int nu = x % nph, b2 = (x / nph) % kMaxW, b1 = (x / (nph * kMaxW)) % nb1, q = x / (nph * kMaxW * nb1);
    double v = 0.0;
    if (b2 < s.info[4 * q + 1]) {
      double2 acc = cmk(0.0, 0.0);
      for (int w2 = 0; w2 < nw; ++w2)
        acc = cadd(acc, cmul(cconj(s.U2[(q * nw + w2) * kMaxW + b2]), s.g4[((q * nph + nu) * kMaxW + b1) * nw + w2]));
      v = acc.x * acc.x + acc.y * acc.y;
    }
    s.cs[((q * kMaxW + b1) * kMaxW + b2) * nph + nu] = v;
  }
  __syncthreads();
}

// symmetrizeCoupling (scattering.cpp:1209-1318) of the kQT couplings:
// forward-scan degenerate blocks of b1 (E1), then b2 (E2[q]), then nu (E3[q])
__device__ void pair_symmetrize(const double* E1, int nb1, int nph, const PairSmem& s) {
  const int tid = threadIdx.x, NT = blockDim.x;
  auto C = [&](int q, int b1, int b2, int nu) -> double& {
    return s.cs[((q * kMaxW + b1) * kMaxW + b2) * nph + nu];
  };
  // A forward-scan block of two or more states exists exactly when two
  // neighbouring energies are within the threshold; a pass without one is
  // the identity and is skipped (block-wide votes, which are also barriers).
  const bool n1 = tid + 1 < nb1 && fabs(E1[tid] - E1[tid + 1]) < 1.0e-6;
  bool n2 = false, n3 = false;
  if (tid < kQT * kMaxW) {
    const int q = tid / kMaxW, b = tid % kMaxW;
    n2 = s.info[4 * q] && b + 1 < s.info[4 * q + 1] && fabs(s.E2[q * kMaxW + b] - s.E2[q * kMaxW + b + 1]) < 1.0e-6;
  }
  if (tid < kQT * nph) {
    const int q = tid / nph, nu = tid % nph;
    n3 = s.info[4 * q] && nu + 1 < nph && fabs(s.E3[q * nph + nu] - s.E3[q * nph + nu + 1]) < 1.0e-6;
  }
  if (!__syncthreads_or(n1 || n2 || n3)) return;
  if (__syncthreads_or(n1)) {
    for (int x = tid; x < kQT * kMaxW * nph; x += NT) {
      const int q = x / (kMaxW * nph), b2 = (x / nph) % kMaxW, nu = x % nph;
      if (!s.info[4 * q] || b2 >= s.info[4 * q + 1]) continue;
      for (int ib = 0; ib < nb1;) {
        int deg = 0;
        for (int i = ib; i < nb1; ++i) {
          if (fabs(E1[ib] - E1[i]) < 1.0e-6) ++deg;
          else break;
        }
        if (deg > 1) {
          double t = 0.0;
          for (int i = 0; i < deg; ++i) t += C(q, ib + i, b2, nu);
          for (int i = 0; i < deg; ++i) C(q, ib + i, b2, nu) = t / float(deg);
        }
        ib += deg;
      }
    }
  }
  if (__syncthreads_or(n2)) {
    for (int x = tid; x < kQT * kMaxW * nph; x += NT) {
      const int q = x / (kMaxW * nph), b1 = (x / nph) % kMaxW, nu = x % nph;
      const int nb2 = s.info[4 * q + 1];
      if (!s.info[4 * q] || b1 >= nb1) continue;
      const double* E2 = s.E2 + q * kMaxW;
      for (int ib = 0; ib < nb2;) {
        int deg = 0;
        for (int i = ib; i < nb2; ++i) {
          if (fabs(E2[ib] - E2[i]) < 1.0e-6) ++deg;
          else break;
        }
        if (deg > 1) {
          double t = 0.0;
          for (int i = 0; i < deg; ++i) t += C(q, b1, ib + i, nu);
          for (int i = 0; i < deg; ++i) C(q, b1, ib + i, nu) = t / float(deg);
        }
        ib += deg;
      }
    }
  }
  if (__syncthreads_or(n3)) {
    for (int x = tid; x < kQT * kMaxW * kMaxW; x += NT) {
      const int q = x / (kMaxW * kMaxW), b1 = (x / kMaxW) % kMaxW, b2 = x % kMaxW;
      if (!s.info[4 * q] || b1 >= nb1 || b2 >= s.info[4 * q + 1]) continue;
      const double* E3 = s.E3 + q * nph;
      for (int ib = 0; ib < nph;) {
        int deg = 0;
        for (int i = ib; i < nph; ++i) {
          if (fabs(E3[ib] - E3[i]) < 1.0e-6) ++deg;
          else break;
        }
        if (deg > 1) {
          double t = 0.0;
          for (int i = 0; i < deg; ++i) t += C(q, b1, b2, ib + i);
          for (int i = 0; i < deg; ++i) C(q, b1, b2, ib + i) = t / float(deg);
        }
        ib += deg;
      }
    }
  }
  __syncthreads();
}

struct ElArgs {
  int nw, nph, nRp;
  const double2* cached;   // batch of k1: cached + blockIdx.y * cper
  size_t cper;
  const double* Rp;
  const double* degP;
  int kmesh[3], qmesh[3];
  const double* Ek;        // (nk,nw)
  const double2* Uk;       // (nk,nw,nw)
  const double* vk;        // (nk,nw,3) or null
  const double* kcart;     // (nk,3)
  const int* lo;
  const int* hi;
  const double* Eq;        // (nq,nph)
  const double2* evq;      // (nq,nph,nph)
  int ik1s[kB1], i1s[kB1]; // per blockIdx.y: k1 mesh index and its row in the output
  long long g3offs[kB1];   // per blockIdx.y: offset of its g3 columns in g3in
  int nk1;
  int nT;
  double temps[pairc::kMaxT];
  double mu;
  int smearing;
  double sigma;
  double qT[9];
  double norm;
  double* out;             // (nT, nk1, nw)
  const float2* g3in;      // precomputed g3 of this k1, g3in[x * g3ld + q], or null
  int g3ld;
};

// adaptive width of a (k1 b1, k2 b2) pair from v = v1 - v2 (delta_function.cpp:65-88);
// vzero: |v| == 0
struct ElWidth {
  double sg;
  bool vzero;
};
__device__ __forceinline__ ElWidth el_width(const ElArgs& A, const double v[3]) {
  ElWidth w;
  w.vzero = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) == 0.0;
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double d = A.qT[3 * i] * v[0] + A.qT[3 * i + 1] * v[1] + A.qT[3 * i + 2] * v[2];
    s += d * d;
  }
  w.sg = sqrt(s / 6.0);
  return w;
}


// Delta of the reference (delta_function.cpp:65-96) from a tabulated width:
// w.x the floored sigma with the zero-velocity flag in its sign bit, w.y its
// reciprocal (adaptive), or the fixed Gaussian width's reciprocal ginv; the
// quotients e / sigma and 1 / (sqrt(pi) sigma erf(2)) become products.
template <int SM>
__device__ __forceinline__ double el_delta_tab(double ginv, double e, double2 w) {
  if constexpr (SM == PHX_SMEAR_GAUSSIAN) {
    const double x = e * ginv;
    if (x > 6.0) return 0.0;
    return ginv * (1.0 / phxc::sqrtPi) * exp(-x * x);
  }
  const double sg = fabs(w.x);
  if (signbit(w.x) && e == 0.0) return 1.0;
  if (sg == 0.0) return 0.0;
  if (fabs(e) > 2.0 * sg) return 0.0;
  const double x = e * w.y;   // |x| <= 2 past the cut-off
  return exp(-x * x) * w.y * (1.0 / (phxc::sqrtPi * phxc::erf2));
}

// G3IN: g3 from the tensor-core GEMM (split path); SM: the smearing.  Each
// combination is its own instantiation, which keeps the kernel's code small.
template <bool G3IN, int SM>
__global__ void __launch_bounds__(kPairThreads) el_pair_kernel(ElArgs A) {
  extern __shared__ __align__(16) char sraw[];
  const int nw = A.nw, nph = A.nph, nRp = A.nRp;
  // no phase buffer when g3 comes from the tensor-core GEMM
  const PairSmem s = pair_carve(sraw, G3IN ? 0 : nRp, nph, nw);
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nq = A.qmesh[0] * A.qmesh[1] * A.qmesh[2];
  const int jb = blockIdx.y;
  const int ik1 = A.ik1s[jb], i1 = A.i1s[jb], lo1 = A.lo[ik1], nb1 = A.hi[ik1] - lo1;
  const double2* cached = A.cached + (size_t)jb * A.cper;
  const float2* g3in = G3IN ? A.g3in + A.g3offs[jb] : nullptr;
  const int x1 = ik1 % A.kmesh[0], y1 = (ik1 / A.kmesh[0]) % A.kmesh[1], z1 = ik1 / (A.kmesh[0] * A.kmesh[1]);
  const int f0 = A.kmesh[0] / A.qmesh[0], f1 = A.kmesh[1] / A.qmesh[1], f2 = A.kmesh[2] / A.qmesh[2];
  const double* E1 = A.Ek + (size_t)ik1 * nw + lo1;
  for (int i = tid; i < kMaxW * pairc::kMaxT; i += NT) s.acc[i] = 0.0;
  // final states of this block
  if (tid < kQT) {
    const int iq = blockIdx.x * kQT + tid;
    int valid = 0, nb2 = 0, ik2 = 0;
    if (iq < nq) {
      const int qx = iq % A.qmesh[0], qy = (iq / A.qmesh[0]) % A.qmesh[1], qz = iq / (A.qmesh[0] * A.qmesh[1]);
      ik2 = (x1 + f0 * qx) % A.kmesh[0] +
            A.kmesh[0] * ((y1 + f1 * qy) % A.kmesh[1] + A.kmesh[1] * ((z1 + f2 * qz) % A.kmesh[2]));
      nb2 = A.hi[ik2] - A.lo[ik2];
      valid = nb2 > 0;
    }
    s.info[4 * tid] = valid;
    s.info[4 * tid + 1] = valid ? nb2 : 0;
    s.info[4 * tid + 2] = ik2;
    s.info[4 * tid + 3] = iq;
  }
  __syncthreads();
  int any_valid = 0;
#pragma unroll
  for (int q = 0; q < kQT; ++q) any_valid |= s.info[4 * q];
  if (!any_valid) return;
  // phases e^{+i q3.Rp}/deg with q3 = k2 - k1 (helper_el_scattering.cpp:233-234),
  // not needed when g3 comes from the tensor-core GEMM
  for (int i = tid; i < (G3IN ? 0 : kQT * nRp); i += NT) {
    const int q = i / nRp, r = i % nRp;
    double2 v = cmk(0.0, 0.0);
    if (s.info[4 * q]) {
      const int ik2 = s.info[4 * q + 2];
      double q3[3];
      for (int c = 0; c < 3; ++c) q3[c] = A.kcart[3 * ik2 + c] - A.kcart[3 * ik1 + c];
      double sn, cs;
      sincos(q3[0] * A.Rp[3 * r] + q3[1] * A.Rp[3 * r + 1] + q3[2] * A.Rp[3 * r + 2], &sn, &cs);
      v = cmk(cs / A.degP[r], sn / A.degP[r]);
    }
    s.ph[i] = v;
  }
  for (int i = tid; i < kQT * nw * kMaxW; i += NT) {
    const int q = i / (nw * kMaxW), w = (i / kMaxW) % nw, b2 = i % kMaxW;
    double2 v = cmk(0.0, 0.0);
    if (s.info[4 * q] && b2 < s.info[4 * q + 1]) {
      const int ik2 = s.info[4 * q + 2];
      v = A.Uk[((size_t)ik2 * nw + w) * nw + A.lo[ik2] + b2];
    }
    s.U2[i] = v;
  }
  for (int i = tid; i < kQT * nph * nph; i += NT) {
    const int q = i / (nph * nph);
    s.ev3[i] = s.info[4 * q] ? A.evq[(size_t)s.info[4 * q + 3] * nph * nph + i % (nph * nph)] : cmk(0.0, 0.0);
  }
  for (int i = tid; i < kQT * kMaxW; i += NT) {
    const int q = i / kMaxW, b2 = i % kMaxW;
    s.E2[i] = (s.info[4 * q] && b2 < s.info[4 * q + 1]) ? A.Ek[(size_t)s.info[4 * q + 2] * nw + A.lo[s.info[4 * q + 2]] + b2] : 0.0;
  }
  for (int i = tid; i < kQT * nph; i += NT) {
    const int q = i / nph;
    s.E3[i] = s.info[4 * q] ? A.Eq[(size_t)s.info[4 * q + 3] * nph + i % nph] : 0.0;
  }
  // populations of the final states (el_scattering.cpp:287-300)
  for (int i = tid; i < kQT * kMaxW * A.nT; i += NT) {
    const int t = i % A.nT, b2 = (i / A.nT) % kMaxW, q = i / (A.nT * kMaxW);
    double f = 0.0;
    if (s.info[4 * q] && b2 < s.info[4 * q + 1]) {
      const double T = A.temps[t];
      const int ik2 = s.info[4 * q + 2];
      const double en2 = A.Ek[(size_t)ik2 * nw + A.lo[ik2] + b2];
      if (T <= 0.0) {
        f = en2 <= A.mu ? 1.0 : 0.0;
      } else {
        f = 1.0 / (exp((en2 - A.mu) / T) + 1.0);
        f = fmin(1.0, fmax(0.0, f));
      }
    }
    s.f2[(q * kMaxW + b2) * pairc::kMaxT + t] = f;
  }
  for (int i = tid; i < kQT * nph * A.nT; i += NT) {
    const int t = i % A.nT, nu = (i / A.nT) % nph, q = i / (A.nT * nph);
    double n = 0.0;
    const double T = A.temps[t];
    if (s.info[4 * q] && T > 0.0) {
      n = 1.0 / (exp(A.Eq[(size_t)s.info[4 * q + 3] * nph + nu] / T) - 1.0);
      if (n < 0.0) n = 0.0;
    }
    s.n3[(q * kMaxPh + nu) * pairc::kMaxT + t] = n;
  }
  // adaptive widths of the (b1, b2) pairs (delta_function.cpp:65-88), floored,
  // as (sigma, 1/sigma) with the zero-velocity flag in the sign bit of sigma
  for (int x = tid; x < (SM == PHX_SMEAR_ADAPTIVE ? kQT * kMaxW * kMaxW : 0); x += NT) {
    const int b2 = x % kMaxW, b1 = (x / kMaxW) % kMaxW, q = x / (kMaxW * kMaxW);
    double2 wv = make_double2(0.0, 0.0);
    if (s.info[4 * q] && b1 < nb1 && b2 < s.info[4 * q + 1]) {
      const int ik2 = s.info[4 * q + 2];
      double v[3];
      for (int c = 0; c < 3; ++c)
        v[c] = A.vk[((size_t)ik1 * nw + lo1 + b1) * 3 + c] - A.vk[((size_t)ik2 * nw + A.lo[ik2] + b2) * 3 + c];
      const ElWidth w = el_width(A, v);
      double sg = w.sg;
      if (sg != 0.0 && sg < phxc::adaptiveCutoff) sg = phxc::adaptiveCutoff;
      wv = make_double2(w.vzero ? -0.0 : sg, sg > 0.0 ? 1.0 / sg : 0.0);
    }
    s.wd[x] = wv;
  }
  __syncthreads();
  pair_couplings<G3IN>(cached, nRp, nph, nw, nb1, s, g3in, A.g3ld);
  pair_symmetrize(E1, nb1, nph, s);
  // rates (el_scattering.cpp:268-327), one thread per (b1, q, b2, nu) with b1
  // slowest: when the kQT * kMaxW * nph entries of one b1 fill whole warps
  // (nph even), a warp reduces its rates and adds them once; otherwise every
  // thread adds its own
  const int per_b1 = kQT * kMaxW * nph;
  const bool warp_sums = per_b1 % 32 == 0;
  const double ginv = SM == PHX_SMEAR_GAUSSIAN ? 1.0 / A.sigma : 0.0;
  for (int x = tid; x < nb1 * per_b1; x += NT) {
    const int nu = x % nph, b2 = (x / nph) % kMaxW, q = (x / (nph * kMaxW)) % kQT, b1 = x / per_b1;
    double r[pairc::kMaxT];
#pragma unroll
    for (int t = 0; t < pairc::kMaxT; ++t) r[t] = 0.0;
    const double en3 = s.E3[q * nph + nu];
    if (s.info[4 * q] && b2 < s.info[4 * q + 1] && en3 >= phxc::elPhononCutoff) {
      const double en1 = E1[b1], en2 = s.E2[q * kMaxW + b2];
      const double2 wv = SM == PHX_SMEAR_ADAPTIVE ? s.wd[(q * kMaxW + b1) * kMaxW + b2] : make_double2(0.0, 0.0);
      const double d1 = el_delta_tab<SM>(ginv, en1 - en2 + en3, wv);
      const double d2 = el_delta_tab<SM>(ginv, en1 - en2 - en3, wv);
      if (d1 > 0.0 || d2 > 0.0) {
        const double c = s.cs[((q * kMaxW + b1) * kMaxW + b2) * nph + nu] * A.norm * phxc::pi / en3;
#pragma unroll
        for (int t = 0; t < pairc::kMaxT; ++t) {
          if (t < A.nT) {
            const double fermi2 = s.f2[(q * kMaxW + b2) * pairc::kMaxT + t];
            const double bose3 = s.n3[(q * kMaxPh + nu) * pairc::kMaxT + t];
            r[t] = c * ((fermi2 + bose3) * d1 + (1.0 - fermi2 + bose3) * d2);
          }
        }
      }
    }
#pragma unroll
    for (int t = 0; t < pairc::kMaxT; ++t) {
      if (t < A.nT) {
        double v = r[t];
        if (warp_sums) {
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if ((tid & 31) == 0 && v != 0.0) atomicAdd(&s.acc[b1 * pairc::kMaxT + t], v);
        } else if (v != 0.0) {
          atomicAdd(&s.acc[b1 * pairc::kMaxT + t], v);
        }
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < nb1 * A.nT; i += NT) {
    const int b1 = i / A.nT, t = i % A.nT;
    const double v = s.acc[b1 * pairc::kMaxT + t];
    if (v != 0.0) atomicAdd(&A.out[((size_t)t * A.nk1 + i1) * nw + lo1 + b1], v);
  }
}

// API variant: explicit final states (q3, U2, ev3), |g|^2 written out
__global__ void __launch_bounds__(kPairThreads) elph_api_pair_kernel(
    const double2* __restrict__ cached, int nRp, int nph, int nw, int nb1, const double* __restrict__ Rp,
    const double* __restrict__ degP, int nk2, const double* __restrict__ q3s, const double2* __restrict__ U2s,
    const int* __restrict__ nb2s, int nb2max, const double2* __restrict__ ev3s, double* __restrict__ out) {
  extern __shared__ __align__(16) char sraw[];
  const PairSmem s = pair_carve(sraw, nRp, nph, nw);
  const int tid = threadIdx.x, NT = blockDim.x;
  if (tid < kQT) {
    const int j = blockIdx.x * kQT + tid;
    s.info[4 * tid] = j < nk2;
    s.info[4 * tid + 1] = j < nk2 ? nb2s[j] : 0;
    s.info[4 * tid + 2] = j;
    s.info[4 * tid + 3] = j;
  }
  __syncthreads();
  for (int i = tid; i < kQT * nRp; i += NT) {
    const int q = i / nRp, r = i % nRp, j = blockIdx.x * kQT + q;
    double2 v = cmk(0.0, 0.0);
    if (j < nk2) {
      const double* q3 = q3s + 3 * j;
      double sn, cs;
      sincos(q3[0] * Rp[3 * r] + q3[1] * Rp[3 * r + 1] + q3[2] * Rp[3 * r + 2], &sn, &cs);
      v = cmk(cs / degP[r], sn / degP[r]);
    }
    s.ph[i] = v;
  }
  for (int i = tid; i < kQT * nw * kMaxW; i += NT) {
    const int q = i / (nw * kMaxW), w = (i / kMaxW) % nw, b2 = i % kMaxW, j = blockIdx.x * kQT + q;
    s.U2[i] = (j < nk2 && b2 < nb2s[j]) ? U2s[((size_t)j * nw + w) * nb2max + b2] : cmk(0.0, 0.0);
  }
  for (int i = tid; i < kQT * nph * nph; i += NT) {
    const int q = i / (nph * nph), j = blockIdx.x * kQT + q;
    s.ev3[i] = j < nk2 ? ev3s[(size_t)j * nph * nph + i % (nph * nph)] : cmk(0.0, 0.0);
  }
  __syncthreads();
  pair_couplings<false>(cached, nRp, nph, nw, nb1, s);
  for (int x = tid; x < kQT * nb1 * nb2max * nph; x += NT) {
    const int nu = x % nph, b2 = (x / nph) % nb2max, b1 = (x / (nph * nb2max)) % nb1, q = x / (nph * nb2max * nb1);
    const int j = blockIdx.x * kQT + q;
    if (j >= nk2) continue;
    out[(((size_t)j * nb1 + b1) * nb2max + b2) * nph + nu] =
        b2 < kMaxW ? s.cs[((q * kMaxW + b1) * kMaxW + b2) * nph + nu] : 0.0;
  }
}

__global__ void el_window_kernel(const double* __restrict__ E, int nk, int nw, double mu, double w,
                                 int* __restrict__ lo, int* __restrict__ hi) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
    int l = nw, h = 0;
    for (int b = 0; b < nw; ++b) {
      const double e = E[(size_t)k * nw + b];
      if (e >= mu - w && e <= mu + w) {
        l = min(l, b);
        h = max(h, b + 1);
      }
    }
    if (h <= l) l = h = 0;
    lo[k] = l;
    hi[k] = h;
  }
}

// active-band counts of the k1 list
__global__ void el_k1_bands_kernel(const int* __restrict__ k1s, int nk1, const int* __restrict__ lo,
                                   const int* __restrict__ hi, int* __restrict__ nb1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nk1) nb1[i] = hi[k1s[i]] - lo[k1s[i]];
}

// k1 coordinates, active-band counts and U1 columns lo..hi-1 of a batch of
// active k1 (mesh indices ik[0..nb)); unused slots are zeroed
__global__ void el_batch_gather_kernel(const int* __restrict__ ik, int nb, const int* __restrict__ lo,
                                       const int* __restrict__ hi, const double* __restrict__ kcart,
                                       const double2* __restrict__ Uk, int nw, double* __restrict__ kb,
                                       double2* __restrict__ ub, int* __restrict__ nbb) {
  for (int i = threadIdx.x; i < kB1 * nw * nw; i += blockDim.x) {
    const int j = i / (nw * nw), w = (i / nw) % nw, b = i % nw;
    double2 v = cmk(0.0, 0.0);
    if (j < nb) {
      const int k = ik[j];
      if (b < hi[k] - lo[k]) v = Uk[((size_t)k * nw + w) * nw + lo[k] + b];
    }
    ub[i] = v;
  }
  for (int j = threadIdx.x; j < kB1; j += blockDim.x) {
    const int k = j < nb ? ik[j] : 0;
    nbb[j] = j < nb ? hi[k] - lo[k] : 0;
    for (int c = 0; c < 3; ++c) kb[3 * j + c] = j < nb ? kcart[3 * (size_t)k + c] : 0.0;
  }
}

// degeneracyAveragingLinewidths of temperature row 0 (scattering.cpp:1168-1207)
__global__ void el_degavg_kernel(double* __restrict__ out, int nk1, int nw, const int* __restrict__ k1s,
                                 const double* __restrict__ Ek, const int* __restrict__ lo,
                                 const int* __restrict__ hi) {
  for (int i1 = blockIdx.x * blockDim.x + threadIdx.x; i1 < nk1; i1 += gridDim.x * blockDim.x) {
    const int ik = k1s[i1], l = lo[ik], n = hi[ik] - l;
    if (n <= 0) continue;
    const double* E = Ek + (size_t)ik * nw + l;
    double tmp[kMaxW];
    for (int b1 = 0; b1 < n; ++b1) {
      int cnt = 0;
      double s = 0.0;
      for (int b2 = 0; b2 < n; ++b2)
        if (fabs(E[b2] - E[b1]) < 1.0e-6) {
          ++cnt;
          s += out[(size_t)i1 * nw + l + b2];
        }
      tmp[b1] = s / float(cnt);
    }
    for (int b1 = 0; b1 < n; ++b1) out[(size_t)i1 * nw + l + b1] = tmp[b1];
  }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int elph_reserve(phx_elph* e, size_t bytes) {
  if (e->scratch_bytes >= bytes) return PHX_OK;
  cudaFree(e->d_scratch);
  e->d_scratch = nullptr;
  e->scratch_bytes = 0;
  PHX_CUDA(e->ctx, cudaMalloc(&e->d_scratch, bytes));
  e->scratch_bytes = bytes;
  return PHX_OK;
}

// cacheElPh of nb (<= kB1) k1 points: k1s (device, nb*3), U1s (device, nb*nw*nw, columns
// >= nb1 ignored), nb1s (device) -> cached (device, nb * nRp*nph*nw*nw)
int elph_cache_batch(phx_elph* e, int nb, const double* d_k1s, const double2* d_U1s, const int* d_nb1s,
                     double2* d_g1, double2* d_cached, bool tensor_cores = false) {
  phx_ctx* ctx = e->ctx;
  const size_t N = (size_t)e->nRp * e->nph * e->nw * e->nw;
  if (tensor_cores) {
    // g1 on the tensor cores from the split image of g (built once per coupling object)
    if (!e->d_gimg) {
      PHX_CUDA(ctx, cudaMalloc(&e->d_gimg, phx_el_split_g_image_bytes(e->nRe, (long long)N)));
      PHX_CUDA(ctx, cudaMalloc(&e->d_kimg, phx_el_split_k1_image_bytes()));
      PHX_TRY(phx_el_split_g_image(ctx, e->d_g, e->nRe, (long long)N, e->d_gimg));
    }
    PHX_TRY(phx_el_split_g1(ctx, e->d_gimg, e->nRe, (long long)N, e->d_Re, e->d_degE, nb, d_k1s, e->d_kimg, d_g1));
    elph_rot_kernel<<<std::min<size_t>((N * nb + 255) / 256, (size_t)ctx->num_sms * 16), 256, 0, ctx->stream>>>(
        d_g1, e->nRp * e->nph, e->nw, nb, d_U1s, d_nb1s, d_cached);
    PHX_CUDA(ctx, cudaGetLastError());
    return PHX_OK;
  }
  const size_t smem = sizeof(double2) * kB1 * e->nRe;
  if (smem > 48 * 1024)
    PHX_CUDA(ctx, cudaFuncSetAttribute(elph_g1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<size_t>((N + 255) / 256, (size_t)ctx->num_sms * 8);
  elph_g1_kernel<<<grid, 256, smem, ctx->stream>>>(reinterpret_cast<const float2*>(e->d_g), e->nRe, N, e->d_Re,
                                                   e->d_degE, d_k1s, nb, d_g1);
  PHX_CUDA(ctx, cudaGetLastError());
  elph_rot_kernel<<<std::min<size_t>((N * nb + 255) / 256, (size_t)ctx->num_sms * 16), 256, 0, ctx->stream>>>(
      d_g1, e->nRp * e->nph, e->nw, nb, d_U1s, d_nb1s, d_cached);
  PHX_CUDA(ctx, cudaGetLastError());
  return PHX_OK;
}

size_t pair_smem(const phx_elph* e) {
  size_t off[13];
  return pair_smem_layout(e->nRp, e->nph, e->nw, off);
}

}  // namespace

extern "C" int phx_elph_create(phx_ctx* ctx, int nw, int nph, int nRe, int nRp, const double* Re,
                               const double* degE, const double* Rp, const double* degP, const float* g,
                               phx_elph** out) {
  PHX_ARG(ctx, ctx && Re && degE && Rp && degP && g && out, "phx_elph_create: bad arguments");
  PHX_ARG(ctx, nw > 0 && nw <= kMaxW && nph > 0 && nph <= kMaxPh && nRe > 0 && nRp > 0,
          "phx_elph_create: need 0 < nw <= 8 and 0 < nph <= 12");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  phx_elph* e = new phx_elph;
  e->ctx = ctx;
  e->nw = nw;
  e->nph = nph;
  e->nRe = nRe;
  e->nRp = nRp;
  const size_t ng = (size_t)nRe * nRp * nph * nw * nw;
  cudaError_t err = cudaMalloc(&e->d_Re, sizeof(double) * 3 * nRe);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_degE, sizeof(double) * nRe);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_Rp, sizeof(double) * 3 * nRp);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_degP, sizeof(double) * nRp);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_g, sizeof(float) * 2 * ng);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_cached, sizeof(double) * 2 * (size_t)nRp * nph * nw * nw);
  if (err == cudaSuccess) err = cudaMemcpy(e->d_Re, Re, sizeof(double) * 3 * nRe, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(e->d_degE, degE, sizeof(double) * nRe, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(e->d_Rp, Rp, sizeof(double) * 3 * nRp, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(e->d_degP, degP, sizeof(double) * nRp, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(e->d_g, g, sizeof(float) * 2 * ng, cudaMemcpyHostToDevice);
  if (err != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_elph_create: ") + cudaGetErrorString(err));
    phx_elph_destroy(e);
    return PHX_ERR_CUDA;
  }
  *out = e;
  return PHX_OK;
}

extern "C" int phx_elph_destroy(phx_elph* e) {
  if (!e) return PHX_OK;
  cudaFree(e->d_Re);
  cudaFree(e->d_degE);
  cudaFree(e->d_Rp);
  cudaFree(e->d_degP);
  cudaFree(e->d_g);
  cudaFree(e->d_cached);
  cudaFree(e->d_scratch);
  cudaFree(e->d_gimg);
  cudaFree(e->d_kimg);
  delete e;
  return PHX_OK;
}

extern "C" int phx_elph_cache_k1(phx_elph* e, const double* k1, const double* U1, int nb1) {
  PHX_ARG(e ? e->ctx : nullptr, e && k1 && U1 && nb1 > 0, "phx_elph_cache_k1: bad arguments");
  phx_ctx* ctx = e->ctx;
  PHX_ARG(ctx, nb1 <= e->nw, "phx_elph_cache_k1: nb1 > number of Wannier functions");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nw = e->nw;
  const size_t N = (size_t)e->nRp * e->nph * nw * nw;
  const size_t b_k = align256(sizeof(double) * 3), b_u = align256(sizeof(double2) * nw * nw),
               b_n = align256(sizeof(int)), b_g1 = align256(sizeof(double2) * N);
  PHX_TRY(elph_reserve(e, b_k + b_u + b_n + b_g1));
  char* base = static_cast<char*>(e->d_scratch);
  double* dk = reinterpret_cast<double*>(base);
  double2* dU = reinterpret_cast<double2*>(base + b_k);
  int* dn = reinterpret_cast<int*>(base + b_k + b_u);
  double2* dg1 = reinterpret_cast<double2*>(base + b_k + b_u + b_n);
  // U1 (nw, nb1) -> (nw, nw) with zero columns beyond nb1
  std::vector<double> Upad((size_t)2 * nw * nw, 0.0);
  for (int w = 0; w < nw; ++w)
    for (int b = 0; b < nb1; ++b) {
      Upad[2 * (w * nw + b)] = U1[2 * (w * nb1 + b)];
      Upad[2 * (w * nw + b) + 1] = U1[2 * (w * nb1 + b) + 1];
    }
  PHX_CUDA(ctx, cudaMemcpyAsync(dk, k1, sizeof(double) * 3, cudaMemcpyHostToDevice, ctx->stream));
  PHX_CUDA(ctx, cudaMemcpyAsync(dU, Upad.data(), sizeof(double) * Upad.size(), cudaMemcpyHostToDevice, ctx->stream));
  PHX_CUDA(ctx, cudaMemcpyAsync(dn, &nb1, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  PHX_TRY(elph_cache_batch(e, 1, dk, dU, dn, dg1, reinterpret_cast<double2*>(e->d_cached)));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  e->nb1 = nb1;
  return PHX_OK;
}

extern "C" int phx_elph_couplings_sq(phx_elph* e, int nk2, const double* q3, const double* U2s, const int* nb2s,
                                     int nb2max, const double* ev3s, double* coupling) {
  PHX_ARG(e ? e->ctx : nullptr, e && (nk2 == 0 || (q3 && U2s && nb2s && ev3s && coupling)) && nk2 >= 0,
          "phx_elph_couplings_sq: bad arguments");
  phx_ctx* ctx = e->ctx;
  PHX_ARG(ctx, e->nb1 > 0, "phx_elph_couplings_sq: call phx_elph_cache_k1 first");
  PHX_ARG(ctx, nb2max > 0 && nb2max <= e->nw, "phx_elph_couplings_sq: nb2max out of range");
  for (int i = 0; i < nk2; ++i)
    PHX_ARG(ctx, nb2s[i] >= 0 && nb2s[i] <= nb2max, "phx_elph_couplings_sq: nb2s out of range");
  if (nk2 == 0) return PHX_OK;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nw = e->nw, nph = e->nph, nb1 = e->nb1;
  const size_t N = (size_t)e->nRp * nph * nw * nw;
  const size_t b_q = align256(sizeof(double) * 3 * nk2), b_u = align256(sizeof(double2) * nk2 * nw * nb2max),
               b_n = align256(sizeof(int) * nk2), b_e = align256(sizeof(double2) * nk2 * nph * nph),
               b_o = align256(sizeof(double) * (size_t)nk2 * nb1 * nb2max * nph),
               b_g1 = align256(sizeof(double2) * N);
  PHX_TRY(elph_reserve(e, b_q + b_u + b_n + b_e + b_o + b_g1));
  char* base = static_cast<char*>(e->d_scratch);
  double* dq = reinterpret_cast<double*>(base);
  double2* dU = reinterpret_cast<double2*>(base + b_q);
  int* dn = reinterpret_cast<int*>(base + b_q + b_u);
  double2* dev = reinterpret_cast<double2*>(base + b_q + b_u + b_n);
  double* dout = reinterpret_cast<double*>(base + b_q + b_u + b_n + b_e);
  PHX_CUDA(ctx, cudaMemcpyAsync(dq, q3, sizeof(double) * 3 * nk2, cudaMemcpyHostToDevice, ctx->stream));
  PHX_CUDA(ctx, cudaMemcpyAsync(dU, U2s, sizeof(double2) * nk2 * nw * nb2max, cudaMemcpyHostToDevice, ctx->stream));
  PHX_CUDA(ctx, cudaMemcpyAsync(dn, nb2s, sizeof(int) * nk2, cudaMemcpyHostToDevice, ctx->stream));
  PHX_CUDA(ctx, cudaMemcpyAsync(dev, ev3s, sizeof(double2) * nk2 * nph * nph, cudaMemcpyHostToDevice, ctx->stream));
  const size_t smem = pair_smem(e);
  PHX_ARG(ctx, smem <= 227 * 1024, "phx_elph_couplings_sq: too many phonon Bravais vectors");
  PHX_CUDA(ctx, cudaFuncSetAttribute(elph_api_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  elph_api_pair_kernel<<<(nk2 + kQT - 1) / kQT, kPairThreads, smem, ctx->stream>>>(
      reinterpret_cast<const double2*>(e->d_cached), e->nRp, nph, nw, nb1, e->d_Rp, e->d_degP, nk2, dq, dU, dn,
      nb2max, dev, dout);
  PHX_CUDA(ctx, cudaGetLastError());
  PHX_CUDA(ctx, cudaMemcpyAsync(coupling, dout, sizeof(double) * (size_t)nk2 * nb1 * nb2max * nph,
                                cudaMemcpyDeviceToHost, ctx->stream));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

extern "C" int phx_el_linewidths(phx_elph* e, phx_bands* el, phx_bands* ph, const phx_el_params* p, double* out,
                                 phx_lw_stats* stats) {
  PHX_ARG(e ? e->ctx : nullptr, e && el && ph && p && out, "phx_el_linewidths: bad arguments");
  phx_ctx* ctx = e->ctx;
  PHX_ARG(ctx, el->nb == e->nw && ph->nb == e->nph, "phx_el_linewidths: band counts do not match the coupling");
  PHX_ARG(ctx, p->num_temperatures >= 1 && p->num_temperatures <= pairc::kMaxT && p->temperatures,
          "phx_el_linewidths: 1..4 temperatures");
  PHX_ARG(ctx, p->num_k1 >= 0 && (p->num_k1 == 0 || p->k1_list), "phx_el_linewidths: bad k1 list");
  PHX_ARG(ctx, p->smearing == PHX_SMEAR_GAUSSIAN || p->smearing == PHX_SMEAR_ADAPTIVE,
          "phx_el_linewidths: smearing must be Gaussian or adaptive");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_ADAPTIVE || el->d_vg, "phx_el_linewidths: adaptive smearing needs velocities");
  PHX_ARG(ctx, p->smearing != PHX_SMEAR_GAUSSIAN || p->sigma > 0.0, "phx_el_linewidths: sigma must be > 0");
  for (int i = 0; i < 3; ++i)
    PHX_ARG(ctx, el->mesh[i] % ph->mesh[i] == 0, "phx_el_linewidths: the q mesh must divide the k mesh");
  const int nk = el->nq, nw = e->nw, nph = e->nph, nT = p->num_temperatures, nk1 = p->num_k1;
  for (int i = 0; i < nk1; ++i)
    PHX_ARG(ctx, p->k1_list[i] >= 0 && p->k1_list[i] < nk, "phx_el_linewidths: k1 index out of range");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t N = (size_t)e->nRp * nph * nw * nw;
  const bool split = e->precision != PHX_PREC_FP64;
  // split path: phase image, coupling image of a batch, g3T of a batch (x, q)
  int sKC = 0, sMT = 0;
  phx_el_split_dims(e->nRp, ph->nq, &sKC, &sMT);
  const int xmax = kB1 * nph * nw * nw;
  const size_t b_A = split ? align256(phx_el_split_phase_bytes(e->nRp, ph->nq)) : 0;
  const size_t b_B = split ? align256(phx_el_split_coupling_bytes(e->nRp, xmax)) : 0;
  const size_t b_g3 = split ? align256(sizeof(float2) * (size_t)xmax * sMT * 128) + b_A + b_B : 0;
  const size_t b_lo = align256(sizeof(int) * nk), b_k1 = align256(sizeof(int) * std::max(1, nk1)),
               b_out = align256(sizeof(double) * (size_t)nT * std::max(1, nk1) * nw),
               b_kb = align256(sizeof(double) * 3 * kB1), b_ub = align256(sizeof(double2) * kB1 * nw * nw),
               b_nb = align256(sizeof(int) * kB1), b_g1 = align256(sizeof(double2) * kB1 * N);
  PHX_TRY(elph_reserve(e, 2 * b_lo + 3 * b_k1 + b_out + b_kb + b_ub + b_nb + 2 * b_g1 + b_g3));
  char* base = static_cast<char*>(e->d_scratch);
  int* dlo = reinterpret_cast<int*>(base);
  int* dhi = reinterpret_cast<int*>(base + b_lo);
  int* dk1 = reinterpret_cast<int*>(base + 2 * b_lo);
  double* dout = reinterpret_cast<double*>(base + 2 * b_lo + b_k1);
  char* bb = base + 2 * b_lo + b_k1 + b_out;
  double* dkb = reinterpret_cast<double*>(bb);
  double2* dub = reinterpret_cast<double2*>(bb + b_kb);
  int* dnb = reinterpret_cast<int*>(bb + b_kb + b_ub);
  double2* dg1 = reinterpret_cast<double2*>(bb + b_kb + b_ub + b_nb);
  double2* dcached = reinterpret_cast<double2*>(bb + b_kb + b_ub + b_nb + b_g1);
  uint8_t* dAimg = split ? reinterpret_cast<uint8_t*>(bb + b_kb + b_ub + b_nb + 2 * b_g1) : nullptr;
  uint8_t* dBimg = split ? dAimg + b_A : nullptr;
  float2* dg3 = split ? reinterpret_cast<float2*>(dBimg + b_B) : nullptr;
  int* dnball = reinterpret_cast<int*>(bb + b_kb + b_ub + b_nb + 2 * b_g1 + b_g3);   // (nk1) active bands
  int* dactik = dnball + b_k1 / sizeof(int);                                        // mesh index of active k1
  cudaStream_t st = ctx->stream;
  cudaEvent_t ev0, ev1;
  PHX_CUDA(ctx, cudaEventCreate(&ev0));
  PHX_CUDA(ctx, cudaEventCreate(&ev1));
  PHX_CUDA(ctx, cudaEventRecord(ev0, st));
  int launches = 0;
  PHX_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
  el_window_kernel<<<(nk + 255) / 256, 256, 0, st>>>(el->d_E, nk, nw, p->chemical_potential, p->window, dlo, dhi);
  ++launches;
  PHX_CUDA(ctx, cudaGetLastError());
  if (nk1 > 0) PHX_CUDA(ctx, cudaMemcpyAsync(dk1, p->k1_list, sizeof(int) * nk1, cudaMemcpyHostToDevice, st));
  PHX_CUDA(ctx, cudaMemsetAsync(dout, 0, sizeof(double) * (size_t)nT * std::max(1, nk1) * nw, st));
  // active-band counts of the k1 list: the host needs them to lay out the batches
  std::vector<int> nb1all(std::max(1, nk1), 0);
  if (nk1 > 0) {
    el_k1_bands_kernel<<<(nk1 + 255) / 256, 256, 0, st>>>(dk1, nk1, dlo, dhi, dnball);
    ++launches;
    PHX_CUDA(ctx, cudaGetLastError());
    PHX_CUDA(ctx, cudaMemcpyAsync(nb1all.data(), dnball, sizeof(int) * nk1, cudaMemcpyDeviceToHost, st));
    PHX_CUDA(ctx, cudaStreamSynchronize(st));
  }
  // the k1 with active states, in list order, taken kB1 at a time
  std::vector<int> act, actik;
  for (int i = 0; i < nk1; ++i)
    if (nb1all[i] > 0) {
      act.push_back(i);
      actik.push_back(p->k1_list[i]);
    }
  const int nact = (int)act.size();
  if (nact > 0) PHX_CUDA(ctx, cudaMemcpyAsync(dactik, actik.data(), sizeof(int) * nact, cudaMemcpyHostToDevice, st));
  ElArgs A;
  A.nw = nw;
  A.nph = nph;
  A.nRp = e->nRp;
  A.Rp = e->d_Rp;
  A.degP = e->d_degP;
  for (int i = 0; i < 3; ++i) {
    A.kmesh[i] = el->mesh[i];
    A.qmesh[i] = ph->mesh[i];
  }
  A.Ek = el->d_E;
  A.Uk = reinterpret_cast<const double2*>(el->d_U);
  A.vk = el->d_vg;
  A.kcart = el->d_q;
  A.lo = dlo;
  A.hi = dhi;
  A.Eq = ph->d_E;
  A.evq = reinterpret_cast<const double2*>(ph->d_U);
  A.nk1 = nk1;
  A.nT = nT;
  for (int t = 0; t < pairc::kMaxT; ++t) A.temps[t] = t < nT ? p->temperatures[t] : 0.0;
  A.mu = p->chemical_potential;
  A.smearing = p->smearing;
  A.sigma = p->sigma;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A.qT[i * 3 + j] = el->recip[i * 3 + j] / el->mesh[i];
  A.norm = p->norm;
  A.out = dout;
  A.g3in = nullptr;
  A.g3ld = 0;
  if (split) {
    PHX_ARG(ctx, kB1 <= phx_el_split_max_batch(), "phx_el_linewidths: k1 batch larger than the split GEMM's");
    PHX_TRY(phx_el_split_phases(ctx, ph->nq, ph->d_q, e->nRp, e->d_Rp, e->d_degP, dAimg));
    ++launches;
  }
  size_t soff[13];
  const size_t smem = pair_smem_layout(split ? 0 : e->nRp, nph, nw, soff);
  PHX_ARG(ctx, smem <= 227 * 1024, "phx_el_linewidths: too many phonon Bravais vectors");
  constexpr int ad = PHX_SMEAR_ADAPTIVE, ga = PHX_SMEAR_GAUSSIAN;
  const cudaFuncAttribute fa = cudaFuncAttributeMaxDynamicSharedMemorySize;
  PHX_CUDA(ctx, cudaFuncSetAttribute(el_pair_kernel<false, ad>, fa, (int)smem));
  PHX_CUDA(ctx, cudaFuncSetAttribute(el_pair_kernel<false, ga>, fa, (int)smem));
  PHX_CUDA(ctx, cudaFuncSetAttribute(el_pair_kernel<true, ad>, fa, (int)smem));
  PHX_CUDA(ctx, cudaFuncSetAttribute(el_pair_kernel<true, ga>, fa, (int)smem));
  const int nq = ph->nq;
  const int qblocks = (nq + kQT - 1) / kQT;
  const size_t per = N;
  long long pairs = 0;
  for (int b0 = 0; b0 < nact; b0 += kB1) {
    const int nb = std::min(kB1, nact - b0);
    std::vector<int> rows(act.begin() + b0, act.begin() + b0 + nb);
    std::vector<int> nbb(kB1, 0);
    for (int j = 0; j < nb; ++j) nbb[j] = nb1all[rows[j]];
    // k1 coordinates, band counts and U1 of the batch, gathered on the device
    el_batch_gather_kernel<<<1, 256, 0, st>>>(dactik + b0, nb, dlo, dhi, el->d_q,
                                              reinterpret_cast<const double2*>(el->d_U), nw, dkb, dub, dnb);
    ++launches;
    PHX_CUDA(ctx, cudaGetLastError());
    PHX_TRY(elph_cache_batch(e, nb, dkb, dub, dnb, dg1, dcached, split));
    launches += split ? 3 : 2;
    // the Rp transform of all q and the batch's k1 on the tensor cores (BF16 x3, FP32 accumulation)
    int g3ld = 0;
    std::vector<int> xoff(kB1, 0);
    if (split) {
      PHX_TRY(phx_el_split_g3_batch(ctx, dAimg, dBimg, dcached, per, e->nRp, nph, nw, nq, nb, nbb.data(), dg3,
                                    &g3ld, xoff.data()));
      launches += 2;
    }
    // one launch for the batch: blockIdx.y = k1 of the batch
    A.cached = dcached;
    A.cper = per;
    for (int j = 0; j < nb; ++j) {
      A.ik1s[j] = p->k1_list[rows[j]];
      A.i1s[j] = rows[j];
      A.g3offs[j] = (long long)xoff[j] * g3ld;
    }
    if (split) {
      A.g3in = dg3;
      A.g3ld = g3ld;
    }
    const dim3 grid(qblocks, nb);
    const bool adaptive = A.smearing == PHX_SMEAR_ADAPTIVE;
    if (A.g3in) {
      if (adaptive) el_pair_kernel<true, ad><<<grid, kPairThreads, smem, st>>>(A);
      else el_pair_kernel<true, ga><<<grid, kPairThreads, smem, st>>>(A);
    } else {
      if (adaptive) el_pair_kernel<false, ad><<<grid, kPairThreads, smem, st>>>(A);
      else el_pair_kernel<false, ga><<<grid, kPairThreads, smem, st>>>(A);
    }
    ++launches;
    pairs += (long long)nq * nb;
    PHX_CUDA(ctx, cudaGetLastError());
  }
  if (nk1 > 0) {
    el_degavg_kernel<<<(nk1 + 127) / 128, 128, 0, st>>>(dout, nk1, nw, dk1, el->d_E, dlo, dhi);
    ++launches;
    PHX_CUDA(ctx, cudaGetLastError());
  }
  PHX_CUDA(ctx, cudaEventRecord(ev1, st));
  PHX_CUDA(ctx, cudaMemcpyAsync(out, dout, sizeof(double) * (size_t)nT * nk1 * nw, cudaMemcpyDeviceToHost, st));
  int kst = 0;
  PHX_CUDA(ctx, cudaMemcpyAsync(&kst, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  PHX_CUDA(ctx, cudaStreamSynchronize(st));
  if (kst) {
    cudaMemset(ctx->d_status, 0, sizeof(int));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    phx_set_error(ctx, PHX_ERR_CUDA, "el-ph tensor-core GEMM gave up waiting on its MMA barrier");
    return PHX_ERR_CUDA;
  }
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    stats->ms_total = ms;
    stats->ms_vertex = ms;
    stats->pairs = pairs;
    stats->kernel_launches = launches;
    stats->pair_launches = 0;
    stats->ms_pair = 0.0;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  return PHX_OK;
}

extern "C" int phx_elph_set_precision(phx_elph* e, int precision) {
  PHX_ARG(e ? e->ctx : nullptr, e, "phx_elph_set_precision: null handle");
  PHX_ARG(e->ctx, precision == PHX_PREC_FP64 || precision == PHX_PREC_SPLIT_BF16,
          "phx_elph_set_precision: PHX_PREC_FP64 or PHX_PREC_SPLIT_BF16");
  e->precision = precision;
  return PHX_OK;
}
