// Split-precision (BF16 x3) tensor-core path of the fused 3-phonon builder.
//
// The R3 transform of the vertex (interaction_3ph.cpp:276-289, "tmploop"),
//   T(q1; a,b2,c) = sum_r3 e^{-i q1.R3} Dp(q2)[r3][a][b2][c],
// is a complex GEMM with M = q1 (128 per CTA), K = r3, N = (a,b2,c).  It runs
// on the 5th-generation tensor cores as a real GEMM on [Re | Im] extended
// operands, each operand split as x = hi + lo in BF16 and accumulated as
// hi*hi + hi*lo + lo*hi in FP32 in tensor memory (TMEM).
//
// Per CTA: 4 epilogue warps (one per TMEM lane quarter; thread = q1), one
// producer warp (bulk async copies of pre-laid-out B images), one MMA warp
// (single thread issues tcgen05.mma).  N is processed in three parts of two
// b2 values (144 FP32 columns, an MMA N that is a multiple of 16) that rotate
// through three TMEM regions, so the MMA of one part overlaps the CUDA-core
// epilogue of the others.  The
// epilogue contracts with e1 and e3 in FP32, symmetrises over degenerate
// blocks, and evaluates the delta functions and Bose factors of the + and -
// processes with energy differences formed in FP64, accumulating linewidths
// in FP64.  Triplets whose delta is zero by the reference's own cut-offs are
// skipped before any arithmetic (exactly zero contributions).
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>
#include <vector>

#include "pair_common.cuh"
#include "tc.cuh"

using namespace pairc;

namespace {

constexpr int kM = 128;            // q1 rows per CTA = TMEM lanes
constexpr int kKC = 32;            // K elements per B chunk (2 MMA K-steps)
constexpr int kParts = 3;          // N split into 3 parts of 2 b2 each
constexpr int kB2PerPart = 2;
constexpr int kNH = 144;           // N columns per part: 2 b2 x 36 (a,c) x {re,im}
constexpr int kStages = 2;
constexpr int kRegion = 160;       // TMEM columns per accumulator region (>= kNH)
constexpr int kTmemCols = 512;
constexpr int kEpiWarps = 8;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kPartBytes = kNH * kKC * 2;    // one of hi / lo: 9216 B
constexpr uint32_t kStageBytes = 2 * kPartBytes;  // hi + lo: 18432 B
constexpr uint32_t kBSbo = (kKC / 8) * 128;       // 512 B between 8-row groups

struct TcArgs {
  MeshArgs m;
  int Kp;                      // padded real K (2*nr3 rounded up to 48)
  const uint8_t* Bimg;         // [j][part][kc] x kStageBytes
  const float2* U32;           // (nq, nb, nb) fp32 eigenvectors
  const double* R3;
  int nr3;
  const int* q1_order;         // q1 points in k-space blocks of 4x4x2 (warp coherence)
  int q2_first, q2_count, q2_per_slot;
  double* partial;             // (S, nq, nb, nT)
  int* status;
};

// ---------------------------------------------------------------------------
// B images: Dp (FP64 complex [j][r3][a][b2][c]) -> BF16 hi/lo K-major tiles
// ---------------------------------------------------------------------------
__global__ void convert_b_kernel(const double2* __restrict__ Dp, int nr3, int Kp, int q2_count,
                                 uint8_t* __restrict__ Bimg) {
  const int nkc = Kp / kKC;
  const int j = blockIdx.x;
  const int h = blockIdx.y / nkc, kc = blockIdx.y % nkc;
  if (j >= q2_count) return;
  uint8_t* img = Bimg + ((size_t)(j * kParts + h) * nkc + kc) * kStageBytes;
  const double2* D = Dp + (size_t)j * nr3 * 216;
  for (int e = threadIdx.x; e < kNH * kKC; e += blockDim.x) {
    const int n = e / kKC, kk = e % kKC;
    const int kg = kc * kKC + kk;
    const int ri = n & 1, rest = n >> 1;
    const int bl = rest / 36, a = (rest / 6) % 6, c = rest % 6;
    const int b2 = kB2PerPart * h + bl;
    double v = 0.0;
    if (kg < 2 * nr3) {
      const int part = kg < nr3 ? 0 : 1;
      const int r3 = part ? kg - nr3 : kg;
      const double2 B = D[(size_t)r3 * 216 + a * 36 + b2 * 6 + c];
      v = ri == 0 ? (part == 0 ? B.x : -B.y) : (part == 0 ? B.y : B.x);
    }
    const __nv_bfloat16 hi = __double2bfloat16(v);
    const __nv_bfloat16 lo = __double2bfloat16(v - (double)__bfloat162float(hi));
    const uint32_t off = tc::core_offset(n, kk, kKC, 2);
    *reinterpret_cast<__nv_bfloat16*>(img + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(img + kPartBytes + off) = lo;
  }
}

__global__ void to_fp32_kernel(const double2* __restrict__ U, size_t n, float2* __restrict__ U32) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    U32[i] = make_float2((float)U[i].x, (float)U[i].y);
}

// ---------------------------------------------------------------------------
// epilogue helpers (FP32 contraction, FP64 energies)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sigma_f(const float* qT, float v0, float v1, float v2) {
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float d = qT[3 * i] * v0 + qT[3 * i + 1] * v1 + qT[3 * i + 2] * v2;
    s = fmaf(d, d, s);
  }
  s = sqrtf(s / 6.0f);
  if (s != 0.f && s < (float)phxc::adaptiveCutoff) s = (float)phxc::adaptiveCutoff;
  return s;
}

// delta of one process in FP32 from an FP64 energy difference; 0 when the
// reference's cut-offs make it zero (Gaussian: x > 6; x < -8.5 contributes
// below 1e-31 of the peak and is dropped).
__device__ __forceinline__ float delta_f(int smearing, float sigma, double de, bool vzero) {
  const float e = (float)de;
  if (smearing == PHX_SMEAR_GAUSSIAN) {
    const float x = e / sigma;
    if (x > 6.f || x < -8.5f) return 0.f;
    return __expf(-x * x) / ((float)phxc::sqrtPi * sigma);
  }
  if (vzero && de == 0.0) return 1.f;
  if (sigma == 0.f) return 0.f;
  if (fabsf(e) > 2.f * sigma) return 0.f;
  const float x = e / sigma;
  return __expf(-x * x) / ((float)phxc::sqrtPi * sigma * (float)phxc::erf2);
}

// ---------------------------------------------------------------------------
// the fused pair kernel
// ---------------------------------------------------------------------------
// Warp roles (320 threads): warps 0-7 epilogue (TMEM lane quarter = warp & 3,
// b2 parity = warp >> 2), warp 8 producer, warp 9 MMA issuer.
// Shared-memory plan (bytes), Kp = 96:
//   A hi/lo 48 K | B stages 2 x 18 K | e1 36 K | e3 36 K | E(q1), E(q3) 12 K |
//   v(q3) 9 K | Bose(q3), Bose(q1) 24 K | per-warp q2 data 3.4 K | barriers
struct U2 {             // uniform data of one b2 at q2 and at -q2
  double e2, e2m;
  float v2[3], v2m[3];
  float n2[kMaxT], n2m[kMaxT];
};

struct Smem3 {
  const float2* E1v;   // e1 [36][128]
  const float2* E3v;   // e3 [36][128]
  const double* En1;   // [6][128]
  const double* En3;   // [6][128]
  const float* V3;     // [18][128]
  const float* N3;     // [kMaxT*6][128]
  const float* N1;     // [kMaxT*6][128]
};

// OR the 6x6 mask (bit b1*6+b3) over the degenerate blocks of b1 and b3
// Degenerate blocks of 6 sorted energies packed as 3-bit block starts
// (forward scan of scattering.cpp:1218-1230).
constexpr unsigned kIdentityBlocks = 0u | (1u << 3) | (2u << 6) | (3u << 9) | (4u << 12) | (5u << 15);
__device__ __forceinline__ unsigned pack_blocks(const double* e) {
  unsigned p = 0;
  int start = 0;
#pragma unroll
  for (int b = 0; b < 6; ++b) {
    if (b > start && !(fabs(e[start] - e[b]) < phxc::degThreshold)) start = b;
    if (b == 0) start = 0;
    p |= (unsigned)start << (3 * b);
  }
  return p;
}
__device__ __forceinline__ int blk_start(unsigned p, int b) { return (p >> (3 * b)) & 7; }
__device__ __forceinline__ int blk_size(unsigned p, int b) {
  const int s = blk_start(p, b);
  int n = 0;
#pragma unroll
  for (int k = 0; k < 6; ++k) n += blk_start(p, k) == s;
  return n;
}

// OR the 6x6 mask (bit b1*6+b3) over the degenerate blocks of b1 and b3
__device__ __forceinline__ unsigned long long expand_blocks(unsigned long long m, unsigned gp1,
                                                            unsigned gp3) {
  unsigned long long rows[6];
#pragma unroll
  for (int b1 = 0; b1 < 6; ++b1) rows[b1] = (m >> (6 * b1)) & 63ull;
  unsigned long long out = 0;
#pragma unroll
  for (int b1 = 0; b1 < 6; ++b1) {
    unsigned long long row = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) row |= (blk_start(gp1, k) == blk_start(gp1, b1)) ? rows[k] : 0ull;
    unsigned long long e = 0;
#pragma unroll
    for (int b3 = 0; b3 < 6; ++b3) {
      unsigned long long blk = 0;
#pragma unroll
      for (int k = 0; k < 6; ++k) blk |= (blk_start(gp3, k) == blk_start(gp3, b3)) ? (1ull << k) : 0ull;
      e |= ((row >> b3) & 1ull) ? blk : 0ull;
    }
    out |= e << (6 * b1);
  }
  return out;
}

// Rate factors of one branch triplet (b1,b2,b3) for all temperatures: the
// "+" process of (q1,q2) and the two "-" processes of (q1,-q2), exactly as
// ph_scattering.cpp:338-380 and :466-518 (cut-offs, deltas, Bose factors),
// times 0.5 (the linewidth convention of :433,:574); multiply by |V|^2.
__device__ __forceinline__ void rate_factors(const MeshArgs& M, double en1, const float* n1,
                                             const U2& x, double en3, const float* n3, float sp,
                                             float sm, bool vzp, bool vzm, float* f) {
#pragma unroll
  for (int c = 0; c < kMaxT; ++c) f[c] = 0.f;
  if (en1 < phxc::phExcludeCutoff || en3 < phxc::phEnergyCutoff) return;
  const bool ok2 = x.e2 >= phxc::phExcludeCutoff;
  const bool ok2m = x.e2m >= phxc::phExcludeCutoff;
  const float dplus = ok2 ? delta_f(M.smearing, sp, en1 + x.e2 - en3, vzp) : 0.f;
  float d1 = 0.f, d2 = 0.f;
  if (ok2m) {
    d1 = delta_f(M.smearing, sm, en1 + en3 - x.e2m, vzm);
    d2 = delta_f(M.smearing, sm, x.e2m + en3 - en1, vzm);
  }
  if (dplus <= 0.f && d1 <= 0.f && d2 <= 0.f) return;
  d1 = fmaxf(d1, 0.f);
  d2 = fmaxf(d2, 0.f);
  const float pre = (float)(phxc::pi * 0.25 * 0.5) * (float)M.norm;
  const float fp = dplus > 0.f ? pre * dplus / (float)(en1 * x.e2 * en3) : 0.f;
  const float fm = (d1 > 0.f || d2 > 0.f) ? pre / (float)(en1 * x.e2m * en3) : 0.f;
#pragma unroll
  for (int c = 0; c < kMaxT; ++c) {
    if (c >= M.nT) break;
    float r = 0.f;
    if (fp > 0.f) r += fp * n1[c] * x.n2[c] * (n3[c] + 1.f);
    if (fm > 0.f) r += fm * (n3[c] * n1[c] * (x.n2m[c] + 1.f) * d1 + x.n2m[c] * n3[c] * (n1[c] + 1.f) * d2);
    f[c] = r;
  }
}

__device__ __forceinline__ void sigmas(const MeshArgs& M, const float* qT, const U2& x,
                                       const float* V3, int m, int b3, float& sp, float& sm,
                                       bool& vzp, bool& vzm) {
  sp = sm = (float)M.sigma;
  vzp = vzm = false;
  if (M.smearing != PHX_SMEAR_ADAPTIVE) return;
  const float v30 = V3[(b3 * 3) * 128 + m], v31 = V3[(b3 * 3 + 1) * 128 + m],
              v32 = V3[(b3 * 3 + 2) * 128 + m];
  const float dp0 = x.v2[0] - v30, dp1 = x.v2[1] - v31, dp2 = x.v2[2] - v32;
  const float dm0 = x.v2m[0] - v30, dm1 = x.v2m[1] - v31, dm2 = x.v2m[2] - v32;
  vzp = dp0 == 0.f && dp1 == 0.f && dp2 == 0.f;
  vzm = dm0 == 0.f && dm1 == 0.f && dm2 == 0.f;
  sp = sigma_f(qT, dp0, dp1, dp2);
  sm = sigma_f(qT, dm0, dm1, dm2);
}

// Block-averaged rate factors G(b1, block(b2), block(b3)) used when any of
// the three points has degenerate bands: by the symmetry of the block
// average, sum S(W) F = sum W S(F), so |V|^2 never has to be symmetrised.
__device__ __forceinline__ void rate_block(const MeshArgs& M, const float* qT, const Smem3& S,
                                        const U2* u2, int m, int b1, int b2s, int b2n, int b3s,
                                        int b3n, float* g) {
#pragma unroll
  for (int c = 0; c < kMaxT; ++c) g[c] = 0.f;
  const double en1 = S.En1[b1 * 128 + m];
  float n1[kMaxT];
#pragma unroll
  for (int c = 0; c < kMaxT; ++c) n1[c] = S.N1[(c * 6 + b1) * 128 + m];
  for (int bb = b2s; bb < b2s + b2n; ++bb) {
    const U2 x = u2[bb];
    for (int b3 = b3s; b3 < b3s + b3n; ++b3) {
      float sp, sm;
      bool vzp, vzm;
      sigmas(M, qT, x, S.V3, m, b3, sp, sm, vzp, vzm);
      float n3[kMaxT];
#pragma unroll
      for (int c = 0; c < kMaxT; ++c) n3[c] = S.N3[(c * 6 + b3) * 128 + m];
      float f[kMaxT];
      rate_factors(M, en1, n1, x, S.En3[b3 * 128 + m], n3, sp, sm, vzp, vzm, f);
#pragma unroll
      for (int c = 0; c < kMaxT; ++c) g[c] += f[c];
    }
  }
  const float inv = 1.f / (float)(b2n * b3n);
#pragma unroll
  for (int c = 0; c < kMaxT; ++c) g[c] *= inv;
}

// Liveness of (b1, b2, b3) for all b1, b3 at one b2 (bit b1*6+b3), in FP32
// with a margin for rounding; the rate stage re-applies the exact tests.
__device__ __forceinline__ unsigned long long live_mask(const MeshArgs& M, const float* qT,
                                                       const Smem3& S, const U2& x, int m,
                                                       const float* E1f, unsigned ok1) {
  const bool ok2 = x.e2 >= phxc::phExcludeCutoff;
  const bool ok2m = x.e2m >= phxc::phExcludeCutoff;
  if (!ok2 && !ok2m) return 0ull;
  const float tol = 4.0e-9f;  // bound on the FP32 error of an energy difference (Ry)
  const float e2f = (float)x.e2, e2mf = (float)x.e2m;
  unsigned long long msk = 0;
#pragma unroll 1
  for (int b3 = 0; b3 < 6; ++b3) {
    const double en3 = S.En3[b3 * 128 + m];
    if (!(en3 >= phxc::phEnergyCutoff)) continue;
    const float e3f = (float)en3;
    float sp, sm;
    bool vzp, vzm;
    sigmas(M, qT, x, S.V3, m, b3, sp, sm, vzp, vzm);
    float hip, lop, him, lom;
    if (M.smearing == PHX_SMEAR_ADAPTIVE) {
      hip = 2.f * sp + tol;
      lop = -hip;
      him = 2.f * sm + tol;
      lom = -him;
    } else {
      hip = 6.f * sp + tol;
      lop = -8.5f * sp - tol;
      him = 6.f * sm + tol;
      lom = -8.5f * sm - tol;
    }
    if (!ok2) { hip = -1.f; lop = 1.f; }
    if (!ok2m) { him = -1.f; lom = 1.f; }
    const float cp = e2f - e3f, cm1 = e3f - e2mf, cm2 = e2mf + e3f;
    unsigned long long col = 0;
#pragma unroll
    for (int b1 = 0; b1 < 6; ++b1) {
      const float dp = E1f[b1] + cp, d1 = E1f[b1] + cm1, d2 = cm2 - E1f[b1];
      const bool live = (dp <= hip && dp >= lop) || (d1 <= him && d1 >= lom) || (d2 <= him && d2 >= lom);
      col |= (live && ((ok1 >> b1) & 1u)) ? (1ull << (b1 * 6)) : 0ull;
    }
    msk |= col << b3;
  }
  return msk;
}

__global__ void __launch_bounds__(kThreads, 1) pair_tc_kernel(TcArgs P) {
  const MeshArgs& M = P.m;
  extern __shared__ __align__(1024) uint8_t smem[];
  const int Kp = P.Kp, nkc = Kp / kKC;
  const uint32_t aPart = (uint32_t)kM * Kp * 2;
  uint8_t* sA = smem;                                                   // [hi | lo]
  uint8_t* sB = sA + 2 * aPart;                                         // stages
  float2* sE1 = reinterpret_cast<float2*>(sB + kStages * kStageBytes);  // [36][128]
  float2* sE3 = sE1 + 36 * kM;                                          // [36][128]
  double* sEn1 = reinterpret_cast<double*>(sE3 + 36 * kM);              // [6][128]
  double* sEn3 = sEn1 + 6 * kM;                                         // [6][128]
  float* sV3 = reinterpret_cast<float*>(sEn3 + 6 * kM);                 // [18][128]
  float* sN3 = sV3 + 18 * kM;                                           // [kMaxT*6][128]
  float* sN1 = sN3 + kMaxT * 6 * kM;                                    // [kMaxT*6][128]
  U2* sU2 = reinterpret_cast<U2*>(sN1 + kMaxT * 6 * kM);               // [8 warps][6]
  float* sQT = reinterpret_cast<float*>(sU2 + kEpiWarps * 6);           // [9] adaptive qTensor
  uint64_t* bars = reinterpret_cast<uint64_t*>(sQT + 10);
  uint64_t* full = bars;
  uint64_t* empty = bars + kStages;
  uint64_t* accf = bars + 2 * kStages;
  uint64_t* acce = accf + kParts;
  uint64_t* done = acce + kParts;
  uint64_t* stg = done + 1;        // [4] q3 data staged by both parities of a quarter
  uint64_t* rel = stg + 4;         // [4] q3 data released by both parities
  uint32_t* tslot = reinterpret_cast<uint32_t*>(rel + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nq = M.nq, n0 = M.n0, n1 = M.n1, n2 = M.n2, nT = M.nT;
  const int tile0 = blockIdx.x * kM;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int r = 0; r < kParts; ++r) {
      tc::mbar_init(&accf[r], 1);
      tc::mbar_init(&acce[r], kEpiWarps);
    }
    tc::mbar_init(done, 1);
    for (int q = 0; q < 4; ++q) {
      tc::mbar_init(&stg[q], 64);
      tc::mbar_init(&rel[q], 64);
    }
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (tid < 9) sQT[tid] = (float)M.qT[tid];
  if (warp == 0) {
    tc::tmem_alloc(tslot, kTmemCols);
    tc::tmem_relinquish();
  }
  // A operand: [cos(theta) | sin(theta) | 0] with theta = -q1.R3, split hi/lo
  for (int e = tid; e < kM * Kp; e += kThreads) {
    const int mm = e / Kp, k = e % Kp;
    const int q = P.q1_order[min(tile0 + mm, nq - 1)];
    double v = 0.0;
    if (k < 2 * P.nr3) {
      const int r = k < P.nr3 ? k : k - P.nr3;
      const double* qc = M.qcart + 3 * q;
      double sn, cs;
      sincos(-(qc[0] * P.R3[3 * r] + qc[1] * P.R3[3 * r + 1] + qc[2] * P.R3[3 * r + 2]), &sn, &cs);
      v = k < P.nr3 ? cs : sn;
    }
    const __nv_bfloat16 hi = __double2bfloat16(v);
    const __nv_bfloat16 lo = __double2bfloat16(v - (double)__bfloat162float(hi));
    const uint32_t off = tc::core_offset(mm, k, Kp, 2);
    *reinterpret_cast<__nv_bfloat16*>(sA + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(sA + aPart + off) = lo;
  }
  for (int e = tid; e < 36 * kM; e += kThreads) {
    const int el = e / kM, mm = e % kM;
    const int q = P.q1_order[min(tile0 + mm, nq - 1)];
    sE1[e] = P.U32[(size_t)q * 36 + el];
  }
  for (int e = tid; e < kMaxT * 6 * kM; e += kThreads) {
    const int f = e / kM, mm = e % kM, c = f / 6, b = f % 6;
    const int q = P.q1_order[min(tile0 + mm, nq - 1)];
    sN1[e] = c < nT ? (float)M.bose[((size_t)c * nq + q) * 6 + b] : 0.f;
  }
  for (int e = tid; e < 6 * kM; e += kThreads) {
    const int b = e / kM, mm = e % kM;
    const int q = P.q1_order[min(tile0 + mm, nq - 1)];
    sEn1[e] = M.E[(size_t)q * 6 + b];
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;

  const int jbeg = blockIdx.y * P.q2_per_slot;
  const int jend = min(P.q2_count, jbeg + P.q2_per_slot);
  const int nunits = kParts * max(0, jend - jbeg);

  if (warp == kEpiWarps) {
    // ---------------- producer ----------------
    if (lane == 0) {
      int it = 0;
      for (int u = 0; u < nunits && !*abort_flag; ++u) {
        const int j = jbeg + u / kParts, h = u % kParts;
        for (int kc = 0; kc < nkc; ++kc, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (!tc::mbar_wait_sleep(&empty[s], ph ^ 1, P.status, 1)) { *abort_flag = 1; break; }
          tc::mbar_arrive_expect_tx(&full[s], kStageBytes);
          tc::bulk_g2s(sB + s * kStageBytes, P.Bimg + ((size_t)(j * kParts + h) * nkc + kc) * kStageBytes,
                       kStageBytes, &full[s]);
        }
      }
    }
  } else if (warp == kEpiWarps + 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_bf16_f32(kM, kNH);
      const uint32_t sbA = (uint32_t)(Kp / 8) * 128;
      const uint32_t aHi = tc::smem_u32(sA), aLo = tc::smem_u32(sA + aPart);
      int it = 0;
      for (int u = 0; u < nunits && !*abort_flag; ++u) {
        const int r = u % kParts, k = u / kParts;
        if (!tc::mbar_wait_sleep(&acce[r], (k & 1) ^ 1, P.status, 2)) { *abort_flag = 1; break; }
        tc::tc_fence_after();
        const uint32_t d = tmem + r * kRegion;
        bool ok = true;
        for (int kc = 0; kc < nkc; ++kc, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (!tc::mbar_wait_sleep(&full[s], ph, P.status, 4)) { ok = false; break; }
          tc::tc_fence_after();
          const uint32_t bHi = tc::smem_u32(sB + s * kStageBytes);
          const uint32_t bLo = bHi + kPartBytes;
#pragma unroll
          for (int ks = 0; ks < kKC / 16; ++ks) {
            const int kg = kc * (kKC / 16) + ks;
            const uint64_t dAh = tc::smem_desc(aHi + kg * 256, 128, sbA);
            const uint64_t dAl = tc::smem_desc(aLo + kg * 256, 128, sbA);
            const uint64_t dBh = tc::smem_desc(bHi + ks * 256, 128, kBSbo);
            const uint64_t dBl = tc::smem_desc(bLo + ks * 256, 128, kBSbo);
            tc::mma_bf16(d, dAh, dBh, idesc, (kc | ks) != 0);
            tc::mma_bf16(d, dAh, dBl, idesc, 1);
            tc::mma_bf16(d, dAl, dBh, idesc, 1);
          }
          tc::mma_commit(&empty[s]);
        }
        if (!ok) { *abort_flag = 1; break; }
        tc::mma_commit(&accf[r]);
      }
      // drain: wait until every issued MMA has completed
      tc::mma_commit(done);
      tc::mbar_wait_sleep(done, 0, P.status, 8);
    }
  } else {
    // ---------------- epilogue: thread = (q1, b2 parity) ----------------
    const int qd = warp & 3, par = warp >> 2;
    const int m = qd * 32 + lane;
    const bool valid = tile0 + m < nq;
    const int q1c = P.q1_order[min(tile0 + m, nq - 1)];
    const unsigned FULL = 0xffffffffu;
    float E1f[6];
    unsigned ok1 = 0;
    unsigned gp1;  // packed block starts of q1 (3 bits per band)
    {
      double e1d[6];
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        e1d[b] = sEn1[b * kM + m];
        E1f[b] = (float)e1d[b];
        ok1 |= (e1d[b] >= phxc::phExcludeCutoff && valid) ? (1u << b) : 0u;
      }
      gp1 = pack_blocks(e1d);
    }
    const bool deg1 = gp1 != kIdentityBlocks;
    const float* qT = sQT;
    double acc[6][kMaxT];
#pragma unroll
    for (int b = 0; b < 6; ++b)
#pragma unroll
      for (int c = 0; c < kMaxT; ++c) acc[b][c] = 0.0;
    unsigned long long need[3];   // own b2 = par + 2j
    unsigned gp2 = kIdentityBlocks, gp3 = kIdentityBlocks;
    float Wd[36];                 // |V|^2 of triplets at degenerate points (deferred)
    unsigned long long dmask = 0;
    bool deg = false;
    U2* u2 = sU2 + warp * 6;
    const uint32_t lane_base = (uint32_t)(qd * 32) << 16;
    for (int u = 0; u < nunits; ++u) {
      const int h = u % kParts, k = u / kParts;
      if (h == 0) {
        // ---- new q2: stage q3 data (shared by both parities of the quarter)
        const int iq2 = P.q2_first + jbeg + k;
        const int iq2m = mesh_neg(iq2, n0, n1, n2);
        const int iq3 = mesh_add(q1c, iq2, n0, n1, n2);
        // both parities must be done with the previous q2's staged data
        if (k > 0 && !tc::mbar_wait_sleep(&rel[qd], (k - 1) & 1, P.status, 32)) { *abort_flag = 1; break; }
        if (par == 0) {
          const float2* src = P.U32 + (size_t)iq3 * 36;
#pragma unroll 6
          for (int e = 0; e < 36; ++e) sE3[e * kM + m] = src[e];
#pragma unroll
          for (int b = 0; b < 6; ++b) sEn3[b * kM + m] = M.E[(size_t)iq3 * 6 + b];
        } else {
          if (M.smearing == PHX_SMEAR_ADAPTIVE) {
#pragma unroll 6
            for (int i = 0; i < 18; ++i) sV3[i * kM + m] = (float)M.vg[(size_t)iq3 * 18 + i];
          }
          for (int c = 0; c < nT; ++c) {
#pragma unroll
            for (int b = 0; b < 6; ++b) sN3[(c * 6 + b) * kM + m] = (float)M.bose[((size_t)c * nq + iq3) * 6 + b];
          }
        }
        if (lane < 6) {
          U2 x;
          x.e2 = M.E[(size_t)iq2 * 6 + lane];
          x.e2m = M.E[(size_t)iq2m * 6 + lane];
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            x.v2[i] = M.smearing == PHX_SMEAR_ADAPTIVE ? (float)M.vg[((size_t)iq2 * 6 + lane) * 3 + i] : 0.f;
            x.v2m[i] = M.smearing == PHX_SMEAR_ADAPTIVE ? (float)M.vg[((size_t)iq2m * 6 + lane) * 3 + i] : 0.f;
          }
#pragma unroll
          for (int c = 0; c < kMaxT; ++c) {
            x.n2[c] = c < nT ? (float)M.bose[((size_t)c * nq + iq2) * 6 + lane] : 0.f;
            x.n2m[c] = c < nT ? (float)M.bose[((size_t)c * nq + iq2m) * 6 + lane] : 0.f;
          }
          u2[lane] = x;
        }
        tc::mbar_arrive(&stg[qd]);  // staged data visible to both parities
        if (!tc::mbar_wait(&stg[qd], k & 1, P.status, 64)) { *abort_flag = 1; break; }
        {
          double e2d[6], e3d[6];
#pragma unroll
          for (int b = 0; b < 6; ++b) {
            e2d[b] = u2[b].e2;
            e3d[b] = sEn3[b * kM + m];
          }
          gp2 = pack_blocks(e2d);
          gp3 = pack_blocks(e3d);
        }
        const bool deg2 = gp2 != kIdentityBlocks, deg3 = gp3 != kIdentityBlocks;
        deg = deg1 || deg2 || deg3;
        // liveness masks of the own b2 values, expanded over degenerate blocks
#pragma unroll
        for (int j = 0; j < 3; ++j) need[j] = 0ull;
#pragma unroll 1
        for (int bx = 0; bx < 6; ++bx) {
          if (!deg2 && (bx & 1) != par) continue;
          Smem3 S;
          S.En3 = sEn3; S.V3 = sV3;
          const unsigned long long mk = live_mask(M, qT, S, u2[bx], m, E1f, ok1);
#pragma unroll
          for (int j = 0; j < 3; ++j)
            if (blk_start(gp2, bx) == blk_start(gp2, par + 2 * j)) need[j] |= mk;
        }
        if (deg1 || deg3) {
#pragma unroll
          for (int j = 0; j < 3; ++j) need[j] = expand_blocks(need[j], gp1, gp3);
        }
      }
      // ---- this part holds b2 = 2h and 2h+1; this thread takes b2 = 2h + par
      const int b2 = 2 * h + par;
      unsigned long long nb2 = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j)
        if (j == h) nb2 = need[j];
      unsigned rows = 0;
#pragma unroll
      for (int b1 = 0; b1 < 6; ++b1) rows |= ((nb2 >> (6 * b1)) & 63ull) ? (1u << b1) : 0u;
      const unsigned wrows = __reduce_or_sync(FULL, rows);
      if (!tc::mbar_wait_sleep(&accf[h], k & 1, P.status, 16)) { *abort_flag = 1; break; }
      tc::tc_fence_after();
      const uint32_t col0 = tmem + lane_base + h * kRegion + par * 72;
      const U2& x = u2[b2];
#pragma unroll 1
      for (int hb = 0; hb < 2; ++hb) {
        const unsigned hrows = (wrows >> (3 * hb)) & 7u;
        if (!hrows) continue;
        // X(b1,c) = sum_a e1(a,b1) T(a,c) for b1 = 3hb..3hb+2; T read from TMEM one a-row at a time
        float2 X[3][6];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int c = 0; c < 6; ++c) X[i][c] = make_float2(0.f, 0.f);
#pragma unroll
        for (int a = 0; a < 6; ++a) {
          float t[12];
          __syncwarp();
          tc::tmem_ld8(col0 + a * 12, t);
          tc::tmem_ld4(col0 + a * 12 + 8, t + 8);
          tc::tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            if (!((hrows >> i) & 1u)) continue;
            const float2 e = sE1[(a * 6 + 3 * hb + i) * kM + m];
#pragma unroll
            for (int c = 0; c < 6; ++c) cfmaf(X[i][c], e, make_float2(t[2 * c], t[2 * c + 1]));
          }
        }
        // V(b1,b3) = sum_c X(b1,c) conj(e3(c,b3)); rates of the needed triplets
#pragma unroll 1
        for (int b3 = 0; b3 < 6; ++b3) {
          unsigned cols = 0;
#pragma unroll
          for (int i = 0; i < 3; ++i) cols |= ((nb2 >> (6 * (3 * hb + i) + b3)) & 1ull) ? (1u << i) : 0u;
          const unsigned wcols = __reduce_or_sync(FULL, cols);
          if (!wcols) continue;
          float2 ec[6];
#pragma unroll
          for (int c = 0; c < 6; ++c) ec[c] = sE3[(c * 6 + b3) * kM + m];
          float sp, sm;
          bool vzp, vzm;
          sigmas(M, qT, x, sV3, m, b3, sp, sm, vzp, vzm);
          const double en3 = sEn3[b3 * kM + m];
          float n3[kMaxT];
#pragma unroll
          for (int c = 0; c < kMaxT; ++c) n3[c] = sN3[(c * 6 + b3) * kM + m];
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            if (!((wcols >> i) & 1u)) continue;
            float2 v = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 6; ++c) cfmacf(v, X[i][c], ec[c]);
            const float w = fmaf(v.x, v.x, v.y * v.y);
            if (!((cols >> i) & 1u)) continue;
            const int b1 = 3 * hb + i;
            if (!deg) {
              float n1v[kMaxT], f[kMaxT];
#pragma unroll
              for (int c = 0; c < kMaxT; ++c) n1v[c] = sN1[(c * 6 + b1) * kM + m];
              rate_factors(M, sEn1[b1 * kM + m], n1v, x, en3, n3, sp, sm, vzp, vzm, f);
              if (hb == 0) {
#pragma unroll
                for (int c = 0; c < kMaxT; ++c) acc[i][c] += (double)(w * f[c]);
              } else {
#pragma unroll
                for (int c = 0; c < kMaxT; ++c) acc[3 + i][c] += (double)(w * f[c]);
              }
            } else {
              // degenerate points: defer (W is spread over blocks after X is released)
              Wd[b1 * 6 + b3] = w;
              dmask |= 1ull << (b1 * 6 + b3);
            }
          }
        }
      }
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&acce[h]);
      if (dmask) {
        // degenerate points: spread W over the block of b1 with block-averaged
        // rate factors (sum S(W) F = sum W S(F) for the block average S)
        Smem3 S;
        S.E1v = sE1; S.E3v = sE3; S.En1 = sEn1; S.En3 = sEn3; S.V3 = sV3; S.N3 = sN3; S.N1 = sN1;
        const int b2s = blk_start(gp2, b2), b2n = blk_size(gp2, b2);
        while (dmask) {
          const int bit = __ffsll((long long)dmask) - 1;
          dmask &= dmask - 1;
          const int b1 = bit / 6, b3 = bit % 6;
          const float w = Wd[bit];
          const int b3s = blk_start(gp3, b3), b3n = blk_size(gp3, b3);
          const int b1s = blk_start(gp1, b1), b1n = blk_size(gp1, b1);
          for (int bt = b1s; bt < b1s + b1n; ++bt) {
            float g[kMaxT];
            rate_block(M, qT, S, u2, m, bt, b2s, b2n, b3s, b3n, g);
#pragma unroll
            for (int bb = 0; bb < 6; ++bb)
              if (bb == bt) {
#pragma unroll
                for (int c = 0; c < kMaxT; ++c) acc[bb][c] += (double)(w * g[c] / (float)b1n);
              }
          }
        }
      }
      if (h == kParts - 1) tc::mbar_arrive(&rel[qd]);  // done with this q2's staged data
      if (*abort_flag) break;
    }
    // each parity owns its own partial-sum slot (2 slots per CTA row)
    if (valid) {
      double* out = P.partial + ((size_t)(2 * blockIdx.y + par) * nq + q1c) * 6 * nT;
#pragma unroll
      for (int b1 = 0; b1 < 6; ++b1)
#pragma unroll
        for (int c = 0; c < kMaxT; ++c)
          if (c < nT) out[b1 * nT + c] += acc[b1][c];
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// self-test GEMM: one 128 x N tile through the same layouts and split MMAs
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) diag_gemm_kernel(int N, int Kp, const float* __restrict__ A,
                                                           const float* __restrict__ B,
                                                           float* __restrict__ C, int* status) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t aPart = 128u * Kp * 2, bPart = (uint32_t)N * Kp * 2;
  uint8_t* sA = smem;
  uint8_t* sB = sA + 2 * aPart;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + 2 * bPart);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, 256);
    tc::tmem_relinquish();
  }
  for (int e = tid; e < 128 * Kp; e += 128) {
    const int m = e / Kp, k = e % Kp;
    const float v = A[e];
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    const uint32_t off = tc::core_offset(m, k, Kp, 2);
    *reinterpret_cast<__nv_bfloat16*>(sA + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(sA + aPart + off) = lo;
  }
  for (int e = tid; e < N * Kp; e += 128) {
    const int n = e / Kp, k = e % Kp;
    const float v = B[e];
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    const uint32_t off = tc::core_offset(n, k, Kp, 2);
    *reinterpret_cast<__nv_bfloat16*>(sB + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(sB + bPart + off) = lo;
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    const uint32_t idesc = tc::idesc_bf16_f32(128, N);
    const uint32_t sb = (uint32_t)(Kp / 8) * 128;
    const uint32_t aHi = tc::smem_u32(sA), aLo = aHi + aPart;
    const uint32_t bHi = tc::smem_u32(sB), bLo = bHi + bPart;
    for (int kg = 0; kg < Kp / 16; ++kg) {
      tc::mma_bf16(tmem, tc::smem_desc(aHi + kg * 256, 128, sb), tc::smem_desc(bHi + kg * 256, 128, sb),
                   idesc, kg != 0);
      tc::mma_bf16(tmem, tc::smem_desc(aHi + kg * 256, 128, sb), tc::smem_desc(bLo + kg * 256, 128, sb),
                   idesc, 1);
      tc::mma_bf16(tmem, tc::smem_desc(aLo + kg * 256, 128, sb), tc::smem_desc(bHi + kg * 256, 128, sb),
                   idesc, 1);
    }
    tc::mma_commit(bar);
  }
  __syncwarp();
  const bool ok = tc::mbar_wait(bar, 0, status, 1);
  tc::tc_fence_after();
  if (ok) {
    for (int c0 = 0; c0 < N; c0 += 8) {
      float v[8];
      tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
      tc::tmem_wait_ld();
      for (int i = 0; i < 8; ++i) C[(size_t)tid * N + c0 + i] = v[i];
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 256);
  }
}

size_t pair_tc_smem(int Kp) {
  return 2 * (size_t)kM * Kp * 2 + (size_t)kStages * kStageBytes + 2 * 36 * kM * sizeof(float2) +
         12 * kM * sizeof(double) + (18 + 2 * kMaxT * 6) * kM * sizeof(float) +
         kEpiWarps * 6 * sizeof(U2) + 10 * sizeof(float) + (2 * kStages + 2 * kParts + 9) * sizeof(uint64_t) +
         16 + 1024;
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int phx_split_kp(int nr3) { return ((2 * nr3 + kKC - 1) / kKC) * kKC; }

size_t phx_split_bimg_bytes(int chunk, int nr3) {
  return (size_t)chunk * kParts * (phx_split_kp(nr3) / kKC) * kStageBytes;
}

// FP32 eigenvectors and the q1 visiting order (k-space blocks of 4x4x2 so
// that the 32 lanes of a warp hold neighbouring q1 with similar energies).
int phx_split_prepare_bands(phx_ctx* ctx, phx_bands* b) {
  if (!b->d_U32) {
    const size_t n = (size_t)b->nq * b->nb * b->nb;
    PHX_CUDA(ctx, cudaMalloc(&b->d_U32, sizeof(float2) * n));
    to_fp32_kernel<<<1024, 256, 0, ctx->stream>>>(reinterpret_cast<const double2*>(b->d_U), n,
                                                  reinterpret_cast<float2*>(b->d_U32));
    PHX_CUDA(ctx, cudaGetLastError());
  }
  if (!b->d_q1_order) {
    const int n0 = b->mesh[0], n1 = b->mesh[1], n2 = b->mesh[2];
    std::vector<long long> key(b->nq);
    std::vector<int> order(b->nq);
    for (int i = 0; i < b->nq; ++i) {
      const int x = i % n0, y = (i / n0) % n1, z = i / (n0 * n1);
      const long long bz = z / 2, by = y / 4, bx = x / 4;
      const long long nbx = (n0 + 3) / 4, nby = (n1 + 3) / 4;
      key[i] = (((bz * nby + by) * nbx + bx) * 32 + (z % 2) * 16 + (y % 4) * 4 + (x % 4));
      order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return key[a] < key[c]; });
    PHX_CUDA(ctx, cudaMalloc(&b->d_q1_order, sizeof(int) * b->nq));
    PHX_CUDA(ctx, cudaMemcpy(b->d_q1_order, order.data(), sizeof(int) * b->nq, cudaMemcpyHostToDevice));
  }
  return PHX_OK;
}

// One chunk of q2: convert the FP64 Dp images to BF16 hi/lo tiles and run the
// fused tensor-core pair kernel over (q1 tiles) x (q2 slots).
int phx_split_pair_chunk(phx_ctx* ctx, const pairc::MeshArgs& M, const phx_v3* v, const phx_bands* b,
                         const double2* Dp, uint8_t* Bimg, int q2_first, int q2_count, int slots,
                         double* partial, int* launches) {
  const int Kp = phx_split_kp(v->nr3);
  const int nkc = Kp / kKC;
  convert_b_kernel<<<dim3(q2_count, kParts * nkc), 256, 0, ctx->stream>>>(Dp, v->nr3, Kp, q2_count, Bimg);
  PHX_CUDA(ctx, cudaGetLastError());
  TcArgs A;
  A.m = M;
  A.Kp = Kp;
  A.Bimg = Bimg;
  A.U32 = reinterpret_cast<const float2*>(b->d_U32);
  A.R3 = v->d_R3;
  A.nr3 = v->nr3;
  A.q1_order = b->d_q1_order;
  A.q2_first = q2_first;
  A.q2_count = q2_count;
  A.q2_per_slot = (q2_count + slots - 1) / slots;
  A.partial = partial;
  A.status = ctx->d_status;
  const size_t smem = pair_tc_smem(Kp);
  PHX_CUDA(ctx, cudaFuncSetAttribute(pair_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  const int tiles = (M.nq + kM - 1) / kM;
  pair_tc_kernel<<<dim3(tiles, slots), kThreads, smem, ctx->stream>>>(A);
  PHX_CUDA(ctx, cudaGetLastError());
  *launches += 2;
  return PHX_OK;
}

size_t phx_split_smem_bytes(int nr3) { return pair_tc_smem(phx_split_kp(nr3)); }

extern "C" int phx_diag_tc_gemm(phx_ctx* ctx, int N, int Kp, const float* A, const float* B, float* C) {
  PHX_ARG(ctx, ctx && A && B && C, "phx_diag_tc_gemm: bad arguments");
  PHX_ARG(ctx, N >= 16 && N <= 256 && N % 16 == 0 && Kp >= 16 && Kp <= 256 && Kp % 16 == 0,
          "phx_diag_tc_gemm: N in [16,256] and Kp in [16,256], multiples of 16");
  PHX_ARG(ctx, 4 * (128 + (size_t)N) * Kp + 1088 <= 227 * 1024,
          "phx_diag_tc_gemm: tile does not fit in shared memory");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  float *dA = nullptr, *dB = nullptr, *dC = nullptr;
  int rc = PHX_OK;
  cudaError_t e = cudaMalloc(&dA, sizeof(float) * 128 * Kp);
  if (e == cudaSuccess) e = cudaMalloc(&dB, sizeof(float) * N * Kp);
  if (e == cudaSuccess) e = cudaMalloc(&dC, sizeof(float) * 128 * N);
  if (e == cudaSuccess) e = cudaMemcpy(dA, A, sizeof(float) * 128 * Kp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dB, B, sizeof(float) * N * Kp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
  const size_t smem = 2 * 128 * (size_t)Kp * 2 + 2 * (size_t)N * Kp * 2 + 64 + 1024;
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(diag_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    diag_gemm_kernel<<<1, 128, smem, ctx->stream>>>(N, Kp, dA, dB, dC, ctx->d_status);
    e = cudaGetLastError();
  }
  int st = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(C, dC, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_diag_tc_gemm: ") + cudaGetErrorString(e));
    rc = PHX_ERR_CUDA;
  } else if (st) {
    phx_set_error(ctx, PHX_ERR_CUDA, "phx_diag_tc_gemm: MMA completion wait timed out");
    rc = PHX_ERR_CUDA;
  }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dC);
  return rc;
}
