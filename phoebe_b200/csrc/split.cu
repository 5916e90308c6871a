// Split-precision (BF16 x3) tensor-core path of the fused 3-phonon builder.
//
// The R3 transform of the vertex (interaction_3ph.cpp:276-289, "tmploop"),
//   X(q1; a,b2,c) = sum_r3 e^{-i q1.R3} Dp(q2)[r3][a][b2][c],
// is a complex GEMM with M = q1 (128 per CTA), K = r3, N = (a,b2,c).  It runs
// on the 5th-generation tensor cores as a real GEMM on [Re | Im] extended
// operands, each operand split as x = hi + lo in BF16 and accumulated as
// hi*hi + hi*lo + lo*hi in FP32 in tensor memory (TMEM).  N is processed in
// three parts of two b2 values (144 FP32 columns) that live in three fixed
// TMEM regions, so the MMA of one part overlaps the CUDA-core epilogue of the
// others.
//
// Epilogue (12 warps; TMEM lane quarter = warp & 3 = 32 q1 rows, k = warp >> 2):
//  * the three warps of a quarter stage the records of q3 = q1 + q2 for their
//    rows (one 592-byte record per mesh point: FP32 eigenvectors, energies,
//    velocity projections, Bose factors, degenerate blocks);
//  * warp k decides, for b2 = 2k, 2k+1 and every (b1, b3), whether any of the
//    three delta functions of the triplet can be non-zero (FP32 windows with a
//    rounding margin); the masks are shared in shared memory;
//  * warp k handles the rows (b1, b2) with (b1 + b2) % 3 == k: it contracts
//    the rows of X it needs with e1 and e3 in FP32 and queues the live
//    triplets (|V|^2 and indices) in shared memory; 32 queued triplets at a
//    time get their delta functions and Bose factors with every lane busy,
//    and their rates go to FP32 accumulators of the current q2, which are
//    folded into FP64 registers once per q2.
// Degenerate points need no symmetrised |V|^2: with S the block average over
// the degenerate blocks of b1, b2 and b3 (scattering.cpp:1209-1318),
//   Gamma(b1) = sum_{b2,b3} S(W) F = sum_{b1' in blk(b1), b2, b3} W(b1',b2,b3) G(b1,b2,b3) / n1,
// where G is the average of the rate factors F over blk(b2) x blk(b3).  Each
// owner therefore contracts the rows of its b1 block and averages F, and the
// triplets whose delta is zero by the reference's own cut-offs are skipped.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <vector>

#include "pair_common.cuh"
#include "tc.cuh"

using namespace pairc;

namespace {

constexpr int kM = 128;            // q1 rows per CTA = TMEM lanes
constexpr int kKC = 16;            // K elements per B stage (one MMA K-step)
constexpr int kParts = 3;          // N split into 3 parts of 2 b2 each
constexpr int kNH = 144;           // N columns per part: 2 b2 x 36 (a,c) x {re,im}
constexpr int kStages = 2;
constexpr int kRegion = 160;       // TMEM columns per accumulator region (>= kNH)
constexpr int kTmemCols = 512;
constexpr int kEpiWarps = 12;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kPartBytes = kNH * kKC * 2;    // one of hi / lo: 4608 B
constexpr uint32_t kStageBytes = 2 * kPartBytes;  // hi + lo: 9216 B
constexpr uint32_t kBSbo = (kKC / 8) * 128;       // 256 B between 8-row groups

// Per-point record, 37 chunks of 16 bytes:
//   chunks 0-17   e(a, b) (FP32 complex) band-major: element b*6+a, two per
//                 chunk, so band b's six components are chunks 3b .. 3b+2
//   chunks 18+3b  band b: words 0-1 E (FP64), 2-4 P = qT.v (FP32), 5 1/E,
//                 6-9 Bose factors of up to 4 temperatures, 10-11 unused
//   chunk 36      word 0: degenerate blocks of the 6 bands (3 bits each)
constexpr int kRecChunks = 37;
constexpr int kChBand = 18;
constexpr int kChGp = 36;
constexpr int kU2Chunks = kRecChunks - kChBand;   // band blocks + blocks word
// Sizes that depend on the number of temperatures NT:
//  * kAccRow: FP32 rate accumulators of a quarter, one row of 6 b1 x NT per
//    q1, padded to an odd stride so that the rows of a warp fall in distinct
//    banks;
//  * kQueue: live-triplet queue entries per warp (a push round adds at most
//    32 to fewer than 32 queued).
template <int NT>
struct Pcfg {
  static constexpr int kAccRow = 6 * NT + 1;
  static constexpr int kQueue = 64;
};

struct TcArgs {
  MeshArgs m;
  int Kp;                      // padded real K (2*nr3 rounded up to kKC)
  const uint8_t* Bimg;         // [j][part][kc] x kStageBytes
  const uint4* rec;            // (nq, kRecChunks) per-point records
  const double* R3;
  int nr3;
  const int* q1_order;         // q1 points in k-space blocks of 4x4x2 (warp coherence)
  int q2_first, q2_count, q2_per_slot;
  float tol;                   // margin of the FP32 liveness windows (Ry)
  double* partial;             // (S, nq, nb, nT)
  int* status;
  int fp16;                    // operands FP16 hi/lo (B scaled by a power of 2) instead of BF16 hi/lo
  const unsigned* dmax;        // FP16: bits of max |Dp| of the chunk (written by the fold)
  struct EdgeEvent* edges;     // near-cut-off processes, re-decided in FP64 by edge_fix_kernel
  unsigned* edge_count;
  unsigned edge_cap;
  unsigned* edge_peak;         // largest event count of the call's launches
  unsigned* edge_overflow;     // set when this launch's events exceeded edge_cap (none applied)
  int edge_only;               // 1: rates off, only the near-cut-off events (re-run of an overflowed chunk)
  phx_split_matrix mat;        // matrix modes: mat.plus != null
};

// A queued triplet one of whose adaptive deltas sat within 1e-5 of the
// |E| > 2 sigma cut-off: the queue entry and where it was evaluated.
struct EdgeEvent {
  unsigned where;    // tile << 12 | slot << 7 | row
  int iq2;
  uint2 entry;       // the queue entry (|V|^2 / n1, meta)
};

// Power-of-2 scale of the B operand for FP16 hi/lo: max |Dp| * scale in [0.5, 1]
__device__ __forceinline__ float fp16_scale(unsigned maxbits) {
  const float m = __uint_as_float(maxbits);
  if (!(m > 0.f)) return 1.f;
  int e;
  frexpf(m, &e);
  return ldexpf(1.f, -e);
}

// hi/lo split of v into two 16-bit values of the operand format
__device__ __forceinline__ void split16(double v, bool fp16, uint16_t* hi, uint16_t* lo) {
  if (fp16) {
    const __half h = __double2half(v);
    const __half l = __double2half(v - (double)__half2float(h));
    *hi = __half_as_ushort(h);
    *lo = __half_as_ushort(l);
  } else {
    const __nv_bfloat16 h = __double2bfloat16(v);
    const __nv_bfloat16 l = __double2bfloat16(v - (double)__bfloat162float(h));
    *hi = __bfloat16_as_ushort(h);
    *lo = __bfloat16_as_ushort(l);
  }
}

// ---------------------------------------------------------------------------
// degenerate blocks of 6 sorted energies, packed as 3-bit block starts
// (forward scan of scattering.cpp:1218-1230)
// ---------------------------------------------------------------------------
constexpr unsigned kIdentityBlocks = 0u | (1u << 3) | (2u << 6) | (3u << 9) | (4u << 12) | (5u << 15);
__host__ __device__ __forceinline__ unsigned pack_blocks(const double* e) {
  unsigned p = 0;
  int start = 0;
  for (int b = 0; b < 6; ++b) {
    if (b > start && !(fabs(e[start] - e[b]) < phxc::degThreshold)) start = b;
    p |= (unsigned)start << (3 * b);
  }
  return p;
}
__device__ __forceinline__ int blk_start(unsigned p, int b) { return (p >> (3 * b)) & 7; }
// bit mask of the bands in the block of band b
__device__ __forceinline__ unsigned blk_mask(unsigned p, int b) {
  const int s = blk_start(p, b);
  unsigned m = 0;
#pragma unroll
  for (int k = 0; k < 6; ++k) m |= (blk_start(p, k) == s) ? (1u << k) : 0u;
  return m;
}

// ---------------------------------------------------------------------------
// records and B images
// ---------------------------------------------------------------------------
// A velocity projection p is kept as its FP32 value ph and, in FP16, the
// residual (p - ph) relative to |ph| 2^-24 (|r| <= 1): together ~35 bits,
// enough to settle the reference's |E| > 2 sigma cut-off like FP64 does
// when the FP32 comparison is too close to call.
__device__ __forceinline__ uint16_t proj_residual(double p, float ph) {
  if (ph == 0.f) return 0;
  const double r = (p - (double)ph) / fabs((double)ph) * 16777216.0;
  return __half_as_ushort(__double2half(r));
}
__device__ __forceinline__ double proj_fp64(float ph, unsigned r) {
  return (double)ph + (double)__half2float(__ushort_as_half((unsigned short)r)) * fabs((double)ph) * 5.9604644775390625e-8;
}

__global__ void pack_records_kernel(MeshArgs M, uint4* __restrict__ rec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= M.nq) return;
  uint32_t w[kRecChunks * 4];
#pragma unroll 1
  for (int el = 0; el < 36; ++el) {
    const double2 u = M.U[(size_t)q * 36 + el];   // e(a, b), el = a*6 + b
    const int t = (el % 6) * 6 + el / 6;
    w[2 * t] = __float_as_uint((float)u.x);
    w[2 * t + 1] = __float_as_uint((float)u.y);
  }
  double e[6];
#pragma unroll 1
  for (int b = 0; b < 6; ++b) {
    e[b] = M.E[(size_t)q * 6 + b];
    uint32_t* o = w + 4 * (kChBand + 3 * b);
    const unsigned long long eb = (unsigned long long)__double_as_longlong(e[b]);
    o[0] = (uint32_t)eb;
    o[1] = (uint32_t)(eb >> 32);
    uint16_t plo[3];
    for (int i = 0; i < 3; ++i) {
      double p = 0.0;
      if (M.smearing == PHX_SMEAR_ADAPTIVE && M.vg)
        for (int j = 0; j < 3; ++j) p += M.qT[3 * i + j] * M.vg[((size_t)q * 6 + b) * 3 + j];
      const float ph = (float)p;
      o[i < 2 ? 2 + i : 4] = __float_as_uint(ph);
      plo[i] = proj_residual(p, ph);
    }
    o[5] = __float_as_uint(e[b] > 0.0 ? (float)(1.0 / e[b]) : 0.f);
    for (int t = 0; t < kMaxT; ++t)
      o[6 + t] = __float_as_uint(t < M.nT ? (float)M.bose[((size_t)t * M.nq + q) * 6 + b] : 0.f);
    // fingerprint of the FP64 velocity: the reference's adaptive width is zero
    // only when two velocities are equal in FP64, which FP32 projections
    // cannot tell from a tiny non-zero difference (then floored at 1e-4 eV)
    unsigned long long h = 0x9E3779B97F4A7C15ull;
    if (M.smearing == PHX_SMEAR_ADAPTIVE && M.vg)
      for (int j = 0; j < 3; ++j) {
        const double vj = M.vg[((size_t)q * 6 + b) * 3 + j] + 0.0;   // -0 -> +0
        h ^= (unsigned long long)__double_as_longlong(vj);
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 31;
      }
    o[10] = ((uint32_t)(h ^ (h >> 32)) & 0xFFFFu) | ((uint32_t)plo[2] << 16);
    o[11] = (uint32_t)plo[0] | ((uint32_t)plo[1] << 16);
  }
  w[4 * kChGp] = pack_blocks(e);
  w[4 * kChGp + 1] = w[4 * kChGp + 2] = w[4 * kChGp + 3] = 0u;
  uint4* dst = rec + (size_t)q * kRecChunks;
#pragma unroll 1
  for (int c = 0; c < kRecChunks; ++c) dst[c] = make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
}

// Dp (FP64 complex [j][r3][a][b2][c]) -> BF16 (or scaled FP16) hi/lo K-major tiles
__global__ void convert_b_kernel(const double2* __restrict__ Dp, int nr3, int Kp, int q2_count,
                                 uint8_t* __restrict__ Bimg, int fp16, const unsigned* __restrict__ dmax) {
  const int nkc = Kp / kKC;
  const double sc = fp16 ? (double)fp16_scale(*dmax) : 1.0;
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
    const int b2 = 2 * h + bl;
    double v = 0.0;
    if (kg < 2 * nr3) {
      const int part = kg < nr3 ? 0 : 1;
      const int r3 = part ? kg - nr3 : kg;
      const double2 B = D[(size_t)r3 * 216 + a * 36 + b2 * 6 + c];
      v = (ri == 0 ? (part == 0 ? B.x : -B.y) : (part == 0 ? B.y : B.x)) * sc;
    }
    uint16_t hi, lo;
    split16(v, fp16 != 0, &hi, &lo);
    const uint32_t off = tc::core_offset(n, kk, kKC, 2);
    *reinterpret_cast<uint16_t*>(img + off) = hi;
    *reinterpret_cast<uint16_t*>(img + kPartBytes + off) = lo;
  }
}

// ---------------------------------------------------------------------------
// epilogue helpers
// ---------------------------------------------------------------------------
// 16-byte asynchronous global -> shared copy (L2 only) and its completion wait
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct Band {            // one band of one point
  double E;
  float P[3];            // qT.v (adaptive smearing), FP32
  float iE;              // 1/E
  float N[kMaxT];        // Bose factors
  unsigned vf;           // 16-bit fingerprint of the FP64 velocity
};

// c0 points at the band's first chunk, the next two follow at stride st
template <int NT>
__device__ __forceinline__ Band load_band(const uint4* c0, int st) {
  const uint4 a = c0[0], b = c0[st];
  Band x;
  x.E = __hiloint2double((int)a.y, (int)a.x);
  x.P[0] = __uint_as_float(a.z);
  x.P[1] = __uint_as_float(a.w);
  x.P[2] = __uint_as_float(b.x);
  x.iE = __uint_as_float(b.y);
  x.N[0] = __uint_as_float(b.z);
  x.N[1] = __uint_as_float(b.w);
  const uint4 c = c0[2 * st];
  x.N[2] = NT > 2 ? __uint_as_float(c.x) : 0.f;
  x.N[3] = NT > 2 ? __uint_as_float(c.y) : 0.f;
  x.vf = c.z & 0xFFFFu;
  return x;
}

struct Sig {
  float s, inv;   // sigma and 1/sigma
  bool vz;        // velocity difference exactly zero
};

// AdaptiveGaussianDeltaFunction::getSmearing (delta_function.cpp:71-83) from
// the projections P = qT.v: sigma^2 = |P2 - P3|^2 / 6, floored at 1e-4 eV.
// The width is zero only for velocities equal in FP64 (same fingerprint and
// same projections); a difference lost in the FP32 projections is below the
// floor, which is what the FP64 width would be raised to.
__device__ __forceinline__ Sig sigma_ad(const float* P2, const float* P3, unsigned f2, unsigned f3) {
  const float d0 = P2[0] - P3[0], d1 = P2[1] - P3[1], d2 = P2[2] - P3[2];
  float s2 = fmaf(d0, d0, fmaf(d1, d1, d2 * d2)) * (1.f / 6.f);
  Sig g;
  g.vz = f2 == f3 && d0 == 0.f && d1 == 0.f && d2 == 0.f;
  constexpr float kCut = (float)phxc::adaptiveCutoff;
  if (!g.vz && s2 < kCut * kCut) s2 = kCut * kCut;
  const float r = s2 > 0.f ? rsqrtf(s2) : 0.f;
  g.s = s2 * r;
  g.inv = r;
  return g;
}

// |de| > 2 sigma decided with the FP64 width of the projections refined by
// their residuals (floored as the reference does)
// The bands' records: three consecutive chunks from a and from b.  Word 10
// (chunk 2 .z) holds the fingerprint and above it the FP16 residual of P[2],
// word 11 (.w) the residuals of P[0] and P[1].
__device__ bool beyond_two_sigma(double de, const uint4* a, const uint4* b) {
  const uint4 a0 = a[0], a1 = a[1], a2 = a[2];
  const uint4 b0 = b[0], b1 = b[1], b2 = b[2];
  const float pa[3] = {__uint_as_float(a0.z), __uint_as_float(a0.w), __uint_as_float(a1.x)};
  const float pb[3] = {__uint_as_float(b0.z), __uint_as_float(b0.w), __uint_as_float(b1.x)};
  const unsigned ra[3] = {a2.w & 0xFFFFu, a2.w >> 16, a2.z >> 16};
  const unsigned rb[3] = {b2.w & 0xFFFFu, b2.w >> 16, b2.z >> 16};
  double s2 = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double d = proj_fp64(pa[i], ra[i]) - proj_fp64(pb[i], rb[i]);
    s2 += d * d;
  }
  double sg = sqrt(s2 / 6.0);
  if (sg != 0.0 && sg < phxc::adaptiveCutoff) sg = phxc::adaptiveCutoff;
  return fabs(de) > 2.0 * sg;
}

// Adaptive delta of one process from the FP32 width and the FP64 energy
// difference, with the reference's cut-offs (delta_function.cpp:65-96).  The
// cut-off |E| > 2 sigma is discontinuous; `near` is set when the FP32
// comparison is within 1e-5 of it, and the caller then re-decides in FP64.
// Evaluated without branches (the exponential always, then selects), so the
// lanes of a warp stay together whatever their triplets.
__device__ __forceinline__ float delta_ad(const Sig& g, double de, bool& near) {
  const float e = (float)de;
  const float two_s = 2.f * g.s;
  near = g.s != 0.f && fabsf(fabsf(e) - two_s) <= two_s * 1e-5f;
  const float x = e * g.inv;
  float d = __expf(-x * x) * g.inv * (float)(1.0 / (phxc::sqrtPi * phxc::erf2));
  d = (g.s == 0.f || fabsf(e) > two_s) ? 0.f : d;
  return (g.vz && de == 0.0) ? 1.f : d;
}
__device__ __forceinline__ float delta_ga(float inv, double de) {
  const float x = (float)de * inv;
  if (x > 6.f || x < -8.5f) return 0.f;
  return __expf(-x * x) * inv * (float)(1.0 / phxc::sqrtPi);
}

// Rate factors of one branch triplet for all temperatures: the "+" process
// of (q1,q2) and the two "-" processes of (q1,-q2), as ph_scattering.cpp:338-380
// and :466-518 (cut-offs, deltas, Bose factors), times 0.5 (the linewidth
// convention of :433,:574); multiply by |V|^2.
// The three deltas of one triplet; `near` gets a bit per adaptive process
// whose FP32 cut-off decision was too close to call (+, -1, -2).
__device__ __forceinline__ void deltas3(int smearing, float ginv, double E1, const Band& x2, const Band& x2m,
                                        const Band& x3, const Sig& gp, const Sig& gm, float& dp, float& d1,
                                        float& d2, unsigned& near) {
  const bool ok2 = x2.E >= phxc::phExcludeCutoff, ok2m = x2m.E >= phxc::phExcludeCutoff;
  dp = d1 = d2 = 0.f;
  near = 0u;
  if (smearing == PHX_SMEAR_ADAPTIVE) {
    bool np = false, n1 = false, n2 = false;
    if (ok2) dp = delta_ad(gp, E1 + x2.E - x3.E, np);
    if (ok2m) {
      d1 = delta_ad(gm, E1 + x3.E - x2m.E, n1);
      d2 = delta_ad(gm, x2m.E + x3.E - E1, n2);
    }
    near = (np ? 1u : 0u) | (n1 ? 2u : 0u) | (n2 ? 4u : 0u);
  } else {
    if (ok2) dp = delta_ga(ginv, E1 + x2.E - x3.E);
    if (ok2m) {
      d1 = delta_ga(ginv, E1 + x3.E - x2m.E);
      d2 = delta_ga(ginv, x2m.E + x3.E - E1);
    }
  }
}

template <int NT>
__device__ __forceinline__ void rate_combine(float pre, float iE1, const float* n1, const Band& x2,
                                             const Band& x2m, const Band& x3, float dp, float d1, float d2,
                                             float* f) {
  const float fp = pre * dp * iE1 * x2.iE * x3.iE;
  const float fm = pre * iE1 * x2m.iE * x3.iE;
#pragma unroll
  for (int t = 0; t < NT; ++t)
    f[t] = fp * n1[t] * x2.N[t] * (x3.N[t] + 1.f) +
           fm * x3.N[t] * (d1 * n1[t] * (x2m.N[t] + 1.f) + d2 * x2m.N[t] * (n1[t] + 1.f));
}

// The "+" and "-" parts of rate_combine separately (matrix modes: the "+"
// process goes to the column of q2, the "-" ones to the column of -q2).
template <int NT>
__device__ __forceinline__ void rate_combine2(float pre, float iE1, const float* n1, const Band& x2,
                                              const Band& x2m, const Band& x3, float dp, float d1, float d2,
                                              float* fplus, float* fminus) {
  const float fp = pre * dp * iE1 * x2.iE * x3.iE;
  const float fm = pre * iE1 * x2m.iE * x3.iE;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    fplus[t] = fp * n1[t] * x2.N[t] * (x3.N[t] + 1.f);
    fminus[t] = fm * x3.N[t] * (d1 * n1[t] * (x2m.N[t] + 1.f) + d2 * x2m.N[t] * (n1[t] + 1.f));
  }
}

// Adds the matrix elements of one row (q1 b1) and one c2: the "+" sums to
// column (q2, c2), minus the "-" sums to column (-q2, c2) (the full matrix),
// or to the two slabs of the chunk.  The rates carry the linewidth's 1/2.
template <int NT>
__device__ __forceinline__ void add_matrix(const TcArgs& P, int q1, int b1, int iq2, int c2, double scale,
                                           const float* gp, const float* gm) {
  const phx_split_matrix& X = P.mat;
  const size_t row = (size_t)q1 * 6 + b1;
  if (X.full) {
    const int iq2m = mesh_neg(iq2, P.m.n0, P.m.n1, P.m.n2);
    if (gp[0] != 0.f) atomicAdd(X.plus + (size_t)(iq2 * 6 + c2) * X.ld + row, 2.0 * scale * (double)gp[0]);
    if (gm[0] != 0.f) atomicAdd(X.plus + (size_t)(iq2m * 6 + c2) * X.ld + row, -2.0 * scale * (double)gm[0]);
    return;
  }
  const size_t col = (size_t)((iq2 - P.q2_first) * 6 + c2) * X.ld + row;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    if (gp[t] != 0.f) atomicAdd(X.plus + t * X.tstride + col, 2.0 * scale * (double)gp[t]);
    if (gm[t] != 0.f) atomicAdd(X.minus + t * X.tstride + col, 2.0 * scale * (double)gm[t]);
  }
}

template <int NT>
__device__ __forceinline__ void rate_f(int smearing, float ginv, float pre, double E1, float iE1,
                                       const float* n1, const Band& x2, const Band& x2m,
                                       const Band& x3, const Sig& gp, const Sig& gm, float* f,
                                       unsigned& near) {
#pragma unroll
  for (int t = 0; t < NT; ++t) f[t] = 0.f;
  near = 0u;
  if (!(x3.E >= phxc::phEnergyCutoff)) return;
  float dp, d1, d2;
  deltas3(smearing, ginv, E1, x2, x2m, x3, gp, gm, dp, d1, d2, near);
  rate_combine<NT>(pre, iE1, n1, x2, x2m, x3, dp, d1, d2, f);
}

// OR a 6-bit b3 mask over the degenerate blocks of q3
__device__ __noinline__ unsigned expand_b3(unsigned c, unsigned gp3) {
  unsigned o = 0;
  for (int b = 0; b < 6; ++b)
    if ((c >> b) & 1u) o |= blk_mask(gp3, b);
  return o;
}

// Liveness of (b1, b2, b3) for all b1 at one (b2, b3): bit b1 is set when
// one of the three deltas may be non-zero (FP32 windows widened by tol).
__device__ __forceinline__ unsigned live6(int smearing, float sg, float tol, const float* E1f,
                                          float E2f, float E2mf, const Band& x2, const Band& x2m,
                                          bool ok2, bool ok2m, float E3f, const Band& x3) {
  float hp, hm, cp, c1, c2;
  if (smearing == PHX_SMEAR_ADAPTIVE) {
    hp = 2.f * sigma_ad(x2.P, x3.P, x2.vf, x3.vf).s + tol;
    hm = 2.f * sigma_ad(x2m.P, x3.P, x2m.vf, x3.vf).s + tol;
    cp = E3f - E2f;          // + : E1 + E2 - E3 = E1 - cp
    c1 = E2mf - E3f;         // -1: E1 + E3 - E2m = E1 - c1
    c2 = E2mf + E3f;         // -2: E2m + E3 - E1 = -(E1 - c2)
  } else {
    // x = dE / sigma in [-8.5, 6]: centre -1.25 sigma, half width 7.25 sigma
    hp = hm = 7.25f * sg + tol;
    cp = E3f - E2f - 1.25f * sg;
    c1 = E2mf - E3f - 1.25f * sg;
    c2 = E2mf + E3f + 1.25f * sg;
  }
  if (!ok2) hp = -1.f;
  if (!ok2m) hm = -1.f;
  unsigned msk = 0;
#pragma unroll
  for (int b1 = 0; b1 < 6; ++b1) {
    const bool live = fabsf(E1f[b1] - cp) <= hp || fabsf(E1f[b1] - c1) <= hm || fabsf(E1f[b1] - c2) <= hm;
    msk |= live ? (1u << b1) : 0u;
  }
  return msk;
}

// ---------------------------------------------------------------------------
// the fused pair kernel
// ---------------------------------------------------------------------------

// Warp roles (448 threads): warps 0-11 epilogue, warp 12 producer (bulk
// copies of B stages), warp 13 MMA issuer.
struct Smem {
  uint32_t aPart;
  uint8_t* A;          // [hi | lo] 128 x Kp BF16
  uint8_t* B;          // kStages x kStageBytes
  float2* E1v;         // e1 [36][128]
  double* En1;         // [6][128]
  float* iE1;          // [6][128]
  float* N1;           // [NT*6][128]
  uint4* rec;          // staged q3 records [kRecChunks][128]
  uint4* u2;           // [4 quarters][2: q2, -q2][kU2Chunks]
  unsigned long long* need;  // [6 b2][128] bit b1*6+b3
  uint2* queue;        // [12 warps][kQueue] live triplets awaiting their rates
  float* acc;          // [4 quarters][32 rows][kAccRow: 6 b1 x NT + pad] rates of the current q2
  uint64_t* bars;
};

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

template <int NT>
__host__ __device__ inline size_t smem_layout(int Kp, size_t* off) {
  size_t o = 0;
  const size_t aPart = (size_t)kM * Kp * 2;
  off[0] = o; o += align16(2 * aPart);                         // A
  off[1] = o; o += align16((size_t)kStages * kStageBytes);     // B
  off[2] = o; o += align16(36 * kM * sizeof(float2));          // e1
  off[3] = o; o += align16(6 * kM * sizeof(double));           // E1
  off[4] = o; o += align16(6 * kM * sizeof(float));            // 1/E1
  off[5] = o; o += align16(NT * 6 * kM * sizeof(float));       // N1
  off[6] = o; o += align16((size_t)kRecChunks * kM * 16);      // staged records
  off[7] = o; o += align16(4 * 2 * kU2Chunks * 16);            // q2 bands
  off[8] = o; o += align16(6 * kM * sizeof(unsigned long long));  // masks
  off[9] = o; o += align16(kEpiWarps * Pcfg<NT>::kQueue * sizeof(uint2));   // queues
  off[10] = o; o += align16(4 * 32 * Pcfg<NT>::kAccRow * sizeof(float));  // q2 accumulators
  off[11] = o; o += align16(32 * sizeof(uint64_t));            // barriers, tmem slot, flag
  return o;
}

template <int NT>
__device__ __forceinline__ Smem carve(uint8_t* base, int Kp) {
  size_t off[12];
  smem_layout<NT>(Kp, off);
  Smem s;
  s.aPart = (uint32_t)kM * Kp * 2;
  s.A = base + off[0];
  s.B = base + off[1];
  s.E1v = reinterpret_cast<float2*>(base + off[2]);
  s.En1 = reinterpret_cast<double*>(base + off[3]);
  s.iE1 = reinterpret_cast<float*>(base + off[4]);
  s.N1 = reinterpret_cast<float*>(base + off[5]);
  s.rec = reinterpret_cast<uint4*>(base + off[6]);
  s.u2 = reinterpret_cast<uint4*>(base + off[7]);
  s.need = reinterpret_cast<unsigned long long*>(base + off[8]);
  s.queue = reinterpret_cast<uint2*>(base + off[9]);
  s.acc = reinterpret_cast<float*>(base + off[10]);
  s.bars = reinterpret_cast<uint64_t*>(base + off[11]);
  return s;
}

// Rate of one queued live triplet, added to the FP32 accumulator of its row
// and b1.  Kept out of line: the kernel's loop calls it from two places (a
// full queue, the end of a q2), and one copy of its code keeps the hot loop
// within the instruction cache.  Entry: x = weight |V|^2 / (n1 n2 n3),
// y = lane of the q1 row | b1 << 5 | b2 << 8 | b3 << 11, where b2 and b3 are
// single bands (degenerate blocks were expanded when the entry was queued).
// The shared arrays are found from the dynamic shared memory, not passed: the
// fewer arguments, the fewer registers the caller holds across the call
// (20^3 step 95.3 -> 94.0 ms, and no spills in the adaptive instantiation).
template <int NT, bool MAT, int SM>
__device__ __noinline__ void rate_entry(uint2 e, int qd, float ginv, float pre, const TcArgs& P, int iq2) {
  constexpr int smearing = SM;   // each smearing has its own instantiation
  extern __shared__ __align__(1024) uint8_t smem[];
  const Smem S = carve<NT>(smem, P.Kp);
  const double* En1 = S.En1;
  const float* iE1s = S.iE1;
  const float* N1 = S.N1;
  const uint4* rec = S.rec;
  const uint4* u2 = S.u2 + qd * 2 * kU2Chunks;
  float* qacc = S.acc + qd * 32 * Pcfg<NT>::kAccRow;
  const float wn = __uint_as_float(e.x);
  const int r = e.y & 31, b1 = (e.y >> 5) & 7, b2 = (e.y >> 8) & 7, b3 = (e.y >> 11) & 7;
  const int mm = qd * 32 + r;
  const double E1 = En1[b1 * kM + mm];
  const float iE1 = iE1s[b1 * kM + mm];
  float n1v[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) n1v[t] = N1[(t * 6 + b1) * kM + mm];
  const Band x2 = load_band<NT>(u2 + 3 * b2, 1);
  const Band x2m = load_band<NT>(u2 + kU2Chunks + 3 * b2, 1);
  const Band x3 = load_band<NT>(rec + mm + (kChBand + 3 * b3) * kM, kM);
  Sig gp, gm;
  if (smearing == PHX_SMEAR_ADAPTIVE) {
    gp = sigma_ad(x2.P, x3.P, x2.vf, x3.vf);
    gm = sigma_ad(x2m.P, x3.P, x2m.vf, x3.vf);
  }
  float f[NT];
  unsigned near = 0u;
  if constexpr (MAT) {
    // matrix modes: the "+" rates go to column (q2, b2), the "-" ones to (-q2, b2)
    float fpv[NT], fmv[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) fpv[t] = fmv[t] = 0.f;
    if (x3.E >= phxc::phEnergyCutoff) {
      float dp, d1, d2;
      deltas3(smearing, ginv, E1, x2, x2m, x3, gp, gm, dp, d1, d2, near);
      rate_combine2<NT>(pre, iE1, n1v, x2, x2m, x3, dp, d1, d2, fpv, fmv);
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) f[t] = fpv[t] + fmv[t];
    add_matrix<NT>(P, P.q1_order[blockIdx.x * kM + mm], b1, iq2, b2, (double)wn, fpv, fmv);
  } else {
    rate_f<NT>(smearing, ginv, pre, E1, iE1, n1v, x2, x2m, x3, gp, gm, f, near);
  }
  if (near) {
    // a cut-off decision too close for FP32: edge_fix_kernel re-decides the entry in FP64
    const unsigned i = atomicAdd(P.edge_count, 1u);
    if (i < P.edge_cap) P.edges[i] = EdgeEvent{(blockIdx.x << 12) | (blockIdx.y << 7) | (unsigned)mm, iq2, e};
  }
  constexpr int AR = Pcfg<NT>::kAccRow;
#pragma unroll
  for (int t = 0; t < NT; ++t) atomicAdd(&qacc[r * AR + b1 * NT + t], wn * f[t]);
}

template <int NT, bool MAT, int SM>
__global__ void __launch_bounds__(kThreads, 1) pair_tc_kernel(TcArgs P) {
  const MeshArgs& M = P.m;
  extern __shared__ __align__(1024) uint8_t smem[];
  const int Kp = P.Kp, nkc = Kp / kKC;
  const Smem S = carve<NT>(smem, Kp);
  uint64_t* full = S.bars;                // [kStages]
  uint64_t* empty = full + kStages;       // [kStages]
  uint64_t* accf = empty + kStages;       // [kParts] MMA of a part done
  uint64_t* acce = accf + kParts;         // [kParts] part released by the 12 epilogue warps
  uint64_t* done = acce + kParts;         // MMA drain
  uint64_t* stg = done + 1;               // [4] q3 records of a quarter staged
  uint64_t* lvb = stg + 4;                // [4] liveness masks of a quarter written
  uint64_t* rel = lvb + 4;                // [4] quarter done with the staged records
  uint32_t* tslot = reinterpret_cast<uint32_t*>(rel + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nq = M.nq, n0 = M.n0, n1 = M.n1, n2 = M.n2;
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
      tc::mbar_init(&stg[q], 96);
      tc::mbar_init(&lvb[q], 96);
      tc::mbar_init(&rel[q], 96);
    }
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
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
    uint16_t hi, lo;
    split16(v, P.fp16 != 0, &hi, &lo);
    const uint32_t off = tc::core_offset(mm, k, Kp, 2);
    *reinterpret_cast<uint16_t*>(S.A + off) = hi;
    *reinterpret_cast<uint16_t*>(S.A + S.aPart + off) = lo;
  }
  // q1 data of the tile from the records
  for (int e = tid; e < 36 * kM; e += kThreads) {
    const int el = e / kM, mm = e % kM;
    const int q = P.q1_order[min(tile0 + mm, nq - 1)];
    const uint2 v = reinterpret_cast<const uint2*>(P.rec + (size_t)q * kRecChunks)[(el % 6) * 6 + el / 6];
    S.E1v[e] = make_float2(__uint_as_float(v.x), __uint_as_float(v.y));   // e1(a, b) at el = a*6 + b
  }
  for (int e = tid; e < 6 * kM; e += kThreads) {
    const int b = e / kM, mm = e % kM;
    const int q = P.q1_order[min(tile0 + mm, nq - 1)];
    const Band x = load_band<kMaxT>(P.rec + (size_t)q * kRecChunks + kChBand + 3 * b, 1);
    S.En1[e] = x.E;
    S.iE1[e] = x.iE;
#pragma unroll
    for (int t = 0; t < NT; ++t) S.N1[(t * 6 + b) * kM + mm] = x.N[t];
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;

  const int jbeg = blockIdx.y * P.q2_per_slot;
  const int jend = min(P.q2_count, jbeg + P.q2_per_slot);
  const int nj = max(0, jend - jbeg);

  if (warp == kEpiWarps) {
    // ---------------- producer ----------------
    if (lane == 0) {
      int it = 0;
      for (int u = 0; u < kParts * nj && !*abort_flag; ++u) {
        const int j = jbeg + u / kParts, h = u % kParts;
        for (int kc = 0; kc < nkc; ++kc, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (!tc::mbar_wait_sleep(&empty[s], ph ^ 1, P.status, 1)) { *abort_flag = 1; break; }
          tc::mbar_arrive_expect_tx(&full[s], kStageBytes);
          tc::bulk_g2s(S.B + s * kStageBytes, P.Bimg + ((size_t)(j * kParts + h) * nkc + kc) * kStageBytes,
                       kStageBytes, &full[s]);
        }
      }
    }
  } else if (warp == kEpiWarps + 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = P.fp16 ? tc::idesc_f16_f32(kM, kNH) : tc::idesc_bf16_f32(kM, kNH);
      const uint32_t sbA = (uint32_t)(Kp / 8) * 128;
      const uint32_t aHi = tc::smem_u32(S.A), aLo = tc::smem_u32(S.A + S.aPart);
      int it = 0;
      for (int u = 0; u < kParts * nj && !*abort_flag; ++u) {
        const int r = u % kParts, jj = u / kParts;
        if (!tc::mbar_wait_sleep(&acce[r], (jj & 1) ^ 1, P.status, 2)) { *abort_flag = 1; break; }
        tc::tc_fence_after();
        const uint32_t d = tmem + r * kRegion;
        bool ok = true;
        for (int kc = 0; kc < nkc; ++kc, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (!tc::mbar_wait_sleep(&full[s], ph, P.status, 4)) { ok = false; break; }
          tc::tc_fence_after();
          const uint32_t bHi = tc::smem_u32(S.B + s * kStageBytes);
          const uint32_t bLo = bHi + kPartBytes;
          const uint64_t dAh = tc::smem_desc(aHi + kc * 256, 128, sbA);
          const uint64_t dAl = tc::smem_desc(aLo + kc * 256, 128, sbA);
          const uint64_t dBh = tc::smem_desc(bHi, 128, kBSbo);
          const uint64_t dBl = tc::smem_desc(bLo, 128, kBSbo);
          tc::mma_bf16(d, dAh, dBh, idesc, kc != 0);
          tc::mma_bf16(d, dAh, dBl, idesc, 1);
          tc::mma_bf16(d, dAl, dBh, idesc, 1);
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
    // ---------------- epilogue ----------------
    // Warp k of quarter qd handles the rows (b1, b2) with (b1 + b2) % 3 == k,
    // so the three warps of a quarter share every b2 and every b1 evenly; the
    // rates go to FP32 accumulators of the quarter (one q2 at a time), which
    // warp k folds into FP64 registers for b1 = k and k + 3.
    const int qd = warp & 3, k = warp >> 2;
    const int m = qd * 32 + lane;
    const bool valid = tile0 + m < nq;
    const int q1c = P.q1_order[min(tile0 + m, nq - 1)];
    const unsigned FULL = 0xffffffffu;
    constexpr int smearing = SM;   // one instantiation per smearing keeps the loop small
    const float sg = (float)M.sigma, ginv = M.sigma > 0.0 ? (float)(1.0 / M.sigma) : 0.f;
    // FP16 operands: |V|^2 carries the square of the B scale, undone here (power of 4)
    float pre = P.edge_only ? 0.f : (float)(phxc::pi * 0.25 * 0.5) * (float)M.norm;
    if (P.fp16) {
      const float sc = fp16_scale(*P.dmax);
      pre *= 1.f / (sc * sc);
    }
    const unsigned gp1 = P.rec[(size_t)q1c * kRecChunks + kChGp].x;
    const bool deg1 = gp1 != kIdentityBlocks;
    unsigned ok1 = 0;
#pragma unroll
    for (int b = 0; b < 6; ++b) ok1 |= (valid && S.En1[b * kM + m] >= phxc::phExcludeCutoff) ? (1u << b) : 0u;
    double acc0[NT], acc1[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc0[t] = acc1[t] = 0.0;
    uint4* u2 = S.u2 + qd * 2 * kU2Chunks;
    const uint4* srow = S.rec + m;
    constexpr int AR = Pcfg<NT>::kAccRow;
    uint2* queue = S.queue + warp * Pcfg<NT>::kQueue;
    float* qacc = S.acc + qd * 32 * AR;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      qacc[lane * AR + k * NT + t] = 0.f;
      qacc[lane * AR + (k + 3) * NT + t] = 0.f;
    }
    int qn = 0;  // queued live triplets (warp-uniform)
    const unsigned lanemask_lt = (1u << lane) - 1u;
    const uint32_t lane_base = (uint32_t)(qd * 32) << 16;
    // fold the quarter's accumulators of b1 = k, k+3 (this lane's row) into FP64
    auto flush = [&]() {
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        acc0[t] += (double)qacc[lane * AR + k * NT + t];
        acc1[t] += (double)qacc[lane * AR + (k + 3) * NT + t];
        qacc[lane * AR + k * NT + t] = 0.f;
        qacc[lane * AR + (k + 3) * NT + t] = 0.f;
      }
    };
    bool failed = false;
    for (int jj = 0; jj < nj; ++jj) {
      // ---- previous q2 done by the whole quarter: fold its rates, then stage
      if (jj > 0) {
        if (!tc::mbar_wait(&rel[qd], (jj - 1) & 1, P.status, 32)) { failed = true; break; }
        flush();
      }
      const int iq2 = P.q2_first + jbeg + jj;
      const int iq2m = mesh_neg(iq2, n0, n1, n2);
      const int iq3 = mesh_add(q1c, iq2, n0, n1, n2);
      {
        const uint4* src = P.rec + (size_t)iq3 * kRecChunks;
#pragma unroll 1
        for (int c = k; c < kRecChunks; c += 3) cp_async16(&S.rec[c * kM + m], src + c);
        if (k == 2 && lane < kU2Chunks) {
          cp_async16(&u2[lane], P.rec + (size_t)iq2 * kRecChunks + kChBand + lane);
          cp_async16(&u2[kU2Chunks + lane], P.rec + (size_t)iq2m * kRecChunks + kChBand + lane);
        }
        cp_async_wait_all();
      }
      tc::mbar_arrive(&stg[qd]);
      if (!tc::mbar_wait(&stg[qd], jj & 1, P.status, 64)) { failed = true; break; }
      const unsigned gp2 = u2[kU2Chunks - 1].x;
      const unsigned gp3 = srow[kChGp * kM].x;
      const bool deg2 = gp2 != kIdentityBlocks, deg3 = gp3 != kIdentityBlocks;
      // ---- liveness of b2 = 2k, 2k+1 for all (b1, b3)
      {
        float E1f[6];
#pragma unroll
        for (int b = 0; b < 6; ++b) E1f[b] = (float)S.En1[b * kM + m];
#pragma unroll 1
        for (int bl = 0; bl < 2; ++bl) {
          const int b2 = 2 * k + bl;
          const Band x2 = load_band<1>(u2 + 3 * b2, 1);
          const Band x2m = load_band<1>(u2 + kU2Chunks + 3 * b2, 1);
          const float E2f = (float)x2.E, E2mf = (float)x2m.E;
          const bool ok2 = x2.E >= phxc::phExcludeCutoff, ok2m = x2m.E >= phxc::phExcludeCutoff;
          unsigned long long nd = 0;
          if (ok2 || ok2m) {
#pragma unroll 1
            for (int b3 = 0; b3 < 6; ++b3) {
              const Band x3 = load_band<1>(srow + (kChBand + 3 * b3) * kM, kM);
              if (!(x3.E >= phxc::phEnergyCutoff)) continue;
              const unsigned c = live6(smearing, sg, P.tol, E1f, E2f, E2mf, x2, x2m, ok2, ok2m,
                                       (float)x3.E, x3) & ok1;
              unsigned long long sp = 0;
#pragma unroll
              for (int b1 = 0; b1 < 6; ++b1) sp |= (unsigned long long)((c >> b1) & 1u) << (6 * b1);
              nd |= sp << b3;
            }
          }
          S.need[b2 * kM + m] = nd;
        }
      }
      tc::mbar_arrive(&lvb[qd]);
      if (!tc::mbar_wait(&lvb[qd], jj & 1, P.status, 128)) { failed = true; break; }
      // ---- the three parts
#pragma unroll 1
      for (int h = 0; h < kParts; ++h) {
        if (!tc::mbar_wait(&accf[h], jj & 1, P.status, 16)) { failed = true; break; }
        tc::tc_fence_after();
#pragma unroll 1
        for (int bl = 0; bl < 2; ++bl) {
          const int b2 = 2 * h + bl;
          const int r0 = (k + 6 - b2 % 3) % 3;       // owned b1 = r0, r0 + 3
          const unsigned bmO0 = deg1 ? blk_mask(gp1, r0) : (1u << r0);
          const unsigned bmO1 = deg1 ? blk_mask(gp1, r0 + 3) : (1u << (r0 + 3));
          // b3 masks of the owned b1 (expanded over the blocks of b2 and b3)
          unsigned long long nsrc = S.need[b2 * kM + m];
          const unsigned bm2 = deg2 ? blk_mask(gp2, b2) : (1u << b2);
          if (bm2 != (1u << b2)) {
            for (int b = 0; b < 6; ++b)
              if (b != b2 && ((bm2 >> b) & 1u)) nsrc |= S.need[b * kM + m];
          }
          unsigned nO0 = (unsigned)(nsrc >> (6 * r0)) & 63u;
          unsigned nO1 = (unsigned)(nsrc >> (6 * (r0 + 3))) & 63u;
          if (deg3) {
            if (nO0) nO0 = expand_b3(nO0, gp3);
            if (nO1) nO1 = expand_b3(nO1, gp3);
          }
          const unsigned R = (nO0 ? bmO0 : 0u) | (nO1 ? bmO1 : 0u);
          unsigned UR = __reduce_or_sync(FULL, R);
          const uint32_t col0 = tmem + lane_base + h * kRegion + bl * 72;
          while (UR) {
            const int row = __ffs(UR) - 1;
            UR &= UR - 1;
            // Y(c) = sum_a e1(a, row) X(a, c), with packed FP32 pairs:
            // R(c) = sum_a Re e1 (Re X, Im X), I(c) = sum_a Im e1 (Re X, Im X),
            // Y = (R.x - I.y, R.y + I.x)
            float2 Y[6], Yi[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) Y[c] = Yi[c] = make_float2(0.f, 0.f);
            // two rows a of X per TMEM wait
#pragma unroll
            for (int a = 0; a < 6; a += 2) {
              float t[24];
              tc::tmem_ld8(col0 + a * 12, t);
              tc::tmem_ld4(col0 + a * 12 + 8, t + 8);
              tc::tmem_ld8(col0 + a * 12 + 12, t + 12);
              tc::tmem_ld4(col0 + a * 12 + 20, t + 20);
              const float2 e0 = S.E1v[(a * 6 + row) * kM + m];
              const float2 e1 = S.E1v[((a + 1) * 6 + row) * kM + m];
              tc::tmem_wait_ld<24>(t);
              const float2 e0r = make_float2(e0.x, e0.x), e0i = make_float2(e0.y, e0.y);
              const float2 e1r = make_float2(e1.x, e1.x), e1i = make_float2(e1.y, e1.y);
#pragma unroll
              for (int c = 0; c < 6; ++c) {
                const float2 x0 = make_float2(t[2 * c], t[2 * c + 1]);
                const float2 x1 = make_float2(t[12 + 2 * c], t[12 + 2 * c + 1]);
                Y[c] = __ffma2_rn(e0r, x0, Y[c]);
                Yi[c] = __ffma2_rn(e0i, x0, Yi[c]);
                Y[c] = __ffma2_rn(e1r, x1, Y[c]);
                Yi[c] = __ffma2_rn(e1i, x1, Yi[c]);
              }
            }
            // Y(c) as broadcast pairs (Re Y, Re Y) and (Im Y, Im Y) for the e3 contraction
#pragma unroll
            for (int c = 0; c < 6; ++c) {
              const float yr = Y[c].x - Yi[c].y, yi = Y[c].y + Yi[c].x;
              Y[c] = make_float2(yr, yr);
              Yi[c] = make_float2(yi, yi);
            }
            const unsigned cols = (((bmO0 >> row) & 1u) ? nO0 : 0u) | (((bmO1 >> row) & 1u) ? nO1 : 0u);
            unsigned UC = __reduce_or_sync(FULL, cols);
            while (UC) {
              const int b3 = __ffs(UC) - 1;
              UC &= UC - 1;
              // V = sum_c Y(c) conj(e3(c, b3)), W = |V|^2; e3(., b3) is record chunks
              // 3 b3 .. 3 b3 + 2 (two components each).  Packed pairs:
              // A = sum Re Y (Re e, Im e), B = sum Im Y (Re e, Im e), V = (A.x + B.y, B.x - A.y)
              float2 va = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
#pragma unroll
              for (int j = 0; j < 3; ++j) {
                const uint4 e = srow[(3 * b3 + j) * kM];
                const float2 ea = make_float2(__uint_as_float(e.x), __uint_as_float(e.y));
                const float2 eb = make_float2(__uint_as_float(e.z), __uint_as_float(e.w));
                va = __ffma2_rn(Y[2 * j], ea, va);
                vb = __ffma2_rn(Yi[2 * j], ea, vb);
                va = __ffma2_rn(Y[2 * j + 1], eb, va);
                vb = __ffma2_rn(Yi[2 * j + 1], eb, vb);
              }
              const float vx = va.x + vb.y, vy = vb.x - va.y;
              const float w = fmaf(vx, vx, vy * vy);
              // Queue the live triplets of the owned b1.  A degenerate b2 or b3
              // averages the rate factors over its block: the entry is queued
              // once per (c2, c3) of the two blocks with weight 1/(n1 n2 n3), so
              // that every queued entry costs one rate evaluation and the lanes
              // of a batch never wait for a degenerate neighbour.
              const unsigned bm3 = deg3 ? blk_mask(gp3, b3) : (1u << b3);
              const bool l0 = ((nO0 >> b3) & 1u) && ((bmO0 >> row) & 1u);
              const bool l1 = ((nO1 >> b3) & 1u) && ((bmO1 >> row) & 1u);
              unsigned orem = (l0 ? 1u : 0u) | (l1 ? 2u : 0u);
              unsigned m2 = bm2, m3 = bm3;
              const int n23 = __popc(bm2) * __popc(bm3);
              unsigned bal;
              while ((bal = __ballot_sync(FULL, orem != 0u)) != 0u) {
                if (orem) {
                  const int o = __ffs(orem) - 1;
                  const int nd = __popc(o ? bmO1 : bmO0) * n23;
                  const float ws = nd == 1 ? w : w / (float)nd;
                  queue[qn + __popc(bal & lanemask_lt)] =
                      make_uint2(__float_as_uint(ws), (unsigned)lane | ((unsigned)(r0 + 3 * o) << 5) |
                                                          ((unsigned)(__ffs(m2) - 1) << 8) |
                                                          ((unsigned)(__ffs(m3) - 1) << 11));
                  m3 &= m3 - 1;
                  if (!m3) {
                    m3 = bm3;
                    m2 &= m2 - 1;
                    if (!m2) {
                      m2 = bm2;
                      orem &= orem - 1;
                    }
                  }
                }
                qn += __popc(bal);
                if (qn >= 32) {
                  __syncwarp();
                  rate_entry<NT, MAT, SM>(queue[lane], qd, ginv, pre, P, iq2);
                  const uint2 rest = lane + 32 < qn ? queue[lane + 32] : make_uint2(0u, 0u);
                  __syncwarp();
                  if (lane + 32 < qn) queue[lane] = rest;
                  qn -= 32;
                  __syncwarp();
                }
              }
            }
          }
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&acce[h]);
      }
      if (failed) break;
      if (qn) {
        __syncwarp();
        if (lane < qn)
          rate_entry<NT, MAT, SM>(queue[lane], qd, ginv, pre, P, iq2);
        qn = 0;
      }
      __syncwarp();
      tc::mbar_arrive(&rel[qd]);  // done with this q2's staged records and accumulators
      if (*abort_flag) break;
    }
    if (failed) *abort_flag = 1;
    // the last q2 of the quarter
    if (!failed && nj > 0 && tc::mbar_wait(&rel[qd], (nj - 1) & 1, P.status, 32)) flush();
    if (valid) {
      double* out = P.partial + ((size_t)blockIdx.y * nq + q1c) * 6 * NT;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        out[k * NT + t] += acc0[t];
        out[(k + 3) * NT + t] += acc1[t];
      }
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
      tc::tmem_wait_ld<8>(v);
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

template <int NT>
size_t pair_tc_smem(int Kp) {
  size_t off[12];
  return smem_layout<NT>(Kp, off) + 1024;
}

template <int NT>
int launch_pair(phx_ctx* ctx, const TcArgs& A, int tiles, int slots) {
  const size_t smem = pair_tc_smem<NT>(A.Kp);   // attribute set by phx_split_set_attributes
  constexpr int ad = PHX_SMEAR_ADAPTIVE, ga = PHX_SMEAR_GAUSSIAN;
  const bool adaptive = A.m.smearing == PHX_SMEAR_ADAPTIVE;
  const dim3 grid(tiles, slots);
  if (A.mat.plus) {
    if (adaptive) pair_tc_kernel<NT, true, ad><<<grid, kThreads, smem, ctx->stream>>>(A);
    else pair_tc_kernel<NT, true, ga><<<grid, kThreads, smem, ctx->stream>>>(A);
  } else {
    if (adaptive) pair_tc_kernel<NT, false, ad><<<grid, kThreads, smem, ctx->stream>>>(A);
    else pair_tc_kernel<NT, false, ga><<<grid, kThreads, smem, ctx->stream>>>(A);
  }
  PHX_CUDA(ctx, cudaGetLastError());
  return PHX_OK;
}

// FP64 re-decision of the adaptive deltas of one queued triplet (q1, q2 and
// its queue entry) whose FP32 cut-off test was too close to call: returns in
// corr[t] the difference of the two rates, times the entry's weight, for the
// partial sum of its row (q1, b1); the matrix modes also correct their
// elements here.
template <int NT>
__device__ __forceinline__ void edge_correction(const TcArgs& P, int q1, int iq2, uint2 e, double* corr) {
  const MeshArgs& M = P.m;
  float pre = (float)(phxc::pi * 0.25 * 0.5) * (float)M.norm;
  if (P.fp16) {
    const float sc = fp16_scale(*P.dmax);
    pre *= 1.f / (sc * sc);
  }
  constexpr float kNorm = (float)(1.0 / (phxc::sqrtPi * phxc::erf2));
  const float wn = __uint_as_float(e.x);
  const int b1 = (e.y >> 5) & 7, b2 = (e.y >> 8) & 7, b3 = (e.y >> 11) & 7;
  const int iq2m = mesh_neg(iq2, M.n0, M.n1, M.n2), iq3 = mesh_add(q1, iq2, M.n0, M.n1, M.n2);
  const uint4* rq2 = P.rec + (size_t)iq2 * kRecChunks;
  const uint4* rq2m = P.rec + (size_t)iq2m * kRecChunks;
  const uint4* rq3 = P.rec + (size_t)iq3 * kRecChunks;
  unsigned bm2 = 1u << b2, bm3 = 1u << b3;
  if ((e.y >> 14) & 1) {
    bm2 = blk_mask(rq2[kChGp].x, b2);
    bm3 = blk_mask(rq3[kChGp].x, b3);
  }
  const Band x1 = load_band<kMaxT>(P.rec + (size_t)q1 * kRecChunks + kChBand + 3 * b1, 1);
  double c[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) c[t] = 0.0;
  const double scale = (double)(wn / (float)(__popc(bm2) * __popc(bm3)));
  for (unsigned m2 = bm2; m2; m2 &= m2 - 1) {
    const int c2 = __ffs(m2) - 1;
    const uint4* r2 = rq2 + kChBand + 3 * c2;
    const uint4* r2m = rq2m + kChBand + 3 * c2;
    const Band x2 = load_band<NT>(r2, 1), x2m = load_band<NT>(r2m, 1);
    float cp[NT], cm[NT];   // matrix modes: corrections of the "+" and "-" sums of this c2
#pragma unroll
    for (int t = 0; t < NT; ++t) cp[t] = cm[t] = 0.f;
    for (unsigned m3 = bm3; m3; m3 &= m3 - 1) {
      const int c3 = __ffs(m3) - 1;
      const uint4* r3 = rq3 + kChBand + 3 * c3;
      const Band x3 = load_band<NT>(r3, 1);
      if (!(x3.E >= phxc::phEnergyCutoff)) continue;
      const Sig gp = sigma_ad(x2.P, x3.P, x2.vf, x3.vf), gm = sigma_ad(x2m.P, x3.P, x2m.vf, x3.vf);
      float dp, d1, d2;
      unsigned near;
      deltas3(PHX_SMEAR_ADAPTIVE, 0.f, x1.E, x2, x2m, x3, gp, gm, dp, d1, d2, near);
      if (!near) continue;
      auto val = [&](double de, float inv) {
        const float x = (float)de * inv;
        return __expf(-x * x) * inv * kNorm;
      };
      const double ep = x1.E + x2.E - x3.E, e1 = x1.E + x3.E - x2m.E, e2 = x2m.E + x3.E - x1.E;
      float fdp = dp, fd1 = d1, fd2 = d2;
      if (near & 1u) fdp = beyond_two_sigma(ep, r2, r3) ? 0.f : val(ep, gp.inv);
      if (near & 2u) fd1 = beyond_two_sigma(e1, r2m, r3) ? 0.f : val(e1, gm.inv);
      if (near & 4u) fd2 = beyond_two_sigma(e2, r2m, r3) ? 0.f : val(e2, gm.inv);
      if (fdp == dp && fd1 == d1 && fd2 == d2) continue;
      float f0[NT], f1[NT];
      rate_combine<NT>(pre, x1.iE, x1.N, x2, x2m, x3, dp, d1, d2, f0);
      rate_combine<NT>(pre, x1.iE, x1.N, x2, x2m, x3, fdp, fd1, fd2, f1);
#pragma unroll
      for (int t = 0; t < NT; ++t) c[t] += (double)f1[t] - (double)f0[t];
      if (P.mat.plus) {
        float p0[NT], m0[NT], p1[NT], m1[NT];
        rate_combine2<NT>(pre, x1.iE, x1.N, x2, x2m, x3, dp, d1, d2, p0, m0);
        rate_combine2<NT>(pre, x1.iE, x1.N, x2, x2m, x3, fdp, fd1, fd2, p1, m1);
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          cp[t] += p1[t] - p0[t];
          cm[t] += m1[t] - m0[t];
        }
      }
    }
    if (P.mat.plus) add_matrix<NT>(P, q1, b1, iq2, c2, scale, cp, cm);
  }
#pragma unroll
  for (int t = 0; t < NT; ++t) corr[t] = scale * c[t];
}

// Re-decides the recorded near-cut-off events of one pair launch (one thread
// per event) and adds their corrections to the partial sums of the event's
// row and slot; records the largest event count of the call.  When the
// launch had more events than the list holds, none is applied and the
// launch is flagged: the host re-runs its q2 in pieces whose events fit
// (events only, rates off) and applies them all there.
template <int NT>
__global__ void edge_fix_kernel(TcArgs P) {
  const unsigned cnt = *P.edge_count;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    atomicMax(P.edge_peak, cnt);
    if (cnt > P.edge_cap && P.edge_overflow) *P.edge_overflow = 1u;
  }
  if (cnt > P.edge_cap) return;
  const unsigned n = cnt;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const EdgeEvent ev = P.edges[i];
    const int tile = ev.where >> 12, slot = (ev.where >> 7) & 31, mm = ev.where & 127;
    const int q1 = P.q1_order[tile * kM + mm];
    const int b1 = (ev.entry.y >> 5) & 7;
    double corr[NT];
    edge_correction<NT>(P, q1, ev.iq2, ev.entry, corr);
    double* out = P.partial + (((size_t)slot * P.m.nq + q1) * 6 + b1) * NT;
#pragma unroll
    for (int t = 0; t < NT; ++t)
      if (corr[t] != 0.0) atomicAdd(out + t, corr[t]);
  }
}

template <int NT>
int launch_edge_fix(phx_ctx* ctx, const TcArgs& A) {
  edge_fix_kernel<NT><<<2 * ctx->num_sms, 128, 0, ctx->stream>>>(A);
  PHX_CUDA(ctx, cudaGetLastError());
  return PHX_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int phx_split_kp(int nr3) { return ((2 * nr3 + kKC - 1) / kKC) * kKC; }

size_t phx_split_bimg_bytes(int chunk, int nr3) {
  return (size_t)chunk * kParts * (phx_split_kp(nr3) / kKC) * kStageBytes;
}

size_t phx_split_rec_bytes(int nq) { return (size_t)nq * kRecChunks * 16; }

// The q1 visiting order: k-space blocks of 4x4x2 so that the 32 lanes of a
// warp hold neighbouring q1 with similar energies and similar q3.
int phx_split_prepare_bands(phx_ctx* ctx, phx_bands* b) {
  if (!b->d_q1_order) {
    const int n0 = b->mesh[0], n1 = b->mesh[1];
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
    PHX_CUDA(ctx, phx_dev_alloc(ctx, (void**)&b->d_q1_order, sizeof(int) * b->nq));
    PHX_CUDA(ctx, cudaMemcpyAsync(b->d_q1_order, order.data(), sizeof(int) * b->nq, cudaMemcpyHostToDevice,
                                  ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return PHX_OK;
}

// Per-point records of one builder call (they hold the Bose factors of its
// temperatures and the velocity projections of its smearing).
int phx_split_pack_records(phx_ctx* ctx, const pairc::MeshArgs& M, void* rec, int* launches) {
  pack_records_kernel<<<(M.nq + 127) / 128, 128, 0, ctx->stream>>>(M, static_cast<uint4*>(rec));
  PHX_CUDA(ctx, cudaGetLastError());
  *launches += 1;
  return PHX_OK;
}

// One chunk of q2: convert the FP64 Dp images to BF16 hi/lo tiles and run the
// fused tensor-core pair kernel over (q1 tiles) x (q2 slots).
int phx_split_pair_chunk(phx_ctx* ctx, const pairc::MeshArgs& M, const phx_v3* v, const phx_bands* b,
                         const double2* Dp, uint8_t* Bimg, const void* rec, double emax, int q2_first,
                         int q2_count, int slots, double* partial, int* launches, cudaEvent_t ev_begin,
                         cudaEvent_t ev_end, int fp16, const unsigned* dmax, void* edges, unsigned* edge_count,
                         unsigned edge_cap, unsigned* edge_peak, unsigned* edge_overflow, int edge_only,
                         const phx_split_matrix* mat) {
  const int Kp = phx_split_kp(v->nr3);
  const int nkc = Kp / kKC;
  convert_b_kernel<<<dim3(q2_count, kParts * nkc), 256, 0, ctx->stream>>>(Dp, v->nr3, Kp, q2_count, Bimg, fp16,
                                                                           dmax);
  PHX_CUDA(ctx, cudaGetLastError());
  TcArgs A;
  A.m = M;
  A.Kp = Kp;
  A.Bimg = Bimg;
  A.rec = static_cast<const uint4*>(rec);
  A.R3 = v->d_R3;
  A.nr3 = v->nr3;
  A.q1_order = b->d_q1_order;
  A.q2_first = q2_first;
  A.q2_count = q2_count;
  A.q2_per_slot = (q2_count + slots - 1) / slots;
  // FP32 energies carry a relative rounding of 2^-24; a window test sums
  // four of them and a sigma: 32 units of the largest energy bound it.
  A.tol = (float)(32.0 * std::max(emax, 1e-6) * 5.9604644775390625e-8);
  A.partial = partial;
  A.status = ctx->d_status;
  A.fp16 = fp16;
  A.dmax = dmax;
  A.edges = static_cast<EdgeEvent*>(edges);
  A.edge_count = edge_count;
  A.edge_cap = edge_cap;
  A.edge_peak = edge_peak;
  A.edge_overflow = edge_overflow;
  A.edge_only = edge_only;
  A.mat = mat ? *mat : phx_split_matrix{nullptr, nullptr, 0, 0, 0};
  PHX_ARG(ctx, slots < 32 && (M.nq + kM - 1) / kM < (1 << 20), "split path: at most 31 slots");
  PHX_CUDA(ctx, cudaMemsetAsync(edge_count, 0, sizeof(unsigned), ctx->stream));
  const int tiles = (M.nq + kM - 1) / kM;
  int rc = PHX_OK;
  if (ev_begin) PHX_CUDA(ctx, phx_record_event(ev_begin, ctx->stream));
  switch (M.nT) {
    case 1: rc = launch_pair<1>(ctx, A, tiles, slots); break;
    case 2: rc = launch_pair<2>(ctx, A, tiles, slots); break;
    case 3: rc = launch_pair<3>(ctx, A, tiles, slots); break;
    default: rc = launch_pair<4>(ctx, A, tiles, slots); break;
  }
  if (rc != PHX_OK) return rc;
  if (ev_end) PHX_CUDA(ctx, phx_record_event(ev_end, ctx->stream));
  switch (M.nT) {
    case 1: rc = launch_edge_fix<1>(ctx, A); break;
    case 2: rc = launch_edge_fix<2>(ctx, A); break;
    case 3: rc = launch_edge_fix<3>(ctx, A); break;
    default: rc = launch_edge_fix<4>(ctx, A); break;
  }
  if (rc != PHX_OK) return rc;
  *launches += 3;
  return PHX_OK;
}

size_t phx_split_smem_bytes(int nr3, int nT) {
  const int Kp = phx_split_kp(nr3);
  switch (nT) {
    case 1: return pair_tc_smem<1>(Kp);
    case 2: return pair_tc_smem<2>(Kp);
    case 3: return pair_tc_smem<3>(Kp);
    default: return pair_tc_smem<4>(Kp);
  }
}

// capacity of the near-cut-off event list of one pair launch (a smaller one
// may be set for tests: a launch with more events is re-run in pieces), and
// the bytes of the list
namespace {
constexpr unsigned kEdgeCapMax = 1u << 18;
std::atomic<unsigned> g_edge_cap{kEdgeCapMax};
}  // namespace
unsigned phx_split_edge_cap() { return g_edge_cap.load(); }
size_t phx_split_edge_bytes() { return sizeof(EdgeEvent) * kEdgeCapMax; }
extern "C" int phx_debug_set_split_edge_cap(unsigned cap) {
  g_edge_cap.store(cap == 0 || cap > kEdgeCapMax ? kEdgeCapMax : cap);
  return PHX_OK;
}

namespace {
template <int NT>
int set_pair_attributes(phx_ctx* ctx, int smem) {
  const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  constexpr int ad = PHX_SMEAR_ADAPTIVE, ga = PHX_SMEAR_GAUSSIAN;
  PHX_CUDA(ctx, cudaFuncSetAttribute(pair_tc_kernel<NT, false, ad>, a, smem));
  PHX_CUDA(ctx, cudaFuncSetAttribute(pair_tc_kernel<NT, false, ga>, a, smem));
  PHX_CUDA(ctx, cudaFuncSetAttribute(pair_tc_kernel<NT, true, ad>, a, smem));
  PHX_CUDA(ctx, cudaFuncSetAttribute(pair_tc_kernel<NT, true, ga>, a, smem));
  return PHX_OK;
}
}  // namespace

// Dynamic shared-memory limit of the pair kernel for nT temperatures; called
// before any launch (and outside graph capture).
int phx_split_set_attributes(phx_ctx* ctx, int nr3, int nT) {
  const int smem = (int)phx_split_smem_bytes(nr3, nT);
  switch (nT) {
    case 1: PHX_TRY(set_pair_attributes<1>(ctx, smem)); break;
    case 2: PHX_TRY(set_pair_attributes<2>(ctx, smem)); break;
    case 3: PHX_TRY(set_pair_attributes<3>(ctx, smem)); break;
    default: PHX_TRY(set_pair_attributes<4>(ctx, smem)); break;
  }
  return PHX_OK;
}

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
