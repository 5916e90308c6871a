// Fused 3-phonon linewidth builder for cells with many branches (any nb up to
// kWideMaxNb; the 15-branch perovskite and the 36-branch 12-atom cell), in
// both precisions, as one persistent kernel per chunk of q2.
//
// Reference: src/bte/ph_scattering.cpp:60-613 (builder, linewidth mode),
// src/interaction/interaction_3ph.cpp:100-405 (cacheD3, getCouplingsSquared),
// src/bte/scattering.cpp:1209-1318 (symmetrizeCoupling).  Same algebra,
// cut-offs and time-reversal pairing as the nb = 6 kernels of builder.cu: the
// "+" vertex of (q1, q2) gives the "+" process of (q1, q2) and the "-" process
// of (q1, -q2).
//
// Why a separate design: a pair's coupling has nb^3 complex entries (373 KB
// at nb = 36), so one b2 slice (nb^2) per q1 is the most a CTA can hold for a
// handful of q1, and the register- or TMEM-lane-per-q1 layouts of the small-nb
// kernels do not fit.  Per work item (one q2, a tile of kWideQ1 q1) and per b2:
//   stage 1  T(q1; a, c)  = sum_r3 e^{-i q1.R3} Dp(q2)[r3][a][b2][c]
//            (the R3 transform, the pair's dominant cost: nb^2 nr3 per b2)
//            FP64 path: CUDA cores; split path: tcgen05 with the (a, c) rows
//            of the folded vertex on the TMEM lanes and the tile's q1 as the
//            N columns (split.cu has q1 on the lanes, which nb = 36 overflows);
//   stage 2  X(q1; b1, c) = sum_a e1(a, b1) T(a, c)          (register tiles)
//   stage 3  W(q1; b1, b3) = |sum_c X(b1, c) conj(e3(c, b3))|^2
//   then W is averaged over the degenerate blocks of b1 and b3 in place, and
//   the degenerate blocks of b2 enter through the rate factors: with S the
//   block average, sum_{b2} S2(Y) F = sum_{b2} Y G, G = F averaged over blk(b2)
//   (the projections are symmetric and commute).
// Work items come from an atomic queue, q2-major, so the CTAs in flight share
// one q2 slab of the folded vertex in L2; tiles whose q1 are all outside the
// window of q2 (and of -q2) are skipped, which balances the uneven windows.
// Linewidths accumulate per item in shared memory and go to global memory
// with FP64 atomics (the order of those additions varies from run to run).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <string>
#include <vector>

#include "cplx.cuh"
#include "pair_common.cuh"
#include "phx_consts.h"
#include "phx_internal.h"
#include "tc.cuh"
#include "wide.cuh"

using namespace pairc;

namespace {

using wide::kMaxNb;
constexpr int kWideQ1 = wide::kQ1;
constexpr int kWideThreads = 256;     // FP64 kernel; split-path epilogue warps x 32
using WideArgs = wide::Args;

// forward-scan degenerate blocks (scattering.cpp:1223,1257,1291): gs[b] = first band of b's block
__device__ inline void wide_blocks(const double* e, int nb, int* gs) {
  int start = 0;
  for (int b = 0; b < nb; ++b) {
    if (b > start && !(fabs(e[start] - e[b]) < phxc::degThreshold)) start = b;
    gs[b] = start;
  }
}
__device__ inline int wide_block_end(const int* gs, int nb, int b) {
  int e = b + 1;
  while (e < nb && gs[e] == gs[b]) ++e;
  return e;
}

// complex helpers on double2 / float2
__device__ __forceinline__ void cfma_t(double2& acc, double2 a, double2 b) { cfma(acc, a, b); }
__device__ __forceinline__ void cfma_t(float2& acc, float2 a, float2 b) { cfmaf(acc, a, b); }
__device__ __forceinline__ void cfmac_t(double2& acc, double2 a, double2 b) { cfmac(acc, a, b); }
__device__ __forceinline__ void cfmac_t(float2& acc, float2 a, float2 b) { cfmacf(acc, a, b); }

// FP32 register tiles on packed FMAs: acc[i][k] += a[i] b[k] (cmac_tile) and
// acc[i][k] += a[i] conj(b[k]) (cmacc_tile), each complex product as
// (Re p, Re p) q + (Im p, Im p) q' with q' = i q or -i q, so that the products
// keep the order of cfmaf / cfmacf (same results).
template <int TI>
__device__ __forceinline__ void cmac_tile(float2 (&acc)[TI][TI], const float2 (&a)[TI], const float2 (&b)[TI]) {
  float2 bn[TI];   // i b
#pragma unroll
  for (int k = 0; k < TI; ++k) bn[k] = make_float2(-b[k].y, b[k].x);
#pragma unroll
  for (int i = 0; i < TI; ++i) {
    const float2 r = make_float2(a[i].x, a[i].x), m = make_float2(a[i].y, a[i].y);
#pragma unroll
    for (int k = 0; k < TI; ++k) {
      acc[i][k] = __ffma2_rn(r, b[k], acc[i][k]);
      acc[i][k] = __ffma2_rn(m, bn[k], acc[i][k]);
    }
  }
}
template <int TI>
__device__ __forceinline__ void cmacc_tile(float2 (&acc)[TI][TI], const float2 (&a)[TI], const float2 (&b)[TI]) {
  float2 as[TI];   // -i a
#pragma unroll
  for (int i = 0; i < TI; ++i) as[i] = make_float2(a[i].y, -a[i].x);
#pragma unroll
  for (int k = 0; k < TI; ++k) {
    const float2 r = make_float2(b[k].x, b[k].x), m = make_float2(b[k].y, b[k].y);
#pragma unroll
    for (int i = 0; i < TI; ++i) {
      acc[i][k] = __ffma2_rn(r, a[i], acc[i][k]);
      acc[i][k] = __ffma2_rn(m, as[i], acc[i][k]);
    }
  }
}
template <class C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }

// Per-item state of the tile in shared memory (both kernels).
struct Tile {
  int* q1s;     // [nq1] q1 (-1: none)
  int* q3s;     // [nq1]
  int* inw;     // [nq1] bit 0: q2 in the window of q1, bit 1: -q2
  int* g1s;     // [nq1][nb] blocks of q1
  int* g3s;     // [nq1][nb] blocks of q3
  int* g2s;     // [nb] blocks of q2
  int* dg;      // [nq1] q1 or q3 has a degenerate block (else symmetrizeCoupling changes nothing)
  double* acc;  // [nq1][nb][kMaxT]
};

// symmetrizeCoupling (scattering.cpp:1209-1318) of the W planes q0 .. q0+nq1-1
// of one b2 (W over T): average over the blocks of b3 (rows), then of b1
// (columns); b2 enters the rates.  Starts and ends with a barrier; when no
// plane's q1 or q3 has a degenerate block the averages change nothing and
// only the ending barrier is taken.
template <class R>
__device__ void wide_symmetrize(const Tile& t, int q0, int nq1, int nb, void* Tv, int tid, int nthreads, int bar_id) {
  const int nbb = nb * nb;
  R* W = reinterpret_cast<R*>(Tv);
  int any_dg = 0;
  for (int q = q0; q < q0 + nq1; ++q) any_dg |= t.dg[q];
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
  if (!any_dg) return;
  for (int u = tid; u < nq1 * nb; u += nthreads) {
    const int q = q0 + u / nb, b1 = u % nb;
    if (t.q1s[q] < 0 || !t.inw[q]) continue;
    R* w = W + (size_t)q * nbb + (size_t)b1 * nb;
    const int* g = t.g3s + q * nb;
    for (int s0 = 0; s0 < nb;) {
      const int s1 = wide_block_end(g, nb, s0);
      if (s1 - s0 > 1) {
        R sum = 0;
        for (int k = s0; k < s1; ++k) sum += w[k];
        for (int k = s0; k < s1; ++k) w[k] = sum / (R)(s1 - s0);
      }
      s0 = s1;
    }
  }
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
  for (int u = tid; u < nq1 * nb; u += nthreads) {
    const int q = q0 + u / nb, b3 = u % nb;
    if (t.q1s[q] < 0 || !t.inw[q]) continue;
    R* w = W + (size_t)q * nbb + b3;
    const int* g = t.g1s + q * nb;
    for (int s0 = 0; s0 < nb;) {
      const int s1 = wide_block_end(g, nb, s0);
      if (s1 - s0 > 1) {
        R sum = 0;
        for (int k = s0; k < s1; ++k) sum += w[(size_t)k * nb];
        for (int k = s0; k < s1; ++k) w[(size_t)k * nb] = sum / (R)(s1 - s0);
      }
      s0 = s1;
    }
  }
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
}

// wide_contract's FP32 4 x 4 tiles when nb is a multiple of 4: no bounds
// checks, and the four consecutive complex values of a tile row (e1, T, e3)
// move as two 16-byte accesses, a row of W as one.
__device__ __forceinline__ float4 ld4(const float2* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ldg4(const float2* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
// TI complex values from a 16-byte aligned address, through L1 (G) or shared memory
template <int TI, bool G>
__device__ __forceinline__ void ldc(float2 (&v)[TI], const float2* p) {
#pragma unroll
  for (int j = 0; j < TI; j += 2) {
    const float4 x = G ? ldg4(p + j) : ld4(p + j);
    v[j] = make_float2(x.x, x.y);
    v[j + 1] = make_float2(x.z, x.w);
  }
}
// stage-2 tile: X(b10 + i, c0 + k) = sum_a e1(a, b10 + i) T(a, c0 + k); e1 = U + q1 nbb + b10,
// Tq = T plane + c0, Xq = X plane + b10 ldx + c0
template <int TI>
__device__ __forceinline__ void f4_x_tile(const float2* __restrict__ e1, const float2* Tq, float2* Xq, int nb,
                                          int ldx) {
  float2 acc[TI][TI];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int k = 0; k < TI; ++k) acc[i][k] = make_float2(0.f, 0.f);
#pragma unroll 2
  for (int a = 0; a < nb; ++a) {
    float2 ev[TI], tv[TI];
    ldc<TI, true>(ev, e1 + a * nb);
    ldc<TI, false>(tv, Tq + a * nb);
    cmac_tile<TI>(acc, ev, tv);
  }
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int k = 0; k < TI; ++k) Xq[i * ldx + k] = acc[i][k];
}
// stage-3 tile: W(b10 + i, b30 + k) = |sum_c X(b10 + i, c) conj(e3(c, b30 + k))|^2; e3 = U + q3 nbb
// + b30, Xq = X plane + b10 ldx, Wq = W plane + b10 nb + b30
template <int TI>
__device__ __forceinline__ void f4_w_tile(const float2* __restrict__ e3, const float2* Xq, float* Wq, int nb,
                                          int ldx) {
  float2 acc[TI][TI];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int k = 0; k < TI; ++k) acc[i][k] = make_float2(0.f, 0.f);
#pragma unroll 2
  for (int c = 0; c < nb; ++c) {
    float2 xv[TI], ev[TI];
#pragma unroll
    for (int i = 0; i < TI; ++i) xv[i] = Xq[i * ldx + c];
    ldc<TI, true>(ev, e3 + c * nb);
    cmacc_tile<TI>(acc, xv, ev);
  }
#pragma unroll
  for (int i = 0; i < TI; ++i) {
    float w[TI];
#pragma unroll
    for (int k = 0; k < TI; ++k) w[k] = acc[i][k].x * acc[i][k].x + acc[i][k].y * acc[i][k].y;
    if constexpr (TI == 4)
      *reinterpret_cast<float4*>(Wq + i * nb) = make_float4(w[0], w[1], w[2], w[3]);
    else
      *reinterpret_cast<float2*>(Wq + i * nb) = make_float2(w[0], w[1]);
  }
}
// Units of both stages: the 4 x 4 tiles of the planes, whole in full rounds
// over the threads; the tiles of a last, partial round are cut into four 2 x 2
// tiles, so that no thread has a second 4 x 4 tile while others idle (nb = 36,
// 8 planes, 512 threads: 648 tiles, at most 24 outputs a thread instead of 32).
__device__ __forceinline__ int f4_whole_tiles(int units, int nthreads) {
  return units >= nthreads ? units - units % nthreads : units;
}
__device__ void wide_contract_f4(const Tile& t, int q0, int nq1, int nb, const float2* __restrict__ U, float2* T,
                                 float2* X, int ldx, int tid, int nthreads, int bar_id) {
  const int nt = nb / 4, per_q = nt * nt, nbb = nb * nb;
  const int units = nq1 * per_q, whole = f4_whole_tiles(units, nthreads), subs = 4 * (units - whole);
  for (int v = tid; v < whole + subs; v += nthreads) {
    const int u = v < whole ? v : whole + (v - whole) / 4, sub = v < whole ? 0 : (v - whole) % 4;
    const int q = q0 + u / per_q, r = u % per_q;
    const int b10 = (r / nt) * 4 + (sub >> 1) * 2, c0 = (r % nt) * 4 + (sub & 1) * 2;
    const int q1 = t.q1s[q];
    if (q1 < 0 || !t.inw[q]) continue;
    const float2* e1 = U + (size_t)q1 * nbb + b10;
    const float2* Tq = T + (size_t)q * nbb + c0;
    float2* Xq = X + (size_t)(q - q0) * nb * ldx + (size_t)b10 * ldx + c0;
    if (v < whole)
      f4_x_tile<4>(e1, Tq, Xq, nb, ldx);
    else
      f4_x_tile<2>(e1, Tq, Xq, nb, ldx);
  }
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
  float* W = reinterpret_cast<float*>(T);
  for (int v = tid; v < whole + subs; v += nthreads) {
    const int u = v < whole ? v : whole + (v - whole) / 4, sub = v < whole ? 0 : (v - whole) % 4;
    const int q = q0 + u / per_q, r = u % per_q;
    const int b10 = (r / nt) * 4 + (sub >> 1) * 2, b30 = (r % nt) * 4 + (sub & 1) * 2;
    if (t.q1s[q] < 0 || !t.inw[q]) continue;
    const float2* e3 = U + (size_t)t.q3s[q] * nbb + b30;
    const float2* Xq = X + (size_t)(q - q0) * nb * ldx + (size_t)b10 * ldx;
    float* Wq = W + (size_t)q * nbb + (size_t)b10 * nb + b30;
    if (v < whole)
      f4_w_tile<4>(e3, Xq, Wq, nb, ldx);
    else
      f4_w_tile<2>(e3, Xq, Wq, nb, ldx);
  }
  wide_symmetrize<float>(t, q0, nq1, nb, T, tid, nthreads, bar_id);
}

// Stages 2 and 3 for one b2 of every q1 of the item, on CUDA cores: T (a, c)
// -> X (b1, c) -> W (b1, b3) = |V|^2, W written over T (as R).  Register
// tiles of RT x RT outputs per thread.
//   The q1 planes q0 .. q0+nq1-1 are contracted in this call, X holds nq1
// planes (X[q - q0], rows of ldx >= nb elements: an odd stride keeps the
// stage-3 row reads of a warp in distinct banks); W plane q lands in the
// first half of T's plane q / 2 (R is half of C), i.e. on planes already
// consumed when calls run in increasing q0.  e1 and e3 come from E1s / E3s
// (the caller's shared-memory copies [q - q0][row][col], rows of nb) when
// given, else from the global table U through L1.
template <class R, class C, int RT>
__device__ void wide_contract(const Tile& t, int q0, int nq1, int nb, const C* __restrict__ U, const C* E1s,
                              const C* E3s, C* T, C* X, int ldx, int tid, int nthreads, int bar_id) {
  const int nt = (nb + RT - 1) / RT, per_q = nt * nt, nbb = nb * nb;
  if constexpr (RT == 4 && sizeof(C) == 8) {
    if ((nb & 3) == 0 && !E1s) {
      wide_contract_f4(t, q0, nq1, nb, reinterpret_cast<const float2*>(U), reinterpret_cast<float2*>(T),
                       reinterpret_cast<float2*>(X), ldx, tid, nthreads, bar_id);
      return;
    }
  }
  // stage 2: X[q][b1][c] = sum_a e1(a, b1) T[q][a][c]
  for (int u = tid; u < nq1 * per_q; u += nthreads) {
    const int q = q0 + u / per_q, r = u % per_q, b10 = (r / nt) * RT, c0 = (r % nt) * RT;
    const int q1 = t.q1s[q];
    if (q1 < 0 || !t.inw[q]) continue;
    const C* e1 = E1s ? E1s + (size_t)(q - q0) * nbb : U + (size_t)q1 * nbb;
    const C* Tq = T + (size_t)q * nbb;
    C acc[RT][RT];
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int k = 0; k < RT; ++k) acc[i][k] = czero<C>();
#pragma unroll 2
    for (int a = 0; a < nb; ++a) {
      C ev[RT], tv[RT];
#pragma unroll
      for (int i = 0; i < RT; ++i) ev[i] = b10 + i < nb ? e1[a * nb + b10 + i] : czero<C>();
#pragma unroll
      for (int k = 0; k < RT; ++k) tv[k] = c0 + k < nb ? Tq[a * nb + c0 + k] : czero<C>();
#pragma unroll
      for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int k = 0; k < RT; ++k) cfma_t(acc[i][k], ev[i], tv[k]);
    }
    C* Xq = X + (size_t)(q - q0) * nb * ldx;
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int k = 0; k < RT; ++k)
        if (b10 + i < nb && c0 + k < nb) Xq[(b10 + i) * ldx + c0 + k] = acc[i][k];
  }
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
  // stage 3: W[q][b1][b3] = |sum_c X[q][b1][c] conj(e3(c, b3))|^2, over T
  R* W = reinterpret_cast<R*>(T);
  for (int u = tid; u < nq1 * per_q; u += nthreads) {
    const int q = q0 + u / per_q, r = u % per_q, b10 = (r / nt) * RT, b30 = (r % nt) * RT;
    if (t.q1s[q] < 0 || !t.inw[q]) continue;
    const C* e3 = E3s ? E3s + (size_t)(q - q0) * nbb : U + (size_t)t.q3s[q] * nbb;
    const C* Xq = X + (size_t)(q - q0) * nb * ldx;
    C acc[RT][RT];
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int k = 0; k < RT; ++k) acc[i][k] = czero<C>();
#pragma unroll 2
    for (int c = 0; c < nb; ++c) {
      C xv[RT], ev[RT];
#pragma unroll
      for (int i = 0; i < RT; ++i) xv[i] = b10 + i < nb ? Xq[(b10 + i) * ldx + c] : czero<C>();
#pragma unroll
      for (int k = 0; k < RT; ++k) ev[k] = b30 + k < nb ? e3[c * nb + b30 + k] : czero<C>();
#pragma unroll
      for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int k = 0; k < RT; ++k) cfmac_t(acc[i][k], xv[i], ev[k]);
    }
    R* Wq = W + (size_t)q * nbb;
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int k = 0; k < RT; ++k)
        if (b10 + i < nb && b30 + k < nb) Wq[(b10 + i) * nb + b30 + k] = acc[i][k].x * acc[i][k].x + acc[i][k].y * acc[i][k].y;
  }
  wide_symmetrize<R>(t, q0, nq1, nb, T, tid, nthreads, bar_id);
}

// Segments of b3 per (q1, b1) row in the rate loop: the count that minimises
// the work of the busiest thread, (rounds of units over the threads) x
// (cells per segment + one cell's worth for the unit's set-up and atomics),
// the smallest such count on ties.  Each thread runs whole segments, so the
// lanes of a warp stay in step.  nb = 36, 8 planes, 512 threads: 3 segments
// of 12 cells (4 segments: 3 rounds of 9); nb = 15: 4 segments, one round.
__device__ inline int wide_rate_segments(int nq1, int nb, int nthreads) {
  const int rows = nq1 * nb;
  int best = 1, best_cost = 1 << 30;
  for (int sg = 1; sg <= nb; ++sg) {
    const int cost = ((sg * rows + nthreads - 1) / nthreads) * ((nb + sg - 1) / sg + 1);
    if (cost < best_cost) {
      best_cost = cost;
      best = sg;
    }
  }
  return best;
}

// Adaptive delta (delta_function.cpp:65-96) from a tabulated width: sigma,
// its reciprocal and whether the velocity difference is exactly zero.
// exp(-x^2) / (sqrt(pi) sigma erf(2)) with x = e / sigma as products.  The
// cut-off decisions stay FP64; F32EXP evaluates the Gaussian itself in FP32
// (relative error ~1e-7, for the split path, whose |V|^2 carries ~1e-6).
template <bool F32EXP>
__device__ __forceinline__ double delta_tab(double sigma, double inv, bool vz, double e) {
  if (vz && e == 0.0) return 1.0;
  if (sigma == 0.0) return 0.0;
  if (fabs(e) > 2.0 * sigma) return 0.0;
  const double x = e * inv;   // |x| <= 2 past the cut-off
  const double g = F32EXP ? (double)expf((float)(-x * x)) : exp(-x * x);
  return g * inv * (1.0 / (phxc::sqrtPi * phxc::erf2));
}

// Rates of the b2 plane (ph_scattering.cpp:338-380, 466-518), FP64, with the
// rate factors averaged over the degenerate block of b2: "+" of (q1, q2) and
// "-" of (q1, -q2).  Units (segment of b3, q1, b1), segs segments per row
// (wide_rate_segments); one shared-memory atomic per unit and temperature.
// W scaled by wscale (split FP16 operands).
//   With adaptive smearing the widths of the pairs (q3 b3, q2 c2) and
// (q3 b3, -q2 c2), which every b1 of a plane shares, are tabulated first in
// `sig` (sig_bytes of shared memory that is free during this phase: the X
// slab), as (sigma, 1/sigma) with the zero-velocity flag in the sign bit of
// sigma; a block of b2 too large for the table computes them per cell.
// Called by all nthreads threads of named barrier bar_id.
template <class R>
__device__ void wide_rates(const Tile& t, const MeshArgs& M, int nq1, int b2, int iq2, int iq2m, const R* W,
                           double wscale, int segs, double* sig, size_t sig_bytes, int tid, int nthreads,
                           int bar_id) {
  const int nb = M.nb, nbb = nb * nb, nT = M.nT, nq = M.nq;
  const int seg = (nb + segs - 1) / segs;
  const int* g2 = t.g2s;
  const int s0 = g2[b2], s1 = wide_block_end(g2, nb, s0), nblk = s1 - s0;
  const double inv2 = 1.0 / (double)nblk;
  const bool adaptive = M.smearing == PHX_SMEAR_ADAPTIVE;
  const bool tab = adaptive && sizeof(double) * 4 * (size_t)nq1 * nb * nblk <= sig_bytes;
  auto widths = [&](int iq3, int b3, int c2, double& sp, bool& vzp, double& sm, bool& vzm) {
    const double* v3 = M.vg + ((size_t)iq3 * nb + b3) * 3;
    const double* v2 = M.vg + ((size_t)iq2 * nb + c2) * 3;
    const double* v2m = M.vg + ((size_t)iq2m * nb + c2) * 3;
    const double dp0 = v2[0] - v3[0], dp1 = v2[1] - v3[1], dp2 = v2[2] - v3[2];
    const double dm0 = v2m[0] - v3[0], dm1 = v2m[1] - v3[1], dm2 = v2m[2] - v3[2];
    vzp = (dp0 * dp0 + dp1 * dp1 + dp2 * dp2) == 0.0;
    vzm = (dm0 * dm0 + dm1 * dm1 + dm2 * dm2) == 0.0;
    sp = floor_sigma(adaptive_sigma(M.qT, dp0, dp1, dp2));
    sm = floor_sigma(adaptive_sigma(M.qT, dm0, dm1, dm2));
  };
  if (tab) {
    for (int e = tid; e < nq1 * nb * nblk; e += nthreads) {
      const int q = e / (nb * nblk), b3 = (e / nblk) % nb, c2 = s0 + e % nblk;
      if (t.q1s[q] < 0 || !t.inw[q]) continue;
      double sp, sm;
      bool vzp, vzm;
      widths(t.q3s[q], b3, c2, sp, vzp, sm, vzm);
      sig[4 * e] = vzp ? -0.0 : sp;   // zero width when the velocities agree
      sig[4 * e + 1] = sp > 0.0 ? 1.0 / sp : 0.0;
      sig[4 * e + 2] = vzm ? -0.0 : sm;
      sig[4 * e + 3] = sm > 0.0 ? 1.0 / sm : 0.0;
    }
    asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
  }
  for (int u = tid; u < segs * nq1 * nb; u += nthreads) {
    const int sg = u / (nq1 * nb), rest = u % (nq1 * nb), q = rest / nb, b1 = rest % nb;
    const int q1 = t.q1s[q];
    if (q1 < 0 || !t.inw[q]) continue;
    const double en1 = M.E[(size_t)q1 * nb + b1];
    if (en1 < phxc::phExcludeCutoff || en1 < phxc::phEnergyCutoff) continue;
    const int iq3 = t.q3s[q];
    double r[kMaxT];
#pragma unroll
    for (int c = 0; c < kMaxT; ++c) r[c] = 0.0;
    const int b3b = sg * seg, b3e = min(nb, b3b + seg);
    for (int b3 = b3b; b3 < b3e; ++b3) {
      const double w = (double)W[(size_t)q * nbb + (size_t)b1 * nb + b3] * wscale;
      if (w == 0.0) continue;
      const double en3 = M.E[(size_t)iq3 * nb + b3];
      if (en3 < phxc::phEnergyCutoff) continue;
      const double* sg4 = sig + (size_t)(q * nb + b3) * nblk * 4;
      for (int c2 = s0; c2 < s1; ++c2) {
        const double en2 = M.E[(size_t)iq2 * nb + c2];
        const double en2m = M.E[(size_t)iq2m * nb + c2];
        const bool ok2 = (t.inw[q] & 1) && en2 >= phxc::phExcludeCutoff && en2 >= phxc::phEnergyCutoff;
        const bool ok2m = (t.inw[q] & 2) && en2m >= phxc::phExcludeCutoff && en2m >= phxc::phEnergyCutoff;
        if (!ok2 && !ok2m) continue;
        double dlt = 0.0, d1 = 0.0, d2 = 0.0;
        if (tab) {
          const double* e4 = sg4 + (c2 - s0) * 4;
          const double sp = e4[0], ip = e4[1], sm = e4[2], im = e4[3];
          if (ok2) dlt = delta_tab<sizeof(R) == 4>(fabs(sp), ip, signbit(sp), en1 + en2 - en3);
          if (ok2m) {
            d1 = delta_tab<sizeof(R) == 4>(fabs(sm), im, signbit(sm), en1 + en3 - en2m);
            d2 = delta_tab<sizeof(R) == 4>(fabs(sm), im, signbit(sm), en2m + en3 - en1);
          }
        } else {
          double sp = M.sigma, sm = M.sigma;
          bool vzp = false, vzm = false;
          if (adaptive) widths(iq3, b3, c2, sp, vzp, sm, vzm);
          if (ok2) dlt = delta_fn(M.smearing, sp, en1 + en2 - en3, vzp);
          if (ok2m) {
            d1 = delta_fn(M.smearing, sm, en1 + en3 - en2m, vzm);
            d2 = delta_fn(M.smearing, sm, en2m + en3 - en1, vzm);
          }
        }
        if (ok2 && dlt > 0.0) {
          const double f = phxc::pi * 0.25 * w * dlt * M.norm / (en1 * en2 * en3) * inv2;
#pragma unroll
          for (int c = 0; c < kMaxT; ++c)
            if (c < nT) {
              const double n1 = M.bose[((size_t)c * nq + q1) * nb + b1];
              const double n2 = M.bose[((size_t)c * nq + iq2) * nb + c2];
              const double n3 = M.bose[((size_t)c * nq + iq3) * nb + b3];
              r[c] += 0.5 * (f * n1 * n2 * (n3 + 1.0));
            }
        }
        if (ok2m && (d1 > 0.0 || d2 > 0.0)) {
          d1 = fmax(d1, 0.0);
          d2 = fmax(d2, 0.0);
          const double f = phxc::pi * 0.25 * w * M.norm / (en1 * en2m * en3) * inv2;
#pragma unroll
          for (int c = 0; c < kMaxT; ++c)
            if (c < nT) {
              const double n1 = M.bose[((size_t)c * nq + q1) * nb + b1];
              const double n2m = M.bose[((size_t)c * nq + iq2m) * nb + c2];
              const double n3 = M.bose[((size_t)c * nq + iq3) * nb + b3];
              r[c] += 0.5 * (f * n3 * n1 * (n2m + 1.0) * d1 + f * n2m * n3 * (n1 + 1.0) * d2);
            }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < kMaxT; ++c)
      if (c < nT && r[c] != 0.0) atomicAdd(&t.acc[(q * nb + b1) * kMaxT + c], r[c]);
  }
}

// Loads the tile of the current item: q1, q3, window flags, blocks; returns
// (block-uniform, after a barrier) whether any q1 of the tile pairs with q2 or -q2.
__device__ bool wide_load_tile(const Tile& t, const WideArgs& P, int tile, int iq2, int iq2m, int tid,
                               int nthreads, int bar_id) {
  const MeshArgs& M = P.m;
  const int nb = M.nb, nq1 = P.nq1;
  if (tid < nq1) {
    const int i = tile * nq1 + tid;
    const int q1 = i < M.nq ? P.q1_order[i] : -1;
    int f = 0;
    if (q1 >= 0 && !(P.skip && P.skip[(size_t)(iq2 - P.skip_base) * M.nq + q1])) {
      f |= (!P.win_energy || P.win_energy[iq2] <= P.win_cut[q1]) ? 1 : 0;
      f |= (!P.win_energy || P.win_energy[iq2m] <= P.win_cut[q1]) ? 2 : 0;
    }
    t.q1s[tid] = q1;
    t.inw[tid] = f;
    t.q3s[tid] = mesh_add(max(q1, 0), iq2, M.n0, M.n1, M.n2);
    t.dg[tid] = 0;
  }
  // zeroed before the early return too: the split kernel flushes every item
  for (int i = tid; i < nq1 * nb * kMaxT; i += nthreads) t.acc[i] = 0.0;
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
  int any = 0;
  for (int q = 0; q < nq1; ++q) any |= t.inw[q];
  if (!any) return false;
  if (tid < nq1) {
    const int q1 = max(t.q1s[tid], 0);
    int* g1 = t.g1s + tid * nb;
    int* g3 = t.g3s + tid * nb;
    wide_blocks(M.E + (size_t)q1 * nb, nb, g1);
    wide_blocks(M.E + (size_t)t.q3s[tid] * nb, nb, g3);
    int d = 0;
    for (int b = 0; b < nb; ++b) d |= (g1[b] != b) | (g3[b] != b);
    t.dg[tid] = d;
  } else if (tid == nq1) {
    wide_blocks(M.E + (size_t)iq2 * nb, nb, t.g2s);
  }
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
  return true;
}

__device__ void wide_flush(const Tile& t, const WideArgs& P, int tid, int nthreads) {
  const int nb = P.m.nb, nT = P.m.nT;
  for (int i = tid; i < P.nq1 * nb * nT; i += nthreads) {
    const int q = i / (nb * nT), rest = i % (nb * nT), b1 = rest / nT, c = rest % nT;
    const int q1 = t.q1s[q];
    const double v = t.acc[(q * nb + b1) * kMaxT + c];
    if (q1 >= 0 && v != 0.0) atomicAdd(&P.lw[((size_t)q1 * nb + b1) * nT + c], v);
  }
}

__host__ __device__ inline size_t wide_tile_bytes(int nq1, int nb) {
  return sizeof(double) * (size_t)nq1 * nb * kMaxT + sizeof(int) * ((size_t)4 * nq1 + 2 * (size_t)nq1 * nb + nb);
}
__device__ inline Tile carve_tile(char* p, int nq1, int nb) {
  Tile t;
  t.acc = reinterpret_cast<double*>(p);
  t.q1s = reinterpret_cast<int*>(t.acc + (size_t)nq1 * nb * kMaxT);
  t.q3s = t.q1s + nq1;
  t.inw = t.q3s + nq1;
  t.g1s = t.inw + nq1;
  t.g3s = t.g1s + nq1 * nb;
  t.g2s = t.g3s + nq1 * nb;
  t.dg = t.g2s + nb;
  return t;
}

// ---------------------------------------------------------------------------
// FP64 kernel: stage 1 on CUDA cores (each thread owns columns (a, c) and
// accumulates them for every q1 of the tile: one read of the folded vertex per
// tile), T / X / W in FP64 shared memory.
// ---------------------------------------------------------------------------
__host__ __device__ inline int wide_ldx(int nb) { return nb | 1; }   // odd row stride of X
__host__ __device__ inline size_t wide_fp64_smem(int nq1, int nb, int nr3) {
  const size_t nbb = (size_t)nb * nb;
  return sizeof(double2) * ((size_t)nq1 * nr3 + (size_t)nq1 * nbb + (size_t)nq1 * nb * wide_ldx(nb)) +
         wide_tile_bytes(nq1, nb) + 16;
}

template <int NQ1, int RT>
__global__ void __launch_bounds__(kWideThreads) wide_fp64_kernel(WideArgs P) {
  const MeshArgs& M = P.m;
  extern __shared__ __align__(16) char sraw[];
  const int nb = M.nb, nbb = nb * nb, nr3 = P.nr3;
  double2* ph = reinterpret_cast<double2*>(sraw);    // [NQ1][nr3]
  double2* T = ph + NQ1 * nr3;                       // [NQ1][nb][nb]: T (a, c), then W (b1, b3)
  double2* X = T + NQ1 * nbb;                        // [NQ1][nb][ldx]
  double2* Xend = X + (size_t)NQ1 * nb * wide_ldx(nb);
  const Tile t = carve_tile(reinterpret_cast<char*>(Xend), NQ1, nb);
  int* item_s = reinterpret_cast<int*>(reinterpret_cast<char*>(Xend) + wide_tile_bytes(NQ1, nb));
  const int tid = threadIdx.x;
  const unsigned total = (unsigned)P.q2_count * P.ntiles;
  const int segs = wide_rate_segments(NQ1, nb, kWideThreads);
  for (;;) {
    if (tid == 0) *item_s = (int)atomicAdd(P.counter, 1u);
    __syncthreads();
    const unsigned item = (unsigned)*item_s;
    if (item >= total) break;
    const int j = item / P.ntiles, tile = item % P.ntiles;
    const int iq2 = P.q2_first + j, iq2m = mesh_neg(iq2, M.n0, M.n1, M.n2);
    if (!wide_load_tile(t, P, tile, iq2, iq2m, tid, kWideThreads, 1)) continue;
    for (int e = tid; e < NQ1 * nr3; e += kWideThreads) {
      const int q = e / nr3, r = e % nr3;
      const double* qc = M.qcart + 3 * max(t.q1s[q], 0);
      double sn, cs;
      sincos(-(qc[0] * P.R3[3 * r] + qc[1] * P.R3[3 * r + 1] + qc[2] * P.R3[3 * r + 2]), &sn, &cs);
      ph[e] = cmk(cs, sn);
    }
    __syncthreads();
    const double2* D = P.Dp + (size_t)j * nr3 * nbb * nb;
    for (int b2 = 0; b2 < nb; ++b2) {
      // stage 1: T[q][a][c] = sum_r3 ph[q][r3] Dp[r3][a][b2][c]
      for (int col = tid; col < nbb; col += kWideThreads) {
        const int a = col / nb, c = col % nb;
        const double2* d = D + ((size_t)a * nb + b2) * nb + c;
        double2 acc[NQ1];
#pragma unroll
        for (int q = 0; q < NQ1; ++q) acc[q] = cmk(0.0, 0.0);
#pragma unroll 2
        for (int r = 0; r < nr3; ++r) {
          const double2 v = __ldg(d + (size_t)r * nbb * nb);
#pragma unroll
          for (int q = 0; q < NQ1; ++q) cfma(acc[q], ph[q * nr3 + r], v);
        }
#pragma unroll
        for (int q = 0; q < NQ1; ++q) T[(size_t)q * nbb + col] = acc[q];
      }
      __syncthreads();
      wide_contract<double, double2, RT>(t, 0, NQ1, nb, M.U, nullptr, nullptr, T, X, wide_ldx(nb), tid, kWideThreads,
                                         1);
      wide_rates<double>(t, M, NQ1, b2, iq2, iq2m, reinterpret_cast<const double*>(T), 1.0, segs,
                         reinterpret_cast<double*>(X), sizeof(double2) * (size_t)NQ1 * nb * wide_ldx(nb), tid,
                         kWideThreads, 0);
      __syncthreads();
    }
    wide_flush(t, P, tid, kWideThreads);
    __syncthreads();
  }
}

// Sparse R2 fold of the folded vertex for many branches: one block per
// (r3, a, 4 consecutive q2) over the r2 with a non-zero (r3, r2) block only;
//   Y(q2)[b][c]  = sum_{r2 in list(r3)} D3w(r3, r2, a, b, c) e^{+i q2.R2}
//   Dp(q2)[r3][a][b2][c] = e^{-i q2.R3} sum_b e2(b, b2) Y(q2)[b][c]
// (the reference's cacheD3 with the e2 contraction and the q2 phases folded).
constexpr int kFoldWQ = 4;
__global__ void __launch_bounds__(256) fold_wide_kernel(int nb, int nr2, int nr3, const double* __restrict__ D3w,
                                                        const int* __restrict__ r2_ofs, const int* __restrict__ r2_list,
                                                        const double* __restrict__ R2, const double* __restrict__ R3,
                                                        const double* __restrict__ qcart, const double2* __restrict__ U,
                                                        int q2_first, int q2_count, double2* __restrict__ Dp,
                                                        unsigned* __restrict__ dmax) {
  extern __shared__ __align__(16) char sraw[];
  const int nbb = nb * nb, nb3 = nbb * nb;
  const int r3 = blockIdx.y / nb, a = blockIdx.y % nb;
  const int rb = r2_ofs[r3], re = r2_ofs[r3 + 1], nl = re - rb;
  double2* ph2 = reinterpret_cast<double2*>(sraw);   // [kFoldWQ][nl]
  double2* Y = ph2 + kFoldWQ * nl;                   // [kFoldWQ][nb][nb]
  double2* p3 = Y + kFoldWQ * nbb;                   // [kFoldWQ]
  const int j0 = blockIdx.x * kFoldWQ, nj = min(kFoldWQ, q2_count - j0);
  for (int e = threadIdx.x; e < kFoldWQ * nl; e += blockDim.x) {
    const int jl = e / nl, l = e % nl, r = r2_list[rb + l];
    double2 v = cmk(0.0, 0.0);
    if (jl < nj) {
      const double* q = qcart + 3 * (q2_first + j0 + jl);
      double sn, cs;
      sincos(q[0] * R2[3 * r] + q[1] * R2[3 * r + 1] + q[2] * R2[3 * r + 2], &sn, &cs);
      v = cmk(cs, sn);
    }
    ph2[e] = v;
  }
  if (threadIdx.x < kFoldWQ) {
    double2 v = cmk(0.0, 0.0);
    if ((int)threadIdx.x < nj) {
      const double* q = qcart + 3 * (q2_first + j0 + threadIdx.x);
      double sn, cs;
      sincos(-(q[0] * R3[3 * r3] + q[1] * R3[3 * r3 + 1] + q[2] * R3[3 * r3 + 2]), &sn, &cs);
      v = cmk(cs, sn);
    }
    p3[threadIdx.x] = v;
  }
  __syncthreads();
  const double* d0 = D3w + ((size_t)r3 * nr2) * nb3 + (size_t)a * nbb;
  for (int bc = threadIdx.x; bc < nbb; bc += blockDim.x) {
    double2 acc[kFoldWQ];
#pragma unroll
    for (int jl = 0; jl < kFoldWQ; ++jl) acc[jl] = cmk(0.0, 0.0);
    for (int l = 0; l < nl; ++l) {
      const double x = __ldg(d0 + (size_t)r2_list[rb + l] * nb3 + bc);
#pragma unroll
      for (int jl = 0; jl < kFoldWQ; ++jl) {
        const double2 p = ph2[jl * nl + l];
        acc[jl].x = fma(x, p.x, acc[jl].x);
        acc[jl].y = fma(x, p.y, acc[jl].y);
      }
    }
#pragma unroll
    for (int jl = 0; jl < kFoldWQ; ++jl) Y[jl * nbb + bc] = acc[jl];
  }
  __syncthreads();
  float m = 0.f;
  for (int e = threadIdx.x; e < nj * nbb; e += blockDim.x) {
    const int jl = e / nbb, b2 = (e / nb) % nb, c = e % nb;
    const double2* u = U + (size_t)(q2_first + j0 + jl) * nbb + b2;
    const double2* y = Y + jl * nbb + c;
    double2 z = cmk(0.0, 0.0);
    for (int b = 0; b < nb; ++b) cfma(z, __ldg(u + b * nb), y[b * nb]);
    const double2 d = cmul(z, p3[jl]);
    Dp[(((size_t)(j0 + jl) * nr3 + r3) * nb + a) * nbb + b2 * nb + c] = d;
    m = fmaxf(m, (float)fmax(fabs(d.x), fabs(d.y)));
  }
  if (dmax) {
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(dmax, __float_as_uint(m));
  }
}
__host__ inline size_t fold_wide_smem(int nb, int maxl) {
  return sizeof(double2) * ((size_t)kFoldWQ * maxl + (size_t)kFoldWQ * nb * nb + kFoldWQ);
}

// Non-zero (r3, r2) blocks of the folded vertex: flags[r3 * nr2 + r2] = 1.
__global__ void nonzero_blocks_kernel(int nb3, int nblocks, const double* __restrict__ D3w, int* __restrict__ flags) {
  for (int blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
    const double* d = D3w + (size_t)blk * nb3;
    int nz = 0;
    for (int i = threadIdx.x; i < nb3 && !nz; i += blockDim.x) nz = d[i] != 0.0;
    nz = __syncthreads_or(nz);
    if (threadIdx.x == 0) flags[blk] = nz;
  }
}

// ---------------------------------------------------------------------------
// Split-precision kernel: stage 1 on the tensor cores.
//   D[128 rows (a, c) of one b2][16 columns: re/im of 8 q1] =
//     A[rows][K = Re r3 | Im r3] (the chunk's image of Dp, FP16 or BF16 hi/lo)
//   x B[16 columns][K]: column 2i = [cos | -sin] of -q1_i.R3, 2i+1 = [sin | cos],
// hi*hi + hi*lo + lo*hi with FP32 accumulation in TMEM, one M tile per 128 rows
// of the nb^2 (a, c); two TMEM buffers, so the MMAs of the next b2 overlap
// the epilogue of this one.
// Warps: 0-15 epilogue (drain TMEM to the T slab, stages 2 and 3 in FP32,
// rates in FP64), 16 producer (work queue, bulk copies of the A tiles), 17 MMA.
// Control decisions of the epilogue (waits, items) are taken by its thread 0
// and broadcast through a named barrier, so its warps never diverge on them.
// 16 epilogue warps (4 per scheduler) hide the latency of the contractions'
// shared and L1 loads; the register budget is 112 per thread.
// Every wait is bounded; on timeout the kernel records a status bit and all
// roles leave their loops.
// ---------------------------------------------------------------------------
constexpr int kSplitEpiWarps = 16;
constexpr int kSplitThreads = (kSplitEpiWarps + 2) * 32;
constexpr int kAKC = 16;                                // K per A stage (one MMA K-step)
constexpr int kAStages = 2;
constexpr uint32_t kAPart = 128 * kAKC * 2;             // one of hi / lo: 4096 B
constexpr uint32_t kAStage = 2 * kAPart;                // hi + lo
constexpr int kN = 2 * kWideQ1;                         // MMA N
constexpr int kItemSlots = 4;

__host__ __device__ inline int split_nt(int nb) { return (nb * nb + 127) / 128; }
__host__ __device__ inline size_t split_offsets_qp(int nb, int Kp, int qp, size_t* o);
// q1 planes contracted per pass: all 8 when shared memory allows (one pass,
// the most work units per barrier), else 4, else 2
__host__ __device__ inline int split_qp(int nb, int Kp) {
  size_t o[8];
  for (int qp = kWideQ1; qp > 2; qp /= 2)
    if (split_offsets_qp(nb, Kp, qp, o) + 1024 <= 227 * 1024) return qp;
  return 2;
}
__host__ __device__ inline uint32_t split_tmem_cols(int nb) {
  const uint32_t need = 2u * split_nt(nb) * kN;
  uint32_t c = 32;
  while (c < need) c <<= 1;
  return c;
}

struct SplitSmem {
  uint8_t* A;        // [kAStages][hi, lo]
  uint8_t* B;        // [2][hi, lo] x kN rows x Kp
  float2* T;         // [kWideQ1][nb][nb]
  float2* X;         // [qp][nb][ldx]
  float2* E1s;       // shared copies of e1 / e3 (not used: read through L1)
  float2* E3s;
  char* tile;
  uint64_t* bars;
  int* items;        // [kItemSlots]
  int* ctl;          // epilogue broadcasts: [0] item, [1] ok
  uint32_t* tslot;
  volatile int* abort_flag;
};
__host__ __device__ inline size_t split_offsets_qp(int nb, int Kp, int qp, size_t* o) {
  const size_t nbb = (size_t)nb * nb;
  size_t x = 0;
  o[0] = x; x += (size_t)kAStages * kAStage;                       // A ring (1024-aligned start)
  o[1] = x; x += 2 * (size_t)kN * Kp * 2 * 2;                      // B: 2 buffers x hi/lo
  o[2] = x; x += sizeof(float2) * kWideQ1 * nbb;                   // T
  o[3] = x; x += sizeof(float2) * qp * nb * wide_ldx(nb);           // X
  o[7] = x;                                                        // (no shared copies of e1, e3)
  x = (x + 15) & ~size_t(15);
  o[4] = x; x += wide_tile_bytes(kWideQ1, nb);
  x = (x + 7) & ~size_t(7);
  o[5] = x; x += sizeof(uint64_t) * 32;                            // barriers
  o[6] = x; x += sizeof(int) * (kItemSlots + 4 + 4);               // items, ctl, tslot, abort
  return x;
}
__device__ inline SplitSmem carve_split(uint8_t* base, int nb, int Kp, int qp) {
  size_t o[8];
  split_offsets_qp(nb, Kp, qp, o);
  SplitSmem s;
  s.A = base + o[0];
  s.B = base + o[1];
  s.T = reinterpret_cast<float2*>(base + o[2]);
  s.X = reinterpret_cast<float2*>(base + o[3]);
  s.E1s = nullptr;
  s.E3s = nullptr;
  s.tile = reinterpret_cast<char*>(base + o[4]);
  s.bars = reinterpret_cast<uint64_t*>(base + o[5]);
  s.items = reinterpret_cast<int*>(base + o[6]);
  s.ctl = s.items + kItemSlots;
  s.tslot = reinterpret_cast<uint32_t*>(s.ctl + 4);
  s.abort_flag = reinterpret_cast<volatile int*>(s.tslot + 1);
  return s;
}

// Power-of-2 scale of the FP16 A operand: max |Dp| * scale in [0.5, 1]
__device__ __forceinline__ float wide_fp16_scale(const unsigned* dmax) {
  const float m = __uint_as_float(*dmax);
  if (!(m > 0.f)) return 1.f;
  int e;
  frexpf(m, &e);
  return ldexpf(1.f, -e);
}
__device__ __forceinline__ void wide_split16(double v, bool fp16, uint16_t* hi, uint16_t* lo) {
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

// is any q1 of tile t paired with q2 or -q2 (the producer's item filter)
__device__ bool tile_live(const WideArgs& P, int tile, int iq2, int iq2m) {
  if (!P.win_energy && !P.skip) return true;
  for (int i = 0; i < P.nq1; ++i) {
    const int k = tile * P.nq1 + i;
    if (k >= P.m.nq) break;
    const int q1 = P.q1_order[k];
    if (P.skip && P.skip[(size_t)(iq2 - P.skip_base) * P.m.nq + q1]) continue;
    if (!P.win_energy || P.win_energy[iq2] <= P.win_cut[q1] || P.win_energy[iq2m] <= P.win_cut[q1]) return true;
  }
  return false;
}

// Epilogue-side bounded wait by thread 0, broadcast to the 8 warps: true if
// the barrier completed and nobody aborted.
__device__ bool epi_wait(uint64_t* bar, uint32_t parity, const SplitSmem& S, const WideArgs& P, int code, int tid) {
  if (tid == 0) {
    bool ok = !*S.abort_flag && tc::mbar_wait(bar, parity, P.status, code);
    if (!ok) *S.abort_flag = 1;
    S.ctl[1] = ok ? 1 : 0;
  }
  asm volatile("bar.sync 1, %0;" ::"r"(kSplitEpiWarps * 32) : "memory");
  const bool ok = S.ctl[1] != 0;
  asm volatile("bar.sync 1, %0;" ::"r"(kSplitEpiWarps * 32) : "memory");
  return ok;
}

template <int RT>
__global__ void __launch_bounds__(kSplitThreads, 1) wide_split_kernel(WideArgs P) {
  const MeshArgs& M = P.m;
  extern __shared__ __align__(1024) uint8_t smem[];
  const int nb = M.nb, nbb = nb * nb, nr3 = P.nr3, Kp = P.Kp, nkc = Kp / kAKC, mt_n = P.mtiles;
  const SplitSmem S = carve_split(smem, nb, Kp, P.qp);
  uint64_t* full = S.bars;                 // [kAStages] A stage loaded
  uint64_t* empty = full + kAStages;       // [kAStages] A stage consumed
  uint64_t* tfull = empty + kAStages;      // [2] TMEM buffer written by the MMAs
  uint64_t* tfree = tfull + 2;             // [2] TMEM buffer drained by the epilogue
  uint64_t* bready = tfree + 2;            // [2] B (phases) of an item written
  uint64_t* bfree = bready + 2;            // [2] B of an item no longer read by the MMAs
  uint64_t* ifull = bfree + 2;             // [kItemSlots]
  uint64_t* iempty = ifull + kItemSlots;   // [kItemSlots]
  uint64_t* done = iempty + kItemSlots;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned total = (unsigned)P.q2_count * P.ntiles;
  const uint32_t tcols = split_tmem_cols(nb);
  const uint32_t bufcols = (uint32_t)mt_n * kN;

  if (tid == 0) {
    for (int i = 0; i < kAStages; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&tfull[i], 1);
      tc::mbar_init(&tfree[i], 1);
      tc::mbar_init(&bready[i], 1);
      tc::mbar_init(&bfree[i], 1);
    }
    for (int i = 0; i < kItemSlots; ++i) {
      tc::mbar_init(&ifull[i], 1);
      tc::mbar_init(&iempty[i], 2);
    }
    tc::mbar_init(done, 1);
    *S.abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(S.tslot, tcols);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *S.tslot;

  if (warp == kSplitEpiWarps) {
    // ---------------- producer: work queue and A tiles ----------------
    if (lane == 0) {
      int it = 0;
      for (int n = 0;; ++n) {
        const int slot = n % kItemSlots;
        if (!tc::mbar_wait_sleep(&iempty[slot], ((n / kItemSlots) & 1) ^ 1, P.status, 1 << 8)) {
          *S.abort_flag = 1;
          break;
        }
        unsigned item;
        for (;;) {
          item = *S.abort_flag ? total : atomicAdd(P.counter, 1u);
          if (item >= total) break;
          const int j = item / P.ntiles, tl = item % P.ntiles;
          const int iq2 = P.q2_first + j;
          if (tile_live(P, tl, iq2, mesh_neg(iq2, M.n0, M.n1, M.n2))) break;
        }
        S.items[slot] = item < total ? (int)item : -1;
        tc::mbar_arrive(&ifull[slot]);
        if (item >= total) break;
        const int j = item / P.ntiles;
        bool ok = true;
        for (int b2 = 0; b2 < nb && ok; ++b2)
          for (int mt = 0; mt < mt_n && ok; ++mt)
            for (int kc = 0; kc < nkc; ++kc, ++it) {
              const int st = it % kAStages;
              if (!tc::mbar_wait_sleep(&empty[st], ((it / kAStages) & 1) ^ 1, P.status, 1 << 9) || *S.abort_flag) {
                ok = false;
                break;
              }
              tc::mbar_arrive_expect_tx(&full[st], kAStage);
              tc::bulk_g2s(S.A + st * kAStage,
                           P.img + ((((size_t)j * nb + b2) * mt_n + mt) * nkc + kc) * kAStage, kAStage, &full[st]);
            }
        if (!ok) {
          *S.abort_flag = 1;
          break;
        }
      }
    }
  } else if (warp == kSplitEpiWarps + 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = P.fp16 ? tc::idesc_f16_f32(128, kN) : tc::idesc_bf16_f32(128, kN);
      const uint32_t sbB = (uint32_t)(Kp / 8) * 128;
      const uint32_t bBytes = (uint32_t)kN * Kp * 2;   // one of hi / lo
      int it = 0, s = 0;
      bool ok = true;
      for (int n = 0; ok; ++n) {
        const int slot = n % kItemSlots;
        if (!tc::mbar_wait_sleep(&ifull[slot], (n / kItemSlots) & 1, P.status, 1 << 10)) { ok = false; break; }
        const int item = S.items[slot];
        tc::mbar_arrive(&iempty[slot]);
        if (item < 0) break;
        const int bb = n & 1;
        if (!tc::mbar_wait_sleep(&bready[bb], (n >> 1) & 1, P.status, 1 << 11)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t bHi = tc::smem_u32(S.B + (size_t)bb * 2 * bBytes), bLo = bHi + bBytes;
        for (int b2 = 0; b2 < nb && ok; ++b2, ++s) {
          const int buf = s & 1;
          if (!tc::mbar_wait_sleep(&tfree[buf], ((s >> 1) & 1) ^ 1, P.status, 1 << 12)) { ok = false; break; }
          tc::tc_fence_after();
          for (int mt = 0; mt < mt_n && ok; ++mt) {
            const uint32_t d = tmem + (uint32_t)buf * bufcols + (uint32_t)mt * kN;
            for (int kc = 0; kc < nkc; ++kc, ++it) {
              const int st = it % kAStages;
              if (!tc::mbar_wait_sleep(&full[st], (it / kAStages) & 1, P.status, 1 << 13) || *S.abort_flag) {
                ok = false;
                break;
              }
              tc::tc_fence_after();
              const uint32_t aHi = tc::smem_u32(S.A + st * kAStage), aLo = aHi + kAPart;
              const uint64_t dAh = tc::smem_desc(aHi, 128, 256), dAl = tc::smem_desc(aLo, 128, 256);
              const uint64_t dBh = tc::smem_desc(bHi + kc * 256, 128, sbB);
              const uint64_t dBl = tc::smem_desc(bLo + kc * 256, 128, sbB);
              tc::mma_bf16(d, dAh, dBh, idesc, kc != 0);
              tc::mma_bf16(d, dAh, dBl, idesc, 1);
              tc::mma_bf16(d, dAl, dBh, idesc, 1);
              tc::mma_commit(&empty[st]);
            }
          }
          if (ok) tc::mma_commit(&tfull[buf]);
        }
        if (ok) tc::mma_commit(&bfree[bb]);
      }
      if (!ok) *S.abort_flag = 1;
      tc::mma_commit(done);
      tc::mbar_wait_sleep(done, 0, P.status, 1 << 14);
    }
  } else {
    // ---------------- epilogue (8 warps, named barrier 1) ----------------
    const int nth = kSplitEpiWarps * 32;
    const Tile t = carve_tile(S.tile, kWideQ1, nb);
    const int qd = warp & 3, grp = warp >> 2;   // TMEM lane quarter; group of M tiles drained
    const uint32_t bBytes = (uint32_t)kN * Kp * 2;
    const int qp = P.qp;
    const double sc = P.fp16 ? (double)wide_fp16_scale(P.dmax) : 1.0;
    const double wscale = 1.0 / (sc * sc);
    const int segs = wide_rate_segments(kWideQ1, nb, nth);
    int s = 0;
    for (int n = 0;; ++n) {
      const int slot = n % kItemSlots;
      if (!epi_wait(&ifull[slot], (n / kItemSlots) & 1, S, P, 1 << 15, tid)) break;
      const int item = S.items[slot];
      asm volatile("bar.sync 1, %0;" ::"r"(nth) : "memory");
      if (tid == 0) tc::mbar_arrive(&iempty[slot]);
      if (item < 0) break;
      const int j = item / P.ntiles, tl = item % P.ntiles;
      const int iq2 = P.q2_first + j, iq2m = mesh_neg(iq2, M.n0, M.n1, M.n2);
      wide_load_tile(t, P, tl, iq2, iq2m, tid, nth, 1);
      // phases of the item's q1 into B buffer n & 1, once the MMAs of item n - 2 are done with it
      const int bb = n & 1;
      if (!epi_wait(&bfree[bb], ((n >> 1) & 1) ^ 1, S, P, 1 << 16, tid)) break;
      uint8_t* Bh = S.B + (size_t)bb * 2 * bBytes;
      for (int e = tid; e < kWideQ1 * Kp; e += nth) {
        const int q = e / Kp, k = e % Kp;
        double re = 0.0, im = 0.0;
        if (k < 2 * nr3) {
          const int r = k < nr3 ? k : k - nr3;
          const double* qc = M.qcart + 3 * max(t.q1s[q], 0);
          double sn, cs;
          sincos(-(qc[0] * P.R3[3 * r] + qc[1] * P.R3[3 * r + 1] + qc[2] * P.R3[3 * r + 2]), &sn, &cs);
          re = k < nr3 ? cs : -sn;   // column 2q: Tr = sum Dr cos - Di sin
          im = k < nr3 ? sn : cs;    // column 2q + 1: Ti = sum Dr sin + Di cos
        }
        uint16_t h, l;
        wide_split16(re, P.fp16 != 0, &h, &l);
        uint32_t off = tc::core_offset(2 * q, k, Kp, 2);
        *reinterpret_cast<uint16_t*>(Bh + off) = h;
        *reinterpret_cast<uint16_t*>(Bh + bBytes + off) = l;
        wide_split16(im, P.fp16 != 0, &h, &l);
        off = tc::core_offset(2 * q + 1, k, Kp, 2);
        *reinterpret_cast<uint16_t*>(Bh + off) = h;
        *reinterpret_cast<uint16_t*>(Bh + bBytes + off) = l;
      }
      tc::fence_proxy_async_smem();
      asm volatile("bar.sync 1, %0;" ::"r"(nth) : "memory");
      if (tid == 0) tc::mbar_arrive(&bready[bb]);
      bool ok = true;
      for (int b2 = 0; b2 < nb; ++b2, ++s) {
        const int buf = s & 1;
        if (!epi_wait(&tfull[buf], (s >> 1) & 1, S, P, 1 << 17, tid)) { ok = false; break; }
        tc::tc_fence_after();
        // drain: TMEM lane = row (a, c) of an M tile, column 2q + re/im
        for (int mt = grp; mt < mt_n; mt += kSplitEpiWarps / 4) {
          float v[kN];
          const uint32_t ta = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)buf * bufcols + (uint32_t)mt * kN;
          tc::tmem_ld8(ta, v);
          tc::tmem_ld8(ta + 8, v + 8);
          tc::tmem_wait_ld<16>(v);
          const int row = mt * 128 + qd * 32 + lane;
          if (row < nbb) {
#pragma unroll
            for (int q = 0; q < kWideQ1; ++q) S.T[(size_t)q * nbb + row] = make_float2(v[2 * q], v[2 * q + 1]);
          }
        }
        tc::tc_fence_before();
        asm volatile("bar.sync 1, %0;" ::"r"(nth) : "memory");
        if (tid == 0) tc::mbar_arrive(&tfree[buf]);
        for (int q0 = 0; q0 < kWideQ1; q0 += qp)
          wide_contract<float, float2, RT>(t, q0, qp, nb, P.U32, nullptr, nullptr, S.T, S.X, wide_ldx(nb), tid, nth, 1);
        wide_rates<float>(t, M, kWideQ1, b2, iq2, iq2m, reinterpret_cast<const float*>(S.T), wscale, segs,
                          reinterpret_cast<double*>(S.X), sizeof(float2) * (size_t)qp * nb * wide_ldx(nb), tid, nth,
                          1);
        asm volatile("bar.sync 1, %0;" ::"r"(nth) : "memory");
      }
      if (!ok) break;
      wide_flush(t, P, tid, nth);
      asm volatile("bar.sync 1, %0;" ::"r"(nth) : "memory");
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, tcols);
  }
}

// FP64 Dp of a chunk -> A tiles [j][b2][mt][kc] (hi block, lo block; K-major
// core-matrix layout): row = (a, c) = mt * 128 + r, K = [Re r3 | Im r3 | 0].
// One thread per (row, 8 consecutive K) of a tile.
__global__ void convert_wide_kernel(int nb, int nr3, int Kp, int q2_count, const double2* __restrict__ Dp,
                                    uint8_t* __restrict__ img, int fp16, const unsigned* __restrict__ dmax) {
  const int nbb = nb * nb, nkc = Kp / kAKC, mt_n = split_nt(nb);
  const float sc = fp16 ? wide_fp16_scale(dmax) : 1.f;
  const size_t tiles = (size_t)q2_count * nb * mt_n * nkc;
  for (size_t u = (size_t)blockIdx.x * blockDim.x + threadIdx.x; u < tiles * 256; u += (size_t)gridDim.x * blockDim.x) {
    const size_t tile = u / 256;
    const int w = (int)(u % 256), r = w % 128, kh = w / 128;   // row, which 8-element K half
    const int kc = (int)(tile % nkc), mt = (int)((tile / nkc) % mt_n), b2 = (int)((tile / ((size_t)nkc * mt_n)) % nb);
    const int j = (int)(tile / ((size_t)nkc * mt_n * nb));
    const int row = mt * 128 + r;
    uint16_t hi[8], lo[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = kc * kAKC + kh * 8 + i;
      double v = 0.0;
      if (row < nbb && k < 2 * nr3) {
        const int r3 = k < nr3 ? k : k - nr3, a = row / nb, c = row % nb;
        const double2 d = Dp[(((size_t)j * nr3 + r3) * nb + a) * nbb + (size_t)b2 * nb + c];
        v = (k < nr3 ? d.x : d.y) * (double)sc;
      }
      wide_split16(v, fp16 != 0, &hi[i], &lo[i]);
    }
    uint8_t* base = img + tile * kAStage;
    const uint32_t off = tc::core_offset(r, kh * 8, kAKC, 2);
    uint4 h, l;
    h.x = hi[0] | ((uint32_t)hi[1] << 16); h.y = hi[2] | ((uint32_t)hi[3] << 16);
    h.z = hi[4] | ((uint32_t)hi[5] << 16); h.w = hi[6] | ((uint32_t)hi[7] << 16);
    l.x = lo[0] | ((uint32_t)lo[1] << 16); l.y = lo[2] | ((uint32_t)lo[3] << 16);
    l.z = lo[4] | ((uint32_t)lo[5] << 16); l.w = lo[6] | ((uint32_t)lo[7] << 16);
    *reinterpret_cast<uint4*>(base + off) = h;
    *reinterpret_cast<uint4*>(base + kAPart + off) = l;
  }
}

// Screening features of the pairs (q1, q2) of a q2 range, 12 per pair: the
// fractional coordinates of q1, q2 and q3 = q1 + q2, and the lowest phonon
// energy at each of the three over the largest of the mesh.
__global__ void pair_features_kernel(int nq, int nb, int n0, int n1, int n2, const double* __restrict__ E,
                                     double emax, int q2_first, int q2_count, float* __restrict__ X) {
  const size_t n = (size_t)q2_count * nq;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int q1 = (int)(i % nq), iq2 = q2_first + (int)(i / nq);
    const int iq3 = mesh_add(q1, iq2, n0, n1, n2);
    float* x = X + i * wide::kPairFeatures;
    const int qs[3] = {q1, iq2, iq3};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int q = qs[k];
      x[3 * k] = (float)(q % n0) / n0;
      x[3 * k + 1] = (float)((q / n0) % n1) / n1;
      x[3 * k + 2] = (float)(q / (n0 * n1)) / n2;
      double e = E[(size_t)q * nb];
      for (int b = 1; b < nb; ++b) e = fmin(e, E[(size_t)q * nb + b]);
      x[9 + k] = (float)(e / emax);
    }
  }
}

__global__ void screen_mask_kernel(size_t n, const float* __restrict__ y, float thr, uint8_t* __restrict__ skip,
                                   unsigned long long* __restrict__ nskip) {
  unsigned long long c = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint8_t s = y[i] < thr ? 1 : 0;
    skip[i] = s;
    c += s;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(nskip, c);
}

// FP32 copy of the eigenvector table (the split kernel's contractions)
__global__ void u32_kernel(const double2* __restrict__ U, float2* __restrict__ U32, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    U32[i] = make_float2((float)U[i].x, (float)U[i].y);
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
namespace wide {

int fp64_q1(int nb, int nr3) {
  for (int q : {8, 4, 2})
    if (wide_fp64_smem(q, nb, nr3) <= 227 * 1024) return q;
  return 0;
}
size_t fp64_smem(int nq1, int nb, int nr3) { return wide_fp64_smem(nq1, nb, nr3); }
int split_kp(int nr3) { return ((2 * nr3 + kAKC - 1) / kAKC) * kAKC; }
int split_mtiles(int nb) { return split_nt(nb); }
size_t split_smem(int nb, int Kp, int qp) {
  size_t o[8];
  const size_t b = split_offsets_qp(nb, Kp, qp, o) + 1024;   // + alignment slack of the dynamic base
  return b <= 227 * 1024 ? b : 0;
}
int split_default_qp(int nb, int Kp) { return split_qp(nb, Kp); }
size_t split_img_bytes(int nb, int Kp) { return (size_t)nb * split_nt(nb) * (Kp / kAKC) * kAStage; }

cudaError_t set_attributes(int nb, int nr3, bool split) {
  const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (split) {
    const int sm = (int)split_smem(nb, split_kp(nr3), split_qp(nb, split_kp(nr3)));
    cudaError_t e = cudaFuncSetAttribute(wide_split_kernel<4>, a, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(wide_split_kernel<2>, a, sm);
    return e;
  }
  const int q = fp64_q1(nb, nr3);
  const int sm = (int)wide_fp64_smem(q, nb, nr3);
  cudaError_t e = cudaSuccess;
  if (q == 8) e = cudaFuncSetAttribute(wide_fp64_kernel<8, 2>, a, sm);
  if (q == 4) e = cudaFuncSetAttribute(wide_fp64_kernel<4, 4>, a, sm);
  if (q == 2) e = cudaFuncSetAttribute(wide_fp64_kernel<2, 4>, a, sm);
  return e;
}

int blocks_per_sm(int nb, int nr3, bool split) {
  int n = 0;
  if (split) return 1;   // one CTA (and one TMEM allocation) per SM keeps the buffers whole
  const int q = fp64_q1(nb, nr3);
  const int sm = (int)wide_fp64_smem(q, nb, nr3);
  if (q == 8) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wide_fp64_kernel<8, 2>, kWideThreads, sm);
  if (q == 4) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wide_fp64_kernel<4, 4>, kWideThreads, sm);
  if (q == 2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wide_fp64_kernel<2, 4>, kWideThreads, sm);
  return std::max(1, n);
}

cudaError_t launch_fp64(const Args& A, int grid, cudaStream_t st) {
  const int nb = A.m.nb;
  const size_t sm = wide_fp64_smem(A.nq1, nb, A.nr3);
  if (A.nq1 == 8) wide_fp64_kernel<8, 2><<<grid, kWideThreads, sm, st>>>(A);
  else if (A.nq1 == 4) wide_fp64_kernel<4, 4><<<grid, kWideThreads, sm, st>>>(A);
  else wide_fp64_kernel<2, 4><<<grid, kWideThreads, sm, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_split(const Args& A, int grid, cudaStream_t st) {
  const size_t sm = split_smem(A.m.nb, A.Kp, A.qp);
  if (!sm) return cudaErrorInvalidValue;
  if (A.rt == 4) wide_split_kernel<4><<<grid, kSplitThreads, sm, st>>>(A);
  else wide_split_kernel<2><<<grid, kSplitThreads, sm, st>>>(A);
  return cudaGetLastError();
}

size_t fold_smem(int nb, int max_list) { return fold_wide_smem(nb, max_list); }

cudaError_t launch_fold(int nb, int nr2, int nr3, const double* D3w, const int* r2_ofs, const int* r2_list,
                        int max_list, const double* R2, const double* R3, const double* qcart, const double2* U,
                        int q2_first, int q2_count, double2* Dp, unsigned* dmax, cudaStream_t st) {
  const size_t sm = fold_wide_smem(nb, max_list);
  if (sm > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(fold_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
  }
  dim3 g((q2_count + kFoldWQ - 1) / kFoldWQ, nr3 * nb);
  fold_wide_kernel<<<g, 256, sm, st>>>(nb, nr2, nr3, D3w, r2_ofs, r2_list, R2, R3, qcart, U, q2_first, q2_count, Dp,
                                       dmax);
  return cudaGetLastError();
}

cudaError_t launch_convert(int nb, int nr3, int Kp, int q2_count, const double2* Dp, uint8_t* img, int fp16,
                           const unsigned* dmax, cudaStream_t st) {
  const size_t work = (size_t)q2_count * nb * split_nt(nb) * (Kp / kAKC) * 256;
  const int grid = (int)std::min<size_t>((work + 255) / 256, 148 * 32);
  convert_wide_kernel<<<grid, 256, 0, st>>>(nb, nr3, Kp, q2_count, Dp, img, fp16, dmax);
  return cudaGetLastError();
}

cudaError_t launch_u32(const double2* U, float2* U32, size_t n, cudaStream_t st) {
  u32_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 64), 256, 0, st>>>(U, U32, n);
  return cudaGetLastError();
}

cudaError_t launch_pair_features(int nq, int nb, int n0, int n1, int n2, const double* E, double emax, int q2_first,
                                 int q2_count, float* X, cudaStream_t st) {
  const size_t n = (size_t)q2_count * nq;
  pair_features_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 64), 256, 0, st>>>(
      nq, nb, n0, n1, n2, E, emax, q2_first, q2_count, X);
  return cudaGetLastError();
}

cudaError_t launch_screen_mask(size_t n, const float* y, float log10_threshold, uint8_t* skip,
                               unsigned long long* nskip, cudaStream_t st) {
  screen_mask_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 64), 256, 0, st>>>(n, y, log10_threshold,
                                                                                         skip, nskip);
  return cudaGetLastError();
}

cudaError_t launch_nonzero_blocks(int nb, int nr3, int nr2, const double* D3w, int* flags, cudaStream_t st) {
  const int n = nr3 * nr2;
  nonzero_blocks_kernel<<<std::min(n, 4096), 256, 0, st>>>(nb * nb * nb, n, D3w, flags);
  return cudaGetLastError();
}

}  // namespace wide
