// Split-precision (BF16 x3) tensor-core form of the dominant step of
// calcCouplingSquared (interaction_elph.cpp:364-374): for a batch of k1 and
// every q of the phonon mesh,
//   g3(q; k1, nu, b1, w2) = sum_Rp e^{+i q3.Rp}/deg_Rp cached_k1(Rp; nu, b1, w2),  q3 = k2 - k1,
// as one real GEMM  D[q][n] = sum_k A[q][k] B[n][k]  with
//   A[q][k]  = [cos | sin](q.Rp)/deg_Rp            (K = 2 nRp, padded to kKC)
//   B[2x][k] = [Re c ; -Im c],  B[2x+1][k] = [Im c ; Re c]   x = (k1, nu, b1, w2)
// so D[q][2x] + i D[q][2x+1] = g3(q; x).  The phase depends on q3 only modulo
// a reciprocal lattice vector (Rp are Bravais vectors), and k2 - k1 equals the
// phonon mesh point q modulo one, so A is built once per call and shared by
// every k1.
//
// Both operands are split x = hi + lo in BF16 and laid out in global memory as
// the shared-memory images of their tiles (K-major core matrices), so that one
// bulk copy moves a tile's K chunk.  The GEMM is persistent and warp
// specialised: one producer warp (bulk copies into a kStages ring), one MMA
// warp (hi*hi + hi*lo + lo*hi per K step, FP32 accumulators in tensor memory,
// two buffers of 256 columns) and four epilogue warps that drain a buffer
// while the next tile accumulates into the other.  The epilogue writes g3
// transposed, g3T[x][q] (complex FP32), so that a warp stores 32 consecutive
// q of one x and the pair kernel reads its q of one x contiguously.
#include <algorithm>
#include <cuda_bf16.h>

#include "phx_internal.h"
#include "tc.cuh"

namespace {

constexpr int kM = 128;        // q per tile
constexpr int kN = 256;        // real columns per tile
constexpr int kKC = 32;        // K per stage (two MMA K-steps)
constexpr int kStages = 4;
constexpr uint32_t kABytes = kM * kKC * 2 * 2;   // hi + lo
constexpr uint32_t kBBytes = kN * kKC * 2 * 2;
constexpr uint32_t kStageBytes = kABytes + kBBytes;
constexpr int kThreads = 192;  // producer, MMA, 4 epilogue warps
constexpr int kMaxBatch = 16;

__device__ __forceinline__ void split8(const double* v, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat16 h0 = __double2bfloat16(v[2 * i]), h1 = __double2bfloat16(v[2 * i + 1]);
    const __nv_bfloat16 l0 = __double2bfloat16(v[2 * i] - (double)__bfloat162float(h0));
    const __nv_bfloat16 l1 = __double2bfloat16(v[2 * i + 1] - (double)__bfloat162float(h1));
    h[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
    l[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// A image: tile (mt, kc) = [hi 128 x kKC | lo 128 x kKC]; one thread per
// 16-byte chunk (8 consecutive k of one q).
__global__ void el_phase_image_kernel(int nq, const double* __restrict__ qcart, int nRp, const double* __restrict__ Rp, const double* __restrict__ degP,
                                      int nKC, uint8_t* __restrict__ img, int nMT) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)nMT * nKC * kM * (kKC / 8);
  if (t >= total) return;
  const int ch = (int)(t % (kKC / 8));
  const int m = (int)((t / (kKC / 8)) % kM);
  const int kc = (int)((t / (kKC / 8 * kM)) % nKC);
  const int mt = (int)(t / ((long long)kKC / 8 * kM * nKC));
  const int iq = mt * kM + m;
  double v[8];
  double qc[3] = {0.0, 0.0, 0.0};
  if (iq < nq)
    for (int c = 0; c < 3; ++c) qc[c] = qcart[3 * iq + c];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = kc * kKC + ch * 8 + i;
    v[i] = 0.0;
    if (iq < nq && k < 2 * nRp) {
      const int r = k < nRp ? k : k - nRp;
      double sn, cs;
      sincos(qc[0] * Rp[3 * r] + qc[1] * Rp[3 * r + 1] + qc[2] * Rp[3 * r + 2], &sn, &cs);
      v[i] = (k < nRp ? cs : sn) / degP[r];
    }
  }
  uint4 hi, lo;
  split8(v, hi, lo);
  uint8_t* tile = img + ((size_t)mt * nKC + kc) * kABytes;
  const uint32_t off = tc::core_offset(m, ch * 8, kKC, 2);
  *reinterpret_cast<uint4*>(tile + off) = hi;
  *reinterpret_cast<uint4*>(tile + kABytes / 2 + off) = lo;
}

struct BatchCols {
  int nb;                       // k1 in the batch
  int xoff[kMaxBatch + 1];      // first complex column of each k1
  int nb1[kMaxBatch];           // active bands of each k1
};

// B image of a batch: tile (nt, kc) = [hi 256 x kKC | lo 256 x kKC]
__global__ void el_coupling_image_kernel(const double2* __restrict__ cached, size_t per, int nRp, int nph, int nw,
                                         BatchCols cols, int nKC, int nNT, uint8_t* __restrict__ img) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)nNT * nKC * kN * (kKC / 8);
  if (t >= total) return;
  const int ch = (int)(t % (kKC / 8));
  const int n = (int)((t / (kKC / 8)) % kN);
  const int kc = (int)((t / (kKC / 8 * kN)) % nKC);
  const int nt = (int)(t / ((long long)kKC / 8 * kN * nKC));
  const int col = nt * kN + n, xg = col >> 1, c = col & 1;
  int j = -1;
  for (int i = 0; i < cols.nb; ++i)
    if (xg >= cols.xoff[i] && xg < cols.xoff[i + 1]) j = i;
  double v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = 0.0;
  if (j >= 0) {
    const int x = xg - cols.xoff[j], nb1 = cols.nb1[j];
    const int w2 = x % nw, b1 = (x / nw) % nb1, nu = x / (nw * nb1);
    const double2* src = cached + (size_t)j * per + ((size_t)nu * nw + b1) * nw + w2;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = kc * kKC + ch * 8 + i;
      if (k < 2 * nRp) {
        const int r = k < nRp ? k : k - nRp;
        const double2 z = src[(size_t)r * nph * nw * nw];
        v[i] = k < nRp ? (c == 0 ? z.x : z.y) : (c == 0 ? -z.y : z.x);
      }
    }
  }
  uint4 hi, lo;
  split8(v, hi, lo);
  uint8_t* tile = img + ((size_t)nt * nKC + kc) * kBBytes;
  const uint32_t off = tc::core_offset(n, ch * 8, kKC, 2);
  *reinterpret_cast<uint4*>(tile + off) = hi;
  *reinterpret_cast<uint4*>(tile + kBBytes / 2 + off) = lo;
}

struct GemmArgs {
  const uint8_t* Aimg;
  const uint8_t* Bimg;
  int nMT, nNT, nKC;
  float2* g3T;        // (xcols, ldq)
  int ldq;            // nMT * kM
  int xcols;          // complex columns written (x < xcols)
  int* status;
};

__global__ void __launch_bounds__(kThreads, 1) el_gemm_kernel(GemmArgs P) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* stage = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* full = bars;                  // [kStages]
  uint64_t* empty = bars + kStages;       // [kStages]
  uint64_t* accf = bars + 2 * kStages;    // [2] accumulator ready
  uint64_t* acce = accf + 2;              // [2] accumulator drained
  uint64_t* done = acce + 2;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&accf[b], 1);
      tc::mbar_init(&acce[b], 4);
    }
    tc::mbar_init(done, 1);
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, 512);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const int ntiles = P.nMT * P.nNT;
  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      int it = 0;
      for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x) {
        const int mt = tile / P.nNT, nt = tile % P.nNT;
        for (int kc = 0; kc < P.nKC; ++kc, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (!tc::mbar_wait_sleep(&empty[s], ph ^ 1, P.status, 1)) { *abort_flag = 1; break; }
          tc::mbar_arrive_expect_tx(&full[s], kStageBytes);
          tc::bulk_g2s(stage + (size_t)s * kStageBytes, P.Aimg + ((size_t)mt * P.nKC + kc) * kABytes, kABytes,
                       &full[s]);
          tc::bulk_g2s(stage + (size_t)s * kStageBytes + kABytes, P.Bimg + ((size_t)nt * P.nKC + kc) * kBBytes,
                       kBBytes, &full[s]);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_bf16_f32(kM, kN);
      const uint32_t sbo = (kKC / 8) * 128;
      int it = 0, lt = 0;
      for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x, ++lt) {
        const int b = lt & 1;
        if (!tc::mbar_wait_sleep(&acce[b], ((lt >> 1) & 1) ^ 1, P.status, 2)) { *abort_flag = 1; break; }
        tc::tc_fence_after();
        const uint32_t d = tmem + b * kN;
        bool ok = true;
        for (int kc = 0; kc < P.nKC; ++kc, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (!tc::mbar_wait_sleep(&full[s], ph, P.status, 4)) { ok = false; break; }
          tc::tc_fence_after();
          const uint32_t aHi = tc::smem_u32(stage + (size_t)s * kStageBytes), aLo = aHi + kABytes / 2;
          const uint32_t bHi = aHi + kABytes, bLo = bHi + kBBytes / 2;
#pragma unroll
          for (int ks = 0; ks < kKC / 16; ++ks) {
            const uint64_t dAh = tc::smem_desc(aHi + ks * 256, 128, sbo);
            const uint64_t dAl = tc::smem_desc(aLo + ks * 256, 128, sbo);
            const uint64_t dBh = tc::smem_desc(bHi + ks * 256, 128, sbo);
            const uint64_t dBl = tc::smem_desc(bLo + ks * 256, 128, sbo);
            tc::mma_bf16(d, dAh, dBh, idesc, (kc | ks) != 0);
            tc::mma_bf16(d, dAh, dBl, idesc, 1);
            tc::mma_bf16(d, dAl, dBh, idesc, 1);
          }
          tc::mma_commit(&empty[s]);
        }
        if (!ok) { *abort_flag = 1; break; }
        tc::mma_commit(&accf[b]);
      }
      // every issued MMA has completed before TMEM is released
      tc::mma_commit(done);
      tc::mbar_wait_sleep(done, 0, P.status, 8);
    }
  } else {
    // ---------------- epilogue: TMEM -> g3T ----------------
    const int qd = warp & 3;
    int lt = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++lt) {
      const int b = lt & 1;
      if (*abort_flag) break;
      if (!tc::mbar_wait_sleep(&accf[b], (lt >> 1) & 1, P.status, 16)) { *abort_flag = 1; break; }
      tc::tc_fence_after();
      const int mt = tile / P.nNT, nt = tile % P.nNT;
      const int iq = mt * kM + qd * 32 + lane;
      const uint32_t base = tmem + ((uint32_t)(qd * 32) << 16) + b * kN;
      const int x0 = nt * (kN / 2);
#pragma unroll 2
      for (int c0 = 0; c0 < kN; c0 += 16) {
        float v[16];
        tc::tmem_ld8(base + c0, v);
        tc::tmem_ld8(base + c0 + 8, v + 8);
        tc::tmem_wait_ld<16>(v);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int x = x0 + c0 / 2 + i;
          if (x < P.xcols) P.g3T[(size_t)x * P.ldq + iq] = make_float2(v[2 * i], v[2 * i + 1]);
        }
      }
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&acce[b]);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------------------
// cacheElPh first step on the tensor cores (interaction_elph.cpp:540-580):
//   g1(k1; x) = sum_Re e^{+i k1.Re}/deg_Re g(Re; x),   x = (Rp, nu, w1, w2)
// as D[x][n] = sum_k A[x][k] B[n][k] with A[x][k] = [Re g | Im g](Re; x)
// (the coupling tensor itself, split once into a BF16 hi/lo image) and
// B[2j] = [cos ; -sin], B[2j+1] = [sin ; cos] of k1 j (32 columns, 16 k1: each
// pass over the 371 MB image of g serves 16 k1).
// The tensor core's FP32 accumulation rounds toward zero, which biases long
// sums; here every 64-deep K chunk goes to its own TMEM buffer (one of
// kG1Bufs in turn) and the epilogue adds the chunk sums in FP64 registers.
// ---------------------------------------------------------------------------
constexpr int kKC1 = 64;
constexpr int kG1Stages = 3;
constexpr int kG1N = 2 * kMaxBatch;                       // 32 real columns
constexpr uint32_t kA1Bytes = kM * kKC1 * 2 * 2;          // 32 KB per (tile, chunk)
constexpr uint32_t kB1Bytes = kG1N * kKC1 * 2 * 2;        // 8 KB per chunk
constexpr int kG1Bufs = 8;
constexpr int kG1MaxKC = 16;                              // nRe <= 512

// A image of the coupling tensor: tile (mt, kc) = [hi 128 x kKC1 | lo 128 x kKC1];
// consecutive threads take consecutive rows, so the reads of g are coalesced.
__global__ void el_g_image_kernel(const float2* __restrict__ g, int nRe, long long N, int nKC, int nMT,
                                  uint8_t* __restrict__ img) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)nMT * nKC * kM * (kKC1 / 8);
  if (t >= total) return;
  const int m = (int)(t % kM);
  const int ch = (int)((t / kM) % (kKC1 / 8));
  const int kc = (int)((t / ((long long)kM * (kKC1 / 8))) % nKC);
  const int mt = (int)(t / ((long long)kM * (kKC1 / 8) * nKC));
  const long long x = (long long)mt * kM + m;
  double v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = kc * kKC1 + ch * 8 + i;
    v[i] = 0.0;
    if (x < N && k < 2 * nRe) {
      const int r = k < nRe ? k : k - nRe;
      const float2 z = g[(size_t)r * N + x];
      v[i] = k < nRe ? (double)z.x : (double)z.y;
    }
  }
  uint4 hi, lo;
  split8(v, hi, lo);
  uint8_t* tile = img + ((size_t)mt * nKC + kc) * kA1Bytes;
  const uint32_t off = tc::core_offset(m, ch * 8, kKC1, 2);
  *reinterpret_cast<uint4*>(tile + off) = hi;
  *reinterpret_cast<uint4*>(tile + kA1Bytes / 2 + off) = lo;
}

// B image of a batch: chunk kc = [hi kG1N x kKC1 | lo kG1N x kKC1]
__global__ void el_k1_phase_image_kernel(const double* __restrict__ k1s, int nb, int nRe,
                                         const double* __restrict__ Re, const double* __restrict__ degE, int nKC,
                                         uint8_t* __restrict__ img) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nKC * kG1N * (kKC1 / 8)) return;
  const int n = t % kG1N, ch = (t / kG1N) % (kKC1 / 8), kc = t / (kG1N * (kKC1 / 8));
  const int j = n >> 1, c = n & 1;
  double v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = kc * kKC1 + ch * 8 + i;
    v[i] = 0.0;
    if (j < nb && k < 2 * nRe) {
      const int r = k < nRe ? k : k - nRe;
      const double* kk = k1s + 3 * j;
      double sn, cs;
      sincos(kk[0] * Re[3 * r] + kk[1] * Re[3 * r + 1] + kk[2] * Re[3 * r + 2], &sn, &cs);
      cs /= degE[r];
      sn /= degE[r];
      v[i] = k < nRe ? (c == 0 ? cs : sn) : (c == 0 ? -sn : cs);
    }
  }
  uint4 hi, lo;
  split8(v, hi, lo);
  uint8_t* tile = img + (size_t)kc * kB1Bytes;
  const uint32_t off = tc::core_offset(n, ch * 8, kKC1, 2);
  *reinterpret_cast<uint4*>(tile + off) = hi;
  *reinterpret_cast<uint4*>(tile + kB1Bytes / 2 + off) = lo;
}

struct G1Args {
  const uint8_t* Aimg;
  const uint8_t* Bimg;
  int nMT, nKC;
  long long N;       // rows x
  int nb;            // k1 in the batch
  double2* g1;       // (nb, N)
  int* status;
};

__global__ void __launch_bounds__(kThreads, 1) el_g1_gemm_kernel(G1Args P) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* stage = smem;                                     // kG1Stages x kA1Bytes
  uint8_t* Bs = smem + kG1Stages * kA1Bytes;                 // nKC x kB1Bytes
  uint64_t* bars = reinterpret_cast<uint64_t*>(Bs + kG1MaxKC * kB1Bytes);
  uint64_t* full = bars;
  uint64_t* empty = full + kG1Stages;
  uint64_t* accf = empty + kG1Stages;                        // [kG1Bufs]
  uint64_t* acce = accf + kG1Bufs;                           // [kG1Bufs]
  uint64_t* bfull = acce + kG1Bufs;
  uint64_t* done = bfull + 1;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < kG1Stages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < kG1Bufs; ++b) {
      tc::mbar_init(&accf[b], 1);
      tc::mbar_init(&acce[b], 4);
    }
    tc::mbar_init(bfull, 1);
    tc::mbar_init(done, 1);
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, kG1Bufs * kG1N);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      tc::mbar_arrive_expect_tx(bfull, P.nKC * kB1Bytes);
      tc::bulk_g2s(Bs, P.Bimg, P.nKC * kB1Bytes, bfull);
      int it = 0;
      for (int mt = blockIdx.x; mt < P.nMT && !*abort_flag; mt += gridDim.x) {
        for (int kc = 0; kc < P.nKC; ++kc, ++it) {
          const int s = it % kG1Stages;
          const uint32_t ph = (it / kG1Stages) & 1;
          if (!tc::mbar_wait_sleep(&empty[s], ph ^ 1, P.status, 1)) { *abort_flag = 1; break; }
          tc::mbar_arrive_expect_tx(&full[s], kA1Bytes);
          tc::bulk_g2s(stage + (size_t)s * kA1Bytes, P.Aimg + ((size_t)mt * P.nKC + kc) * kA1Bytes, kA1Bytes,
                       &full[s]);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_bf16_f32(kM, kG1N);
      const uint32_t sbo = (kKC1 / 8) * 128;
      bool ok = tc::mbar_wait_sleep(bfull, 0, P.status, 2);
      tc::tc_fence_after();
      const uint32_t bBase = tc::smem_u32(Bs);
      int it = 0;
      for (int mt = blockIdx.x; ok && mt < P.nMT && !*abort_flag; mt += gridDim.x) {
        for (int kc = 0; kc < P.nKC; ++kc, ++it) {
          const int buf = it % kG1Bufs, s = it % kG1Stages;
          if (!tc::mbar_wait_sleep(&acce[buf], ((it / kG1Bufs) & 1) ^ 1, P.status, 2)) { ok = false; break; }
          if (!tc::mbar_wait_sleep(&full[s], (it / kG1Stages) & 1, P.status, 4)) { ok = false; break; }
          tc::tc_fence_after();
          const uint32_t aHi = tc::smem_u32(stage + (size_t)s * kA1Bytes), aLo = aHi + kA1Bytes / 2;
          const uint32_t bHi = bBase + kc * kB1Bytes, bLo = bHi + kB1Bytes / 2;
          const uint32_t d = tmem + buf * kG1N;
#pragma unroll
          for (int ks = 0; ks < kKC1 / 16; ++ks) {
            const uint64_t dAh = tc::smem_desc(aHi + ks * 256, 128, sbo);
            const uint64_t dAl = tc::smem_desc(aLo + ks * 256, 128, sbo);
            const uint64_t dBh = tc::smem_desc(bHi + ks * 256, 128, sbo);
            const uint64_t dBl = tc::smem_desc(bLo + ks * 256, 128, sbo);
            tc::mma_bf16(d, dAh, dBh, idesc, ks != 0);
            tc::mma_bf16(d, dAh, dBl, idesc, 1);
            tc::mma_bf16(d, dAl, dBh, idesc, 1);
          }
          tc::mma_commit(&empty[s]);
          tc::mma_commit(&accf[buf]);
        }
      }
      if (!ok) *abort_flag = 1;
      tc::mma_commit(done);
      tc::mbar_wait_sleep(done, 0, P.status, 8);
    }
  } else {
    // ---------------- epilogue: chunk sums -> FP64 registers -> g1 ----------------
    const int qd = warp & 3;
    const uint32_t lanes = (uint32_t)(qd * 32) << 16;
    int it = 0;
    for (int mt = blockIdx.x; mt < P.nMT; mt += gridDim.x) {
      double acc[kG1N];
#pragma unroll
      for (int i = 0; i < kG1N; ++i) acc[i] = 0.0;
      bool ok = true;
      for (int kc = 0; kc < P.nKC; ++kc, ++it) {
        const int buf = it % kG1Bufs;
        if (*abort_flag || !tc::mbar_wait_sleep(&accf[buf], (it / kG1Bufs) & 1, P.status, 16)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        float v[kG1N];
#pragma unroll
        for (int i = 0; i < kG1N; i += 8) tc::tmem_ld8(tmem + lanes + buf * kG1N + i, v + i);
        tc::tmem_wait_ld<kG1N>(v);
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&acce[buf]);
#pragma unroll
        for (int i = 0; i < kG1N; ++i) acc[i] += (double)v[i];
      }
      if (!ok) {
        *abort_flag = 1;
        break;
      }
      const long long x = (long long)mt * kM + qd * 32 + lane;
      if (x < P.N) {
#pragma unroll
        for (int j = 0; j < kMaxBatch; ++j)
          if (j < P.nb) P.g1[(size_t)j * P.N + x] = make_double2(acc[2 * j], acc[2 * j + 1]);
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, kG1Bufs * kG1N);
  }
}

}  // namespace

// Geometry of the split el-ph GEMM for nRp phonon vectors and nq q points.
void phx_el_split_dims(int nRp, int nq, int* nKC, int* nMT) {
  *nKC = (2 * nRp + kKC - 1) / kKC;
  *nMT = (nq + kM - 1) / kM;
}
size_t phx_el_split_phase_bytes(int nRp, int nq) {
  int nKC, nMT;
  phx_el_split_dims(nRp, nq, &nKC, &nMT);
  return (size_t)nMT * nKC * kABytes;
}
// B image and g3T sizes for a batch of up to kMaxBatch k1 with xmax complex columns
size_t phx_el_split_coupling_bytes(int nRp, int xmax) {
  int nKC, nMT;
  phx_el_split_dims(nRp, 1, &nKC, &nMT);
  const int nNT = (2 * xmax + kN - 1) / kN;
  return (size_t)nNT * nKC * kBBytes;
}
int phx_el_split_max_batch() { return kMaxBatch; }

// A image (phases of the nq Cartesian q points of the phonon mesh), once per linewidth call
int phx_el_split_phases(phx_ctx* ctx, int nq, const double* qcart, int nRp, const double* Rp, const double* degP,
                        uint8_t* img) {
  int nKC, nMT;
  phx_el_split_dims(nRp, nq, &nKC, &nMT);
  const long long total = (long long)nMT * nKC * kM * (kKC / 8);
  el_phase_image_kernel<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(
      nq, qcart, nRp, Rp, degP, nKC, img, nMT);
  PHX_CUDA(ctx, cudaGetLastError());
  return PHX_OK;
}

// g3T (xcols, ldq) of a batch of k1: cached (nb, per) of nb1[j] active bands,
// complex column x of k1 j at xoff[j] + (nu, b1, w2).  Two launches.
int phx_el_split_g3_batch(phx_ctx* ctx, const uint8_t* Aimg, uint8_t* Bimg, const double2* cached, size_t per,
                          int nRp, int nph, int nw, int nq, int nb, const int* nb1, float2* g3T, int* ldq_out,
                          int* xoff_out) {
  PHX_ARG(ctx, nb >= 1 && nb <= kMaxBatch, "split el-ph GEMM: batch of 1..16 k1");
  BatchCols cols;
  cols.nb = nb;
  cols.xoff[0] = 0;
  for (int j = 0; j < nb; ++j) {
    cols.nb1[j] = nb1[j];
    cols.xoff[j + 1] = cols.xoff[j] + nph * nb1[j] * nw;
    xoff_out[j] = cols.xoff[j];
  }
  for (int j = nb; j < kMaxBatch; ++j) {
    cols.nb1[j] = 1;
    cols.xoff[j + 1] = cols.xoff[nb];
  }
  const int xcols = cols.xoff[nb];
  int nKC, nMT;
  phx_el_split_dims(nRp, nq, &nKC, &nMT);
  const int nNT = (2 * xcols + kN - 1) / kN;
  const long long total = (long long)nNT * nKC * kN * (kKC / 8);
  el_coupling_image_kernel<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(cached, per, nRp, nph, nw, cols,
                                                                                     nKC, nNT, Bimg);
  PHX_CUDA(ctx, cudaGetLastError());
  GemmArgs G;
  G.Aimg = Aimg;
  G.Bimg = Bimg;
  G.nMT = nMT;
  G.nNT = nNT;
  G.nKC = nKC;
  G.g3T = g3T;
  G.ldq = nMT * kM;
  G.xcols = xcols;
  G.status = ctx->d_status;
  *ldq_out = G.ldq;
  const size_t smem = (size_t)kStages * kStageBytes + 256;
  PHX_CUDA(ctx, cudaFuncSetAttribute(el_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::min(nMT * nNT, std::max(1, ctx->num_sms));
  el_gemm_kernel<<<grid, kThreads, smem, ctx->stream>>>(G);
  PHX_CUDA(ctx, cudaGetLastError());
  return PHX_OK;
}

// ---------------------------------------------------------------------------
// cacheElPh g1 on the tensor cores
// ---------------------------------------------------------------------------
size_t phx_el_split_g_image_bytes(int nRe, long long N) {
  const int nKC = (2 * nRe + kKC1 - 1) / kKC1;
  const long long nMT = (N + kM - 1) / kM;
  return (size_t)nMT * nKC * kA1Bytes;
}
size_t phx_el_split_k1_image_bytes() { return (size_t)kG1MaxKC * kB1Bytes; }

// the split image of the coupling tensor g (nRe, N) complex FP32, built once per coupling object
int phx_el_split_g_image(phx_ctx* ctx, const float* g, int nRe, long long N, uint8_t* img) {
  const int nKC = (2 * nRe + kKC1 - 1) / kKC1;
  PHX_ARG(ctx, nKC <= kG1MaxKC, "split el-ph path: at most 512 electron Bravais vectors");
  const int nMT = (int)((N + kM - 1) / kM);
  const long long total = (long long)nMT * nKC * kM * (kKC1 / 8);
  el_g_image_kernel<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(reinterpret_cast<const float2*>(g),
                                                                              nRe, N, nKC, nMT, img);
  PHX_CUDA(ctx, cudaGetLastError());
  return PHX_OK;
}

// g1 (nb, N) of a batch of nb <= 16 k1 (Cartesian coordinates k1s on the device)
// from the split image of g; kimg is scratch of phx_el_split_k1_image_bytes().  Two launches.
int phx_el_split_g1(phx_ctx* ctx, const uint8_t* gimg, int nRe, long long N, const double* Re, const double* degE,
                    int nb, const double* k1s, uint8_t* kimg, double2* g1) {
  const int nKC = (2 * nRe + kKC1 - 1) / kKC1;
  PHX_ARG(ctx, nKC <= kG1MaxKC && nb >= 1 && nb <= kMaxBatch, "split el-ph g1: nRe <= 512 and 1..16 k1");
  const int nMT = (int)((N + kM - 1) / kM);
  const int tb = nKC * kG1N * (kKC1 / 8);
  el_k1_phase_image_kernel<<<(tb + 255) / 256, 256, 0, ctx->stream>>>(k1s, nb, nRe, Re, degE, nKC, kimg);
  PHX_CUDA(ctx, cudaGetLastError());
  G1Args G;
  G.Aimg = gimg;
  G.Bimg = kimg;
  G.nMT = nMT;
  G.nKC = nKC;
  G.N = N;
  G.nb = nb;
  G.g1 = g1;
  G.status = ctx->d_status;
  const size_t smem = (size_t)kG1Stages * kA1Bytes + (size_t)kG1MaxKC * kB1Bytes + 512;
  PHX_CUDA(ctx, cudaFuncSetAttribute(el_g1_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::min(nMT, std::max(1, ctx->num_sms));
  el_g1_gemm_kernel<<<grid, kThreads, smem, ctx->stream>>>(G);
  PHX_CUDA(ctx, cudaGetLastError());
  return PHX_OK;
}
