// Tensor-core GEMM on FP32 operands in global memory (tcgen05, sm_100a):
//   C[M,N] (ldc) = sum_k A(m,k) B(k,n) / bscale (+ C when accumulate),
//   A(m,k) = TA ? A[k*lda + m] : A[m*lda + k],  B(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n].
// Operands are staged in shared memory as 16-bit hi + lo pairs (BF16, or FP16
// when F16; B is multiplied by bscale first, a power of 2 that keeps FP16 B in
// range).  RB: B is a weight matrix used as its BF16/FP16 rounding (lo = 0),
// so the product is A_hi B + A_lo B; otherwise hi*hi + lo*hi + hi*lo.  One CTA
// of 128 threads per 128 x 64 tile of C; K in 64-deep chunks, each
// accumulated in FP32 in tensor memory and added to FP32 registers (the
// tensor core's FP32 accumulation runs over 64 terms at a time).  Every wait
// is bounded: on timeout the kernel records a status bit and writes nothing.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tc.cuh"

namespace tcgemm {
// internal linkage: every translation unit that includes this header gets its
// own kernels (no device-side linking between units)
namespace {

constexpr int kTM = 128, kTN = 64, kTKC = 64;     // output tile, K chunk
constexpr uint32_t kGA = kTM * kTKC * 2;          // one of hi / lo of the A tile: 16 KB
constexpr uint32_t kGB = kTN * kTKC * 2;          // one of hi / lo of the B tile: 8 KB
constexpr size_t kSmem = 2 * kGA + 2 * kGB + 64;

template <bool F16>
__device__ __forceinline__ void split2(float v, uint16_t* hi, uint16_t* lo) {
  if (F16) {
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    *hi = __half_as_ushort(h);
    *lo = __half_as_ushort(l);
  } else {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    *hi = __bfloat16_as_ushort(h);
    *lo = __bfloat16_as_ushort(l);
  }
}

template <bool TA, bool TB, bool RB, bool F16>
__global__ void __launch_bounds__(128, 1) gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                      const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                      int ldc, int accumulate, float bscale, int* status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* sA = sm;                  // hi, lo
  uint8_t* sB = sm + 2 * kGA;        // hi, lo
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + 2 * kGB);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, kTN);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  float acc[kTN];
#pragma unroll
  for (int j = 0; j < kTN; ++j) acc[j] = 0.f;
  const uint32_t idesc = F16 ? tc::idesc_f16_f32(kTM, kTN) : tc::idesc_bf16_f32(kTM, kTN);
  const uint32_t sbo = (kTKC / 8) * 128;
  bool ok = true;
  int chunk = 0;
  for (int k0 = 0; k0 < K && ok; k0 += kTKC, ++chunk) {
    // stage the chunk: A rows m, B rows n, both K-major core-matrix layout
    for (int e = tid; e < kTM * kTKC; e += 128) {
      const int mm = TA ? e % kTM : e / kTKC, kk = TA ? e / kTM : e % kTKC;
      const int m = m0 + mm, k = k0 + kk;
      float v = 0.f;
      if (m < M && k < K) v = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
      uint16_t h, l;
      split2<F16>(v, &h, &l);
      const uint32_t off = tc::core_offset(mm, kk, kTKC, 2);
      *reinterpret_cast<uint16_t*>(sA + off) = h;
      *reinterpret_cast<uint16_t*>(sA + kGA + off) = l;
    }
    for (int e = tid; e < kTN * kTKC; e += 128) {
      const int nn = TB ? e / kTKC : e % kTN, kk = TB ? e % kTKC : e / kTN;
      const int n = n0 + nn, k = k0 + kk;
      float v = 0.f;
      if (n < N && k < K) v = (TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n]) * bscale;
      uint16_t h, l;
      split2<F16>(v, &h, &l);
      if (RB) l = 0;
      const uint32_t off = tc::core_offset(nn, kk, kTKC, 2);
      *reinterpret_cast<uint16_t*>(sB + off) = h;
      *reinterpret_cast<uint16_t*>(sB + kGB + off) = l;
    }
    tc::fence_proxy_async_smem();
    tc::tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc::tc_fence_after();
      const uint32_t aHi = tc::smem_u32(sA), aLo = aHi + kGA, bHi = tc::smem_u32(sB), bLo = bHi + kGB;
      for (int ks = 0; ks < kTKC / 16; ++ks) {
        const uint32_t o = ks * 256;
        tc::mma_bf16(tmem, tc::smem_desc(aHi + o, 128, sbo), tc::smem_desc(bHi + o, 128, sbo), idesc, ks != 0);
        tc::mma_bf16(tmem, tc::smem_desc(aLo + o, 128, sbo), tc::smem_desc(bHi + o, 128, sbo), idesc, 1);
        if (!RB) tc::mma_bf16(tmem, tc::smem_desc(aHi + o, 128, sbo), tc::smem_desc(bLo + o, 128, sbo), idesc, 1);
      }
      tc::mma_commit(bar);
    }
    __syncwarp();
    ok = tc::mbar_wait(bar, chunk & 1, status, 1 << 20);
    tc::tc_fence_after();
    if (ok) {
#pragma unroll
      for (int c0 = 0; c0 < kTN; c0 += 8) {
        float v[8];
        tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
        tc::tmem_wait_ld<8>(v);
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[c0 + i] += v[i];
      }
    }
    tc::tc_fence_before();
    ok = __syncthreads_and(ok) != 0;   // smem and TMEM are rewritten by the next chunk
  }
  const int m = m0 + tid;
  if (ok && m < M) {
    const float inv = 1.f / bscale;
    float* c = C + (size_t)m * ldc + n0;
#pragma unroll
    for (int j = 0; j < kTN; ++j)
      if (n0 + j < N) c[j] = accumulate ? c[j] + acc[j] * inv : acc[j] * inv;
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, kTN);
  }
}

template <bool TA, bool TB, bool RB, bool F16>
inline cudaError_t launch(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
                          int accumulate, float bscale, int* status, cudaStream_t st) {
  static bool attr = false;   // per instantiation, once per process
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(gemm_kernel<TA, TB, RB, F16>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  if (M <= 0 || N <= 0) return cudaSuccess;
  dim3 grid((N + kTN - 1) / kTN, (M + kTM - 1) / kTM);
  gemm_kernel<TA, TB, RB, F16><<<grid, 128, kSmem, st>>>(M, N, K, A, lda, B, ldb, C, ldc, accumulate, bscale, status);
  return cudaGetLastError();
}

}  // namespace
}  // namespace tcgemm
