// Interaction3Ph on the GPU: construction, cacheD3 and getCouplingsSquared.
//
// Follows src/interaction/interaction_3ph.cpp of mir-group/phoebe:
//   cacheD3 (:100-175):
//     D3+(abc,r3) = sum_r2 D3(abc,r3,r2) e^{+i q2.R2} e^{-i q2.R3} w2(r2,a,b) w3(r3,a,c)
//     D3-(abc,r3) = sum_r2 D3(abc,r3,r2) e^{-i q2.R2} e^{+i q2.R3} w2(r2,a,b) w3(r3,a,c)
//   getCouplingsSquared (:179-405):
//     T+-(abc) = sum_r3 D3+-(abc,r3) e^{-i q1.R3} w3(r3,a,c)   (w3 a second time)
//     V+ = sum T+ e1(a,b1) e2(b,b2) conj(e3+(c,b3))
//     V- = sum T- e1(a,b1) conj(e2(b,b2)) conj(e3-(c,b3));  output |V|^2
// This is the drop-in call-by-call path (one q2, a batch of q1).  The fused
// builder in builder.cu restructures the same arithmetic for whole meshes.
// With a split precision set on the object (phx_v3_set_precision), the R3
// transform of the whole q1 batch runs as one tensor-core GEMM (tcgemm.cuh,
// FP16 or BF16 hi/lo operands, FP32 accumulation) and the contractions with
// the eigenvectors stay in FP64.
#include <algorithm>
#include <cmath>

#include <cstring>

#include "cplx.cuh"
#include "phx_internal.h"
#include "tcgemm.cuh"

namespace {

__global__ void cache_d3_kernel(int nb, int nat, int nr2, int nr3, const double* __restrict__ D3,
                                const double* __restrict__ R2, const double* __restrict__ R3,
                                const double* __restrict__ w2, const double* __restrict__ w3,
                                double q20, double q21, double q22, double2* __restrict__ plus,
                                double2* __restrict__ mins) {
  extern __shared__ double2 ph2[];  // nr2 phases e^{+i q2.R2}
  for (int r = threadIdx.x; r < nr2; r += blockDim.x) {
    double sn, cs;
    sincos(q20 * R2[3 * r] + q21 * R2[3 * r + 1] + q22 * R2[3 * r + 2], &sn, &cs);
    ph2[r] = cmk(cs, sn);
  }
  __syncthreads();
  const long total = (long)nb * nb * nb * nr3;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int ir3 = idx % nr3;
    const long abc = idx / nr3;
    const int i3 = abc % nb, i2 = (abc / nb) % nb, i1 = abc / (nb * nb);
    const int at1 = i1 / 3, at2 = i2 / 3, at3 = i3 / 3;
    double sn, cs;
    sincos(q20 * R3[3 * ir3] + q21 * R3[3 * ir3 + 1] + q22 * R3[3 * ir3 + 2], &sn, &cs);
    const double2 p3p = cmk(cs, -sn), p3m = cmk(cs, sn);
    const double ww3 = w3[((size_t)ir3 * nat + at1) * nat + at3];
    double2 tp = cmk(0, 0), tm = cmk(0, 0);
    const double* d = D3 + idx * nr2;
    for (int r2 = 0; r2 < nr2; ++r2) {
      const double f = d[r2] * w2[((size_t)r2 * nat + at1) * nat + at2] * ww3;
      tp = cadd(tp, cscale(cmul(ph2[r2], p3p), f));
      tm = cadd(tm, cscale(cmul(cconj(ph2[r2]), p3m), f));
    }
    plus[idx] = tp;
    mins[idx] = tm;
  }
}

// One block per q1: stage T+- (nb^3 complex each) in shared memory, then
// contract with e1, e2, e3 and write |V|^2.  Shared memory limits this
// call-by-call path to nb <= 15; wider cells use the fused builder.
// Tg (split precision): T+- of every q1 from the tensor-core GEMM, FP32,
// row iq = [(+, abc, re/im) | (-, abc, re/im)]; null: the FP64 R3 sum here.
__global__ void couplings_kernel(int nb, int nat, int nr3, const double2* __restrict__ plus,
                                 const double2* __restrict__ mins, const double* __restrict__ R3,
                                 const double* __restrict__ w3, const double* __restrict__ q1s,
                                 const double2* __restrict__ ev1, const int* __restrict__ nb1s,
                                 const double2* __restrict__ ev2, int nb2,
                                 const double2* __restrict__ ev3p, const int* __restrict__ nb3ps,
                                 const double2* __restrict__ ev3m, const int* __restrict__ nb3ms,
                                 const long* __restrict__ offP, const long* __restrict__ offM,
                                 double* __restrict__ outP, double* __restrict__ outM,
                                 const float* __restrict__ Tg) {
  extern __shared__ double2 sm[];
  const int iq = blockIdx.x;
  const int n3 = nb * nb * nb;
  double2* tP = sm;
  double2* tM = sm + n3;
  double2* ph = sm + 2 * n3;           // nr3
  double2* xP = ph + nr3;              // (nb1, nb, nb) scratch
  double2* xM = xP + n3;
  const double* q1 = q1s + 3 * iq;
  if (Tg) {
    const float* tg = Tg + (size_t)iq * 4 * n3;
    for (int abc = threadIdx.x; abc < n3; abc += blockDim.x) {
      tP[abc] = cmk((double)tg[2 * abc], (double)tg[2 * abc + 1]);
      tM[abc] = cmk((double)tg[2 * (n3 + abc)], (double)tg[2 * (n3 + abc) + 1]);
    }
  }
  for (int r = threadIdx.x; r < nr3 && !Tg; r += blockDim.x) {
    double sn, cs;
    sincos(-(q1[0] * R3[3 * r] + q1[1] * R3[3 * r + 1] + q1[2] * R3[3 * r + 2]), &sn, &cs);
    ph[r] = cmk(cs, sn);
  }
  __syncthreads();
  for (int abc = threadIdx.x; abc < n3 && !Tg; abc += blockDim.x) {
    const int a3 = abc % nb, a1 = abc / (nb * nb);
    const int at1 = a1 / 3, at3 = a3 / 3;
    double2 sp = cmk(0, 0), sq = cmk(0, 0);
    for (int r = 0; r < nr3; ++r) {
      const double ww = w3[((size_t)r * nat + at1) * nat + at3];
      const double2 f = cscale(ph[r], ww);
      cfma(sp, plus[(size_t)abc * nr3 + r], f);
      cfma(sq, mins[(size_t)abc * nr3 + r], f);
    }
    tP[abc] = sp;
    tM[abc] = sq;
  }
  __syncthreads();
  const int nb1 = nb1s[iq], nb3p = nb3ps[iq], nb3m = nb3ms[iq];
  const double2* e1 = ev1 + (size_t)iq * nb * nb;
  const double2* e3p = ev3p + (size_t)iq * nb * nb;
  const double2* e3m = ev3m + (size_t)iq * nb * nb;
  // x(b1, a2, a3) = sum_a1 T(a1,a2,a3) e1(a1,b1)
  for (int idx = threadIdx.x; idx < nb1 * nb * nb; idx += blockDim.x) {
    const int a23 = idx % (nb * nb), b1 = idx / (nb * nb);
    double2 sp = cmk(0, 0), sq = cmk(0, 0);
    for (int a1 = 0; a1 < nb; ++a1) {
      const double2 e = e1[a1 * nb + b1];
      cfma(sp, tP[a1 * nb * nb + a23], e);
      cfma(sq, tM[a1 * nb * nb + a23], e);
    }
    xP[idx] = sp;
    xM[idx] = sq;
  }
  __syncthreads();
  // y(b1, b2, a3) = sum_a2 x(b1,a2,a3) e2(a2,b2)  (conj for minus) -> reuse tP/tM
  for (int idx = threadIdx.x; idx < nb1 * nb2 * nb; idx += blockDim.x) {
    const int a3 = idx % nb, b2 = (idx / nb) % nb2, b1 = idx / (nb * nb2);
    double2 sp = cmk(0, 0), sq = cmk(0, 0);
    for (int a2 = 0; a2 < nb; ++a2) {
      const double2 e = ev2[a2 * nb + b2];
      cfma(sp, xP[(b1 * nb + a2) * nb + a3], e);
      cfmac(sq, xM[(b1 * nb + a2) * nb + a3], e);
    }
    tP[idx] = sp;
    tM[idx] = sq;
  }
  __syncthreads();
  double* oP = outP + offP[iq];
  double* oM = outM + offM[iq];
  for (int idx = threadIdx.x; idx < nb1 * nb2 * nb3p; idx += blockDim.x) {
    const int b3 = idx % nb3p, b12 = idx / nb3p;
    double2 s = cmk(0, 0);
    for (int a3 = 0; a3 < nb; ++a3) cfmac(s, tP[b12 * nb + a3], e3p[a3 * nb + b3]);
    oP[idx] = s.x * s.x + s.y * s.y;
  }
  for (int idx = threadIdx.x; idx < nb1 * nb2 * nb3m; idx += blockDim.x) {
    const int b3 = idx % nb3m, b12 = idx / nb3m;
    double2 s = cmk(0, 0);
    for (int a3 = 0; a3 < nb; ++a3) cfmac(s, tM[b12 * nb + a3], e3m[a3 * nb + b3]);
    oM[idx] = s.x * s.x + s.y * s.y;
  }
}

// Split path of getCouplingsSquared: operands of the R3 transform as one GEMM
//   T(q1; s, abc) = sum_r3 D3s(abc, r3) w3(r3, a, c) e^{-i q1.R3},  s = +, -
// on [Re | Im] extended K = 2 nr3: A row q1 = [cos | sin] of -q1.R3; B row
// (s, abc, re) = [Dr | -Di], row (s, abc, im) = [Di | Dr] of D = D3s w3.
__global__ void couplings_b_kernel(int nb, int nat, int nr3, const double2* __restrict__ plus,
                                   const double2* __restrict__ mins, const double* __restrict__ w3,
                                   float* __restrict__ B, unsigned* __restrict__ bmax) {
  const size_t n3 = (size_t)nb * nb * nb, rows = 4 * n3, K = 2 * (size_t)nr3;
  float m = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows * K; i += (size_t)gridDim.x * blockDim.x) {
    const size_t row = i / K;
    const int k = (int)(i % K), r = k < nr3 ? k : k - nr3;
    const int ri = (int)(row & 1);
    const size_t sa = row >> 1, abc = sa % n3;
    const int a3 = (int)(abc % nb), a1 = (int)(abc / ((size_t)nb * nb));
    const double2 d = (sa < n3 ? plus : mins)[abc * nr3 + r];
    const double ww = w3[((size_t)r * nat + a1 / 3) * nat + a3 / 3];
    double v;
    if (ri == 0) v = k < nr3 ? d.x * ww : -d.y * ww;
    else v = k < nr3 ? d.y * ww : d.x * ww;
    B[i] = (float)v;
    m = fmaxf(m, fabsf((float)v));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(bmax, __float_as_uint(m));
}

__global__ void couplings_a_kernel(int nq1, int nr3, const double* __restrict__ q1s, const double* __restrict__ R3,
                                   float* __restrict__ A) {
  const size_t K = 2 * (size_t)nr3;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)nq1 * K; i += (size_t)gridDim.x * blockDim.x) {
    const int q = (int)(i / K), k = (int)(i % K), r = k < nr3 ? k : k - nr3;
    const double* q1 = q1s + 3 * q;
    double sn, cs;
    sincos(-(q1[0] * R3[3 * r] + q1[1] * R3[3 * r + 1] + q1[2] * R3[3 * r + 2]), &sn, &cs);
    A[i] = (float)(k < nr3 ? cs : sn);
  }
}

template <typename T>
int dmalloc(phx_ctx* ctx, T** p, size_t n) {
  cudaError_t e = phx_dev_alloc(ctx, reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(n, 1));
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("device allocation: ") + cudaGetErrorString(e));
    return PHX_ERR_CUDA;
  }
  return PHX_OK;
}

// D3w[r3][r2][a][b][c] = D3(a,b,c,r3,r2) w2(r2,at_a,at_b) w3(r3,at_a,at_c)^2:
// the reference applies w3 in cacheD3 and again in the R3 sum
// (interaction_3ph.cpp:166-169,284-285), folded here once with w2.
__global__ void fold_weights_kernel(int nat, int nr2, int nr3, const double* __restrict__ D3,
                                    const double* __restrict__ w2, const double* __restrict__ w3,
                                    double* __restrict__ D3w) {
  const int nb = 3 * nat;
  const size_t nb3 = (size_t)nb * nb * nb, n = nb3 * nr3 * nr2;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t abc = i % nb3, rr = i / nb3;
    const int r2 = (int)(rr % nr2), r3 = (int)(rr / nr2);
    const int i3 = (int)(abc % nb), i2 = (int)((abc / nb) % nb), i1 = (int)(abc / ((size_t)nb * nb));
    const int at1 = i1 / 3, at2 = i2 / 3, at3 = i3 / 3;
    const double ww3 = w3[((size_t)r3 * nat + at1) * nat + at3];
    D3w[i] = D3[(abc * nr3 + r3) * nr2 + r2] * w2[((size_t)r2 * nat + at1) * nat + at2] * ww3 * ww3;
  }
}

}  // namespace

extern "C" int phx_v3_create(phx_ctx* ctx, int nat, int nr2, int nr3, const double* D3,
                             const double* R2, const double* R3, const double* w2,
                             const double* w3, phx_v3** out) {
  PHX_ARG(ctx, ctx && out && nat > 0 && nat <= 21 && nr2 > 0 && nr3 > 0 && D3 && R2 && R3 && w2 &&
                   w3,
          "phx_v3_create: bad arguments");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  phx_v3* v = new phx_v3;
  v->ctx = ctx;
  v->nat = nat;
  v->nb = 3 * nat;
  v->nr2 = nr2;
  v->nr3 = nr3;
  v->R2.assign(R2, R2 + 3 * (size_t)nr2);
  v->R3.assign(R3, R3 + 3 * (size_t)nr3);
  const int nb = v->nb;
  const size_t nb3 = (size_t)nb * nb * nb;
  int rc = PHX_OK;
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_D3w, nb3 * nr3 * nr2);
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_D3raw, nb3 * nr3 * nr2);
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_w2, (size_t)nr2 * nat * nat);
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_w3, (size_t)nr3 * nat * nat);
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_R2, 3 * (size_t)nr2);
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_R3, 3 * (size_t)nr3);
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_plus, 2 * nb3 * nr3);
  if (rc == PHX_OK) rc = dmalloc(ctx, &v->d_mins, 2 * nb3 * nr3);
  if (rc != PHX_OK) {
    phx_v3_destroy(v);
    return rc;
  }
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(v->d_D3raw, D3, sizeof(double) * nb3 * nr3 * nr2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(v->d_w2, w2, sizeof(double) * nr2 * nat * nat, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(v->d_w3, w3, sizeof(double) * nr3 * nat * nat, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(v->d_R2, R2, sizeof(double) * 3 * nr2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(v->d_R3, R3, sizeof(double) * 3 * nr3, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    const size_t n = nb3 * nr3 * nr2;
    fold_weights_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 64), 256, 0, st>>>(
        nat, nr2, nr3, v->d_D3raw, v->d_w2, v->d_w3, v->d_D3w);
    e = cudaGetLastError();
  }
  // the caller may free or reuse its host arrays on return
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_v3_create: ") + cudaGetErrorString(e));
    phx_v3_destroy(v);
    return PHX_ERR_CUDA;
  }
  *out = v;
  return PHX_OK;
}

extern "C" int phx_v3_destroy(phx_v3* v) {
  if (!v) return PHX_OK;
  if (v->ctx) cudaSetDevice(v->ctx->device);
  phx_builder_release(v);
  if (v->ctx) {
    phx_dev_free(v->ctx, v->d_D3w);
    phx_dev_free(v->ctx, v->d_D3raw);
    phx_dev_free(v->ctx, v->d_w2);
    phx_dev_free(v->ctx, v->d_w3);
    phx_dev_free(v->ctx, v->d_R2);
    phx_dev_free(v->ctx, v->d_R3);
    phx_dev_free(v->ctx, v->d_plus);
    phx_dev_free(v->ctx, v->d_mins);
    phx_dev_free(v->ctx, v->d_r2_ofs);
    phx_dev_free(v->ctx, v->d_r2_list);
  }
  delete v;
  return PHX_OK;
}

extern "C" int phx_v3_set_precision(phx_v3* v, int prec) {
  PHX_ARG(nullptr, v, "null v3 handle");
  PHX_ARG(v->ctx, prec != PHX_PREC_SPLIT_TF32, "phx_v3_set_precision: the TF32 split is not built (use PHX_PREC_SPLIT_FP16)");
  PHX_ARG(v->ctx, prec == PHX_PREC_FP64 || prec == PHX_PREC_SPLIT_BF16 || prec == PHX_PREC_SPLIT_FP16,
          "phx_v3_set_precision: unknown precision");
  v->precision = prec;
  return PHX_OK;
}

extern "C" int phx_v3_cache_d3(phx_v3* v, const double* q2) {
  PHX_ARG(nullptr, v && q2, "phx_v3_cache_d3: bad arguments");
  phx_ctx* ctx = v->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const long total = (long)v->nb * v->nb * v->nb * v->nr3;
  const int threads = 256;
  const int blocks = (int)std::min<long>((total + threads - 1) / threads, (long)ctx->num_sms * 8);
  cache_d3_kernel<<<blocks, threads, sizeof(double2) * v->nr2, ctx->stream>>>(
      v->nb, v->nat, v->nr2, v->nr3, v->d_D3raw, v->d_R2, v->d_R3, v->d_w2, v->d_w3, q2[0], q2[1],
      q2[2], reinterpret_cast<double2*>(v->d_plus), reinterpret_cast<double2*>(v->d_mins));
  PHX_CUDA(ctx, cudaGetLastError());
  v->cached = true;
  for (int i = 0; i < 3; ++i) v->q2_cached[i] = q2[i];
  return PHX_OK;
}

extern "C" int phx_v3_couplings_sq(phx_v3* v, int nq1, const double* q1s, const double* ev1,
                                   const int* nb1s, const double* ev2, int nb2,
                                   const double* ev3p, const int* nb3ps, const double* ev3m,
                                   const int* nb3ms, double* outP, double* outM) {
  PHX_ARG(nullptr, v, "null v3 handle");
  phx_ctx* ctx = v->ctx;
  PHX_ARG(ctx, nq1 >= 0 && (nq1 == 0 || (q1s && ev1 && nb1s && ev2 && ev3p && nb3ps && ev3m &&
                                         nb3ms && outP && outM)),
          "phx_v3_couplings_sq: bad arguments");
  if (!v->cached) {
    phx_set_error(ctx, PHX_ERR_STATE, "phx_v3_couplings_sq called before phx_v3_cache_d3");
    return PHX_ERR_STATE;
  }
  if (nq1 == 0) return PHX_OK;
  const int nb = v->nb;
  PHX_ARG(ctx, nb2 >= 1 && nb2 <= nb, "nb2 out of range");
  std::vector<long> offP(nq1 + 1, 0), offM(nq1 + 1, 0);
  for (int i = 0; i < nq1; ++i) {
    PHX_ARG(ctx, nb1s[i] >= 1 && nb1s[i] <= nb && nb3ps[i] >= 1 && nb3ps[i] <= nb &&
                     nb3ms[i] >= 1 && nb3ms[i] <= nb,
            "band counts out of range");
    offP[i + 1] = offP[i] + (long)nb1s[i] * nb2 * nb3ps[i];
    offM[i + 1] = offM[i] + (long)nb1s[i] * nb2 * nb3ms[i];
  }
  const size_t n3 = (size_t)nb * nb * nb;
  const size_t smem = sizeof(double2) * (4 * n3 + v->nr3);
  PHX_ARG(ctx, smem <= 220 * 1024, "phx_v3_couplings_sq: cell too large for the call-by-call path");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t mm = (size_t)nb * nb * 2;
  double *dq, *de1, *de2, *de3p, *de3m, *doP, *doM;
  int *dn1, *dn3p, *dn3m;
  long *dofP, *dofM;
  int rc = PHX_OK;
  dq = de1 = de2 = de3p = de3m = doP = doM = nullptr;
  dn1 = dn3p = dn3m = nullptr;
  dofP = dofM = nullptr;
  if (rc == PHX_OK) rc = dmalloc(ctx, &dq, 3 * (size_t)nq1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &de1, mm * nq1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &de2, mm);
  if (rc == PHX_OK) rc = dmalloc(ctx, &de3p, mm * nq1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &de3m, mm * nq1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &doP, offP[nq1]);
  if (rc == PHX_OK) rc = dmalloc(ctx, &doM, offM[nq1]);
  if (rc == PHX_OK) rc = dmalloc(ctx, &dn1, nq1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &dn3p, nq1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &dn3m, nq1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &dofP, nq1 + 1);
  if (rc == PHX_OK) rc = dmalloc(ctx, &dofM, nq1 + 1);
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (rc == PHX_OK) {
    e = cudaMemcpyAsync(dq, q1s, sizeof(double) * 3 * nq1, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(de1, ev1, sizeof(double) * mm * nq1, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(de2, ev2, sizeof(double) * mm, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(de3p, ev3p, sizeof(double) * mm * nq1, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(de3m, ev3m, sizeof(double) * mm * nq1, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dn1, nb1s, sizeof(int) * nq1, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dn3p, nb3ps, sizeof(int) * nq1, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dn3m, nb3ms, sizeof(int) * nq1, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dofP, offP.data(), sizeof(long) * (nq1 + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dofM, offM.data(), sizeof(long) * (nq1 + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && smem > 48 * 1024)
      e = cudaFuncSetAttribute(couplings_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // split precision: T+- of the whole batch from one tensor-core GEMM
    const bool split = v->precision != PHX_PREC_FP64;
    const bool f16 = v->precision == PHX_PREC_SPLIT_FP16;
    const int K = 2 * v->nr3, N = (int)(4 * n3);
    float *dA = nullptr, *dB = nullptr, *dT = nullptr;
    unsigned* dmx = nullptr;
    if (e == cudaSuccess && split) {
      if (rc == PHX_OK) rc = dmalloc(ctx, &dA, (size_t)nq1 * K);
      if (rc == PHX_OK) rc = dmalloc(ctx, &dB, (size_t)N * K);
      if (rc == PHX_OK) rc = dmalloc(ctx, &dT, (size_t)nq1 * N);
      if (rc == PHX_OK) rc = dmalloc(ctx, &dmx, 1);
      if (rc != PHX_OK) e = cudaErrorMemoryAllocation;
      unsigned mx = 0;
      if (e == cudaSuccess) e = cudaMemsetAsync(dmx, 0, sizeof(unsigned), st);
      if (e == cudaSuccess) {
        couplings_b_kernel<<<std::min<size_t>(((size_t)N * K + 255) / 256, (size_t)ctx->num_sms * 16), 256, 0, st>>>(
            nb, v->nat, v->nr3, reinterpret_cast<const double2*>(v->d_plus),
            reinterpret_cast<const double2*>(v->d_mins), v->d_w3, dB, dmx);
        couplings_a_kernel<<<std::min<size_t>(((size_t)nq1 * K + 255) / 256, (size_t)ctx->num_sms * 16), 256, 0, st>>>(
            nq1, v->nr3, dq, v->d_R3, dA);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(&mx, dmx, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      // FP16 hi/lo: B scaled by a power of 2 so that its largest entry lies in [0.5, 1]
      float bscale = 1.f;
      float bm = 0.f;
      std::memcpy(&bm, &mx, sizeof(bm));
      if (f16 && bm > 0.f) {
        int ex;
        std::frexp(bm, &ex);
        bscale = std::ldexp(1.f, -ex);
      }
      if (e == cudaSuccess)
        e = f16 ? tcgemm::launch<false, true, false, true>(nq1, N, K, dA, K, dB, K, dT, N, 0, bscale, ctx->d_status, st)
                : tcgemm::launch<false, true, false, false>(nq1, N, K, dA, K, dB, K, dT, N, 0, 1.f, ctx->d_status, st);
    }
    if (e == cudaSuccess) {
      couplings_kernel<<<nq1, 256, smem, st>>>(
          nb, v->nat, v->nr3, reinterpret_cast<const double2*>(v->d_plus),
          reinterpret_cast<const double2*>(v->d_mins), v->d_R3, v->d_w3, dq,
          reinterpret_cast<const double2*>(de1), dn1, reinterpret_cast<const double2*>(de2), nb2,
          reinterpret_cast<const double2*>(de3p), dn3p, reinterpret_cast<const double2*>(de3m),
          dn3m, dofP, dofM, doP, doM, split ? dT : nullptr);
      e = cudaGetLastError();
    }
    int kst = 0;
    if (e == cudaSuccess && split) e = cudaMemcpyAsync(&kst, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && split) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && kst) {
      cudaMemset(ctx->d_status, 0, sizeof(int));
      e = cudaErrorLaunchFailure;
    }
    phx_dev_free(ctx, dA);
    phx_dev_free(ctx, dB);
    phx_dev_free(ctx, dT);
    phx_dev_free(ctx, dmx);
    if (e == cudaSuccess) e = cudaMemcpyAsync(outP, doP, sizeof(double) * offP[nq1], cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(outM, doM, sizeof(double) * offM[nq1], cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_v3_couplings_sq: ") + cudaGetErrorString(e));
      rc = PHX_ERR_CUDA;
    }
  }
  cudaFree(dq); cudaFree(de1); cudaFree(de2); cudaFree(de3p); cudaFree(de3m);
  cudaFree(doP); cudaFree(doM); cudaFree(dn1); cudaFree(dn3p); cudaFree(dn3m);
  cudaFree(dofP); cudaFree(dofM);
  return rc;
}

extern "C" int phx_v3_estimate_num_batches(phx_v3* v, int nq1, int nb2, int* num_batches) {
  PHX_ARG(nullptr, v && num_batches && nq1 >= 0, "bad arguments");
  phx_ctx* ctx = v->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  size_t freeb = 0, totalb = 0;
  PHX_CUDA(ctx, cudaMemGetInfo(&freeb, &totalb));
  const double nb = v->nb;
  // memory of one q1 on the call-by-call path: eigenvectors, outputs, q1
  const double perq1 = 16.0 * nb * nb * 3 + 8.0 * nb * nb2 * nb * 2 + 24.0 + 24.0;
  const double avail = 0.8 * (double)freeb;
  if (avail < perq1) {
    phx_set_error(ctx, PHX_ERR_ARG, "Insufficient memory!");
    return PHX_ERR_ARG;
  }
  *num_batches = std::max(1, (int)std::ceil(perq1 * nq1 / avail));
  return PHX_OK;
}
