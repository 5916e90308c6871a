// Electronic Wannier Hamiltonian on the GPU: Fourier interpolation
// H(k) = sum_R e^{+i k.R} / deg_R H(R), batched Hermitian eigensolve, and the
// group velocities of the Hellmann-Feynman velocity operator
// U^H [(H(k+d) - H(k-d)) / 2d]_herm U with d = 1e-8, degenerate subspaces
// (|dE| <= 1 micro-eV) rediagonalised, zero at |k| < 1e-6.
//
// Reference behaviour followed (mir-group/phoebe):
//   * batchedBuildHamiltonians, no shifted vectors  electron_h0_wannier.cpp:160-184
//   * batchedDiagonalizeFromCoordinates             electron_h0_wannier.cpp:222-235
//   * batchedDiagonalizeWithVelocities              electron_h0_wannier.cpp:633-760
//
// One thread-block team per k point; the team builds H(k) in shared memory
// (phases of 256 Bravais vectors at a time) and runs the shared team Jacobi
// solver (jacobi.cuh) in FP64.
#include <cmath>
#include <vector>

#include "cplx.cuh"
#include "jacobi.cuh"
#include "phx_consts.h"
#include "phx_internal.h"

namespace {

using namespace hjac;

struct ElDev {
  int nw, nR;
  const double* R;     // (nR,3)
  const double* deg;   // (nR)
  const double2* H;    // (nR,nw,nw)
};

// H(k) into s.H (row-major nw x nw); the sum over R runs in ascending order
__device__ void build_ham(const ElDev& h, const double k[3], const Smem& s) {
  const int nw = h.nw, m = nw * nw;
  const int tid = threadIdx.x, NT = blockDim.x;
  for (int e = tid; e < m; e += NT) s.H[e] = cmk(0.0, 0.0);
  __syncthreads();
  for (int c0 = 0; c0 < h.nR; c0 += kPhaseChunk) {
    const int c1 = min(h.nR, c0 + kPhaseChunk);
    for (int r = c0 + tid; r < c1; r += NT) {
      const double arg = k[0] * h.R[3 * r] + k[1] * h.R[3 * r + 1] + k[2] * h.R[3 * r + 2];
      double sn, cs;
      sincos(arg, &sn, &cs);
      s.ph[r - c0] = cmk(cs / h.deg[r], sn / h.deg[r]);
    }
    __syncthreads();
    for (int e = tid; e < m; e += NT) {
      double2 acc = s.H[e];
      for (int r = c0; r < c1; ++r) acc = cadd(acc, cmul(s.ph[r - c0], h.H[(size_t)r * m + e]));
      s.H[e] = acc;
    }
    __syncthreads();
  }
}

__global__ void el_bands_kernel(ElDev h, int nk, const double* __restrict__ ks, double* __restrict__ Eout,
                                double2* __restrict__ Uout, double* __restrict__ vgout, int* status) {
  extern __shared__ __align__(16) char smem_raw[];
  const int nw = h.nw, tid = threadIdx.x, NT = blockDim.x;
  Smem s = carve(smem_raw, nw, NT);
  const double delta = 1.0e-8;
  const double degThr = 0.000001 / phxc::energyRyToEv;  // 1 micro-eV
  for (int pt = blockIdx.x; pt < nk; pt += gridDim.x) {
    const double k[3] = {ks[3 * pt], ks[3 * pt + 1], ks[3 * pt + 2]};
    build_ham(h, k, s);
    if (team_jacobi(nw, nw, s) < 0 && tid == 0) atomicOr(status, 1);
    for (int b = tid; b < nw; b += NT) {
      s.E0[b] = s.E1[b];
      Eout[(size_t)pt * nw + b] = s.E1[b];
    }
    for (int e = tid; e < nw * nw; e += NT) {
      s.U0[e] = s.V[e];
      Uout[(size_t)pt * nw * nw + e] = s.V[e];
    }
    __syncthreads();
    if (!vgout) continue;
    const bool gamma = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]) < 1.0e-6;
    if (gamma) {
      for (int e = tid; e < 3 * nw; e += NT) vgout[(size_t)pt * nw * 3 + e] = 0.0;
      __syncthreads();
      continue;
    }
    for (int dir = 0; dir < 3; ++dir) {
      double kk[3] = {k[0], k[1], k[2]};
      kk[dir] += delta;
      build_ham(h, kk, s);
      for (int e = tid; e < nw * nw; e += NT) s.DER[e] = s.H[e];
      __syncthreads();
      kk[dir] = k[dir] - delta;
      build_ham(h, kk, s);
      // der = (H+ - H-) / 2d, hermitised into T
      for (int e = tid; e < nw * nw; e += NT) s.DER[e] = cscale(csub(s.DER[e], s.H[e]), 1.0 / (2.0 * delta));
      __syncthreads();
      for (int e = tid; e < nw * nw; e += NT) {
        const int i = e / nw, j = e % nw;
        s.T[e] = cscale(cadd(s.DER[i * nw + j], cconj(s.DER[j * nw + i])), 0.5);
      }
      __syncthreads();
      // velocity operator U0^H T U0 (H = T U0 as a temporary)
      for (int e = tid; e < nw * nw; e += NT) {
        const int i = e / nw, j = e % nw;
        double2 acc = cmk(0.0, 0.0);
        for (int l = 0; l < nw; ++l) acc = cadd(acc, cmul(s.T[i * nw + l], s.U0[l * nw + j]));
        s.H[e] = acc;
      }
      __syncthreads();
      for (int e = tid; e < nw * nw; e += NT) {
        const int i = e / nw, j = e % nw;
        double2 acc = cmk(0.0, 0.0);
        for (int l = 0; l < nw; ++l) acc = cadd(acc, cmul(cconj(s.U0[l * nw + i]), s.H[l * nw + j]));
        s.DER[e] = acc;
      }
      __syncthreads();
      for (int b = tid; b < nw; b += NT) s.VG[b] = s.DER[b * nw + b].x;
      __syncthreads();
      // degenerate subspaces: ascending eigenvalues of the hermitised block
      for (int ib = 0; ib < nw;) {
        int size = 1;
        for (int ib2 = ib + 1; ib2 < nw; ++ib2) {
          if (fabs(s.E0[ib] - s.E0[ib2]) > degThr) break;
          ++size;
        }
        if (size > 1) {
          for (int e = tid; e < size * size; e += NT) {
            const int i = e / size, j = e % size;
            s.H[i * nw + j] = cscale(cadd(s.DER[(ib + i) * nw + ib + j], cconj(s.DER[(ib + j) * nw + ib + i])), 0.5);
          }
          __syncthreads();
          if (team_jacobi(size, nw, s) < 0 && tid == 0) atomicOr(status, 1);
          for (int i = tid; i < size; i += NT) s.VG[ib + i] = s.E1[i];
          __syncthreads();
        }
        ib += size;
      }
      for (int b = tid; b < nw; b += NT) vgout[((size_t)pt * nw + b) * 3 + dir] = s.VG[b];
      __syncthreads();
    }
  }
}

int el_team_threads(int nw) { return nw <= 8 ? 32 : (nw <= 24 ? 64 : 128); }

void inv3_transpose_2pi(const double* A, double* B) {
  // B = 2 pi inv(A)^T  (columns of B are the reciprocal vectors of the columns of A)
  const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                     A[2] * (A[3] * A[7] - A[4] * A[6]);
  double inv[9];
  inv[0] = (A[4] * A[8] - A[5] * A[7]) / det;
  inv[1] = (A[2] * A[7] - A[1] * A[8]) / det;
  inv[2] = (A[1] * A[5] - A[2] * A[4]) / det;
  inv[3] = (A[5] * A[6] - A[3] * A[8]) / det;
  inv[4] = (A[0] * A[8] - A[2] * A[6]) / det;
  inv[5] = (A[2] * A[3] - A[0] * A[5]) / det;
  inv[6] = (A[3] * A[7] - A[4] * A[6]) / det;
  inv[7] = (A[1] * A[6] - A[0] * A[7]) / det;
  inv[8] = (A[0] * A[4] - A[1] * A[3]) / det;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i * 3 + j] = 2.0 * M_PI * inv[j * 3 + i];
}

}  // namespace

int phx_launch_el_bands(phx_el_h0* h, int nk, const double* d_k, double* d_E, double* d_U, double* d_vg) {
  phx_ctx* ctx = h->ctx;
  ElDev dev{h->nw, h->nR, h->d_R, h->d_deg, reinterpret_cast<const double2*>(h->d_H)};
  const int NT = el_team_threads(h->nw);
  const size_t smem = smem_bytes(h->nw, NT);
  const int grid = std::max(1, std::min(nk, ctx->num_sms * 16));
  PHX_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  el_bands_kernel<<<grid, NT, smem, ctx->stream>>>(dev, nk, d_k, d_E, reinterpret_cast<double2*>(d_U), d_vg,
                                                   ctx->d_status);
  PHX_CUDA(ctx, cudaGetLastError());
  int st = 0;
  PHX_CUDA(ctx, cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st) {
    phx_set_error(ctx, PHX_ERR_NOCONV, "Jacobi eigensolver did not converge within its sweep cap");
    return PHX_ERR_NOCONV;
  }
  return PHX_OK;
}

extern "C" int phx_el_h0_create(phx_ctx* ctx, int nw, int nR, const double* cell, const double* R,
                                const double* deg, const double* H, phx_el_h0** out) {
  PHX_ARG(ctx, ctx && cell && R && deg && H && out && nw > 0 && nw <= 64 && nR > 0,
          "phx_el_h0_create: bad arguments");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  for (int r = 0; r < nR; ++r) PHX_ARG(ctx, deg[r] > 0.0, "phx_el_h0_create: degeneracies must be > 0");
  phx_el_h0* h = new phx_el_h0;
  h->ctx = ctx;
  h->nw = nw;
  h->nR = nR;
  for (int i = 0; i < 9; ++i) h->cell[i] = cell[i];
  inv3_transpose_2pi(cell, h->recip);
  cudaError_t e = cudaMalloc(&h->d_R, sizeof(double) * 3 * nR);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_deg, sizeof(double) * nR);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_H, sizeof(double) * 2 * (size_t)nR * nw * nw);
  if (e == cudaSuccess) e = cudaMemcpy(h->d_R, R, sizeof(double) * 3 * nR, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->d_deg, deg, sizeof(double) * nR, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(h->d_H, H, sizeof(double) * 2 * (size_t)nR * nw * nw, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_el_h0_create: ") + cudaGetErrorString(e));
    phx_el_h0_destroy(h);
    return PHX_ERR_CUDA;
  }
  *out = h;
  return PHX_OK;
}

extern "C" int phx_el_h0_destroy(phx_el_h0* h) {
  if (!h) return PHX_OK;
  cudaFree(h->d_R);
  cudaFree(h->d_deg);
  cudaFree(h->d_H);
  delete h;
  return PHX_OK;
}

extern "C" int phx_el_h0_num_bands(const phx_el_h0* h) { return h ? h->nw : 0; }

extern "C" int phx_el_diag(phx_el_h0* h, int nk, const double* k, double* E, double* U, double* vg) {
  PHX_ARG(h ? h->ctx : nullptr, h && k && E && U && nk >= 0, "phx_el_diag: bad arguments");
  phx_ctx* ctx = h->ctx;
  if (nk == 0) return PHX_OK;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t nw = h->nw;
  double *dk = nullptr, *dE = nullptr, *dU = nullptr, *dv = nullptr;
  int rc = PHX_OK;
  cudaError_t e = cudaMalloc(&dk, sizeof(double) * 3 * nk);
  if (e == cudaSuccess) e = cudaMalloc(&dE, sizeof(double) * nk * nw);
  if (e == cudaSuccess) e = cudaMalloc(&dU, sizeof(double) * 2 * nk * nw * nw);
  if (e == cudaSuccess && vg) e = cudaMalloc(&dv, sizeof(double) * 3 * nk * nw);
  if (e == cudaSuccess) e = cudaMemcpy(dk, k, sizeof(double) * 3 * nk, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_el_diag: ") + cudaGetErrorString(e));
    rc = PHX_ERR_CUDA;
  }
  if (rc == PHX_OK) rc = phx_launch_el_bands(h, nk, dk, dE, dU, dv);
  if (rc == PHX_OK) {
    e = cudaMemcpy(E, dE, sizeof(double) * nk * nw, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(U, dU, sizeof(double) * 2 * nk * nw * nw, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && vg) e = cudaMemcpy(vg, dv, sizeof(double) * 3 * nk * nw, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_el_diag: ") + cudaGetErrorString(e));
      rc = PHX_ERR_CUDA;
    }
  }
  cudaFree(dk);
  cudaFree(dE);
  cudaFree(dU);
  cudaFree(dv);
  return rc;
}

extern "C" int phx_el_bands_create_mesh(phx_el_h0* h, const int* mesh, int with_velocities, phx_bands** out) {
  PHX_ARG(h ? h->ctx : nullptr, h && mesh && out, "phx_el_bands_create_mesh: bad arguments");
  phx_ctx* ctx = h->ctx;
  PHX_ARG(ctx, mesh[0] > 0 && mesh[1] > 0 && mesh[2] > 0, "phx_el_bands_create_mesh: bad mesh");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  phx_bands* b = new phx_bands;
  b->ctx = ctx;
  b->nb = h->nw;
  b->nq = mesh[0] * mesh[1] * mesh[2];
  for (int i = 0; i < 3; ++i) b->mesh[i] = mesh[i];
  for (int i = 0; i < 9; ++i) b->recip[i] = h->recip[i];
  std::vector<double> k;
  phx_mesh_cartesian(mesh, h->recip, k);
  const size_t nk = b->nq, nw = b->nb;
  cudaError_t e = cudaMalloc(&b->d_E, sizeof(double) * nk * nw);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_U, sizeof(double) * 2 * nk * nw * nw);
  if (e == cudaSuccess && with_velocities) e = cudaMalloc(&b->d_vg, sizeof(double) * 3 * nk * nw);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_q, sizeof(double) * 3 * nk);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_q, k.data(), sizeof(double) * 3 * nk, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
    phx_bands_destroy(b);
    return PHX_ERR_CUDA;
  }
  const int rc = phx_launch_el_bands(h, b->nq, b->d_q, b->d_E, b->d_U, b->d_vg);
  if (rc != PHX_OK) {
    phx_bands_destroy(b);
    return rc;
  }
  *out = b;
  return PHX_OK;
}
