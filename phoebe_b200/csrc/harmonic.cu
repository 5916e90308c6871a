// Phonon harmonic Hamiltonian on the GPU: Fourier interpolation of the
// dynamical matrix, batched Hermitian eigensolve, finite-difference velocity
// operator.
//
// Reference behaviour followed (mir-group/phoebe):
//   * D(q) = sum_R exp(-i q.R) w_R mat2R(R)      phonon_h0.cpp:773-813
//   * D <- (D + D^H)/2,  D_ij /= sqrt(m_i m_j)   phonon_h0.cpp:836-855
//   * w2 ascending, omega = sign(w2) sqrt|w2|,
//     eigenvectors / sqrt(m) when mass-scaled    phonon_h0.cpp:346-387,858-877
//   * velocity operator: U^H [ (S(q+d)-S(q-d))/2d ]_herm U with
//     S = U diag(omega) U^H, d = 1e-8, degenerate blocks (|dw| <= 1e-4 cm^-1)
//     rediagonalised, zero at |q| < 1e-6        phonon_h0.cpp:895-1070
//
// Design: one thread-block team per q-point (grid-stride over points).  The
// team builds D(q) in shared memory from the Wigner-Seitz list grouped by
// atom pair (each R carries one 3x3 block, so the sum skips the zeros of the
// reference's dense (nb,nb,numR) tensor), then runs a parallel cyclic Jacobi
// sweep (round-robin pairing: nb/2 disjoint complex rotations per step, rows
// then columns updated by the whole team) entirely in shared memory, FP64.
// The eigensolver is bounded: after a sweep cap it sets a status flag and the
// host reports PHX_ERR_NOCONV.
#include <cmath>
#include <algorithm>

#include "cplx.cuh"
#include "phx_consts.h"
#include "phx_internal.h"
#include "jacobi.cuh"

namespace {

using namespace hjac;

struct H0Dev {
  int nb, nat, numR;
  const int* pofs;      // (nat*nat+1) ranges into the R list, grouped by atom pair
  const double* R;      // (numR,3)
  const double* wblk;   // (numR,9) w_R * 3x3 block of the pair
  const double* masses; // (nb)
};

// Dynamical matrix at q, hermitised and mass-divided, into H (row-major).
__device__ void build_dyn(const H0Dev& h, const double q[3], const Smem& s) {
  const int nb = h.nb, nat = h.nat, m = nb * nb;
  const int tid = threadIdx.x, NT = blockDim.x;
  for (int e = tid; e < m; e += NT) s.T[e] = cmk(0.0, 0.0);
  __syncthreads();
  for (int c0 = 0; c0 < h.numR; c0 += kPhaseChunk) {
    const int c1 = min(h.numR, c0 + kPhaseChunk);
    for (int k = c0 + tid; k < c1; k += NT) {
      const double arg = q[0] * h.R[3 * k] + q[1] * h.R[3 * k + 1] + q[2] * h.R[3 * k + 2];
      double sn, cs;
      sincos(arg, &sn, &cs);
      s.ph[k - c0] = cmk(cs, -sn);  // exp(-i q.R)
    }
    __syncthreads();
    for (int e = tid; e < m; e += NT) {
      const int row = e / nb, col = e % nb;
      const int a = row / 3, i = row % 3, b = col / 3, j = col % 3;
      const int pr = a * nat + b;
      const int k0 = max(h.pofs[pr], c0), k1 = min(h.pofs[pr + 1], c1);
      double2 acc = s.T[e];
      for (int k = k0; k < k1; ++k) {
        const double v = h.wblk[9 * k + 3 * i + j];
        acc.x = fma(v, s.ph[k - c0].x, acc.x);
        acc.y = fma(v, s.ph[k - c0].y, acc.y);
      }
      s.T[e] = acc;
    }
    __syncthreads();
  }
  for (int e = tid; e < m; e += NT) {
    const int i = e / nb, j = e % nb;
    double2 x = cadd(s.T[i * nb + j], cconj(s.T[j * nb + i]));
    x = cscale(x, 0.5);
    x = cscale(x, 1.0 / sqrt(h.masses[i] * h.masses[j]));
    s.H[e] = x;
  }
  __syncthreads();
}

__global__ void ph_bands_kernel(H0Dev h, int nq, const double* __restrict__ qs,
                                double* __restrict__ Eout, double2* __restrict__ Uout,
                                double* __restrict__ vgout, int mass_scaling, int* status) {
  extern __shared__ __align__(16) char smem_raw[];
  const int nb = h.nb, tid = threadIdx.x, NT = blockDim.x;
  Smem s = carve(smem_raw, nb, NT);
  const double delta = 1.0e-8;
  const double degThr = phxc::velDegThreshold;
  for (int pt = blockIdx.x; pt < nq; pt += gridDim.x) {
    const double q[3] = {qs[3 * pt], qs[3 * pt + 1], qs[3 * pt + 2]};
    build_dyn(h, q, s);
    if (team_jacobi(nb, nb, s) < 0 && tid == 0) atomicOr(status, 1);
    for (int b = tid; b < nb; b += NT) {
      const double w2 = s.E1[b];
      const double en = w2 < 0 ? -sqrt(-w2) : sqrt(w2);
      s.E0[b] = en;
      Eout[(size_t)pt * nb + b] = en;
    }
    for (int e = tid; e < nb * nb; e += NT) {
      s.U0[e] = s.V[e];
      double2 u = s.V[e];
      if (mass_scaling) u = cscale(u, 1.0 / sqrt(h.masses[e / nb]));
      Uout[(size_t)pt * nb * nb + e] = u;
    }
    __syncthreads();
    if (!vgout) continue;
    const bool gamma = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) < 1.0e-6;
    for (int dir = 0; dir < 3; ++dir) {
      for (int e = tid; e < nb * nb; e += NT) s.DER[e] = cmk(0.0, 0.0);
      __syncthreads();
      for (int sgn = 0; sgn < 2; ++sgn) {
        double qq[3] = {q[0], q[1], q[2]};
        qq[dir] += sgn == 0 ? delta : -delta;
        build_dyn(h, qq, s);
        if (team_jacobi(nb, nb, s) < 0 && tid == 0) atomicOr(status, 1);
        for (int b = tid; b < nb; b += NT) {
          const double w2 = s.E1[b];
          s.E1[b] = w2 < 0 ? -sqrt(-w2) : sqrt(w2);
        }
        __syncthreads();
        // DER +/-= V diag(omega) V^H
        const double sg = sgn == 0 ? 1.0 : -1.0;
        for (int e = tid; e < nb * nb; e += NT) {
          const int i = e / nb, j = e % nb;
          double2 acc = cmk(0.0, 0.0);
          for (int l = 0; l < nb; ++l) cfmac(acc, cscale(s.V[i * nb + l], s.E1[l]), s.V[j * nb + l]);
          s.DER[e] = cadd(s.DER[e], cscale(acc, sg));
        }
        __syncthreads();
      }
      // hermitise (der/2d), then T = DERh U0 and H = U0^H T
      for (int e = tid; e < nb * nb; e += NT) {
        const int i = e / nb, j = e % nb;
        const double2 a = cscale(s.DER[i * nb + j], 1.0 / (2.0 * delta));
        const double2 b = cscale(s.DER[j * nb + i], 1.0 / (2.0 * delta));
        s.H[e] = cscale(cadd(a, cconj(b)), 0.5);
      }
      __syncthreads();
      for (int e = tid; e < nb * nb; e += NT) {
        const int i = e / nb, j = e % nb;
        double2 acc = cmk(0.0, 0.0);
        for (int l = 0; l < nb; ++l) cfma(acc, s.H[i * nb + l], s.U0[l * nb + j]);
        s.T[e] = acc;
      }
      __syncthreads();
      for (int e = tid; e < nb * nb; e += NT) {
        const int i = e / nb, j = e % nb;
        double2 acc = cmk(0.0, 0.0);
        for (int l = 0; l < nb; ++l) cfma(acc, cconj(s.U0[l * nb + i]), s.T[l * nb + j]);
        s.DER[e] = acc;  // velocity operator for this direction
      }
      __syncthreads();
      for (int b = tid; b < nb; b += NT) s.VG[b] = s.DER[b * nb + b].x;
      __syncthreads();
      // degenerate subspaces: ascending eigenvalues of the hermitised block
      for (int ib = 0; ib < nb;) {
        int size = 1;
        for (int ib2 = ib + 1; ib2 < nb; ++ib2) {
          if (fabs(s.E0[ib] - s.E0[ib2]) > degThr) break;
          ++size;
        }
        if (size > 1) {
          for (int e = tid; e < size * size; e += NT) {
            const int i = e / size, j = e % size;
            const double2 a = s.DER[(ib + i) * nb + ib + j];
            const double2 b = s.DER[(ib + j) * nb + ib + i];
            s.H[i * nb + j] = cscale(cadd(a, cconj(b)), 0.5);
          }
          __syncthreads();
          if (team_jacobi(size, nb, s) < 0 && tid == 0) atomicOr(status, 1);
          for (int i = tid; i < size; i += NT) s.VG[ib + i] = s.E1[i];
          __syncthreads();
        }
        ib += size;
      }
      for (int b = tid; b < nb; b += NT)
        vgout[((size_t)pt * nb + b) * 3 + dir] = gamma ? 0.0 : s.VG[b];
      __syncthreads();
    }
  }
}

int team_threads(int nb) { return nb <= 8 ? 32 : (nb <= 24 ? 64 : 128); }

}  // namespace

// ---------------------------------------------------------------------------
// ABI
// ---------------------------------------------------------------------------
extern "C" int phx_ph_h0_create(phx_ctx* ctx, int nat, const double* cell, const double* pos,
                                const double* masses, const int* grid, const double* fc,
                                phx_ph_h0** out) {
  PHX_ARG(ctx, ctx && out && nat > 0 && nat <= 21 && cell && pos && masses && grid && fc,
          "phx_ph_h0_create: bad arguments (nat must be 1..21)");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  int numR = 0;
  PHX_TRY(phx_ws_reorder(nat, cell, pos, grid, fc, &numR, nullptr, nullptr, nullptr));
  const int nb = 3 * nat;
  std::vector<double> R(3 * (size_t)numR), w(numR), M((size_t)numR * nb * nb);
  PHX_TRY(phx_ws_reorder(nat, cell, pos, grid, fc, &numR, R.data(), w.data(), M.data()));
  // group the (R, atom pair) list by atom pair; fold the weight into the block
  std::vector<int> pofs(nat * nat + 1, 0);
  std::vector<int> pairOf(numR);
  for (int k = 0; k < numR; ++k) {
    int found = -1;
    const double* Mk = &M[(size_t)k * nb * nb];
    for (int a = 0; a < nat && found < 0; ++a)
      for (int b = 0; b < nat && found < 0; ++b)
        for (int i = 0; i < 3 && found < 0; ++i)
          for (int j = 0; j < 3; ++j)
            if (Mk[(3 * a + i) * nb + 3 * b + j] != 0.0) { found = a * nat + b; break; }
    pairOf[k] = found < 0 ? 0 : found;
  }
  // each R entry of the reference list belongs to exactly one atom pair; an
  // all-zero block carries no information and is dropped
  std::vector<double> Rc, wb;
  for (int pr = 0; pr < nat * nat; ++pr) {
    pofs[pr] = (int)(Rc.size() / 3);
    const int a = pr / nat, b = pr % nat;
    for (int k = 0; k < numR; ++k) {
      if (pairOf[k] != pr) continue;
      const double* Mk = &M[(size_t)k * nb * nb];
      bool nz = false;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) nz |= Mk[(3 * a + i) * nb + 3 * b + j] != 0.0;
      if (!nz) continue;
      Rc.insert(Rc.end(), &R[3 * k], &R[3 * k] + 3);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) wb.push_back(w[k] * Mk[(3 * a + i) * nb + 3 * b + j]);
    }
  }
  pofs[nat * nat] = (int)(Rc.size() / 3);
  phx_ph_h0* h = new phx_ph_h0;
  h->ctx = ctx;
  h->nat = nat;
  h->nb = nb;
  h->numR = pofs[nat * nat];
  for (int i = 0; i < 9; ++i) h->cell[i] = cell[i];
  {
    // reciprocal = 2 pi (A^-1)^T, columns = b vectors (crystal.cpp:290-293)
    const double* A = cell;
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
    const double tp = 2.0 * 3.14159265358979323846;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) h->recip[i * 3 + j] = tp * inv[j * 3 + i];
  }
  h->masses.resize(nb);
  for (int a = 0; a < nat; ++a)
    for (int i = 0; i < 3; ++i) h->masses[3 * a + i] = masses[a];
  cudaError_t e = cudaSuccess;
  cudaStream_t st = ctx->stream;
  e = phx_dev_alloc(ctx, (void**)&h->d_R, sizeof(double) * std::max<size_t>(1, Rc.size()));
  if (e == cudaSuccess) e = phx_dev_alloc(ctx, (void**)&h->d_wblk, sizeof(double) * std::max<size_t>(1, wb.size()));
  if (e == cudaSuccess) e = phx_dev_alloc(ctx, (void**)&h->d_pofs, sizeof(int) * pofs.size());
  if (e == cudaSuccess) e = phx_dev_alloc(ctx, (void**)&h->d_masses, sizeof(double) * nb);
  if (e == cudaSuccess && !Rc.empty())
    e = cudaMemcpyAsync(h->d_R, Rc.data(), sizeof(double) * Rc.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !wb.empty())
    e = cudaMemcpyAsync(h->d_wblk, wb.data(), sizeof(double) * wb.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->d_pofs, pofs.data(), sizeof(int) * pofs.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->d_masses, h->masses.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_ph_h0_create: ") + cudaGetErrorString(e));
    phx_ph_h0_destroy(h);
    return PHX_ERR_CUDA;
  }
  *out = h;
  return PHX_OK;
}

extern "C" int phx_ph_h0_destroy(phx_ph_h0* h) {
  if (!h) return PHX_OK;
  if (h->ctx) {
    cudaSetDevice(h->ctx->device);
    phx_dev_free(h->ctx, h->d_R);
    phx_dev_free(h->ctx, h->d_pofs);
    phx_dev_free(h->ctx, h->d_wblk);
    phx_dev_free(h->ctx, h->d_masses);
  }
  delete h;
  return PHX_OK;
}

extern "C" int phx_ph_h0_num_bands(const phx_ph_h0* h) { return h ? h->nb : 0; }

int phx_launch_ph_bands(phx_ph_h0* h0, int nq, const double* d_q, double* d_E, double* d_U,
                        double* d_vg, int mass_scaling) {
  phx_ctx* ctx = h0->ctx;
  if (nq <= 0) return PHX_OK;
  H0Dev hd;
  hd.nb = h0->nb;
  hd.nat = h0->nat;
  hd.numR = h0->numR;
  hd.pofs = h0->d_pofs;
  hd.R = h0->d_R;
  hd.wblk = h0->d_wblk;
  hd.masses = h0->d_masses;
  const int NT = team_threads(h0->nb);
  const size_t smem = smem_bytes(h0->nb, NT);
  if (smem > 48 * 1024)
    PHX_CUDA(ctx, cudaFuncSetAttribute(ph_bands_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
  PHX_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  const int blocks = std::min(nq, ctx->num_sms * 16);
  ph_bands_kernel<<<blocks, NT, smem, ctx->stream>>>(hd, nq, d_q, d_E,
                                                     reinterpret_cast<double2*>(d_U), d_vg,
                                                     mass_scaling, ctx->d_status);
  PHX_CUDA(ctx, cudaGetLastError());
  int st = 0;
  PHX_CUDA(ctx, cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st) {
    phx_set_error(ctx, PHX_ERR_NOCONV, "Jacobi eigensolver reached its sweep cap");
    return PHX_ERR_NOCONV;
  }
  return PHX_OK;
}

static int diag_common(phx_ph_h0* h0, int nq, const double* q, int mass_scaling, double* E,
                       double* U, double* vg) {
  PHX_ARG(nullptr, h0 && h0->ctx, "null PhononH0 handle");
  phx_ctx* ctx = h0->ctx;
  PHX_ARG(ctx, nq >= 0 && (nq == 0 || (q && E && U)), "phx_ph_diag: bad arguments");
  if (nq == 0) return PHX_OK;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nb = h0->nb;
  double *dq = nullptr, *dE = nullptr, *dU = nullptr, *dv = nullptr;
  int rc = PHX_OK;
  cudaError_t e = cudaMalloc(&dq, sizeof(double) * 3 * nq);
  if (e == cudaSuccess) e = cudaMalloc(&dE, sizeof(double) * nq * nb);
  if (e == cudaSuccess) e = cudaMalloc(&dU, sizeof(double) * 2 * (size_t)nq * nb * nb);
  if (e == cudaSuccess && vg) e = cudaMalloc(&dv, sizeof(double) * 3 * (size_t)nq * nb);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dq, q, sizeof(double) * 3 * nq, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
    rc = PHX_ERR_CUDA;
  }
  if (rc == PHX_OK) rc = phx_launch_ph_bands(h0, nq, dq, dE, dU, dv, mass_scaling);
  if (rc == PHX_OK || rc == PHX_ERR_NOCONV) {
    e = cudaMemcpyAsync(E, dE, sizeof(double) * nq * nb, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(U, dU, sizeof(double) * 2 * (size_t)nq * nb * nb, cudaMemcpyDeviceToHost,
                          ctx->stream);
    if (e == cudaSuccess && vg)
      e = cudaMemcpyAsync(vg, dv, sizeof(double) * 3 * (size_t)nq * nb, cudaMemcpyDeviceToHost,
                          ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, cudaGetErrorString(e));
      rc = PHX_ERR_CUDA;
    }
  }
  cudaFree(dq);
  cudaFree(dE);
  cudaFree(dU);
  cudaFree(dv);
  return rc;
}

extern "C" int phx_ph_diag(phx_ph_h0* h0, int nq, const double* q, int mass_scaling, double* E,
                           double* U) {
  return diag_common(h0, nq, q, mass_scaling, E, U, nullptr);
}

extern "C" int phx_ph_diag_velocities(phx_ph_h0* h0, int nq, const double* q, double* E,
                                      double* U, double* vg) {
  PHX_ARG(h0 ? h0->ctx : nullptr, vg != nullptr, "phx_ph_diag_velocities: vg is NULL");
  return diag_common(h0, nq, q, 1, E, U, vg);
}
