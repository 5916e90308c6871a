// Team eigensolver shared by the phonon and Wannier band kernels: one thread
// block per k (or q) point builds its Hermitian matrix in shared memory and
// diagonalises it with a parallel cyclic Jacobi sweep (round-robin pairing:
// n/2 disjoint complex rotations per step), FP64, bounded by a sweep cap.
#pragma once
#include <cmath>
#include <cstdint>

#include "cplx.cuh"

namespace hjac {

constexpr int kMaxSweeps = 60;
constexpr int kPhaseChunk = 256;

struct Rot {
  int p, q, active;
  double c, s, ap, dq;
  double2 ph;  // exp(i phi) of H_pq
};

// Shared-memory carve-up for one team.
struct Smem {
  double2 *H, *V, *U0, *DER, *T;
  double *E0, *E1, *VG, *red;
  int* perm;
  Rot* rot;
  double2* ph;
};

__device__ __forceinline__ Smem carve(char* base, int nb, int NT) {
  Smem s;
  size_t m = (size_t)nb * nb;
  double2* c = reinterpret_cast<double2*>(base);
  s.H = c;
  s.V = c + m;
  s.U0 = c + 2 * m;
  s.DER = c + 3 * m;
  s.T = c + 4 * m;
  s.ph = c + 5 * m;
  double* d = reinterpret_cast<double*>(s.ph + kPhaseChunk);
  s.E0 = d;
  s.E1 = d + nb;
  s.VG = d + 2 * nb;
  s.red = d + 3 * nb;
  // Rot holds a double2: round up to 16 bytes (3 nb + NT doubles need not be)
  const uintptr_t ra = (reinterpret_cast<uintptr_t>(s.red + NT) + 15) & ~uintptr_t(15);
  Rot* r = reinterpret_cast<Rot*>(ra);
  s.rot = r;
  s.perm = reinterpret_cast<int*>(r + (nb / 2 + 1));
  return s;
}

inline size_t smem_bytes(int nb, int NT) {
  size_t m = (size_t)nb * nb;
  // + 64: the 16-byte alignment of the Rot array (at most 8 bytes) and slack
  return sizeof(double2) * (5 * m + kPhaseChunk) + sizeof(double) * (3 * nb + NT) +
         sizeof(Rot) * (nb / 2 + 1) + sizeof(int) * nb + 64;
}

__device__ inline double team_reduce_max(double v, double* red) {
  const int tid = threadIdx.x, NT = blockDim.x;
  red[tid] = v;
  __syncthreads();
  for (int off = NT / 2; off > 0; off >>= 1) {
    if (tid < off) red[tid] = fmax(red[tid], red[tid + off]);
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}

// Cyclic parallel Jacobi on the n x n Hermitian matrix H (smem, row-major,
// leading dimension ld).  On exit: E1[0..n) ascending eigenvalues, V columns
// the matching eigenvectors (leading dimension ld).  Returns sweeps used or
// -1 when the sweep cap was reached.
__device__ inline int team_jacobi(int n, int ld, const Smem& s) {
  const int tid = threadIdx.x, NT = blockDim.x;
  double2* H = s.H;
  double2* V = s.V;
  for (int e = tid; e < n * n; e += NT) {
    const int i = e / n, j = e % n;
    V[i * ld + j] = cmk(i == j ? 1.0 : 0.0, 0.0);
  }
  double fro = 0.0;
  for (int e = tid; e < n * n; e += NT) fro = fmax(fro, cabs2(H[(e / n) * ld + e % n]));
  fro = sqrt(team_reduce_max(fro, s.red)) * n;
  const double thr = 1.0e-18 * fro;
  const int np = n + (n & 1);
  const int npair = np / 2;
  int sweep = 0;
  bool done = (n < 2);
  while (!done) {
    if (sweep >= kMaxSweeps) return -1;
    double rotated = 0.0;
    for (int r = 0; r < np - 1; ++r) {
      for (int k = tid; k < npair; k += NT) {
        int p, q;
        if (k == 0) {
          p = r;
          q = np - 1;
        } else {
          p = (r + k) % (np - 1);
          q = (r - k + np - 1) % (np - 1);
        }
        if (p > q) { int t = p; p = q; q = t; }
        Rot ro;
        ro.p = p;
        ro.q = q;
        ro.active = 0;
        if (q < n) {
          const double2 b = H[p * ld + q];
          const double mb = sqrt(cabs2(b));
          if (mb > thr) {
            const double a = H[p * ld + p].x, d = H[q * ld + q].x;
            const double theta = (d - a) / (2.0 * mb);
            double t;
            if (fabs(theta) > 1.0e150) t = 0.5 / theta;
            else t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            ro.c = 1.0 / sqrt(1.0 + t * t);
            ro.s = t * ro.c;
            ro.ph = cmk(b.x / mb, b.y / mb);
            ro.ap = a - t * mb;
            ro.dq = d + t * mb;
            ro.active = 1;
          }
        }
        s.rot[k] = ro;
      }
      __syncthreads();
      // rows: p' = c p - s e^{i phi} q ; q' = s e^{-i phi} p + c q
      for (int idx = tid; idx < npair * n; idx += NT) {
        const Rot ro = s.rot[idx / n];
        if (!ro.active) continue;
        const int j = idx % n;
        const double2 hp = H[ro.p * ld + j], hq = H[ro.q * ld + j];
        const double2 eq = cmul(ro.ph, hq);
        const double2 ep = cmulc(hp, ro.ph);  // hp * conj(ph)
        H[ro.p * ld + j] = cmk(ro.c * hp.x - ro.s * eq.x, ro.c * hp.y - ro.s * eq.y);
        H[ro.q * ld + j] = cmk(ro.s * ep.x + ro.c * hq.x, ro.s * ep.y + ro.c * hq.y);
      }
      __syncthreads();
      // columns of H and V: p' = c p - s e^{-i phi} q ; q' = s e^{i phi} p + c q
      for (int idx = tid; idx < npair * n; idx += NT) {
        const Rot ro = s.rot[idx / n];
        if (!ro.active) continue;
        const int i = idx % n;
        {
          const double2 hp = H[i * ld + ro.p], hq = H[i * ld + ro.q];
          const double2 eq = cmulc(hq, ro.ph);
          const double2 ep = cmul(hp, ro.ph);
          H[i * ld + ro.p] = cmk(ro.c * hp.x - ro.s * eq.x, ro.c * hp.y - ro.s * eq.y);
          H[i * ld + ro.q] = cmk(ro.s * ep.x + ro.c * hq.x, ro.s * ep.y + ro.c * hq.y);
        }
        {
          const double2 vp = V[i * ld + ro.p], vq = V[i * ld + ro.q];
          const double2 eq = cmulc(vq, ro.ph);
          const double2 ep = cmul(vp, ro.ph);
          V[i * ld + ro.p] = cmk(ro.c * vp.x - ro.s * eq.x, ro.c * vp.y - ro.s * eq.y);
          V[i * ld + ro.q] = cmk(ro.s * ep.x + ro.c * vq.x, ro.s * ep.y + ro.c * vq.y);
        }
      }
      __syncthreads();
      for (int k = tid; k < npair; k += NT) {
        const Rot ro = s.rot[k];
        if (!ro.active) continue;
        H[ro.p * ld + ro.p] = cmk(ro.ap, 0.0);
        H[ro.q * ld + ro.q] = cmk(ro.dq, 0.0);
        H[ro.p * ld + ro.q] = cmk(0.0, 0.0);
        H[ro.q * ld + ro.p] = cmk(0.0, 0.0);
        rotated = 1.0;
      }
      __syncthreads();
    }
    ++sweep;
    done = team_reduce_max(rotated, s.red) == 0.0;
  }
  // ascending order (stable rank sort)
  for (int i = tid; i < n; i += NT) {
    const double ei = H[i * ld + i].x;
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double ej = H[j * ld + j].x;
      rank += (ej < ei) || (ej == ei && j < i);
    }
    s.perm[rank] = i;
  }
  __syncthreads();
  for (int i = tid; i < n; i += NT) s.E1[i] = H[s.perm[i] * ld + s.perm[i]].x;
  // permute V columns through T
  for (int e = tid; e < n * n; e += NT) {
    const int i = e / n, j = e % n;
    s.T[i * ld + j] = V[i * ld + s.perm[j]];
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += NT) {
    const int i = e / n, j = e % n;
    V[i * ld + j] = s.T[i * ld + j];
  }
  __syncthreads();
  return sweep;
}

}  // namespace hjac
