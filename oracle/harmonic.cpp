// Oracle: phonon harmonic Hamiltonian (test infrastructure only).
//
// Restates, in plain C++ with OpenMP over q-points:
//   * PhononH0::setAcousticSumRule "simple" (src/harmonic/phonon_h0_sum_rule.cpp:45-79)
//   * PhononH0::wsInit / wsWeight (src/harmonic/phonon_h0.cpp:426-535)
//   * PhononH0::reorderDynamicalMatrix (src/harmonic/phonon_h0.cpp:672-771)
//   * PhononH0::shortRangeTerm + dynDiagonalize + mass scaling
//     (src/harmonic/phonon_h0.cpp:346-387,773-886)
//   * PhononH0::diagonalizeVelocityFromCoordinates (src/harmonic/phonon_h0.cpp:895-1070)
// The dipole long-range term (phonon_h0.cpp:536-670) is not restated: the
// workloads carry no Born charges, and the one reference fixture that does
// (test/data/444_silicon.fc) has charges that the simple sum rule zeroes.
#include "oracle_common.h"
#include <cstring>
#include <cstdio>

using namespace orc;

namespace {

double ws_weight(const double r[3], const std::vector<double>& rws) {
  // phonon_h0.cpp:506-534
  int nreq = 1;
  int n = (int)rws.size() / 3;
  for (int ir = 0; ir < n; ++ir) {
    const double* g = &rws[3 * ir];
    double rrt = r[0] * g[0] + r[1] * g[1] + r[2] * g[2];
    double ck = rrt - (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) / 2.0;
    if (ck > 1.0e-5) return 0.0;
    if (std::fabs(ck) <= 1.0e-5) nreq += 1;
  }
  return 1.0 / (double)nreq;
}

inline int pmod(int a, int b) { return ((a % b) + b) % b; }

}  // namespace

extern "C" {

// ASR "simple" + Wigner-Seitz reorder.  fc is (3,3,n1,n2,n3,nat,nat) C-order,
// cell is 3x3 C-order with lattice vectors as columns (cell[i*3+j] = a_j[i]),
// pos is (nat,3).  Pass R/w/mat2R = NULL to query numR.  mat2R is written as
// [iR][nb][nb] with nb = 3*nat (row 3*na+i, column 3*nb+j).
int orc_ws_reorder(int nat, const double* cell, const double* pos, const int* grid,
                   const double* fc_in, int* numR_out, double* R, double* w, double* mat2R) {
  const int n1 = grid[0], n2 = grid[1], n3 = grid[2];
  const int nbnd = 3 * nat;
  auto FC = [&](int i, int j, int m1, int m2, int m3, int a, int b) -> size_t {
    return ((((((size_t)i * 3 + j) * n1 + m1) * n2 + m2) * n3 + m3) * nat + a) * nat + b;
  };
  std::vector<double> fc(fc_in, fc_in + (size_t)9 * n1 * n2 * n3 * nat * nat);
  // sum rule, phonon_h0_sum_rule.cpp:64-78
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int na = 0; na < nat; ++na) {
        double sum = 0.0;
        for (int nb = 0; nb < nat; ++nb)
          for (int a = 0; a < n1; ++a)
            for (int b = 0; b < n2; ++b)
              for (int c = 0; c < n3; ++c) sum += fc[FC(i, j, a, b, c, na, nb)];
        fc[FC(i, j, 0, 0, 0, na, na)] -= sum;
      }
  // wsInit, phonon_h0.cpp:426-503 (supercell vectors as WS neighbours)
  double sup[3][3];
  for (int i = 0; i < 3; ++i) {
    sup[i][0] = cell[i * 3 + 0] * n1;
    sup[i][1] = cell[i * 3 + 1] * n2;
    sup[i][2] = cell[i * 3 + 2] * n3;
  }
  std::vector<double> rws;
  for (int ir = -2; ir <= 2; ++ir)
    for (int jr = -2; jr <= 2; ++jr)
      for (int kr = -2; kr <= 2; ++kr) {
        double t[3];
        for (int i = 0; i < 3; ++i) t[i] = sup[i][0] * ir + sup[i][1] * jr + sup[i][2] * kr;
        if (t[0] * t[0] + t[1] * t[1] + t[2] * t[2] > 1.0e-6) rws.insert(rws.end(), t, t + 3);
      }
  const int b1 = 2 * n1, b2 = 2 * n2, b3 = 2 * n3;
  const int s1 = 2 * b1 + 1, s2 = 2 * b2 + 1, s3 = 2 * b3 + 1;
  std::vector<double> cache((size_t)s1 * s2 * s3 * nat * nat, 0.0);
  auto CI = [&](int m3, int m2, int m1, int nb, int na) -> size_t {
    return ((((size_t)m3 * s2 + m2) * s1 + m1) * nat + nb) * nat + na;
  };
  for (int na = 0; na < nat; ++na)
    for (int nb = 0; nb < nat; ++nb) {
      double total = 0.0;
      for (int m1 = -b1; m1 <= b1; ++m1)
        for (int m2 = -b2; m2 <= b2; ++m2)
          for (int m3 = -b3; m3 <= b3; ++m3) {
            double r[3];
            for (int i = 0; i < 3; ++i)
              r[i] = m1 * cell[i * 3 + 0] + m2 * cell[i * 3 + 1] + m3 * cell[i * 3 + 2] +
                     pos[na * 3 + i] - pos[nb * 3 + i];
            double x = ws_weight(r, rws);
            cache[CI(m3 + b3, m2 + b2, m1 + b1, nb, na)] = x;
            total += x;
          }
      if (std::fabs(total - n1 * n2 * n3) > 1.0e-8) return 2;
    }
  // reorderDynamicalMatrix, phonon_h0.cpp:704-764 (loop order n3,n2,n1,nb,na)
  int iR = 0;
  for (int m3 = -b3; m3 <= b3; ++m3)
    for (int m2 = -b2; m2 <= b2; ++m2)
      for (int m1 = -b1; m1 <= b1; ++m1)
        for (int nb = 0; nb < nat; ++nb)
          for (int na = 0; na < nat; ++na) {
            double weight = cache[CI(m3 + b3, m2 + b2, m1 + b1, nb, na)];
            if (weight > 0.0) {
              if (R) {
                w[iR] = weight;
                for (int i = 0; i < 3; ++i)
                  R[iR * 3 + i] = m1 * cell[i * 3 + 0] + m2 * cell[i * 3 + 1] + m3 * cell[i * 3 + 2];
                double* M = mat2R + (size_t)iR * nbnd * nbnd;
                std::memset(M, 0, sizeof(double) * nbnd * nbnd);
                int c1 = pmod(m1, n1), c2 = pmod(m2, n2), c3 = pmod(m3, n3);
                for (int j = 0; j < 3; ++j)
                  for (int i = 0; i < 3; ++i)
                    M[(3 * na + i) * nbnd + 3 * nb + j] += fc[FC(i, j, c1, c2, c3, na, nb)];
              }
              ++iR;
            }
          }
  *numR_out = iR;
  return 0;
}

// Dynamical matrix FT + diagonalisation at nq Cartesian wavevectors.
// energies: (nq,nb); eigvecs: (nq,nb,nb) complex, U[a][band].
// masses: per band (nb).  with_mass_scaling divides rows by sqrt(m).
int orc_ph_diag(int nbnd, int numR, const double* R, const double* w, const double* mat2R,
                const double* masses, int nq, const double* q, int with_mass_scaling,
                double* energies, double* eigvecs) {
  int err = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : err)
  for (int iq = 0; iq < nq; ++iq) {
    std::vector<cd> D(nbnd * nbnd, cd(0, 0)), Dh(nbnd * nbnd), Z(nbnd * nbnd);
    std::vector<double> w2(nbnd);
    const double* qq = q + 3 * iq;
    // shortRangeTerm, phonon_h0.cpp:773-813
    for (int ir = 0; ir < numR; ++ir) {
      double arg = qq[0] * R[3 * ir] + qq[1] * R[3 * ir + 1] + qq[2] * R[3 * ir + 2];
      cd phase = std::exp(cd(0.0, -arg));
      const double* M = mat2R + (size_t)ir * nbnd * nbnd;
      for (int k = 0; k < nbnd * nbnd; ++k) D[k] += M[k] * phase * w[ir];
    }
    // dynDiagonalize, phonon_h0.cpp:815-886: hermitise, divide by sqrt(m_i m_j)
    for (int i = 0; i < nbnd; ++i)
      for (int j = 0; j < nbnd; ++j) {
        cd x = D[i * nbnd + j] + std::conj(D[j * nbnd + i]);
        x *= 0.5;
        x /= std::sqrt(masses[i] * masses[j]);
        Dh[i * nbnd + j] = x;
      }
    if (hermitian_eig(nbnd, Dh.data(), w2.data(), Z.data())) err |= 1;
    for (int b = 0; b < nbnd; ++b)
      energies[(size_t)iq * nbnd + b] = w2[b] < 0 ? -std::sqrt(-w2[b]) : std::sqrt(w2[b]);
    double* ev = eigvecs + (size_t)iq * nbnd * nbnd * 2;
    for (int a = 0; a < nbnd; ++a)
      for (int b = 0; b < nbnd; ++b) {
        cd z = Z[a * nbnd + b];
        if (with_mass_scaling) z /= std::sqrt(masses[a]);
        ev[2 * (a * nbnd + b)] = z.real();
        ev[2 * (a * nbnd + b) + 1] = z.imag();
      }
  }
  return err;
}

// Velocity operator (phonon_h0.cpp:895-1070), returning group velocities
// (nq,nb,3) = Re diag of the velocity operator after the degenerate-subspace
// rediagonalisation, plus optionally the full operator (nq,nb,nb,3) complex.
int orc_ph_velocities(int nbnd, int numR, const double* R, const double* w, const double* mat2R,
                      const double* masses, int nq, const double* q, double* vgroup,
                      double* vfull) {
  const double deltaQ = 1.0e-8;
  const double degThr = 0.0001 / ryToCmm1;
  int err = 0;
#pragma omp parallel for schedule(dynamic, 2) reduction(| : err)
  for (int iq = 0; iq < nq; ++iq) {
    const int n = nbnd;
    std::vector<double> E0(n), Ep(n), Em(n);
    std::vector<double> U0(2 * n * n), Up(2 * n * n), Um(2 * n * n);
    std::vector<cd> vel((size_t)n * n * 3);
    const double* qq = q + 3 * iq;
    err |= orc_ph_diag(n, numR, R, w, mat2R, masses, 1, qq, 0, E0.data(), U0.data());
    auto U = [](const std::vector<double>& u, int n, int a, int b) {
      return cd(u[2 * (a * n + b)], u[2 * (a * n + b) + 1]);
    };
    for (int ic = 0; ic < 3; ++ic) {
      double qp[3] = {qq[0], qq[1], qq[2]}, qm[3] = {qq[0], qq[1], qq[2]};
      qp[ic] += deltaQ;
      qm[ic] -= deltaQ;
      err |= orc_ph_diag(n, numR, R, w, mat2R, masses, 1, qp, 0, Ep.data(), Up.data());
      err |= orc_ph_diag(n, numR, R, w, mat2R, masses, 1, qm, 0, Em.data(), Um.data());
      std::vector<cd> der(n * n), der2(n * n), tmp(n * n);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          cd sp = 0.0, sm = 0.0;
          for (int l = 0; l < n; ++l) {
            sp += U(Up, n, i, l) * Ep[l] * std::conj(U(Up, n, j, l));
            sm += U(Um, n, i, l) * Em[l] * std::conj(U(Um, n, j, l));
          }
          der[i * n + j] = (sp - sm) / (2.0 * deltaQ);
        }
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          der2[i * n + j] = 0.5 * (der[i * n + j] + std::conj(der[j * n + i]));
      // der = U0^H der U0
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          cd s = 0.0;
          for (int l = 0; l < n; ++l) s += der2[i * n + l] * U(U0, n, l, j);
          tmp[i * n + j] = s;
        }
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          cd s = 0.0;
          for (int l = 0; l < n; ++l) s += std::conj(U(U0, n, l, i)) * tmp[l * n + j];
          vel[((size_t)i * n + j) * 3 + ic] = s;
        }
    }
    // degenerate subspaces, phonon_h0.cpp:1008-1055
    for (int ib = 0; ib < n; ++ib) {
      int size = 1;
      for (int ib2 = ib + 1; ib2 < n; ++ib2) {
        if (std::fabs(E0[ib] - E0[ib2]) > degThr) break;
        size += 1;
      }
      if (size > 1) {
        for (int ic = 0; ic < 3; ++ic) {
          std::vector<cd> sub(size * size), sub2(size * size), Z(size * size), t(size * size);
          std::vector<double> ev(size);
          for (int i = 0; i < size; ++i)
            for (int j = 0; j < size; ++j) sub[i * size + j] = vel[((size_t)(ib + i) * n + ib + j) * 3 + ic];
          for (int i = 0; i < size; ++i)
            for (int j = 0; j < size; ++j)
              sub2[i * size + j] = 0.5 * (sub[i * size + j] + std::conj(sub[j * size + i]));
          sub = sub2;
          if (hermitian_eig(size, sub2.data(), ev.data(), Z.data())) err |= 1;
          // sub = Z^H sub Z, hermitised
          for (int i = 0; i < size; ++i)
            for (int j = 0; j < size; ++j) {
              cd s = 0.0;
              for (int l = 0; l < size; ++l) s += sub[i * size + l] * Z[l * size + j];
              t[i * size + j] = s;
            }
          for (int i = 0; i < size; ++i)
            for (int j = 0; j < size; ++j) {
              cd s = 0.0;
              for (int l = 0; l < size; ++l) s += std::conj(Z[l * size + i]) * t[l * size + j];
              sub2[i * size + j] = s;
            }
          for (int i = 0; i < size; ++i)
            for (int j = 0; j < size; ++j)
              vel[((size_t)(ib + i) * n + ib + j) * 3 + ic] =
                  0.5 * (sub2[i * size + j] + std::conj(sub2[j * size + i]));
        }
      }
      ib += size - 1;
    }
    if (std::sqrt(qq[0] * qq[0] + qq[1] * qq[1] + qq[2] * qq[2]) < 1.0e-6)
      for (auto& x : vel) x = 0.0;
    for (int b = 0; b < n; ++b)
      for (int ic = 0; ic < 3; ++ic)
        vgroup[((size_t)iq * n + b) * 3 + ic] = vel[((size_t)b * n + b) * 3 + ic].real();
    if (vfull)
      for (size_t k = 0; k < vel.size(); ++k) {
        vfull[(size_t)iq * n * n * 3 * 2 + 2 * k] = vel[k].real();
        vfull[(size_t)iq * n * n * 3 * 2 + 2 * k + 1] = vel[k].imag();
      }
  }
  return err;
}

}  // extern "C"
