// Electron-phonon Wannier path of the oracle (TEST INFRASTRUCTURE ONLY; see
// oracle_common.h).  CPU FP64 restatement of:
//   * ElectronH0Wannier::batchedBuildHamiltonians / batchedDiagonalizeFromCoordinates
//     (src/harmonic/electron_h0_wannier.cpp:160-235) and
//     batchedDiagonalizeWithVelocities (:633-760)
//   * InteractionElPhWan::cacheElPh (src/interaction/interaction_elph.cpp:492-701,
//     single-process branch) and calcCouplingSquared (:229-448, no polar term)
//   * ElScatteringMatrix::builder, linewidth mode (src/bte/el_scattering.cpp:38-405)
//     with HelperElScattering::get on a common mesh (src/bte/helper_el_scattering.cpp:230-288),
//     symmetrizeCoupling (src/bte/scattering.cpp:1209-1318) and
//     degeneracyAveragingLinewidths (:1168-1207).
// Arrays are C-order; complex arrays interleaved (re, im).  Electron eigenvectors
// are U[w][b] (row = Wannier orbital, column = band); phonon eigenvectors
// U[a][nu] (row = 3*atom + cartesian, column = branch).
#include "oracle_common.h"
#include <algorithm>
#include <cstring>

namespace {

using orc::cd;

// H(k) = sum_R e^{+i k.R} / deg_R H(R)   (electron_h0_wannier.cpp:166-184)
void build_h(int nw, int nR, const double* R, const double* deg, const double* H, const double* k,
             cd* out) {
  const int m2 = nw * nw;
  std::vector<cd> ph(nR);
  for (int ir = 0; ir < nR; ++ir) {
    const double arg = k[0] * R[3 * ir] + k[1] * R[3 * ir + 1] + k[2] * R[3 * ir + 2];
    ph[ir] = cd(std::cos(arg), std::sin(arg)) / deg[ir];
  }
  for (int e = 0; e < m2; ++e) {
    cd acc(0.0, 0.0);
    for (int ir = 0; ir < nR; ++ir)
      acc += ph[ir] * cd(H[2 * ((size_t)ir * m2 + e)], H[2 * ((size_t)ir * m2 + e) + 1]);
    out[e] = acc;
  }
}

// degenerate subspace of the velocity operator (electron_h0_wannier.cpp:710-757):
// the group velocities of a block are the ascending eigenvalues of its hermitised part
void degenerate_fix(int n, const double* E, double thr, const std::vector<cd>& vop, double* vg) {
  for (int ib = 0; ib < n;) {
    int size = 1;
    for (int ib2 = ib + 1; ib2 < n; ++ib2) {
      if (std::fabs(E[ib] - E[ib2]) > thr) break;
      ++size;
    }
    if (size > 1) {
      std::vector<cd> sub(size * size), Z(size * size);
      std::vector<double> w(size);
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j)
          sub[i * size + j] = 0.5 * (vop[(ib + i) * n + ib + j] + std::conj(vop[(ib + j) * n + ib + i]));
      orc::hermitian_eig(size, sub.data(), w.data(), Z.data());
      for (int i = 0; i < size; ++i) vg[ib + i] = w[i];
    } else {
      vg[ib] = vop[ib * n + ib].real();
    }
    ib += size;
  }
}

double gauss_delta(double sigma, double e) {
  // delta_function.cpp:40-45 (one-sided cut-off)
  const double x = e / sigma;
  if (x > 6.0) return 0.0;
  return 1.0 / sigma / std::sqrt(orc::pi) * std::exp(-x * x);
}

double adaptive_delta(const double qT[9], double e, const double v[3]) {
  // delta_function.cpp:65-96 (same order of tests as the phonon oracle)
  const double cutoff = 0.0001 / orc::energyRyToEv;
  const double vn = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (vn == 0.0 && e == 0.0) return 1.0;
  double s = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double d = qT[3 * i] * v[0] + qT[3 * i + 1] * v[1] + qT[3 * i + 2] * v[2];
    s += d * d;
  }
  double sigma = 1.0 * std::sqrt(s / 6.0);
  if (sigma == 0.0) return 0.0;
  if (sigma < cutoff) sigma = cutoff;
  if (std::fabs(e) > 2.0 * sigma) return 0.0;
  const double x = e / sigma;
  if (x > 6.0) return 0.0;
  return std::exp(-x * x) / std::sqrt(orc::pi) / sigma / 0.9953222650189527;
}

// symmetrizeCoupling (scattering.cpp:1209-1318) on c(nb1, nb2, nb3)
void symmetrize3(double* c, int nb1, int nb2, int nb3, const double* e1, const double* e2,
                 const double* e3) {
  auto C = [&](int i, int j, int k) -> double& { return c[((size_t)i * nb2 + j) * nb3 + k]; };
  for (int ib1 = 0; ib1 < nb1; ++ib1) {
    int deg = 0;
    for (int i = ib1; i < nb1; ++i) {
      if (std::fabs(e1[ib1] - e1[i]) < 1.0e-6) deg++;
      else break;
    }
    std::vector<double> tmp((size_t)nb2 * nb3, 0.0);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb2; ++j)
        for (int k = 0; k < nb3; ++k) tmp[j * nb3 + k] += C(ib1 + i, j, k);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb2; ++j)
        for (int k = 0; k < nb3; ++k) C(ib1 + i, j, k) = tmp[j * nb3 + k] / float(deg);
    ib1 += deg - 1;
  }
  for (int ib2 = 0; ib2 < nb2; ++ib2) {
    int deg = 0;
    for (int i = ib2; i < nb2; ++i) {
      if (std::fabs(e2[ib2] - e2[i]) < 1.0e-6) deg++;
      else break;
    }
    std::vector<double> tmp((size_t)nb1 * nb3, 0.0);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb1; ++j)
        for (int k = 0; k < nb3; ++k) tmp[j * nb3 + k] += C(j, ib2 + i, k);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb1; ++j)
        for (int k = 0; k < nb3; ++k) C(j, ib2 + i, k) = tmp[j * nb3 + k] / float(deg);
    ib2 += deg - 1;
  }
  for (int ib3 = 0; ib3 < nb3; ++ib3) {
    int deg = 0;
    for (int i = ib3; i < nb3; ++i) {
      if (std::fabs(e3[ib3] - e3[i]) < 1.0e-6) deg++;
      else break;
    }
    std::vector<double> tmp((size_t)nb1 * nb2, 0.0);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb1; ++j)
        for (int k = 0; k < nb2; ++k) tmp[j * nb2 + k] += C(j, k, ib3 + i);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb1; ++j)
        for (int k = 0; k < nb2; ++k) C(j, k, ib3 + i) = tmp[j * nb2 + k] / float(deg);
    ib3 += deg - 1;
  }
}

int pmod(int a, int n) { return ((a % n) + n) % n; }

}  // namespace

extern "C" {

// ElectronH0Wannier: energies (nk,nw) ascending, eigvecs (nk,nw,nw) U[w][b],
// optionally group velocities (nk,nw,3) (may be NULL).
int orc_el_diag(int nw, int nR, const double* R, const double* deg, const double* H, int nk,
                const double* k, double* energies, double* eigvecs, double* vgroup) {
  const double delta = 1.0e-8;
  const double thr = 0.000001 / orc::energyRyToEv;  // 1 micro-eV
  int err = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : err)
  for (int ik = 0; ik < nk; ++ik) {
    const int n = nw;
    std::vector<cd> Hk(n * n), Z(n * n);
    std::vector<double> w(n);
    const double* kk = k + 3 * ik;
    build_h(nw, nR, R, deg, H, kk, Hk.data());
    if (orc::hermitian_eig(n, Hk.data(), w.data(), Z.data())) err |= 1;
    for (int b = 0; b < n; ++b) energies[(size_t)ik * n + b] = w[b];
    for (int e = 0; e < n * n; ++e) {
      eigvecs[2 * ((size_t)ik * n * n + e)] = Z[e].real();
      eigvecs[2 * ((size_t)ik * n * n + e) + 1] = Z[e].imag();
    }
    if (!vgroup) continue;
    const bool gamma = std::sqrt(kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2]) < 1.0e-6;
    for (int ic = 0; ic < 3; ++ic) {
      if (gamma) {
        for (int b = 0; b < n; ++b) vgroup[((size_t)ik * n + b) * 3 + ic] = 0.0;
        continue;
      }
      double kp[3] = {kk[0], kk[1], kk[2]}, km[3] = {kk[0], kk[1], kk[2]};
      kp[ic] += delta;
      km[ic] -= delta;
      std::vector<cd> Hp(n * n), Hm(n * n), der(n * n), derh(n * n), tmp(n * n), vop(n * n);
      build_h(nw, nR, R, deg, H, kp, Hp.data());
      build_h(nw, nR, R, deg, H, km, Hm.data());
      for (int e = 0; e < n * n; ++e) der[e] = (Hp[e] - Hm[e]) / (2.0 * delta);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) derh[i * n + j] = 0.5 * (der[i * n + j] + std::conj(der[j * n + i]));
      // U^H der U
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          cd acc(0.0, 0.0);
          for (int l = 0; l < n; ++l) acc += derh[i * n + l] * Z[l * n + j];
          tmp[i * n + j] = acc;
        }
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          cd acc(0.0, 0.0);
          for (int l = 0; l < n; ++l) acc += std::conj(Z[l * n + i]) * tmp[l * n + j];
          vop[i * n + j] = acc;
        }
      std::vector<double> vg(n);
      degenerate_fix(n, w.data(), thr, vop, vg.data());
      for (int b = 0; b < n; ++b) vgroup[((size_t)ik * n + b) * 3 + ic] = vg[b];
    }
  }
  return err;
}

// cacheElPh: cached(Rp, nu, b1, w2) = sum_w1 U1[w1][b1] sum_Re g(Re,Rp,nu,w1,w2) e^{+i k1.Re}/deg_e.
// g is FP32 complex (nRe, nRp, nph, nw, nw); U1 is (nw, nb1) complex.
int orc_elph_cache(int nw, int nph, int nRe, int nRp, const double* Re, const double* degE,
                   const float* g, const double* k1, const double* U1, int nb1, double* cached) {
  const size_t inner = (size_t)nRp * nph * nw * nw;
  std::vector<cd> ph(nRe);
  for (int ir = 0; ir < nRe; ++ir) {
    const double arg = k1[0] * Re[3 * ir] + k1[1] * Re[3 * ir + 1] + k1[2] * Re[3 * ir + 2];
    ph[ir] = cd(std::cos(arg), std::sin(arg)) / degE[ir];
  }
  std::vector<cd> g1(inner, cd(0.0, 0.0));
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < (long long)inner; ++e) {
    cd acc(0.0, 0.0);
    for (int ir = 0; ir < nRe; ++ir) {
      const float* x = g + 2 * ((size_t)ir * inner + e);
      acc += cd((double)x[0], (double)x[1]) * ph[ir];
    }
    g1[e] = acc;
  }
  for (int irp = 0; irp < nRp; ++irp)
    for (int nu = 0; nu < nph; ++nu)
      for (int b1 = 0; b1 < nb1; ++b1)
        for (int w2 = 0; w2 < nw; ++w2) {
          cd acc(0.0, 0.0);
          for (int w1 = 0; w1 < nw; ++w1)
            acc += g1[(((size_t)irp * nph + nu) * nw + w1) * nw + w2] *
                   cd(U1[2 * (w1 * nb1 + b1)], U1[2 * (w1 * nb1 + b1) + 1]);
          const size_t o = (((size_t)irp * nph + nu) * nb1 + b1) * nw + w2;
          cached[2 * o] = acc.real();
          cached[2 * o + 1] = acc.imag();
        }
  return 0;
}

// calcCouplingSquared for nk2 final states: coupling (nk2, nb1, nb2max, nph) = |g|^2 with
// g(b1, b2, nu) = sum_w2 conj(U2[w2][b2]) sum_nu' ev3[nu'][nu] sum_Rp e^{+i q3.Rp}/deg_p cached(Rp,nu',b1,w2).
//   U2s (nk2, nw, nb2max) complex, nb2s (nk2); ev3s (nk2, nph, nph) complex U[a][nu]; q3s (nk2,3)
int orc_elph_couplings(int nw, int nph, int nRp, const double* Rp, const double* degP,
                       const double* cached, int nb1, int nk2, const double* q3s, const double* U2s,
                       const int* nb2s, int nb2max, const double* ev3s, double* coupling) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int ik = 0; ik < nk2; ++ik) {
    const double* q = q3s + 3 * ik;
    std::vector<cd> ph(nRp);
    for (int ir = 0; ir < nRp; ++ir) {
      const double arg = q[0] * Rp[3 * ir] + q[1] * Rp[3 * ir + 1] + q[2] * Rp[3 * ir + 2];
      ph[ir] = std::exp(cd(0.0, 1.0) * arg) / degP[ir];
    }
    std::vector<cd> g3((size_t)nph * nb1 * nw), g4((size_t)nph * nb1 * nw);
    for (int nu = 0; nu < nph; ++nu)
      for (int b1 = 0; b1 < nb1; ++b1)
        for (int w2 = 0; w2 < nw; ++w2) {
          cd acc(0.0, 0.0);
          for (int ir = 0; ir < nRp; ++ir) {
            const size_t o = (((size_t)ir * nph + nu) * nb1 + b1) * nw + w2;
            acc += ph[ir] * cd(cached[2 * o], cached[2 * o + 1]);
          }
          g3[((size_t)nu * nb1 + b1) * nw + w2] = acc;
        }
    const double* E3 = ev3s + (size_t)ik * nph * nph * 2;
    for (int nu2 = 0; nu2 < nph; ++nu2)
      for (int b1 = 0; b1 < nb1; ++b1)
        for (int w2 = 0; w2 < nw; ++w2) {
          cd acc(0.0, 0.0);
          for (int nu = 0; nu < nph; ++nu)
            acc += g3[((size_t)nu * nb1 + b1) * nw + w2] * cd(E3[2 * (nu * nph + nu2)], E3[2 * (nu * nph + nu2) + 1]);
          g4[((size_t)nu2 * nb1 + b1) * nw + w2] = acc;
        }
    const double* U2 = U2s + (size_t)ik * nw * nb2max * 2;
    for (int b1 = 0; b1 < nb1; ++b1)
      for (int b2 = 0; b2 < nb2max; ++b2)
        for (int nu = 0; nu < nph; ++nu) {
          double v = 0.0;
          if (b2 < nb2s[ik]) {
            cd acc(0.0, 0.0);
            for (int w2 = 0; w2 < nw; ++w2)
              acc += std::conj(cd(U2[2 * (w2 * nb2max + b2)], U2[2 * (w2 * nb2max + b2) + 1])) *
                     g4[((size_t)nu * nb1 + b1) * nw + w2];
            v = acc.real() * acc.real() + acc.imag() * acc.imag();
          }
          coupling[(((size_t)ik * nb1 + b1) * nb2max + b2) * nph + nu] = v;
        }
  }
  return 0;
}

// ElScatteringMatrix::builder, linewidth mode, on a Gamma-centred k mesh with
// k2 = k1 + q for every q of a q mesh that divides the k mesh.
//   kmesh/qmesh (3); Ek (nk,nw), Uk (nk,nw,nw), vk (nk,nw,3) electron data on the k mesh;
//   lo/hi (nk): active band range [lo, hi) of every k point (energy window);
//   Eq (nq,nph), evq (nq,nph,nph), phonon data on the q mesh; kcart (nk,3);
//   recipk: reciprocal cell 3x3 C-order (columns = b vectors);
//   k1list (nk1): outer k points; temps (nT), mu; smearing 0 gaussian / 1 adaptive;
//   norm: prefactor of every rate (1/N of the summed mesh).
//   out (nT, nk1, nw): linewidths of the active states (zero elsewhere), after
//   degeneracy averaging of row 0 (scattering.cpp:1168-1207).
int orc_el_linewidths(int nw, int nph, int nRe, int nRp, const double* Re, const double* degE,
                      const double* Rp, const double* degP, const float* g, const int* kmesh,
                      const int* qmesh, const double* Ek, const double* Uk, const double* vk,
                      const int* lo, const int* hi, const double* Eq, const double* evq,
                      const double* kcart, const double* recipk, int nk1, const int* k1list,
                      int nT, const double* temps, double mu, int smearing, double sigma,
                      double norm, double* out) {
  const int nq = qmesh[0] * qmesh[1] * qmesh[2];
  int f[3];
  for (int i = 0; i < 3; ++i) {
    if (kmesh[i] % qmesh[i]) return 1;
    f[i] = kmesh[i] / qmesh[i];
  }
  double qT[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) qT[i * 3 + j] = recipk[i * 3 + j] / kmesh[i];
  const double phononCutoff = 5.0 / orc::ryToCmm1;  // el_scattering.cpp:127
  std::memset(out, 0, sizeof(double) * (size_t)nT * nk1 * nw);
  auto fermi = [&](double e, double T) {
    if (T <= 0.0) return e <= mu ? 1.0 : 0.0;
    double p = 1.0 / (std::exp((e - mu) / T) + 1.0);
    return std::min(1.0, std::max(0.0, p));
  };
  auto bose = [&](double e, double T) {
    if (T <= 0.0) return 0.0;
    double p = 1.0 / (std::exp(e / T) - 1.0);
    return p < 0.0 ? 0.0 : p;
  };
  for (int i1 = 0; i1 < nk1; ++i1) {
    const int ik1 = k1list[i1];
    const int nb1 = hi[ik1] - lo[ik1];
    if (nb1 <= 0) continue;
    const int x1 = ik1 % kmesh[0], y1 = (ik1 / kmesh[0]) % kmesh[1], z1 = ik1 / (kmesh[0] * kmesh[1]);
    // outer eigenvectors of the active bands
    std::vector<double> U1((size_t)nw * nb1 * 2);
    for (int w = 0; w < nw; ++w)
      for (int b = 0; b < nb1; ++b) {
        U1[2 * (w * nb1 + b)] = Uk[2 * (((size_t)ik1 * nw + w) * nw + lo[ik1] + b)];
        U1[2 * (w * nb1 + b) + 1] = Uk[2 * (((size_t)ik1 * nw + w) * nw + lo[ik1] + b) + 1];
      }
    std::vector<double> cached((size_t)nRp * nph * nb1 * nw * 2);
    orc_elph_cache(nw, nph, nRe, nRp, Re, degE, g, kcart + 3 * ik1, U1.data(), nb1, cached.data());
    // final states k2 = k1 + q with active bands
    std::vector<int> k2s, q3i;
    for (int iq = 0; iq < nq; ++iq) {
      const int qx = iq % qmesh[0], qy = (iq / qmesh[0]) % qmesh[1], qz = iq / (qmesh[0] * qmesh[1]);
      const int ik2 = pmod(x1 + f[0] * qx, kmesh[0]) + kmesh[0] * (pmod(y1 + f[1] * qy, kmesh[1]) +
                                                                  kmesh[1] * pmod(z1 + f[2] * qz, kmesh[2]));
      if (hi[ik2] - lo[ik2] <= 0) continue;
      k2s.push_back(ik2);
      q3i.push_back(iq);
    }
    const int n2 = (int)k2s.size();
    int nb2max = 0;
    for (int ik2 : k2s) nb2max = std::max(nb2max, hi[ik2] - lo[ik2]);
    std::vector<double> q3s((size_t)n2 * 3), U2s((size_t)n2 * nw * nb2max * 2, 0.0),
        ev3s((size_t)n2 * nph * nph * 2);
    std::vector<int> nb2s(n2);
    for (int j = 0; j < n2; ++j) {
      const int ik2 = k2s[j];
      // q3 = k2 - k1 (helper_el_scattering.cpp:233-234)
      for (int i = 0; i < 3; ++i) q3s[3 * j + i] = kcart[3 * ik2 + i] - kcart[3 * ik1 + i];
      nb2s[j] = hi[ik2] - lo[ik2];
      for (int w = 0; w < nw; ++w)
        for (int b = 0; b < nb2s[j]; ++b) {
          U2s[2 * (((size_t)j * nw + w) * nb2max + b)] = Uk[2 * (((size_t)ik2 * nw + w) * nw + lo[ik2] + b)];
          U2s[2 * (((size_t)j * nw + w) * nb2max + b) + 1] =
              Uk[2 * (((size_t)ik2 * nw + w) * nw + lo[ik2] + b) + 1];
        }
      std::memcpy(&ev3s[(size_t)j * nph * nph * 2], evq + (size_t)q3i[j] * nph * nph * 2,
                  sizeof(double) * nph * nph * 2);
    }
    std::vector<double> cpl((size_t)n2 * nb1 * nb2max * nph);
    orc_elph_couplings(nw, nph, nRp, Rp, degP, cached.data(), nb1, n2, q3s.data(), U2s.data(),
                       nb2s.data(), nb2max, ev3s.data(), cpl.data());
    const double* E1 = Ek + (size_t)ik1 * nw + lo[ik1];
    for (int j = 0; j < n2; ++j) {
      const int ik2 = k2s[j], iq = q3i[j], nb2 = nb2s[j];
      const double* E2 = Ek + (size_t)ik2 * nw + lo[ik2];
      const double* E3 = Eq + (size_t)iq * nph;
      // the coupling of this final state, (nb1, nb2, nph), symmetrised
      std::vector<double> c((size_t)nb1 * nb2 * nph);
      for (int b1 = 0; b1 < nb1; ++b1)
        for (int b2 = 0; b2 < nb2; ++b2)
          for (int nu = 0; nu < nph; ++nu)
            c[((size_t)b1 * nb2 + b2) * nph + nu] = cpl[(((size_t)j * nb1 + b1) * nb2max + b2) * nph + nu];
      symmetrize3(c.data(), nb1, nb2, nph, E1, E2, E3);
      for (int b2 = 0; b2 < nb2; ++b2) {
        const double en2 = E2[b2];
        for (int b1 = 0; b1 < nb1; ++b1) {
          const double en1 = E1[b1];
          for (int nu = 0; nu < nph; ++nu) {
            const double en3 = E3[nu];
            if (en3 < phononCutoff) continue;
            double d1, d2;
            if (smearing == 0) {
              d1 = gauss_delta(sigma, en1 - en2 + en3);
              d2 = gauss_delta(sigma, en1 - en2 - en3);
            } else {
              double v[3];
              for (int i = 0; i < 3; ++i)
                v[i] = vk[((size_t)ik1 * nw + lo[ik1] + b1) * 3 + i] - vk[((size_t)ik2 * nw + lo[ik2] + b2) * 3 + i];
              d1 = adaptive_delta(qT, en1 - en2 + en3, v);
              d2 = adaptive_delta(qT, en1 - en2 - en3, v);
            }
            if (d1 <= 0.0 && d2 <= 0.0) continue;
            const double cc = c[((size_t)b1 * nb2 + b2) * nph + nu];
            for (int it = 0; it < nT; ++it) {
              const double fermi2 = fermi(en2, temps[it]);
              const double bose3 = bose(en3, temps[it]);
              const double rate = cc * ((fermi2 + bose3) * d1 + (1.0 - fermi2 + bose3) * d2) * norm / en3 * orc::pi;
              out[((size_t)it * nk1 + i1) * nw + lo[ik1] + b1] += rate;
            }
          }
        }
      }
    }
    // degeneracyAveragingLinewidths, row iCalc = 0 (scattering.cpp:1168-1207)
    std::vector<double> tmp(nb1);
    for (int b1 = 0; b1 < nb1; ++b1) {
      int n = 0;
      double s = 0.0;
      for (int b2 = 0; b2 < nb1; ++b2)
        if (std::fabs(E1[b2] - E1[b1]) < 1.0e-6) {
          ++n;
          s += out[(size_t)i1 * nw + lo[ik1] + b2];
        }
      tmp[b1] = s / float(n);
    }
    for (int b1 = 0; b1 < nb1; ++b1) out[(size_t)i1 * nw + lo[ik1] + b1] = tmp[b1];
  }
  return 0;
}

}  // extern "C"
