// Oracle: 3-phonon vertex and RTA linewidth builder (test infrastructure only).
//
// Restates, in plain C++ with OpenMP where the reference runs Kokkos or
// OpenMP loops:
//   * Interaction3Ph::cacheD3 (src/interaction/interaction_3ph.cpp:100-175)
//   * Interaction3Ph::getCouplingsSquared (src/interaction/interaction_3ph.cpp:179-405),
//     including the weights3 factor applied in both stages (:166-169, :284-285)
//   * ScatteringMatrix::symmetrizeCoupling (src/bte/scattering.cpp:1209-1318)
//   * PhScatteringMatrix::builder (src/bte/ph_scattering.cpp:60-935) in its three
//     modes without symmetries: switchCase 2 (linewidths), 0 (matrix in memory,
//     :382-406, :520-547, :714-738, :846-847, :864-890, :910-933) and 1 (matrix-vector
//     product, :408-431, :549-572, :741-759, :849-855, :891-897), with
//     Helper3rdState case 1 (src/bte/helper_3rd_state.cpp:128-170)
//   * ScatteringMatrix::dot / offDiagonalDot of a stored matrix (src/bte/scattering.cpp:
//     180-265, 266-330)
//   * GaussianDeltaFunction / AdaptiveGaussianDeltaFunction (src/delta_function.cpp:34-96)
//   * Particle::getPopulation / getPopPopPm1 / getDndt (src/particle.cpp:64-128)
//   * ScatteringMatrix::degeneracyAveragingLinewidths (src/bte/scattering.cpp:1168-1207),
//     getSingleModeTimes (:484-527), BulkTDrift (src/bte/drift.cpp:3-29) and
//     PhononThermalConductivity::calcFromPopulation (src/observable/phonon_thermal_cond.cpp:64-113)
// The serial "HOT LOOP 3" of the builder stays serial, as in the reference.
#include "oracle_common.h"
#include <algorithm>
#include <cstring>

using namespace orc;

namespace {

struct V3 {
  int nb, nat, nr2, nr3;
  std::vector<double> D3;   // (nb,nb,nb,nr3,nr2)
  std::vector<double> R2, R3, w2, w3;
  std::vector<cd> plus, mins;  // cached (nb,nb,nb,nr3)
};

double bose(double e, double t) {
  // particle.cpp:64-96, chemical potential 0
  if (t <= 0.0) return e <= 0.0 ? 1.0 : 0.0;
  double y = e / t;
  double n = 1.0 / (std::exp(y) - 1.0);
  return n < 0.0 ? 0.0 : n;
}

double poppm1(double e, double t) {
  // particle.cpp:117-128
  double x = std::sinh(e / 2.0 / t);
  return 0.25 / x / x;
}

void cache_d3(V3& v, const double* q2) {
  const int nb = v.nb, nr2 = v.nr2, nr3 = v.nr3;
  std::vector<cd> pp2(nr2), pm2(nr2), pp3(nr3), pm3(nr3);
  for (int ir = 0; ir < nr2; ++ir) {
    double a = q2[0] * v.R2[3 * ir] + q2[1] * v.R2[3 * ir + 1] + q2[2] * v.R2[3 * ir + 2];
    pp2[ir] = std::exp(cd(0, a));
    pm2[ir] = std::exp(cd(0, -a));
  }
  for (int ir = 0; ir < nr3; ++ir) {
    double a = q2[0] * v.R3[3 * ir] + q2[1] * v.R3[3 * ir + 1] + q2[2] * v.R3[3 * ir + 2];
    pp3[ir] = std::exp(cd(0, -a));
    pm3[ir] = std::exp(cd(0, a));
  }
  v.plus.assign((size_t)nb * nb * nb * nr3, 0.0);
  v.mins.assign((size_t)nb * nb * nb * nr3, 0.0);
  const int nat = v.nat;
#pragma omp parallel for collapse(2)
  for (int i1 = 0; i1 < nb; ++i1)
    for (int i2 = 0; i2 < nb; ++i2)
      for (int i3 = 0; i3 < nb; ++i3)
        for (int ir3 = 0; ir3 < nr3; ++ir3) {
          int at1 = i1 / 3, at2 = i2 / 3, at3 = i3 / 3;
          cd tp = 0.0, tm = 0.0;
          size_t base = ((((size_t)i1 * nb + i2) * nb + i3) * nr3 + ir3) * nr2;
          for (int ir2 = 0; ir2 < nr2; ++ir2) {
            double d = v.D3[base + ir2];
            double ww = v.w2[((size_t)ir2 * nat + at1) * nat + at2] *
                        v.w3[((size_t)ir3 * nat + at1) * nat + at3];
            tp += d * pp2[ir2] * pp3[ir3] * ww;
            tm += d * pm2[ir2] * pm3[ir3] * ww;
          }
          size_t o = (((size_t)i1 * nb + i2) * nb + i3) * nr3 + ir3;
          v.plus[o] = tp;
          v.mins[o] = tm;
        }
}

inline cd EV(const double* ev, int nb, int a, int b) {
  return cd(ev[2 * (a * nb + b)], ev[2 * (a * nb + b) + 1]);
}

// One q1 of getCouplingsSquared (full bands).  outP/outM: (nb1,nb2,nb3).
void couplings_one(const V3& v, const double* q1, const double* ev1, int nb1, const double* ev2,
                   int nb2, const double* ev3p, int nb3p, const double* ev3m, int nb3m,
                   double* outP, double* outM) {
  const int nb = v.nb, nr3 = v.nr3, nat = v.nat;
  std::vector<cd> ph(nr3);
  for (int ir = 0; ir < nr3; ++ir) {
    double a = -(q1[0] * v.R3[3 * ir] + q1[1] * v.R3[3 * ir + 1] + q1[2] * v.R3[3 * ir + 2]);
    ph[ir] = std::exp(cd(0, a));
  }
  const size_t nb3 = (size_t)nb * nb * nb;
  std::vector<cd> tP(nb3), tM(nb3);
  for (int a1 = 0; a1 < nb; ++a1)
    for (int a2 = 0; a2 < nb; ++a2)
      for (int a3 = 0; a3 < nb; ++a3) {
        int at1 = a1 / 3, at3 = a3 / 3;
        cd sp = 0.0, sm = 0.0;
        size_t base = (((size_t)a1 * nb + a2) * nb + a3) * nr3;
        for (int ir = 0; ir < nr3; ++ir) {
          double ww = v.w3[((size_t)ir * nat + at1) * nat + at3];
          sp += v.plus[base + ir] * ph[ir] * ww;
          sm += v.mins[base + ir] * ph[ir] * ww;
        }
        tP[((size_t)a1 * nb + a2) * nb + a3] = sp;
        tM[((size_t)a1 * nb + a2) * nb + a3] = sm;
      }
  // tmp1(ib1, a3, a2) = sum_a1 tmp(a1,a2,a3) ev1(a1,ib1)
  std::vector<cd> t1P((size_t)nb1 * nb * nb), t1M((size_t)nb1 * nb * nb);
  for (int ib1 = 0; ib1 < nb1; ++ib1)
    for (int a2 = 0; a2 < nb; ++a2)
      for (int a3 = 0; a3 < nb; ++a3) {
        cd sp = 0.0, sm = 0.0;
        for (int a1 = 0; a1 < nb; ++a1) {
          cd e = EV(ev1, nb, a1, ib1);
          sp += tP[((size_t)a1 * nb + a2) * nb + a3] * e;
          sm += tM[((size_t)a1 * nb + a2) * nb + a3] * e;
        }
        t1P[((size_t)ib1 * nb + a3) * nb + a2] = sp;
        t1M[((size_t)ib1 * nb + a3) * nb + a2] = sm;
      }
  // tmp2(ib1, ib2, a3) = sum_a2 tmp1(ib1,a3,a2) ev2(a2,ib2) [conj for minus]
  std::vector<cd> t2P((size_t)nb1 * nb2 * nb), t2M((size_t)nb1 * nb2 * nb);
  for (int ib1 = 0; ib1 < nb1; ++ib1)
    for (int ib2 = 0; ib2 < nb2; ++ib2)
      for (int a3 = 0; a3 < nb; ++a3) {
        cd sp = 0.0, sm = 0.0;
        for (int a2 = 0; a2 < nb; ++a2) {
          cd e = EV(ev2, nb, a2, ib2);
          sp += t1P[((size_t)ib1 * nb + a3) * nb + a2] * e;
          sm += t1M[((size_t)ib1 * nb + a3) * nb + a2] * std::conj(e);
        }
        t2P[((size_t)ib1 * nb2 + ib2) * nb + a3] = sp;
        t2M[((size_t)ib1 * nb2 + ib2) * nb + a3] = sm;
      }
  for (int ib1 = 0; ib1 < nb1; ++ib1)
    for (int ib2 = 0; ib2 < nb2; ++ib2) {
      for (int ib3 = 0; ib3 < nb3p; ++ib3) {
        cd s = 0.0;
        for (int a3 = 0; a3 < nb; ++a3)
          s += t2P[((size_t)ib1 * nb2 + ib2) * nb + a3] * std::conj(EV(ev3p, nb, a3, ib3));
        outP[((size_t)ib1 * nb2 + ib2) * nb3p + ib3] = s.real() * s.real() + s.imag() * s.imag();
      }
      for (int ib3 = 0; ib3 < nb3m; ++ib3) {
        cd s = 0.0;
        for (int a3 = 0; a3 < nb; ++a3)
          s += t2M[((size_t)ib1 * nb2 + ib2) * nb + a3] * std::conj(EV(ev3m, nb, a3, ib3));
        outM[((size_t)ib1 * nb2 + ib2) * nb3m + ib3] = s.real() * s.real() + s.imag() * s.imag();
      }
    }
}

void symmetrize(double* c, int nb1, int nb2, int nb3, const double* e1, const double* e2,
                const double* e3) {
  // scattering.cpp:1209-1318: forward-scan degenerate blocks along each index
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
        for (int k = 0; k < nb3; ++k) tmp[j * nb3 + k] += C(ib1 + i, j, k) / float(deg);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb2; ++j)
        for (int k = 0; k < nb3; ++k) C(ib1 + i, j, k) = tmp[j * nb3 + k];
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
        for (int k = 0; k < nb3; ++k) tmp[j * nb3 + k] += C(j, ib2 + i, k) / float(deg);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb1; ++j)
        for (int k = 0; k < nb3; ++k) C(j, ib2 + i, k) = tmp[j * nb3 + k];
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
        for (int k = 0; k < nb2; ++k) tmp[j * nb2 + k] += C(j, k, ib3 + i) / float(deg);
    for (int i = 0; i < deg; ++i)
      for (int j = 0; j < nb1; ++j)
        for (int k = 0; k < nb2; ++k) C(j, k, ib3 + i) = tmp[j * nb2 + k];
    ib3 += deg - 1;
  }
}

struct Smearing {
  int type;            // 0 gaussian, 1 adaptive
  double sigma;        // gaussian width
  double qT[3][3];     // adaptive: reciprocal cell with row i divided by mesh(i)
  double cutoff;       // adaptive: broadening floor (1e-4 eV)
  double gauss(double e) const {
    // delta_function.cpp:40-45 (one-sided cutoff)
    double x = e / sigma;
    if (x > 6.0) return 0.0;
    return 1.0 / sigma / std::sqrt(pi) * std::exp(-x * x);
  }
  double adaptive(double e, const double v[3]) const {
    // delta_function.cpp:65-96
    double vn = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (vn == 0.0 && e == 0.0) return 1.0;
    double s = 0.0;
    for (int i = 0; i < 3; ++i) {
      double d = qT[i][0] * v[0] + qT[i][1] * v[1] + qT[i][2] * v[2];
      s += d * d;
    }
    double sig = 1.0 * std::sqrt(s / 6.0);
    if (sig == 0.0) return 0.0;
    if (sig < cutoff) sig = cutoff;
    if (std::fabs(e) > 2.0 * sig) return 0.0;
    double x = e / sig;
    if (x > 6.0) return 0.0;
    return std::exp(-x * x) / sqrtPi / sig / 0.9953222650189527;
  }
};

// Where the builder's rates go (ph_scattering.cpp, the three switchCase branches of
// each process).  sign: +1 for the "+" process, -1 for the "-" processes and
// isotope scattering; dfac: the linewidth share (1/2 for 3-phonon rates, 1 for
// isotope rates).
struct Sink {
  int mode = 2;            // 2 linewidths, 0 matrix, 1 matrix-vector product
  size_t ns = 0;
  int nT = 0;
  double* lw = nullptr;    // (nT, ns): modes 2 and 0
  double* mat = nullptr;   // (ns, ns) row-major: mode 0
  int nvec = 0;            // mode 1: x, y (nvec, nT, 3, ns)
  const double* x = nullptr;
  double* y = nullptr;
  void add(int c, size_t s1, size_t s2, double rate, double sign, double dfac) const {
    if (mode == 2) {
      lw[c * ns + s1] += dfac * rate;
    } else if (mode == 0) {
      lw[c * ns + s1] += dfac * rate;
      mat[s1 * ns + s2] += sign * rate;
    } else {
      for (int v = 0; v < nvec; ++v)
        for (int i = 0; i < 3; ++i) {
          const size_t o = (((size_t)v * nT + c) * 3 + i) * ns;
          if (s1 != s2) y[o + s1] += sign * rate * x[o + s2];
          y[o + s1] += dfac * rate * x[o + s1];
        }
    }
  }
};

int builder(void* p, int nq, const int* mesh, const double* E, const double* ev, const double* vg,
            const double* qcart, const double* recip, int nT, const double* Tk_ry, int smearing, double sigma,
            int nq2, const int* q2_list, int finalize, const Sink& sink, const double* win_energy,
            const double* win_cut, const double* iso, double boundary_length);

}  // namespace

extern "C" {

struct orc_v3;

void* orc_v3_create(int nat, int nr2, int nr3, const double* D3, const double* R2,
                    const double* R3, const double* w2, const double* w3) {
  V3* v = new V3;
  v->nat = nat;
  v->nb = 3 * nat;
  v->nr2 = nr2;
  v->nr3 = nr3;
  size_t n = (size_t)v->nb * v->nb * v->nb * nr3 * nr2;
  v->D3.assign(D3, D3 + n);
  v->R2.assign(R2, R2 + 3 * nr2);
  v->R3.assign(R3, R3 + 3 * nr3);
  v->w2.assign(w2, w2 + (size_t)nr2 * nat * nat);
  v->w3.assign(w3, w3 + (size_t)nr3 * nat * nat);
  return v;
}

void orc_v3_destroy(void* p) { delete (V3*)p; }

void orc_v3_cache_d3(void* p, const double* q2) { cache_d3(*(V3*)p, q2); }

// Batched getCouplingsSquared for full bands (nb1 = nb2 = nb3 = nb).
// ev1s, ev3ps, ev3ms: (nq1,nb,nb) complex; ev2: (nb,nb) complex.
// outP/outM: (nq1,nb,nb,nb).
void orc_v3_couplings(void* p, int nq1, const double* q1s, const double* ev1s, const double* ev2,
                      const double* ev3ps, const double* ev3ms, double* outP, double* outM) {
  V3& v = *(V3*)p;
  const int nb = v.nb;
  const size_t m = (size_t)nb * nb * 2, o = (size_t)nb * nb * nb;
#pragma omp parallel for schedule(dynamic, 8)
  for (int i = 0; i < nq1; ++i)
    couplings_one(v, q1s + 3 * i, ev1s + i * m, nb, ev2, nb, ev3ps + i * m, nb, ev3ms + i * m, nb,
                  outP + i * o, outM + i * o);
}

void orc_symmetrize_coupling(double* c, int nb1, int nb2, int nb3, const double* e1,
                             const double* e2, const double* e3) {
  symmetrize(c, nb1, nb2, nb3, e1, e2, e3);
}

// PhScatteringMatrix::builder in linewidth mode on a full Gamma-centred mesh.
//   E (nq,nb), ev (nq,nb,nb,2) mass-scaled, vg (nq,nb,3), qcart (nq,3)
//   recip: reciprocal cell 3x3 C-order (columns = b vectors)
//   smearing: 0 gaussian (sigma), 1 adaptive
//   q2_list: which q2 to process (NULL -> all), nq2 its length
//   out: A_out (nT, nq*nb), accumulated (not zeroed here when accumulate=1)
//   finalize: 1 -> degeneracy averaging of row 0 and zeroing excluded states
//   win_energy / win_cut (nq) or NULL: the pair (q1, q2) is skipped unless
//     win_energy[q2] <= win_cut[q1] (per-q1 window of the batched-instance
//     workload; no counterpart in the reference)
//   iso (nat) or NULL: isotope scattering with massVariance iso (ph_scattering.cpp:616-793)
//   boundary_length > 0: boundary scattering after the averaging (ph_scattering.cpp:819-860)
int orc_ph_linewidths(void* p, int nq, const int* mesh, const double* E, const double* ev,
                      const double* vg, const double* qcart, const double* recip, int nT,
                      const double* Tk_ry, int smearing, double sigma, int nq2,
                      const int* q2_list, int finalize, double* out, const double* win_energy,
                      const double* win_cut, const double* iso, double boundary_length) {
  Sink sk;
  sk.mode = 2;
  sk.ns = (size_t)nq * ((V3*)p)->nb;
  sk.nT = nT;
  sk.lw = out;
  return builder(p, nq, mesh, E, ev, vg, qcart, recip, nT, Tk_ry, smearing, sigma, nq2, q2_list, finalize, sk,
                 win_energy, win_cut, iso, boundary_length);
}

// switchCase 0: the scattering matrix (ns, ns) row-major and its diagonal
// linewidth row lw (ns), for one temperature (scattering.cpp:105-111).
// Accumulates into mat and lw (zero them first).
int orc_ph_smatrix(void* p, int nq, const int* mesh, const double* E, const double* ev, const double* vg,
                   const double* qcart, const double* recip, const double* Tk_ry, int smearing, double sigma,
                   int nq2, const int* q2_list, int finalize, double* lw, double* mat, const double* iso,
                   double boundary_length) {
  Sink sk;
  sk.mode = 0;
  sk.ns = (size_t)nq * ((V3*)p)->nb;
  sk.nT = 1;
  sk.lw = lw;
  sk.mat = mat;
  return builder(p, nq, mesh, E, ev, vg, qcart, recip, 1, Tk_ry, smearing, sigma, nq2, q2_list, finalize, sk,
                 nullptr, nullptr, iso, boundary_length);
}

// switchCase 1: y += A x for nvec input vectors x (nvec, nT, 3, ns), one matrix
// per temperature, without storing A.  Accumulates into y (zero it first).
int orc_ph_smatrix_dot(void* p, int nq, const int* mesh, const double* E, const double* ev, const double* vg,
                       const double* qcart, const double* recip, int nT, const double* Tk_ry, int smearing,
                       double sigma, int nq2, const int* q2_list, int finalize, int nvec, const double* x,
                       double* y, const double* iso, double boundary_length) {
  Sink sk;
  sk.mode = 1;
  sk.ns = (size_t)nq * ((V3*)p)->nb;
  sk.nT = nT;
  sk.nvec = nvec;
  sk.x = x;
  sk.y = y;
  return builder(p, nq, mesh, E, ev, vg, qcart, recip, nT, Tk_ry, smearing, sigma, nq2, q2_list, finalize, sk,
                 nullptr, nullptr, iso, boundary_length);
}

// ScatteringMatrix::dot (off_diagonal = 0; excluded rows and columns skipped,
// scattering.cpp:266-330) and offDiagonalDot (off_diagonal = 1; the diagonal
// skipped, :180-232) of a stored matrix: y (nvec, 3, ns) = A x.
void orc_smatrix_dot(int ns, const double* mat, const double* E, int nvec, const double* x, int off_diagonal,
                     double* y) {
  std::vector<char> excluded(ns, 0);
  for (int s = 0; s < ns; ++s) excluded[s] = E[s] < 0.1 / ryToCmm1;
#pragma omp parallel for
  for (int r = 0; r < ns; ++r)
    for (int v = 0; v < nvec; ++v)
      for (int i = 0; i < 3; ++i) {
        const double* xv = x + ((size_t)v * 3 + i) * ns;
        double acc = 0.0;
        for (int c = 0; c < ns; ++c) {
          if (off_diagonal ? r == c : (excluded[r] || excluded[c])) continue;
          acc += mat[(size_t)r * ns + c] * xv[c];
        }
        y[((size_t)v * 3 + i) * ns + r] = acc;
      }
}

}  // extern "C"

namespace {

int builder(void* p, int nq, const int* mesh, const double* E, const double* ev, const double* vg,
            const double* qcart, const double* recip, int nT, const double* Tk_ry, int smearing, double sigma,
            int nq2, const int* q2_list, int finalize, const Sink& sink, const double* win_energy,
            const double* win_cut, const double* iso, double boundary_length) {
  V3& v = *(V3*)p;
  const int nb = v.nb;
  const size_t ns = (size_t)nq * nb;
  const double energyCutoff = 0.001 / ryToCmm1;
  const double norm = 1.0 / (double)((long)mesh[0] * mesh[1] * mesh[2]);
  Smearing sm;
  sm.type = smearing;
  sm.sigma = sigma;
  sm.cutoff = 0.0001 / energyRyToEv;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) sm.qT[i][j] = recip[i * 3 + j] / mesh[i];
  // excludeIndices, scattering.cpp:30-41
  std::vector<char> excluded(ns, 0);
  for (size_t s = 0; s < ns; ++s)
    if (E[s] < 0.1 / ryToCmm1) excluded[s] = 1;
  // Bose tables, ph_scattering.cpp:98-143
  std::vector<double> boseT((size_t)nT * ns);
  for (int c = 0; c < nT; ++c)
    for (size_t s = 0; s < ns; ++s) boseT[c * ns + s] = bose(E[s], Tk_ry[c]);
  // inverse reciprocal cell for Cartesian -> crystal
  double Bi[3][3];
  {
    const double* b = recip;
    double det = b[0] * (b[4] * b[8] - b[5] * b[7]) - b[1] * (b[3] * b[8] - b[5] * b[6]) +
                 b[2] * (b[3] * b[7] - b[4] * b[6]);
    Bi[0][0] = (b[4] * b[8] - b[5] * b[7]) / det;
    Bi[0][1] = (b[2] * b[7] - b[1] * b[8]) / det;
    Bi[0][2] = (b[1] * b[5] - b[2] * b[4]) / det;
    Bi[1][0] = (b[5] * b[6] - b[3] * b[8]) / det;
    Bi[1][1] = (b[0] * b[8] - b[2] * b[6]) / det;
    Bi[1][2] = (b[2] * b[3] - b[0] * b[5]) / det;
    Bi[2][0] = (b[3] * b[7] - b[4] * b[6]) / det;
    Bi[2][1] = (b[1] * b[6] - b[0] * b[7]) / det;
    Bi[2][2] = (b[0] * b[4] - b[1] * b[3]) / det;
  }
  auto lookup = [&](const double* qc) -> int {
    // points.cpp:404-423 via cartesianToCrystal (points.cpp:461-464)
    double diff = 0.0;
    int pidx[3];
    for (int i = 0; i < 3; ++i) {
      double c = Bi[i][0] * qc[0] + Bi[i][1] * qc[1] + Bi[i][2] * qc[2];
      double x = c * mesh[i];
      double r = std::round(x);
      diff += r - x;
      int ri = (int)r;
      pidx[i] = ((ri % mesh[i]) + mesh[i]) % mesh[i];
    }
    if (diff >= 1.0e-6) return -1;
    return pidx[2] * mesh[0] * mesh[1] + pidx[1] * mesh[0] + pidx[0];
  };
  const size_t m = (size_t)nb * nb * 2, o = (size_t)nb * nb * nb;
  std::vector<int> iq3p(nq), iq3m(nq);
  std::vector<double> cP((size_t)nq * o), cM((size_t)nq * o);
  std::vector<double> ev3p((size_t)nq * m), ev3m((size_t)nq * m);
  for (int ii = 0; ii < nq2; ++ii) {
    const int iq2 = q2_list ? q2_list[ii] : ii;
    const double* q2 = qcart + 3 * iq2;
    int bad = 0;
#pragma omp parallel for reduction(| : bad)
    for (int iq1 = 0; iq1 < nq; ++iq1) {
      double qp[3], qm[3];
      for (int i = 0; i < 3; ++i) {
        qp[i] = qcart[3 * iq1 + i] + q2[i];
        qm[i] = qcart[3 * iq1 + i] - q2[i];
      }
      iq3p[iq1] = lookup(qp);
      iq3m[iq1] = lookup(qm);
      if (iq3p[iq1] < 0 || iq3m[iq1] < 0) {
        bad = 1;
        continue;
      }
      std::memcpy(&ev3p[iq1 * m], ev + (size_t)iq3p[iq1] * m, m * sizeof(double));
      std::memcpy(&ev3m[iq1 * m], ev + (size_t)iq3m[iq1] * m, m * sizeof(double));
    }
    if (bad) return 3;
    cache_d3(v, q2);
    orc_v3_couplings(p, nq, qcart, ev, ev + (size_t)iq2 * m, ev3p.data(), ev3m.data(), cP.data(),
                     cM.data());
#pragma omp parallel for
    for (int iq1 = 0; iq1 < nq; ++iq1) {
      symmetrize(&cP[iq1 * o], nb, nb, nb, E + (size_t)iq1 * nb, E + (size_t)iq2 * nb,
                 E + (size_t)iq3p[iq1] * nb);
      symmetrize(&cM[iq1 * o], nb, nb, nb, E + (size_t)iq1 * nb, E + (size_t)iq2 * nb,
                 E + (size_t)iq3m[iq1] * nb);
    }
    // HOT LOOP 3 (serial in the reference), ph_scattering.cpp:284-613
    for (int iq1 = 0; iq1 < nq; ++iq1) {
      if (win_energy && !(win_energy[iq2] <= win_cut[iq1])) continue;
      const double* c_p = &cP[iq1 * o];
      const double* c_m = &cM[iq1 * o];
      const int q3p = iq3p[iq1], q3m = iq3m[iq1];
      for (int ib1 = 0; ib1 < nb; ++ib1) {
        const size_t s1 = (size_t)iq1 * nb + ib1;
        const double en1 = E[s1];
        if (excluded[s1]) continue;
        for (int ib2 = 0; ib2 < nb; ++ib2) {
          const size_t s2 = (size_t)iq2 * nb + ib2;
          const double en2 = E[s2];
          if (excluded[s2]) continue;
          for (int ib3 = 0; ib3 < nb; ++ib3) {
            const size_t s3 = (size_t)q3p * nb + ib3;
            const double en3 = E[s3];
            const double enProd = en1 * en2 * en3;
            if (en1 < energyCutoff || en2 < energyCutoff || en3 < energyCutoff) continue;
            double delta;
            if (smearing == 0) {
              delta = sm.gauss(en1 + en2 - en3);
            } else {
              double vv[3];
              for (int i = 0; i < 3; ++i) vv[i] = vg[s2 * 3 + i] - vg[s3 * 3 + i];
              delta = sm.adaptive(en1 + en2 - en3, vv);
            }
            if (delta <= 0.0) continue;
            for (int c = 0; c < nT; ++c) {
              double b1 = boseT[c * ns + s1], b2 = boseT[c * ns + s2], b3 = boseT[c * ns + s3];
              double rate = pi * 0.25 * b1 * b2 * (b3 + 1.0) *
                            c_p[((size_t)ib1 * nb + ib2) * nb + ib3] * delta * norm / enProd;
              sink.add(c, s1, s2, rate, 1.0, 0.5);
            }
          }
          for (int ib3 = 0; ib3 < nb; ++ib3) {
            const size_t s3 = (size_t)q3m * nb + ib3;
            const double en3 = E[s3];
            const double enProd = en1 * en2 * en3;
            if (en1 < energyCutoff || en2 < energyCutoff || en3 < energyCutoff) continue;
            double d1, d2;
            if (smearing == 0) {
              d1 = sm.gauss(en1 + en3 - en2);
              d2 = sm.gauss(en2 + en3 - en1);
            } else {
              double vv[3];
              for (int i = 0; i < 3; ++i) vv[i] = vg[s2 * 3 + i] - vg[s3 * 3 + i];
              d1 = sm.adaptive(en1 + en3 - en2, vv);
              d2 = sm.adaptive(en2 + en3 - en1, vv);
            }
            if (d1 <= 0.0 && d2 <= 0.0) continue;
            if (d1 < 0.0) d1 = 0.0;
            if (d2 < 0.0) d2 = 0.0;
            for (int c = 0; c < nT; ++c) {
              double b1 = boseT[c * ns + s1], b2 = boseT[c * ns + s2], b3 = boseT[c * ns + s3];
              double cm = c_m[((size_t)ib1 * nb + ib2) * nb + ib3];
              double r1 = pi * 0.25 * b3 * b1 * (b2 + 1.0) * cm * d1 * norm / enProd;
              double r2 = pi * 0.25 * b2 * b3 * (b1 + 1.0) * cm * d2 * norm / enProd;
              sink.add(c, s1, s2, r1 + r2, -1.0, 0.5);
            }
          }
        }
      }
    }
    // isotope scattering of the (q1, q2) pairs (ph_scattering.cpp:616-793)
    if (iso) {
      const int nat = nb / 3;
      for (int iq1 = 0; iq1 < nq; ++iq1) {
        for (int ib1 = 0; ib1 < nb; ++ib1) {
          const size_t s1 = (size_t)iq1 * nb + ib1;
          const double en1 = E[s1];
          if (excluded[s1] || en1 < energyCutoff) continue;
          for (int ib2 = 0; ib2 < nb; ++ib2) {
            const size_t s2 = (size_t)iq2 * nb + ib2;
            const double en2 = E[s2];
            if (excluded[s2] || en2 < energyCutoff) continue;
            double deltaIso;
            if (smearing == 0) {
              deltaIso = sm.gauss(en1 - en2);
            } else {
              // the reference evaluates the v2 width, overwrites it with the v1 one, halves it
              double v1[3];
              for (int i = 0; i < 3; ++i) v1[i] = vg[s1 * 3 + i];
              deltaIso = 0.5 * sm.adaptive(en1 - en2, v1);
            }
            double termIso = 0.0;
            for (int at = 0; at < nat; ++at) {
              double zr = 0.0, zi = 0.0;
              for (int k = 0; k < 3; ++k) {
                const int a = 3 * at + k;
                const double* u1 = ev + (((size_t)iq1 * nb + a) * nb + ib1) * 2;
                const double* u2 = ev + (((size_t)iq2 * nb + a) * nb + ib2) * 2;
                zr += u1[0] * u2[0] + u1[1] * u2[1];   // conj(u1) u2
                zi += u1[0] * u2[1] - u1[1] * u2[0];
              }
              termIso += (zr * zr + zi * zi) * iso[at];
            }
            termIso *= pi * 0.5 * norm * en1 * en2 * deltaIso;
            for (int c = 0; c < nT; ++c) {
              const double b1 = boseT[c * ns + s1], b2 = boseT[c * ns + s2];
              sink.add(c, s1, s2, termIso * (b1 * b2 + 0.5 * (b1 + b2)), -1.0, 1.0);
            }
          }
        }
      }
    }
  }
  if (finalize && sink.mode == 0) {
    // boundary scattering on the diagonal, exclusions, then the linewidths
    // placed on the diagonal (ph_scattering.cpp:846-847, :864-890, :910-933)
    double* lw = sink.lw;
    if (boundary_length > 0.0)
      for (size_t s = 0; s < ns; ++s) {
        if (excluded[s]) continue;
        const double* u = vg + s * 3;
        lw[s] += std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) / boundary_length * poppm1(E[s], Tk_ry[0]);
      }
    for (size_t s = 0; s < ns; ++s)
      if (excluded[s]) {
        lw[s] = 0.0;
        for (size_t t = 0; t < ns; ++t)
          if (excluded[t]) sink.mat[s * ns + t] = 0.0;
      }
    for (size_t s = 0; s < ns; ++s) sink.mat[s * ns + s] = lw[s];
  }
  if (finalize && sink.mode == 1) {
    // boundary scattering on the diagonal, then excluded rows zeroed (:849-855, :891-897)
    for (int vv = 0; vv < sink.nvec; ++vv)
      for (int c = 0; c < nT; ++c)
        for (int i = 0; i < 3; ++i) {
          const size_t o = (((size_t)vv * nT + c) * 3 + i) * ns;
          for (size_t s = 0; s < ns; ++s) {
            if (excluded[s]) {
              sink.y[o + s] = 0.0;
              continue;
            }
            if (boundary_length > 0.0) {
              const double* u = vg + s * 3;
              const double rate =
                  std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) / boundary_length * poppm1(E[s], Tk_ry[c]);
              sink.y[o + s] += rate * sink.x[o + s];
            }
          }
        }
  }
  if (finalize && sink.mode == 2) {
    double* out = sink.lw;
    // degeneracyAveragingLinewidths, scattering.cpp:1168-1207 (row iCalc=0 only)
    for (int iq = 0; iq < nq; ++iq) {
      std::vector<double> tmp(nb);
      for (int b1 = 0; b1 < nb; ++b1) {
        int n = 0;
        double t2 = 0.0;
        for (int b2 = 0; b2 < nb; ++b2)
          if (std::fabs(E[iq * nb + b2] - E[iq * nb + b1]) < 1.0e-6) {
            n++;
            t2 += out[(size_t)iq * nb + b2];
          }
        tmp[b1] = t2 / float(n);
      }
      for (int b1 = 0; b1 < nb; ++b1) out[(size_t)iq * nb + b1] = tmp[b1];
    }
    // boundary scattering, after the averaging (ph_scattering.cpp:819-860)
    if (boundary_length > 0.0) {
      for (int c = 0; c < nT; ++c)
        for (size_t s = 0; s < ns; ++s) {
          if (excluded[s]) continue;
          const double* v = vg + s * 3;
          const double x = std::sinh(E[s] / 2.0 / Tk_ry[c]);
          out[c * ns + s] += std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / boundary_length * (0.25 / x / x);
        }
    }
    for (int c = 0; c < nT; ++c)
      for (size_t s = 0; s < ns; ++s)
        if (excluded[s]) out[c * ns + s] = 0.0;
  }
  return 0;
}

}  // namespace

extern "C" {

// RTA thermal conductivity from A_out (nT, ns): tau = n(n+1)/A_out,
// popRTA = dn/dT v tau, kappa_ij = sum n_i v_j E / (Nq V) (atomic units;
// multiply by thConductivityAuToSi for W/m/K).  kappa: (nT,3,3).
void orc_rta_kappa(int ns, int nT, const double* Tk_ry, const double* E, const double* vg,
                   const double* Aout, long nqmesh, double volume, double* kappa) {
  for (int c = 0; c < nT; ++c) {
    double k[3][3] = {{0}};
    const double T = Tk_ry[c];
    for (int s = 0; s < ns; ++s) {
      const double en = E[s];
      if (en < 0.1 / ryToCmm1) continue;  // excluded states, phonon_thermal_cond.cpp:93-96
      double pp = poppm1(en, T);
      double tau = pp / Aout[(size_t)c * ns + s];
      double dndt = pp * en / T / T;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          k[i][j] += dndt * vg[s * 3 + i] * tau * vg[s * 3 + j] * en / (double)nqmesh / volume;
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) kappa[c * 9 + i * 3 + j] = k[i][j];
  }
}

}  // extern "C"
