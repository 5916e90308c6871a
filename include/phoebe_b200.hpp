// phoebe_b200.hpp -- C++ host layer over the C ABI (phx_abi.h) with the class
// and method names of mir-group/phoebe's scattering-rate call surface, without
// Eigen or Kokkos types.  Header only (C++17); link with -lphx.
//
//   reference class / method                                  here
//   PhononH0 ctor, diagonalizeFromCoordinates,               phx::PhononH0
//     kokkosBatchedDiagonalizeFromCoordinates / WithVelocities,
//     populate (src/harmonic/phonon_h0.h:76-149)
//   ElectronH0Wannier (src/harmonic/electron_h0_wannier.h:59-205)  phx::ElectronH0Wannier
//   Interaction3Ph ctor, cacheD3, getCouplingsSquared,       phx::Interaction3Ph
//     estimateNumBatches (src/interaction/interaction_3ph.h:92-152)
//   InteractionElPhWan cacheElPh, calcCouplingSquared,       phx::InteractionElPhWan
//     getCouplingSquared (src/interaction/interaction_elph.h:149-205)
//   PhScatteringMatrix / ElScatteringMatrix via setup()      phx::PhScatteringMatrix,
//     (src/bte/ph_scattering.h:37-41, el_scattering.h:31,     phx::ElScatteringMatrix
//      scattering.h:41), getLinewidths, getSingleModeTimes
//
// Matrices are row-major (rows = 3*atom + Cartesian component, or Wannier
// index; columns = bands), complex as std::complex<double>.  Errors throw
// phx::Error carrying the ABI status and message, where the reference calls
// Error(...) (src/exceptions.cpp:6-16).  Objects own their device handles and
// are movable, not copyable (the reference's copy constructors do not copy
// device data either, src/interaction/interaction_3ph.cpp:71-74).
#ifndef PHOEBE_B200_HPP
#define PHOEBE_B200_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "phx_abi.h"

namespace phx {

using cd = std::complex<double>;
using Vec3 = std::array<double, 3>;
using Mesh3 = std::array<int, 3>;

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int rc, const phx_ctx* ctx) {
  if (rc == PHX_OK) return;
  char buf[1024] = {0};
  phx_last_error(ctx, buf, sizeof(buf));
  throw Error(rc, std::string("phx: ") + buf);
}

// Row-major complex matrix (Eigen::MatrixXcd stand-in).
struct ComplexMatrix {
  int rows = 0, cols = 0;
  std::vector<cd> data;
  ComplexMatrix() = default;
  ComplexMatrix(int r, int c) : rows(r), cols(c), data((size_t)r * c) {}
  cd& operator()(int i, int j) { return data[(size_t)i * cols + j]; }
  const cd& operator()(int i, int j) const { return data[(size_t)i * cols + j]; }
};

// Row-major real rank-3 tensor (Eigen::Tensor<double,3> stand-in).
struct Tensor3 {
  std::array<int, 3> dims{0, 0, 0};
  std::vector<double> data;
  Tensor3() = default;
  Tensor3(int a, int b, int c) : dims{a, b, c}, data((size_t)a * b * c) {}
  double& operator()(int i, int j, int k) { return data[((size_t)i * dims[1] + j) * dims[2] + k]; }
  double operator()(int i, int j, int k) const { return data[((size_t)i * dims[1] + j) * dims[2] + k]; }
  int dimension(int i) const { return dims[i]; }
};

namespace detail {
template <class H, int (*Destroy)(H*)>
class Handle {
 public:
  Handle() = default;
  explicit Handle(H* h) : h_(h) {}
  Handle(const Handle&) = delete;
  Handle& operator=(const Handle&) = delete;
  Handle(Handle&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
  Handle& operator=(Handle&& o) noexcept {
    if (this != &o) {
      reset();
      h_ = o.h_;
      o.h_ = nullptr;
    }
    return *this;
  }
  ~Handle() { reset(); }
  void reset() {
    if (h_) Destroy(h_);
    h_ = nullptr;
  }
  H* get() const { return h_; }

 private:
  H* h_ = nullptr;
};

// interleaved (re, im) doubles <-> std::complex<double> (same layout)
inline const double* dptr(const std::vector<cd>& v) { return reinterpret_cast<const double*>(v.data()); }
inline double* dptr(std::vector<cd>& v) { return reinterpret_cast<double*>(v.data()); }
}  // namespace detail

// ---------------------------------------------------------------------------
class Context {
 public:
  explicit Context(int device = 0) {
    phx_ctx* c = nullptr;
    check(phx_ctx_create(device, &c), nullptr);
    h_ = detail::Handle<phx_ctx, phx_ctx_destroy>(c);
  }
  phx_ctx* get() const { return h_.get(); }
  void synchronize() const { check(phx_ctx_synchronize(get()), get()); }
  static std::string version() { return phx_version(); }

 private:
  detail::Handle<phx_ctx, phx_ctx_destroy> h_;
};

// Crystal: lattice vectors as the columns of cell (Bohr), positions (nat,3)
// Bohr, masses per atom in Ry mass units.
struct Crystal {
  std::array<double, 9> cell{};
  std::vector<double> positions;
  std::vector<double> masses;
  int numAtoms() const { return (int)masses.size(); }
  int numBands() const { return 3 * numAtoms(); }
  double volume() const {
    const auto& a = cell;
    return std::fabs(a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]));
  }
};

// ---------------------------------------------------------------------------
// Band structure on a Gamma-centred mesh, resident on the device.
class BandStructure {
 public:
  BandStructure(phx_bands* b, phx_ctx* ctx, Mesh3 mesh, int nb)
      : h_(b), ctx_(ctx), mesh_(mesh), nb_(nb) {}
  // FullBandStructure from host arrays: E (nq,nb), U (nq,nb,nb), vg (nq,nb,3) or empty
  static BandStructure fromHost(const Context& ctx, Mesh3 mesh, const std::array<double, 9>& reciprocalCell,
                                int nb, const std::vector<double>& E, const std::vector<cd>& U,
                                const std::vector<double>& vg = {}) {
    phx_bands* b = nullptr;
    check(phx_bands_create_from_host(ctx.get(), mesh.data(), reciprocalCell.data(), nb, E.data(), detail::dptr(U),
                                     vg.empty() ? nullptr : vg.data(), &b),
          ctx.get());
    return BandStructure(b, ctx.get(), mesh, nb);
  }
  int getNumPoints() const { return phx_bands_num_points(h_.get()); }
  int getNumBands() const { return nb_; }
  Mesh3 getMesh() const { return mesh_; }
  std::vector<double> getEnergies() const {
    std::vector<double> E((size_t)getNumPoints() * nb_);
    check(phx_bands_get(h_.get(), E.data(), nullptr, nullptr), ctx_);
    return E;
  }
  std::vector<cd> getEigenvectors() const {
    std::vector<cd> U((size_t)getNumPoints() * nb_ * nb_);
    check(phx_bands_get(h_.get(), nullptr, detail::dptr(U), nullptr), ctx_);
    return U;
  }
  std::vector<double> getGroupVelocities() const {
    std::vector<double> v((size_t)getNumPoints() * nb_ * 3);
    check(phx_bands_get(h_.get(), nullptr, nullptr, v.data()), ctx_);
    return v;
  }
  phx_bands* get() const { return h_.get(); }

 private:
  detail::Handle<phx_bands, phx_bands_destroy> h_;
  phx_ctx* ctx_;
  Mesh3 mesh_;
  int nb_;
};

// ---------------------------------------------------------------------------
class PhononH0 {
 public:
  // fc2: QE force constants (3,3,n1,n2,n3,nat,nat) Ry/Bohr^2; the "simple"
  // acoustic sum rule and the Wigner-Seitz reordering run in the constructor.
  PhononH0(const Context& ctx, const Crystal& crystal, const std::vector<double>& fc2, Mesh3 fcGrid)
      : ctx_(ctx.get()), nb_(crystal.numBands()) {
    phx_ph_h0* h = nullptr;
    check(phx_ph_h0_create(ctx_, crystal.numAtoms(), crystal.cell.data(), crystal.positions.data(),
                           crystal.masses.data(), fcGrid.data(), fc2.data(), &h),
          ctx_);
    h_ = detail::Handle<phx_ph_h0, phx_ph_h0_destroy>(h);
  }
  int getNumBands() const { return nb_; }

  // energies (nb) and eigenvectors U[a][b] at one Cartesian wavevector
  std::tuple<std::vector<double>, ComplexMatrix> diagonalizeFromCoordinates(const Vec3& q,
                                                                            bool withMassScaling = true) {
    auto r = kokkosBatchedDiagonalizeFromCoordinates({q}, withMassScaling);
    return {std::move(std::get<0>(r)), std::move(std::get<1>(r)[0])};
  }
  // batched: energies (nq*nb) and one eigenvector matrix per point
  std::tuple<std::vector<double>, std::vector<ComplexMatrix>> kokkosBatchedDiagonalizeFromCoordinates(
      const std::vector<Vec3>& q, bool withMassScaling = true) {
    const int nq = (int)q.size();
    std::vector<double> E((size_t)nq * nb_);
    std::vector<cd> U((size_t)nq * nb_ * nb_);
    check(phx_ph_diag(h_.get(), nq, q.empty() ? nullptr : q[0].data(), withMassScaling ? 1 : 0, E.data(),
                      detail::dptr(U)),
          ctx_);
    return {std::move(E), split(U, nq)};
  }
  // batched with group velocities (nq*nb*3); eigenvectors are mass-scaled
  std::tuple<std::vector<double>, std::vector<ComplexMatrix>, std::vector<double>>
  kokkosBatchedDiagonalizeWithVelocities(const std::vector<Vec3>& q) {
    const int nq = (int)q.size();
    std::vector<double> E((size_t)nq * nb_), v((size_t)nq * nb_ * 3);
    std::vector<cd> U((size_t)nq * nb_ * nb_);
    check(phx_ph_diag_velocities(h_.get(), nq, q.empty() ? nullptr : q[0].data(), E.data(), detail::dptr(U),
                                 v.data()),
          ctx_);
    return {std::move(E), split(U, nq), std::move(v)};
  }
  BandStructure populate(Mesh3 mesh, bool withVelocities = true) {
    phx_bands* b = nullptr;
    check(phx_bands_create_mesh(h_.get(), mesh.data(), withVelocities ? 1 : 0, &b), ctx_);
    return BandStructure(b, ctx_, mesh, nb_);
  }

 private:
  std::vector<ComplexMatrix> split(const std::vector<cd>& U, int nq) const {
    std::vector<ComplexMatrix> out(nq, ComplexMatrix(nb_, nb_));
    for (int i = 0; i < nq; ++i)
      std::copy(U.begin() + (size_t)i * nb_ * nb_, U.begin() + (size_t)(i + 1) * nb_ * nb_, out[i].data.begin());
    return out;
  }
  phx_ctx* ctx_;
  int nb_;
  detail::Handle<phx_ph_h0, phx_ph_h0_destroy> h_;
};

// ---------------------------------------------------------------------------
enum class Precision { fp64 = PHX_PREC_FP64, splitBf16 = PHX_PREC_SPLIT_BF16, splitFp16 = PHX_PREC_SPLIT_FP16 };
enum class Smearing { gaussian = PHX_SMEAR_GAUSSIAN, adaptive = PHX_SMEAR_ADAPTIVE };

class Interaction3Ph {
 public:
  // D3 (nb,nb,nb,nr3,nr2) Ry/Bohr^3, R2 (nr2,3), R3 (nr3,3) Bohr, w2 (nr2,nat,nat), w3 (nr3,nat,nat)
  Interaction3Ph(const Context& ctx, int nat, int nr2, int nr3, const std::vector<double>& D3,
                 const std::vector<double>& R2, const std::vector<double>& R3, const std::vector<double>& w2,
                 const std::vector<double>& w3)
      : ctx_(ctx.get()), nb_(3 * nat) {
    phx_v3* h = nullptr;
    check(phx_v3_create(ctx_, nat, nr2, nr3, D3.data(), R2.data(), R3.data(), w2.data(), w3.data(), &h), ctx_);
    h_ = detail::Handle<phx_v3, phx_v3_destroy>(h);
  }
  void setPrecision(Precision p) { check(phx_v3_set_precision(h_.get(), (int)p), ctx_); }
  void cacheD3(const Vec3& q2) { check(phx_v3_cache_d3(h_.get(), q2.data()), ctx_); }

  // |V+|^2 and |V-|^2 per q1, each (nb1s[i], nb2, nb3+-[i]); eigenvector
  // matrices are (nb, nbX) with the used columns first.
  std::tuple<std::vector<Tensor3>, std::vector<Tensor3>> getCouplingsSquared(
      const std::vector<Vec3>& q1s, const Vec3& q2, const std::vector<ComplexMatrix>& ev1s,
      const ComplexMatrix& ev2, const std::vector<ComplexMatrix>& ev3Pluss, const std::vector<ComplexMatrix>& ev3Minss,
      const std::vector<int>& nb1s, int nb2, const std::vector<int>& nb3Pluss, const std::vector<int>& nb3Minss) {
    (void)q2;  // q2 enters through cacheD3, as in the reference
    const int nq1 = (int)q1s.size();
    auto pad = [&](const std::vector<ComplexMatrix>& evs) {
      std::vector<cd> out((size_t)nq1 * nb_ * nb_);
      for (int i = 0; i < nq1; ++i)
        for (int a = 0; a < evs[i].rows; ++a)
          for (int b = 0; b < evs[i].cols; ++b) out[((size_t)i * nb_ + a) * nb_ + b] = evs[i](a, b);
      return out;
    };
    const auto e1 = pad(ev1s), e3p = pad(ev3Pluss), e3m = pad(ev3Minss);
    std::vector<cd> e2((size_t)nb_ * nb_);
    for (int a = 0; a < ev2.rows; ++a)
      for (int b = 0; b < ev2.cols; ++b) e2[(size_t)a * nb_ + b] = ev2(a, b);
    size_t sp = 0, sm = 0;
    for (int i = 0; i < nq1; ++i) {
      sp += (size_t)nb1s[i] * nb2 * nb3Pluss[i];
      sm += (size_t)nb1s[i] * nb2 * nb3Minss[i];
    }
    std::vector<double> outP(std::max<size_t>(sp, 1)), outM(std::max<size_t>(sm, 1));
    check(phx_v3_couplings_sq(h_.get(), nq1, q1s.empty() ? nullptr : q1s[0].data(), detail::dptr(e1), nb1s.data(),
                              detail::dptr(e2), nb2, detail::dptr(e3p), nb3Pluss.data(), detail::dptr(e3m),
                              nb3Minss.data(), outP.data(), outM.data()),
          ctx_);
    std::vector<Tensor3> cp, cm;
    size_t oP = 0, oM = 0;
    for (int i = 0; i < nq1; ++i) {
      Tensor3 p(nb1s[i], nb2, nb3Pluss[i]), m(nb1s[i], nb2, nb3Minss[i]);
      std::copy(outP.begin() + oP, outP.begin() + oP + p.data.size(), p.data.begin());
      std::copy(outM.begin() + oM, outM.begin() + oM + m.data.size(), m.data.begin());
      oP += p.data.size();
      oM += m.data.size();
      cp.push_back(std::move(p));
      cm.push_back(std::move(m));
    }
    return {std::move(cp), std::move(cm)};
  }
  int estimateNumBatches(int nq1, int nb2) {
    int n = 0;
    check(phx_v3_estimate_num_batches(h_.get(), nq1, nb2, &n), ctx_);
    return n;
  }
  phx_v3* get() const { return h_.get(); }
  const phx_ctx* context() const { return ctx_; }

 private:
  phx_ctx* ctx_;
  int nb_;
  detail::Handle<phx_v3, phx_v3_destroy> h_;
};

// ---------------------------------------------------------------------------
// PhScatteringMatrix, linewidth mode: setup() runs the whole builder on the GPU.
class PhScatteringMatrix {
 public:
  PhScatteringMatrix(Interaction3Ph& coupling3Ph, BandStructure& bands, std::vector<double> temperatures,
                     Smearing smearing = Smearing::adaptive, double sigma = 0.0)
      : v3_(coupling3Ph), bands_(bands), T_(std::move(temperatures)), smearing_(smearing), sigma_(sigma) {}

  // isotope scattering: per-atom isotope mass variance x mass^2 (the
  // reference's massVariance); empty disables it
  void setIsotopeCoupling(std::vector<double> massVariance) { iso_ = std::move(massVariance); }
  // boundary scattering |v|/L n(n+1); L <= 0 disables it (Bohr)
  void setBoundaryLength(double L) { boundary_ = L; }
  // the reference's scatteringMatrixInMemory: setup() builds the whole matrix
  // (one temperature) into device memory, dot() multiplies with it
  void setMatrixInMemory(bool inMemory) { inMemory_ = inMemory; }

  // internalDiagonal A_out (nT, nq*nb) = linewidth * n(n+1); [q2Begin, q2End)
  // restricts the outer loop (one rank's share), finalize = false leaves the
  // degeneracy averaging and exclusions to the caller after summing shares.
  // In memory: the matrix too, whose diagonal (not degeneracy-averaged) is
  // then the internalDiagonal.
  void setup(int q2Begin = 0, int q2End = -1, bool finalize = true) {
    const phx_lw_params p = params(q2Begin, q2End, finalize);
    internalDiagonal_.assign(T_.size() * numStates(), 0.0);
    if (inMemory_) {
      phx_smatrix* m = nullptr;
      check(phx_ph_smatrix_create(v3_.get(), bands_.get(), &p, &m, &stats_), v3_.context());
      matrix_ = detail::Handle<phx_smatrix, phx_smatrix_destroy>(m);
      check(phx_smatrix_diagonal(matrix_.get(), internalDiagonal_.data()), v3_.context());
      return;
    }
    check(phx_ph_linewidths(v3_.get(), bands_.get(), &p, internalDiagonal_.data(), &stats_), v3_.context());
  }

  // ScatteringMatrix::dot: A x for nvec vectors x (nvec, nT, 3, numStates);
  // in memory a product with the stored matrix, otherwise one builder pass
  std::vector<double> dot(const std::vector<double>& x, int nvec = 1) {
    std::vector<double> y(x.size(), 0.0);
    if (x.size() != (size_t)nvec * T_.size() * 3 * numStates()) throw Error(PHX_ERR_ARG, "dot: bad vector size");
    if (inMemory_) {
      if (!matrix_.get()) throw Error(PHX_ERR_STATE, "dot: setup() first");
      check(phx_smatrix_dot(matrix_.get(), nvec, x.data(), 0, y.data()), v3_.context());
    } else {
      const phx_lw_params p = params(0, -1, true);
      check(phx_ph_smatrix_dot(v3_.get(), bands_.get(), &p, nvec, x.data(), y.data(), &stats_), v3_.context());
    }
    return y;
  }
  // ScatteringMatrix::offDiagonalDot; without a stored matrix, as the
  // reference, dot(x) - internalDiagonal * x
  std::vector<double> offDiagonalDot(const std::vector<double>& x, int nvec = 1) {
    if (inMemory_) {
      if (!matrix_.get()) throw Error(PHX_ERR_STATE, "offDiagonalDot: setup() first");
      std::vector<double> y(x.size(), 0.0);
      if (x.size() != (size_t)nvec * 3 * numStates()) throw Error(PHX_ERR_ARG, "offDiagonalDot: bad vector size");
      check(phx_smatrix_dot(matrix_.get(), nvec, x.data(), 1, y.data()), v3_.context());
      return y;
    }
    std::vector<double> y = dot(x, nvec);
    const size_t ns = numStates();
    for (size_t v = 0; v < (size_t)nvec; ++v)
      for (size_t t = 0; t < T_.size(); ++t)
        for (size_t i = 0; i < 3; ++i)
          for (size_t s = 0; s < ns; ++s) {
            const size_t o = ((v * T_.size() + t) * 3 + i) * ns + s;
            y[o] -= internalDiagonal_[t * ns + s] * x[o];
          }
    return y;
  }
  // rows row0 .. row0+nrows-1 of the stored matrix, row-major (nrows, numStates)
  std::vector<double> getRows(int row0, int nrows) const {
    if (!matrix_.get()) throw Error(PHX_ERR_STATE, "getRows: no stored matrix");
    std::vector<double> out((size_t)nrows * numStates());
    check(phx_smatrix_get_rows(matrix_.get(), row0, nrows, out.data()), v3_.context());
    return out;
  }
  // A -> (A + A^T) / 2 (ScatteringMatrix::symmetrize)
  void symmetrize() {
    if (!matrix_.get()) throw Error(PHX_ERR_STATE, "symmetrize: no stored matrix");
    check(phx_smatrix_symmetrize(matrix_.get()), v3_.context());
  }
  // ScatteringMatrix::a2Omega (src/bte/scattering.cpp:366-434); internalDiagonal / n(n+1)
  void a2Omega() {
    if (!matrix_.get()) throw Error(PHX_ERR_STATE, "a2Omega: no stored matrix");
    check(phx_smatrix_a2omega(matrix_.get()), v3_.context());
    check(phx_smatrix_diagonal(matrix_.get(), internalDiagonal_.data()), v3_.context());
  }
  // ScatteringMatrix::diagonalize (scattering.cpp:872-910): eigenvalues of the
  // upper triangle, ascending; all (numEigenvalues <= 0) or the smallest
  // numEigenvalues.  The eigenvectors replace the matrix (getRows).
  std::vector<double> diagonalize(int numEigenvalues = 0) {
    if (!matrix_.get()) throw Error(PHX_ERR_STATE, "diagonalize: no stored matrix");
    std::vector<double> ev(numStates());
    int found = 0;
    check(phx_smatrix_diagonalize(matrix_.get(), numEigenvalues, ev.data(), &found), v3_.context());
    ev.resize((size_t)found);
    return ev;
  }
  // Theta diag(1/lambda, lambda > 0) Theta^T x, x (nvec, 3, numStates)
  // (calcFromRelaxons, src/observable/phonon_thermal_cond.cpp:316-380)
  std::vector<double> relaxonSolve(const std::vector<double>& x, int nvec = 1) {
    if (!matrix_.get()) throw Error(PHX_ERR_STATE, "relaxonSolve: no stored matrix");
    if (x.size() != (size_t)nvec * 3 * numStates()) throw Error(PHX_ERR_ARG, "relaxonSolve: bad vector size");
    std::vector<double> y(x.size(), 0.0);
    check(phx_smatrix_relaxon_solve(matrix_.get(), nvec, x.data(), y.data()), v3_.context());
    return y;
  }
  size_t numStates() const { return (size_t)bands_.getNumPoints() * bands_.getNumBands(); }
  const std::vector<double>& internalDiagonal() const { return internalDiagonal_; }
  const phx_lw_stats& stats() const { return stats_; }

  // Gamma = A_out / (n(n+1)) (src/bte/scattering.cpp:529-568)
  std::vector<double> getLinewidths() const { return divide(false); }
  // tau = n(n+1) / A_out (src/bte/scattering.cpp:484-513)
  std::vector<double> getSingleModeTimes() const { return divide(true); }
  // RTA thermal conductivity per temperature (3x3 row-major), atomic units
  std::vector<std::array<double, 9>> thermalConductivity(double volume) const {
    std::vector<std::array<double, 9>> k(T_.size());
    check(phx_ph_rta_kappa(bands_.get(), (int)T_.size(), T_.data(), internalDiagonal_.data(), volume, k[0].data()),
          v3_.context());
    return k;
  }

 private:
  phx_lw_params params(int q2Begin, int q2End, bool finalize) const {
    phx_lw_params p{};
    p.num_temperatures = (int)T_.size();
    p.temperatures = T_.data();
    p.smearing = (int)smearing_;
    p.sigma = sigma_;
    p.finalize = finalize ? 1 : 0;
    p.q2_begin = q2Begin;
    p.q2_end = q2End < 0 ? bands_.getNumPoints() : q2End;
    p.isotope_coupling = iso_.empty() ? nullptr : iso_.data();
    p.boundary_length = boundary_;
    return p;
  }
  std::vector<double> divide(bool invert) const {
    const auto E = bands_.getEnergies();
    const size_t ns = E.size();
    std::vector<double> out(internalDiagonal_.size(), 0.0);
    for (size_t t = 0; t < T_.size(); ++t)
      for (size_t s = 0; s < ns; ++s) {
        const double x = std::sinh(E[s] / 2.0 / T_[t]);
        const double popPop = 0.25 / x / x;
        const double a = internalDiagonal_[t * ns + s];
        out[t * ns + s] = invert ? popPop / a : a / popPop;
      }
    return out;
  }
  Interaction3Ph& v3_;
  BandStructure& bands_;
  std::vector<double> T_;
  Smearing smearing_;
  double sigma_;
  std::vector<double> internalDiagonal_;
  std::vector<double> iso_;
  double boundary_ = 0.0;
  bool inMemory_ = false;
  detail::Handle<phx_smatrix, phx_smatrix_destroy> matrix_;
  phx_lw_stats stats_{};
};

// ---------------------------------------------------------------------------
class ElectronH0Wannier {
 public:
  // H(R) (nR,nw,nw) complex Ry on Bravais vectors R (nR,3) Bohr with degeneracies deg (nR)
  ElectronH0Wannier(const Context& ctx, const std::array<double, 9>& cell, int nw, const std::vector<double>& R,
                    const std::vector<double>& deg, const std::vector<cd>& H)
      : ctx_(ctx.get()), nw_(nw) {
    phx_el_h0* h = nullptr;
    check(phx_el_h0_create(ctx_, nw, (int)deg.size(), cell.data(), R.data(), deg.data(), detail::dptr(H), &h), ctx_);
    h_ = detail::Handle<phx_el_h0, phx_el_h0_destroy>(h);
  }
  int getNumBands() const { return nw_; }
  std::tuple<std::vector<double>, std::vector<ComplexMatrix>> batchedDiagonalizeFromCoordinates(
      const std::vector<Vec3>& k) {
    std::vector<double> v;
    return diag(k, false, v);
  }
  std::tuple<std::vector<double>, std::vector<ComplexMatrix>, std::vector<double>> batchedDiagonalizeWithVelocities(
      const std::vector<Vec3>& k) {
    std::vector<double> v;
    auto r = diag(k, true, v);
    return {std::move(std::get<0>(r)), std::move(std::get<1>(r)), std::move(v)};
  }
  std::tuple<std::vector<double>, ComplexMatrix> diagonalizeFromCoordinates(const Vec3& k) {
    auto r = batchedDiagonalizeFromCoordinates({k});
    return {std::move(std::get<0>(r)), std::move(std::get<1>(r)[0])};
  }
  BandStructure populate(Mesh3 mesh, bool withVelocities = true) {
    phx_bands* b = nullptr;
    check(phx_el_bands_create_mesh(h_.get(), mesh.data(), withVelocities ? 1 : 0, &b), ctx_);
    return BandStructure(b, ctx_, mesh, nw_);
  }

 private:
  std::tuple<std::vector<double>, std::vector<ComplexMatrix>> diag(const std::vector<Vec3>& k, bool vel,
                                                                   std::vector<double>& v) {
    const int nk = (int)k.size();
    std::vector<double> E((size_t)nk * nw_);
    std::vector<cd> U((size_t)nk * nw_ * nw_);
    if (vel) v.assign((size_t)nk * nw_ * 3, 0.0);
    check(phx_el_diag(h_.get(), nk, k.empty() ? nullptr : k[0].data(), E.data(), detail::dptr(U),
                      vel ? v.data() : nullptr),
          ctx_);
    std::vector<ComplexMatrix> Us(nk, ComplexMatrix(nw_, nw_));
    for (int i = 0; i < nk; ++i)
      std::copy(U.begin() + (size_t)i * nw_ * nw_, U.begin() + (size_t)(i + 1) * nw_ * nw_, Us[i].data.begin());
    return {std::move(E), std::move(Us)};
  }
  phx_ctx* ctx_;
  int nw_;
  detail::Handle<phx_el_h0, phx_el_h0_destroy> h_;
};

// ---------------------------------------------------------------------------
class InteractionElPhWan {
 public:
  // g(Re,Rp,nu,w1,w2) complex FP32 (interleaved floats), Re (nRe,3), Rp (nRp,3) Bohr
  InteractionElPhWan(const Context& ctx, int nw, int nph, const std::vector<double>& Re,
                     const std::vector<double>& degE, const std::vector<double>& Rp, const std::vector<double>& degP,
                     const std::vector<float>& g)
      : ctx_(ctx.get()), nw_(nw), nph_(nph) {
    phx_elph* h = nullptr;
    check(phx_elph_create(ctx_, nw, nph, (int)degE.size(), (int)degP.size(), Re.data(), degE.data(), Rp.data(),
                          degP.data(), g.data(), &h),
          ctx_);
    h_ = detail::Handle<phx_elph, phx_elph_destroy>(h);
  }
  // precision of the transforms inside ElScatteringMatrix::setup
  void setPrecision(Precision p) { check(phx_elph_set_precision(h_.get(), (int)p), ctx_); }
  // U1 (nw, nb1): eigenvectors of the active k1 bands
  void cacheElPh(const ComplexMatrix& U1, const Vec3& k1) {
    nb1_ = U1.cols;
    check(phx_elph_cache_k1(h_.get(), k1.data(), detail::dptr(U1.data), nb1_), ctx_);
  }
  // U2s (nw, nb2_i) and phonon eigenvectors ev3s (nph, nph) of each final state, q3 = k2 - k1
  void calcCouplingSquared(const std::vector<ComplexMatrix>& U2s, const std::vector<ComplexMatrix>& ev3s,
                           const std::vector<Vec3>& q3s) {
    const int nk2 = (int)U2s.size();
    int nb2max = 0;
    std::vector<int> nb2s(nk2);
    for (int i = 0; i < nk2; ++i) nb2max = std::max(nb2max, nb2s[i] = U2s[i].cols);
    std::vector<cd> U2((size_t)nk2 * nw_ * std::max(1, nb2max)), ev3((size_t)nk2 * nph_ * nph_);
    for (int i = 0; i < nk2; ++i) {
      for (int w = 0; w < nw_; ++w)
        for (int b = 0; b < nb2s[i]; ++b) U2[((size_t)i * nw_ + w) * nb2max + b] = U2s[i](w, b);
      std::copy(ev3s[i].data.begin(), ev3s[i].data.end(), ev3.begin() + (size_t)i * nph_ * nph_);
    }
    std::vector<double> out((size_t)nk2 * nb1_ * std::max(1, nb2max) * nph_);
    check(phx_elph_couplings_sq(h_.get(), nk2, q3s.empty() ? nullptr : q3s[0].data(), detail::dptr(U2), nb2s.data(),
                                nb2max, detail::dptr(ev3), out.data()),
          ctx_);
    cache_.clear();
    for (int i = 0; i < nk2; ++i) {
      Tensor3 t(nb1_, nb2s[i], nph_);
      for (int b1 = 0; b1 < nb1_; ++b1)
        for (int b2 = 0; b2 < nb2s[i]; ++b2)
          for (int nu = 0; nu < nph_; ++nu) t(b1, b2, nu) = out[(((size_t)i * nb1_ + b1) * nb2max + b2) * nph_ + nu];
      cache_.push_back(std::move(t));
    }
  }
  // |g(b1, b2, nu)|^2 of final state ik2 of the last calcCouplingSquared
  const Tensor3& getCouplingSquared(int ik2) const { return cache_.at(ik2); }
  phx_elph* get() const { return h_.get(); }
  const phx_ctx* context() const { return ctx_; }
  int numWannier() const { return nw_; }

 private:
  phx_ctx* ctx_;
  int nw_, nph_, nb1_ = 0;
  std::vector<Tensor3> cache_;
  detail::Handle<phx_elph, phx_elph_destroy> h_;
};

// ---------------------------------------------------------------------------
// ElScatteringMatrix, linewidth mode, for outer k points of the electron mesh.
class ElScatteringMatrix {
 public:
  ElScatteringMatrix(InteractionElPhWan& elph, BandStructure& elBands, BandStructure& phBands,
                     std::vector<double> temperatures, double chemicalPotential, double window,
                     Smearing smearing = Smearing::adaptive, double sigma = 0.0, double norm = 0.0)
      : elph_(elph),
        el_(elBands),
        ph_(phBands),
        T_(std::move(temperatures)),
        mu_(chemicalPotential),
        window_(window),
        smearing_(smearing),
        sigma_(sigma),
        norm_(norm > 0.0 ? norm : 1.0 / phBands.getNumPoints()) {}
  // linewidths (nT, k1List.size(), nw), zero for inactive states
  std::vector<double> setup(const std::vector<int>& k1List) {
    phx_el_params p{};
    p.num_temperatures = (int)T_.size();
    p.temperatures = T_.data();
    p.chemical_potential = mu_;
    p.window = window_;
    p.smearing = (int)smearing_;
    p.sigma = sigma_;
    p.norm = norm_;
    p.num_k1 = (int)k1List.size();
    p.k1_list = k1List.data();
    std::vector<double> out(T_.size() * k1List.size() * (size_t)elph_.numWannier());
    check(phx_el_linewidths(elph_.get(), el_.get(), ph_.get(), &p, out.data(), &stats_), elph_.context());
    return out;
  }
  const phx_lw_stats& stats() const { return stats_; }

 private:
  InteractionElPhWan& elph_;
  BandStructure& el_;
  BandStructure& ph_;
  std::vector<double> T_;
  double mu_, window_;
  Smearing smearing_;
  double sigma_, norm_;
  phx_lw_stats stats_{};
};

}  // namespace phx

#endif  // PHOEBE_B200_HPP
