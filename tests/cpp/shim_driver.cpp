// Drives the C++ host layer (include/phoebe_b200.hpp) the way Phoebe's
// transport code drives its classes: harmonic phonons, the 3-phonon vertex,
// the linewidth builder and thermal conductivity, the el-ph Wannier path, and
// the error convention.  Inputs are raw little-endian arrays written by
// tests/test_gpu_cpp_shim.py into a directory; outputs go to a second one.
//
//   shim_driver <input dir> <output dir>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "phoebe_b200.hpp"

namespace {

std::string in_dir, out_dir;

template <class T>
std::vector<T> load(const std::string& name) {
  std::ifstream f(in_dir + "/" + name, std::ios::binary | std::ios::ate);
  if (!f) throw std::runtime_error("missing input " + name);
  const std::streamsize n = f.tellg();
  f.seekg(0);
  std::vector<T> v((size_t)n / sizeof(T));
  f.read(reinterpret_cast<char*>(v.data()), n);
  return v;
}

template <class T>
void save(const std::string& name, const T* p, size_t n) {
  std::ofstream f(out_dir + "/" + name, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(*p)));
}
template <class T>
void save(const std::string& name, const std::vector<T>& v) {
  save(name, v.data(), v.size());
}

std::vector<phx::Vec3> vec3s(const std::vector<double>& a) {
  std::vector<phx::Vec3> out(a.size() / 3);
  for (size_t i = 0; i < out.size(); ++i) out[i] = {a[3 * i], a[3 * i + 1], a[3 * i + 2]};
  return out;
}

std::vector<phx::ComplexMatrix> matrices(const std::vector<double>& a, int n, int rows, int cols) {
  std::vector<phx::ComplexMatrix> out(n, phx::ComplexMatrix(rows, cols));
  for (int i = 0; i < n; ++i)
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) {
        const size_t k = (((size_t)i * rows + r) * cols + c) * 2;
        out[i](r, c) = {a[k], a[k + 1]};
      }
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: shim_driver <input dir> <output dir>\n");
    return 2;
  }
  in_dir = argv[1];
  out_dir = argv[2];
  try {
    phx::Context ctx(0);
    // ---- harmonic phonons -------------------------------------------------
    const auto dims = load<int>("dims.i32");  // nat, nr2, nr3, fc grid(3), mesh(3), nq1, nb2, nT, smearing
    const int nat = dims[0], nr2 = dims[1], nr3 = dims[2], nb = 3 * nat;
    phx::Crystal cr;
    const auto cell = load<double>("cell.f64");
    std::copy(cell.begin(), cell.end(), cr.cell.begin());
    cr.positions = load<double>("positions.f64");
    cr.masses = load<double>("masses.f64");
    phx::PhononH0 h0(ctx, cr, load<double>("fc2.f64"), {dims[3], dims[4], dims[5]});
    const auto qs = vec3s(load<double>("q_points.f64"));
    auto [E, U, v] = h0.kokkosBatchedDiagonalizeWithVelocities(qs);
    save("ph_E.f64", E);
    save("ph_v.f64", v);
    std::vector<phx::cd> Uflat;
    for (const auto& m : U) Uflat.insert(Uflat.end(), m.data.begin(), m.data.end());
    save("ph_U.c128", Uflat);
    auto [Esingle, Usingle] = h0.diagonalizeFromCoordinates(qs[0], false);
    save("ph_E_single.f64", Esingle);
    save("ph_U_single.c128", Usingle.data);

    // ---- 3-phonon vertex --------------------------------------------------
    phx::Interaction3Ph v3(ctx, nat, nr2, nr3, load<double>("D3.f64"), load<double>("R2.f64"), load<double>("R3.f64"),
                           load<double>("w2.f64"), load<double>("w3.f64"));
    const int nq1 = dims[9], nb2 = dims[10];
    const auto q1s = vec3s(load<double>("q1s.f64"));
    const auto q2 = vec3s(load<double>("q2.f64"))[0];
    const auto ev1 = matrices(load<double>("ev1.f64"), nq1, nb, nb);
    const auto ev2 = matrices(load<double>("ev2.f64"), 1, nb, nb)[0];
    const auto ev3p = matrices(load<double>("ev3p.f64"), nq1, nb, nb);
    const auto ev3m = matrices(load<double>("ev3m.f64"), nq1, nb, nb);
    const auto nb1s = load<int>("nb1s.i32"), nb3p = load<int>("nb3p.i32"), nb3m = load<int>("nb3m.i32");
    v3.cacheD3(q2);
    auto [cp, cm] = v3.getCouplingsSquared(q1s, q2, ev1, ev2, ev3p, ev3m, nb1s, nb2, nb3p, nb3m);
    std::vector<double> fp, fm;
    for (const auto& t : cp) fp.insert(fp.end(), t.data.begin(), t.data.end());
    for (const auto& t : cm) fm.insert(fm.end(), t.data.begin(), t.data.end());
    save("v3_plus.f64", fp);
    save("v3_mins.f64", fm);
    const int nbatch = v3.estimateNumBatches(nq1, nb2);
    save("v3_batches.i32", &nbatch, 1);

    // ---- linewidth builder and RTA conductivity ----------------------------
    const int nT = dims[11];
    const auto temps = load<double>("temperatures.f64");
    auto bands = h0.populate({dims[6], dims[7], dims[8]}, true);
    phx::PhScatteringMatrix sm(v3, bands, temps, dims[12] == PHX_SMEAR_GAUSSIAN ? phx::Smearing::gaussian
                                                                                 : phx::Smearing::adaptive,
                               load<double>("sigma.f64")[0]);
    sm.setup();
    save("A_out.f64", sm.internalDiagonal());
    save("linewidths.f64", sm.getLinewidths());
    save("times.f64", sm.getSingleModeTimes());
    const auto kappa = sm.thermalConductivity(cr.volume());
    save("kappa.f64", kappa[0].data(), kappa.size() * 9);
    (void)nT;

    // ---- scattering matrix: stored (first temperature) and matrix-free ------
    {
      const auto x = load<double>("smatrix_x.f64");   // (nT, 3, ns)
      const size_t ns = sm.numStates();
      std::vector<double> x0(x.begin(), x.begin() + 3 * ns);
      phx::PhScatteringMatrix mem(v3, bands, {temps[0]}, phx::Smearing::adaptive);
      mem.setMatrixInMemory(true);
      mem.setup();
      save("smatrix_diag.f64", mem.internalDiagonal());
      save("smatrix_rows.f64", mem.getRows(3, 5));
      save("smatrix_dot.f64", mem.dot(x0));
      save("smatrix_offdot.f64", mem.offDiagonalDot(x0));
      mem.symmetrize();
      save("smatrix_sym_rows.f64", mem.getRows(3, 5));
      mem.a2Omega();
      save("omega_diag.f64", mem.internalDiagonal());
      save("relaxon_eigenvalues.f64", mem.diagonalize());
      save("relaxon_solve.f64", mem.relaxonSolve(x0));
      phx::PhScatteringMatrix freeSm(v3, bands, temps, phx::Smearing::adaptive);
      save("smatrix_free_dot.f64", freeSm.dot(x));
    }

    // ---- el-ph Wannier path -----------------------------------------------
    const auto edims = load<int>("el_dims.i32");  // nw, nph, kmesh(3), qmesh(3), nk1, nk2
    const int nw = edims[0], nph = edims[1];
    phx::ElectronH0Wannier wan(ctx, cr.cell, nw, load<double>("el_R.f64"), load<double>("el_deg.f64"),
                               [&] {
                                 const auto h = load<double>("el_H.f64");
                                 std::vector<phx::cd> H(h.size() / 2);
                                 for (size_t i = 0; i < H.size(); ++i) H[i] = {h[2 * i], h[2 * i + 1]};
                                 return H;
                               }());
    phx::InteractionElPhWan elph(ctx, nw, nph, load<double>("elph_Re.f64"), load<double>("elph_degE.f64"),
                                 load<double>("elph_Rp.f64"), load<double>("elph_degP.f64"),
                                 load<float>("elph_g.f32"));
    const auto k1 = vec3s(load<double>("elph_k1.f64"))[0];
    auto [Ek1, Uk1] = wan.diagonalizeFromCoordinates(k1);
    save("el_E_k1.f64", Ek1);
    phx::ComplexMatrix U1(nw, 3);  // bands 2..4 of k1
    for (int w = 0; w < nw; ++w)
      for (int b = 0; b < 3; ++b) U1(w, b) = Uk1(w, 2 + b);
    elph.cacheElPh(U1, k1);
    const int nk2 = edims[9];
    const auto k2s = vec3s(load<double>("elph_k2.f64"));
    auto [Ek2, Uk2] = wan.batchedDiagonalizeFromCoordinates(k2s);
    std::vector<phx::ComplexMatrix> U2s;
    std::vector<phx::Vec3> q3s;
    for (int i = 0; i < nk2; ++i) {
      phx::ComplexMatrix m(nw, 4);  // bands 1..4 of k2
      for (int w = 0; w < nw; ++w)
        for (int b = 0; b < 4; ++b) m(w, b) = Uk2[i](w, 1 + b);
      U2s.push_back(m);
      q3s.push_back({k2s[i][0] - k1[0], k2s[i][1] - k1[1], k2s[i][2] - k1[2]});
    }
    const auto ev3s = matrices(load<double>("elph_ev3.f64"), nk2, nph, nph);
    elph.calcCouplingSquared(U2s, ev3s, q3s);
    std::vector<double> g2;
    for (int i = 0; i < nk2; ++i) {
      const auto& t = elph.getCouplingSquared(i);
      g2.insert(g2.end(), t.data.begin(), t.data.end());
    }
    save("elph_g2.f64", g2);
    auto elBands = wan.populate({edims[2], edims[3], edims[4]}, true);
    auto phBands = h0.populate({edims[5], edims[6], edims[7]}, false);
    const auto el_extra = load<double>("el_params.f64");  // mu, window, temperature
    phx::ElScatteringMatrix esm(elph, elBands, phBands, {el_extra[2]}, el_extra[0], el_extra[1]);
    save("el_linewidths.f64", esm.setup(load<int>("el_k1_list.i32")));

    // ---- error convention -------------------------------------------------
    int status = 0;
    try {
      v3.setPrecision(static_cast<phx::Precision>(7));
    } catch (const phx::Error& e) {
      status = e.status();
    }
    save("error_status.i32", &status, 1);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "shim_driver: %s\n", e.what());
    return 1;
  }
  return 0;
}
