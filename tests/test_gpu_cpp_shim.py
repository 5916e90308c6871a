"""The C++ host layer (include/phoebe_b200.hpp), with the reference's class and
method names, driven by tests/cpp/shim_driver.cpp.

CPU: the header compiles with -Wall -Wextra and the driver links against
libphx.so (every ABI symbol it uses resolves).  GPU: the driver runs the
harmonic, 3-phonon, builder (linewidths, stored matrix, matrix-free
product), conductivity and el-ph paths through the C++ classes, and its outputs equal those of the Python mirror (phoebe_b200.core)
on the same inputs -- both sit on the same C ABI, whose numerics the other GPU
tests pin to the oracle -- and a bad argument surfaces as phx::Error with
PHX_ERR_ARG."""
import os
import subprocess

import numpy as np
import pytest

from phoebe_b200 import constants as C
from phoebe_b200 import lattice, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "phoebe_b200")


def _compile(out_dir):
    exe = os.path.join(out_dir, "shim_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "shim_driver.cpp"), "-L", LIBDIR, "-lphx",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libphx.so")):
        pytest.skip("libphx.so not built")
    exe = _compile(str(tmp_path))
    assert os.path.getsize(exe) > 0


def _w(d, name, a, dtype):
    np.ascontiguousarray(a, dtype=dtype).tofile(os.path.join(d, name))


def _c(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.view(np.float64)


def _r(d, name, dtype):
    return np.fromfile(os.path.join(d, name), dtype=dtype)


@pytest.mark.gpu
def test_shim_matches_python_mirror(ctx, diamond, tmp_path):
    from phoebe_b200.core import (ElectronH0Wannier, ElScatteringMatrix, Interaction3Ph, InteractionElPhWan,
                                  PhononH0, PhScatteringMatrix)
    inp, out = tmp_path / "in", tmp_path / "out"
    inp.mkdir()
    out.mkdir()
    inp, out = str(inp), str(out)
    exe = _compile(str(tmp_path))
    cr, fc2, fc3 = diamond["crystal"], diamond["fc2"], diamond["fc3"]
    rng = np.random.default_rng(11)
    nb = cr.num_bands
    mesh = (4, 4, 4)
    nq1, nb2 = 6, 5
    nb1s = np.array([6, 5, 6, 4, 6, 6], np.int32)
    nb3p = np.array([6, 6, 3, 6, 6, 6], np.int32)
    nb3m = np.array([6, 6, 6, 6, 2, 6], np.int32)
    temps = np.array([C.kelvin_to_ry(300.0), C.kelvin_to_ry(600.0)])
    dims = [cr.num_atoms, fc3.D3.shape[4], fc3.D3.shape[3], *fc2.shape[2:5], *mesh, nq1, nb2, len(temps),
            1]  # adaptive
    _w(inp, "dims.i32", dims, np.int32)
    _w(inp, "cell.f64", cr.direct_cell, np.float64)
    _w(inp, "positions.f64", cr.positions, np.float64)
    _w(inp, "masses.f64", cr.atomic_masses, np.float64)
    _w(inp, "fc2.f64", fc2, np.float64)
    qs = rng.normal(size=(5, 3)) * 0.3
    _w(inp, "q_points.f64", qs, np.float64)
    for name in ("D3", "R2", "R3", "w2", "w3"):
        _w(inp, name + ".f64", getattr(fc3, name), np.float64)

    def unitary(n, k):
        return np.stack([np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))[0] for _ in range(k)])

    q1s = rng.normal(size=(nq1, 3)) * 0.3
    q2 = rng.normal(size=3) * 0.3
    ev1, ev3p, ev3m = unitary(nb, nq1), unitary(nb, nq1), unitary(nb, nq1)
    ev2 = unitary(nb, 1)[0]
    _w(inp, "q1s.f64", q1s, np.float64)
    _w(inp, "q2.f64", q2, np.float64)
    for name, a in (("ev1", ev1), ("ev2", ev2), ("ev3p", ev3p), ("ev3m", ev3m)):
        _w(inp, name + ".f64", _c(a), np.float64)
    for name, a in (("nb1s", nb1s), ("nb3p", nb3p), ("nb3m", nb3m)):
        _w(inp, name + ".i32", a, np.int32)
    _w(inp, "temperatures.f64", temps, np.float64)
    _w(inp, "sigma.f64", [0.0], np.float64)
    # el-ph
    model = synth.elph_model(nw=8, ncell_h=1, ncell_e=1, ncell_p=1)
    kmesh, qmesh = (6, 6, 6), (3, 3, 3)
    nk2 = 5
    k1 = np.array([0.11, -0.23, 0.05])
    k2s = rng.normal(size=(nk2, 3)) * 0.4
    ev3s = unitary(6, nk2)
    _w(inp, "el_dims.i32", [8, 6, *kmesh, *qmesh, 1, nk2], np.int32)
    _w(inp, "el_R.f64", model.Re, np.float64)
    _w(inp, "el_deg.f64", model.degE, np.float64)
    _w(inp, "el_H.f64", _c(model.H), np.float64)
    _w(inp, "elph_Re.f64", model.Re, np.float64)
    _w(inp, "elph_degE.f64", model.degE, np.float64)
    _w(inp, "elph_Rp.f64", model.Rp, np.float64)
    _w(inp, "elph_degP.f64", model.degP, np.float64)
    _w(inp, "elph_g.f32", np.ascontiguousarray(model.g, dtype=np.complex64).view(np.float32), np.float32)
    _w(inp, "elph_k1.f64", k1, np.float64)
    _w(inp, "elph_k2.f64", k2s, np.float64)
    _w(inp, "elph_ev3.f64", _c(ev3s), np.float64)
    wan = ElectronH0Wannier(ctx, cr, model.Re, model.degE, model.H)
    elb = wan.populate(kmesh, withVelocities=True)
    Ek = elb.get(velocities=False)[0]
    mu, window, T_el = float(np.median(Ek)), 0.05, C.kelvin_to_ry(300.0)
    k1_list = np.arange(0, int(np.prod(kmesh)), 2, dtype=np.int32)
    _w(inp, "el_params.f64", [mu, window, T_el], np.float64)
    _w(inp, "el_k1_list.i32", k1_list, np.int32)

    ns_mesh = int(np.prod(mesh)) * nb
    xs = rng.normal(size=(len(temps), 3, ns_mesh))
    _w(inp, "smatrix_x.f64", xs, np.float64)
    r = subprocess.run([exe, inp, out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr

    # ---- the same calls through the Python mirror
    h0 = PhononH0(ctx, cr, fc2)
    E, U, v = h0.diagonalizeWithVelocities(qs)
    np.testing.assert_array_equal(_r(out, "ph_E.f64", np.float64), E.ravel())
    np.testing.assert_array_equal(_r(out, "ph_v.f64", np.float64), v.ravel())
    np.testing.assert_array_equal(_r(out, "ph_U.c128", np.complex128), U.ravel())
    E1, U1 = h0.diagonalizeFromCoordinates(qs[:1], withMassScaling=False)
    np.testing.assert_array_equal(_r(out, "ph_E_single.f64", np.float64), E1.ravel())
    np.testing.assert_array_equal(_r(out, "ph_U_single.c128", np.complex128), U1.ravel())

    v3 = Interaction3Ph(ctx, cr, fc3)
    v3.cacheD3(q2)
    cp, cm = v3.getCouplingsSquared(q1s, q2, [ev1[i][:, :nb1s[i]] for i in range(nq1)], ev2[:, :nb2],
                                    [ev3p[i][:, :nb3p[i]] for i in range(nq1)],
                                    [ev3m[i][:, :nb3m[i]] for i in range(nq1)])
    np.testing.assert_array_equal(_r(out, "v3_plus.f64", np.float64), np.concatenate([c.ravel() for c in cp]))
    np.testing.assert_array_equal(_r(out, "v3_mins.f64", np.float64), np.concatenate([c.ravel() for c in cm]))
    assert _r(out, "v3_batches.i32", np.int32)[0] == v3.estimateNumBatches(nq1, nb2)

    bands = h0.populate(mesh, withVelocities=True)
    sm = PhScatteringMatrix(v3, bands, temps, "adaptive")
    A = sm.setup()
    Eb = bands.get(velocities=False)[0]
    # FP64 atomics: the last bits of a sum depend on the order of arrival
    np.testing.assert_allclose(_r(out, "A_out.f64", np.float64), A.ravel(), rtol=1e-12, atol=0)
    with np.errstate(divide="ignore", invalid="ignore"):
        lw = sm.getLinewidths(Eb).ravel()
        tau = sm.getSingleModeTimes(Eb).ravel()
    ok = np.isfinite(lw) & (A.ravel() != 0)
    np.testing.assert_allclose(_r(out, "linewidths.f64", np.float64)[ok], lw[ok], rtol=1e-12)
    np.testing.assert_allclose(_r(out, "times.f64", np.float64)[ok], tau[ok], rtol=1e-12)
    kappa = sm.thermalConductivity(lattice.calc_volume(cr.direct_cell))
    mem = PhScatteringMatrix(v3, bands, temps[:1], "adaptive", in_memory=True)
    dmem = mem.setup()
    np.testing.assert_array_equal(_r(out, "smatrix_diag.f64", np.float64), dmem.ravel())
    np.testing.assert_array_equal(_r(out, "smatrix_rows.f64", np.float64), mem.getMatrixRows(3, 5).ravel())
    # FP64 atomics: summation order of the products
    yd = mem.dot(xs[None, :1])[0]
    np.testing.assert_allclose(_r(out, "smatrix_dot.f64", np.float64), yd.ravel(), rtol=1e-12,
                               atol=1e-14 * np.abs(yd).max())
    yo = mem.offDiagonalDot(xs[None, :1])[0]
    np.testing.assert_allclose(_r(out, "smatrix_offdot.f64", np.float64), yo.ravel(), rtol=1e-12,
                               atol=1e-14 * np.abs(yo).max())
    mem.symmetrize()
    np.testing.assert_array_equal(_r(out, "smatrix_sym_rows.f64", np.float64), mem.getMatrixRows(3, 5).ravel())
    mem.a2Omega()
    np.testing.assert_array_equal(_r(out, "omega_diag.f64", np.float64), mem.internalDiagonal.ravel())
    lam = mem.diagonalize()
    np.testing.assert_allclose(_r(out, "relaxon_eigenvalues.f64", np.float64), lam, rtol=0,
                               atol=1e-12 * np.abs(lam).max())
    yr = mem.relaxonSolve(xs[0])
    np.testing.assert_allclose(_r(out, "relaxon_solve.f64", np.float64), yr.ravel(), rtol=0,
                               atol=1e-10 * np.abs(yr).max())
    mem.close()
    yf = PhScatteringMatrix(v3, bands, temps, "adaptive").dot(xs)
    np.testing.assert_allclose(_r(out, "smatrix_free_dot.f64", np.float64), yf.ravel(), rtol=1e-12,
                               atol=1e-14 * np.abs(yf).max())
    np.testing.assert_allclose(_r(out, "kappa.f64", np.float64) * C.thConductivityAuToSi, kappa.ravel(),
                               rtol=1e-10, atol=1e-12 * np.abs(kappa).max())

    Ek1, Uk1 = wan.diagonalizeFromCoordinates(k1[None, :])
    np.testing.assert_array_equal(_r(out, "el_E_k1.f64", np.float64), Ek1.ravel())
    elph = InteractionElPhWan(ctx, model.Re, model.degE, model.Rp, model.degP, model.g)
    elph.cacheElPh(Uk1[0][:, 2:5], k1)
    _, Uk2 = wan.diagonalizeFromCoordinates(k2s)
    g2 = elph.calcCouplingSquared([Uk2[i][:, 1:5] for i in range(nk2)], ev3s, k2s - k1)
    np.testing.assert_array_equal(_r(out, "elph_g2.f64", np.float64), np.concatenate([g.ravel() for g in g2]))
    phb = h0.populate(qmesh, withVelocities=False)
    esm = ElScatteringMatrix(elph, elb, phb, np.array([T_el]), mu, window, "adaptive")
    L = esm.setup(k1_list)
    assert np.abs(L).max() > 0
    np.testing.assert_allclose(_r(out, "el_linewidths.f64", np.float64), L.ravel(), rtol=1e-12,
                               atol=1e-14 * np.abs(L).max())

    assert _r(out, "error_status.i32", np.int32)[0] == 1   # PHX_ERR_ARG
    for o in (phb, elph, elb, wan, bands, v3, h0):
        o.close()
