"""JSON output in the reference's formats (src/bte/scattering.cpp:639-815;
src/observable/phonon_thermal_cond.cpp:475-505).

CPU: the relaxation-times file of oracle linewidths has the reference's keys,
units and (nT, nq, nb[, 3]) nesting; its linewidths, times, energies and
velocities are the oracle's values in meV, ps and m/s; excluded states have
linewidth 0 and a null time, and the file is strict JSON; the conductivity
file holds the tensor in W/(m K).  GPU: PhScatteringMatrix.outputToJSON
writes the same file from the GPU linewidths (1e-10 of the oracle)."""
import json

import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, output


def _oracle(diamond, mesh, temps):
    cr = diamond["crystal"]
    h0 = oracle.PhononH0(cr, diamond["fc2"])
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    E, U = h0.diagonalize(q)
    vg = h0.velocities(q)
    A = oracle.Interaction3Ph(cr, diamond["fc3"]).linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, temps,
                                                              "adaptive", 0.0)
    return E, vg, A


def test_relaxation_times_json(diamond, tmp_path):
    mesh = (3, 3, 3)
    temps = np.array([C.kelvin_to_ry(300.0), C.kelvin_to_ry(600.0)])
    E, vg, A = _oracle(diamond, mesh, temps)
    path = tmp_path / "rta_ph_relaxation_times.json"
    output.relaxation_times_json(path, diamond["crystal"], mesh, E, vg, A, temps)
    text = path.read_text()
    assert "Infinity" not in text and "NaN" not in text
    d = json.loads(text)
    assert d["linewidthsUnit"] == "meV" and d["relaxationTimeUnit"] == "ps" and d["energyUnit"] == "meV"
    assert d["velocityUnit"] == "m/s" and d["coordsType"] == "lattice" and d["particleType"] == "phonon"
    np.testing.assert_allclose(d["temperatures"], [300.0, 600.0], rtol=1e-12)
    nq, nb = E.shape
    lw = np.array(d["linewidths"], dtype=float)
    assert lw.shape == (2, nq, nb)
    assert np.array(d["velocities"]).shape == (2, nq, nb, 3)
    assert np.array(d["wavevectorCoordinates"]).shape == (nq, 3)
    np.testing.assert_allclose(np.array(d["wavevectorCoordinates"]), lattice.Mesh(diamond["crystal"], mesh)
                               .crystal_coords(), atol=1e-12)
    x = np.sinh(E[None] / 2 / temps[:, None, None])
    ok = E >= C.phExcludeCutoff
    ref_lw = A.reshape(2, nq, nb) / (0.25 / x / x) * C.energyRyToEv * 1000
    np.testing.assert_allclose(lw[:, ok], ref_lw[:, ok], rtol=1e-13)
    assert np.all(lw[:, ~ok] == 0.0)
    times = np.array(d["relaxationTimes"], dtype=float)          # null -> nan
    np.testing.assert_allclose(times[:, ok], 1.0 / (ref_lw[:, ok] / (C.energyRyToEv * 1000))
                               * C.energyRyToFs / C.twoPi * 1e-3, rtol=1e-12)
    assert np.all(np.isnan(times[:, ~ok]))
    np.testing.assert_allclose(np.array(d["energies"])[1], E * C.energyRyToEv * 1000, rtol=1e-14)
    np.testing.assert_allclose(np.array(d["velocities"])[0], vg * C.velocityRyToSi, rtol=1e-14)
    # keys sorted and indented by 3, as nlohmann::json with std::setw(3)
    assert text.startswith('{\n   "chemicalPotentialUnit"')


def test_thermal_conductivity_json(tmp_path):
    k = np.arange(18, dtype=float).reshape(2, 3, 3)
    d = output.thermal_conductivity_json(tmp_path / "rta_phonon_thermal_cond.json", k,
                                         [C.kelvin_to_ry(100.0), C.kelvin_to_ry(200.0)])
    r = json.loads((tmp_path / "rta_phonon_thermal_cond.json").read_text())
    assert r == d and r["thermalConductivityUnit"] == "W /(m K)"
    np.testing.assert_array_equal(r["thermalConductivity"], k)


@pytest.mark.gpu
def test_gpu_output_json(ctx, diamond, tmp_path):
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr, mesh = diamond["crystal"], (4, 4, 4)
    temps = np.array([C.kelvin_to_ry(300.0)])
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    sm = PhScatteringMatrix(v3, bands, temps, "adaptive")
    sm.setup()
    d = sm.outputToJSON(tmp_path / "gpu.json", cr)
    E, U, vg = bands.get()
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    A = oracle.Interaction3Ph(cr, diamond["fc3"]).linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, temps,
                                                              "adaptive", 0.0)
    r = output.relaxation_times_json(tmp_path / "oracle.json", cr, mesh, E, vg, A, temps)
    a, b = np.array(d["linewidths"], dtype=float), np.array(r["linewidths"], dtype=float)
    np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-14 * np.nanmax(b))
    assert d["energies"] == r["energies"] and d["velocities"] == r["velocities"]
    for o in (v3, bands, h0):
        o.close()
