"""JSON output in the reference's formats.

  * relaxation_times_json: ScatteringMatrix::outputToJSON for phonons
    (src/bte/scattering.cpp:639-815), the file the reference writes as
    rta_ph_relaxation_times.json: linewidths (meV), relaxationTimes (ps),
    velocities (m/s) and energies (meV) as (nT, nq, nb[, 3]) nested lists,
    the temperatures (K), the wavevectors in lattice coordinates;
  * thermal_conductivity_json: PhononThermalConductivity::outputToJSON
    (src/observable/phonon_thermal_cond.cpp:475-505), the files
    rta_phonon_thermal_cond.json, omini_phonon_thermal_cond.json,
    variational_phonon_thermal_cond.json and relaxons_phonon_thermal_cond.json;
  * relaxons_relaxation_times_json: ScatteringMatrix::relaxonsToJSON
    (src/bte/scattering.cpp:816-870), relaxons_relaxation_times.json.

Non-finite numbers (the relaxation time of an excluded state is n(n+1)/0)
are written as null, as nlohmann::json does; the layout is indented by 3 like
the reference's std::setw(3).  Without symmetries every mesh point is
written, in the mesh's index order."""
import json
import math

import numpy as np

from . import constants as C
from . import lattice


def _clean(x):
    """Nested lists with non-finite floats replaced by None."""
    if isinstance(x, list):
        return [_clean(v) for v in x]
    return float(x) if math.isfinite(x) else None


def relaxation_times_json(path, crystal, mesh, E, vg, A_out, temperatures_ry):
    """E (nq, nb) Ry, vg (nq, nb, 3) Ry units, A_out (nT, nq*nb) the
    internalDiagonal (linewidth x n(n+1)), temperatures in Ry."""
    E = np.asarray(E, dtype=np.float64)
    nq, nb = E.shape
    T = np.atleast_1d(np.asarray(temperatures_ry, dtype=np.float64))
    A = np.asarray(A_out, dtype=np.float64).reshape(len(T), nq, nb)
    energy_conv = C.energyRyToEv * 1000.0              # meV
    time_conv = C.energyRyToFs / C.twoPi * 1e-3         # ps
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        x = np.sinh(E[None] / 2.0 / T[:, None, None])
        popterm = 0.25 / x / x
        linewidths = A / popterm                        # getLinewidths (scattering.cpp:529-568)
        times = popterm / A                             # getTimesFromVectorBTE (:484-513)
    m = lattice.Mesh(crystal, mesh)
    coords = m.cartesian_to_crystal(m.cartesian_coords())
    vel = np.asarray(vg, dtype=np.float64).reshape(nq, nb, 3) * C.velocityRyToSi
    out = {
        "temperatures": [float(t * C.temperatureAuToSi) for t in T],
        "temperatureUnit": "K",
        "chemicalPotentials": [0.0] * len(T),
        "chemicalPotentialUnit": "eV",
        "linewidths": _clean((linewidths * energy_conv).tolist()),
        "linewidthsUnit": "meV",
        "relaxationTimes": _clean((times * time_conv).tolist()),
        "relaxationTimeUnit": "ps",
        "velocities": _clean(np.broadcast_to(vel, (len(T), nq, nb, 3)).tolist()),
        "velocityUnit": "m/s",
        "energies": _clean(np.broadcast_to(E * energy_conv, (len(T), nq, nb)).tolist()),
        "energyUnit": "meV",
        "wavevectorCoordinates": _clean(coords.tolist()),
        "coordsType": "lattice",
        "particleType": "phonon",
    }
    with open(path, "w") as f:
        json.dump(out, f, indent=3, sort_keys=True, allow_nan=False)
        f.write("\n")
    return out


def relaxons_relaxation_times_json(path, eigenvalues, temperatures_ry):
    """ScatteringMatrix::relaxonsToJSON (src/bte/scattering.cpp:816-870), the
    file relaxons_relaxation_times.json: the relaxon times 1/lambda of every
    eigenvalue, in fs, once per temperature (the reference writes the same
    list for each; a zero eigenvalue gives null)."""
    T = np.atleast_1d(np.asarray(temperatures_ry, dtype=np.float64))
    lam = np.asarray(eigenvalues, dtype=np.float64).ravel()
    with np.errstate(divide="ignore"):
        times = (1.0 / lam) * C.energyRyToFs
    out = {
        "temperatures": [float(t * C.temperatureAuToSi) for t in T],
        "temperatureUnit": "K",
        "chemicalPotentials": [0.0] * len(T),
        "relaxationTimes": _clean([times.tolist() for _ in T]),
        "relaxationTimeUnit": "fs",
        "particleType": "phonon",
    }
    with open(path, "w") as f:
        json.dump(out, f, indent=3, sort_keys=True, allow_nan=False)
        f.write("\n")
    return out


def thermal_conductivity_json(path, kappa_si, temperatures_ry):
    """kappa_si (nT, 3, 3) in W/(m K)."""
    T = np.atleast_1d(np.asarray(temperatures_ry, dtype=np.float64))
    out = {
        "temperatures": [float(t * C.temperatureAuToSi) for t in T],
        "thermalConductivity": _clean(np.asarray(kappa_si, dtype=np.float64).reshape(len(T), 3, 3).tolist()),
        "temperatureUnit": "K",
        "thermalConductivityUnit": "W /(m K)",
        "particleType": "phonon",
    }
    with open(path, "w") as f:
        json.dump(out, f, indent=3, sort_keys=True, allow_nan=False)
        f.write("\n")
    return out
