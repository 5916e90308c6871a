"""Crystal cell and Gamma-centred wavevector mesh (host side, FP64, numpy).

Mirrors the pieces of Phoebe's ``Crystal`` and ``Points`` classes that the
scattering-rate path touches:

* reciprocal cell = 2*pi*(A^-1)^T with lattice vectors as columns of A
  (src/crystal.cpp:290-293); volume as in src/crystal.cpp:11-21;
* mesh point index = ix + iy*n0 + iz*n0*n1, crystal coordinates i/n + offset
  (src/points.cpp:222-248);
* lookup of a crystal-coordinate point on the mesh, with the reference's
  signed rounding test (src/points.cpp:404-423).
"""
from dataclasses import dataclass, field

import numpy as np


def calc_volume(direct_cell):
    """Unit-cell volume (crystal.cpp:11-21: mean of three |triple products|)."""
    a1, a2, a3 = direct_cell[0, :], direct_cell[1, :], direct_cell[2, :]
    v = abs(a1 @ np.cross(a2, a3)) + abs(a2 @ np.cross(a3, a1)) + abs(a3 @ np.cross(a1, a2))
    return v / 3.0


@dataclass
class Crystal:
    """Direct cell (Bohr, lattice vectors as columns), atoms (Bohr), masses (Ry)."""
    direct_cell: np.ndarray          # (3,3), column i = lattice vector a_i
    positions: np.ndarray            # (nat,3) Cartesian, Bohr
    species: np.ndarray              # (nat,) int species index
    species_masses: np.ndarray       # (nspecies,) Ry mass units
    reciprocal_cell: np.ndarray = field(init=False)
    volume: float = field(init=False)

    def __post_init__(self):
        self.direct_cell = np.asarray(self.direct_cell, dtype=np.float64)
        self.positions = np.asarray(self.positions, dtype=np.float64).reshape(-1, 3)
        self.species = np.asarray(self.species, dtype=np.int32)
        self.species_masses = np.asarray(self.species_masses, dtype=np.float64)
        self.reciprocal_cell = 2.0 * np.pi * np.linalg.inv(self.direct_cell).T
        self.volume = calc_volume(self.direct_cell)

    @property
    def num_atoms(self):
        return self.positions.shape[0]

    @property
    def num_bands(self):
        return 3 * self.num_atoms

    @property
    def atomic_masses(self):
        return self.species_masses[self.species]


def mod(a, b):
    """Python-style modulo for ints (utilities.cpp mod)."""
    return a % b


class Mesh:
    """Gamma-centred (or offset) Monkhorst-Pack mesh over the reciprocal cell."""

    def __init__(self, crystal, mesh, offset=(0.0, 0.0, 0.0)):
        self.crystal = crystal
        self.mesh = np.asarray(mesh, dtype=np.int64)
        self.offset = np.asarray(offset, dtype=np.float64)
        self.num_points = int(np.prod(self.mesh))

    def crystal_coords(self, idx=None):
        """Crystal coordinates of mesh points (points.cpp:233-242)."""
        n0, n1, n2 = (int(x) for x in self.mesh)
        if idx is None:
            idx = np.arange(self.num_points)
        idx = np.asarray(idx, dtype=np.int64)
        ikz = idx // (n0 * n1)
        rem = idx - ikz * n0 * n1
        iky = rem // n0
        ikx = rem % n0
        out = np.empty(idx.shape + (3,), dtype=np.float64)
        out[..., 0] = ikx.astype(np.float64) / float(n0) + self.offset[0]
        out[..., 1] = iky.astype(np.float64) / float(n1) + self.offset[1]
        out[..., 2] = ikz.astype(np.float64) / float(n2) + self.offset[2]
        return out

    def cartesian_coords(self, idx=None):
        """Cartesian wavevectors (1/Bohr): reciprocal_cell @ crystal."""
        c = self.crystal_coords(idx)
        return c @ self.crystal.reciprocal_cell.T

    def cartesian_to_crystal(self, q_cart):
        return np.asarray(q_cart) @ np.linalg.inv(self.crystal.reciprocal_cell).T

    def index_of(self, crys):
        """Mesh index of crystal coordinates, -1 when off-mesh (points.cpp:404-423).

        The reference accumulates the *signed* rounding residual over the three
        axes and rejects only when the sum is >= 1e-6; that quirk is kept.
        """
        crys = np.atleast_2d(np.asarray(crys, dtype=np.float64))
        x = (crys - self.offset) * self.mesh
        r = np.round(x)
        diff = np.sum(r - x, axis=-1)
        p = np.mod(r.astype(np.int64), self.mesh)
        ik = p[:, 2] * self.mesh[0] * self.mesh[1] + p[:, 1] * self.mesh[0] + p[:, 0]
        ik = np.where(diff >= 1.0e-6, -1, ik)
        return ik

    def q3_indices(self, sign=+1):
        """Index table iq3[iq1, iq2] of q1 + sign*q2 (Cartesian sum, then lookup).

        Follows Helper3rdState::get case 1 (src/bte/helper_3rd_state.cpp:134-170):
        q3 is formed in Cartesian coordinates, converted back to crystal
        coordinates and looked up on the same mesh.
        """
        qc = self.cartesian_coords()
        q3 = qc[:, None, :] + sign * qc[None, :, :]
        crys = self.cartesian_to_crystal(q3.reshape(-1, 3))
        return self.index_of(crys).reshape(self.num_points, self.num_points)
