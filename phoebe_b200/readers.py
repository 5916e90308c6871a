"""Readers for the reference's harmonic and anharmonic force-constant files.

* QE ``.fc`` (q2r output): follows QEParser::parsePhHarmonic,
  src/parser/qe_input_parser.cpp:385-560 (lattice from getQELattice,
  :18-110 for ibrav 0-3; masses already in Ry units; atomic positions in alat
  units converted to Bohr; optional dielectric tensor and Born charges; the
  force constants in the (3,3,n1,n2,n3,nat,nat) layout, r1 fastest).
* ShengBTE ``FORCE_CONSTANTS_3RD``: follows IFC3Parser::parseFromShengBTE,
  src/parser/ifc3_parser.cpp:648-840 (cell vectors in Angstrom -> Bohr,
  eV/A^3 -> Ry/Bohr^3, distinct R2 / R3 lists in order of first appearance,
  dense D3(nb,nb,nb,nr3,nr2), unit weights).
"""
import numpy as np

from . import constants as C
from .lattice import Crystal
from .synth import FC3


def _qe_lattice(ibrav, celldm, cell_in):
    a = celldm[0]
    if ibrav == 0:
        return cell_in * (a if a != 0.0 else 1.0)
    if ibrav == 1:
        return a * np.eye(3)
    if ibrav == 2:
        t = a / 2.0
        a1, a2, a3 = [-t, 0, t], [0, t, t], [-t, t, 0]
        return np.array([a1, a2, a3], dtype=np.float64).T
    if abs(ibrav) == 3:
        t = a / 2.0
        a1, a2, a3 = np.full(3, t), np.full(3, t), np.full(3, t)
        if ibrav < 0:
            a1[0], a2[1], a3[2] = -a1[0], -a2[1], -a3[2]
        else:
            a2[0], a3[0] = -a2[0], -a3[0]
            a3[1] = -a3[1]
        return np.array([a1, a2, a3]).T
    raise ValueError("ibrav %d not supported by this reader" % ibrav)


def read_qe_fc(path):
    """Parse a QE ``.fc`` file.

    Returns (crystal, fc, dielectric (3,3), born (nat,3,3)) with fc in the
    reference layout ``forceConstants(ic, jc, r1, r2, r3, iat, jat)``.
    """
    with open(path) as f:
        lines = f.read().splitlines()
    pos = 0

    def nxt():
        nonlocal pos
        line = lines[pos]
        pos += 1
        return line

    head = nxt().split()
    ntyp, nat, ibrav = int(head[0]), int(head[1]), int(head[2])
    celldm = np.array([float(x) for x in head[3:9]])
    cell_in = np.zeros((3, 3))
    if ibrav == 0:
        for i in range(3):
            cell_in[:, i] = [float(x) for x in nxt().split()[:3]]
    cell = _qe_lattice(ibrav, celldm, cell_in)
    masses = np.zeros(ntyp)
    for i in range(ntyp):
        parts = nxt().split("'")
        masses[i] = float(parts[2])
    positions = np.zeros((nat, 3))
    species = np.zeros(nat, dtype=np.int32)
    for i in range(nat):
        p = nxt().split()
        species[i] = int(p[1]) - 1
        positions[i] = celldm[0] * np.array([float(x) for x in p[2:5]])
    has_diel = nxt().strip() == "T"
    diel = np.zeros((3, 3))
    born = np.zeros((nat, 3, 3))
    if has_diel:
        for i in range(3):
            diel[i] = [float(x) for x in nxt().split()[:3]]
        for a in range(nat):
            nxt()
            for i in range(3):
                born[a, i] = [float(x) for x in nxt().split()[:3]]
    grid = [int(x) for x in nxt().split()[:3]]
    fc = np.zeros((3, 3, grid[0], grid[1], grid[2], nat, nat))
    for ic in range(3):
        for jc in range(3):
            for ia in range(nat):
                for ja in range(nat):
                    nxt()
                    for r3 in range(grid[2]):
                        for r2 in range(grid[1]):
                            for r1 in range(grid[0]):
                                fc[ic, jc, r1, r2, r3, ia, ja] = float(nxt().split()[3])
    return Crystal(cell, positions, species, masses), fc, diel, born


def read_shengbte_fc3(path, crystal):
    """Parse ShengBTE ``FORCE_CONSTANTS_3RD`` into the dense D3 layout.

    The reference allocates FC3 as (nb,nb,nb,nr2,nr3) but writes and reads it
    as (...,ir3,ir2) (ifc3_parser.cpp:797,822; interaction_3ph.cpp:53-62);
    the two agree only when nr2 == nr3, which is checked here.
    """
    with open(path) as f:
        toks = f.read().split("\n")
    it = iter(toks)
    ntrip = int(next(it).strip())
    conv = C.distanceBohrToAng ** 3 / C.energyRyToEv
    nat = crystal.num_atoms
    nb = 3 * nat
    cellpos = np.zeros((ntrip, 2, 3))
    atoms = np.zeros((ntrip, 3), dtype=np.int64)
    blocks = np.zeros((ntrip, 3, 3, 3))
    for t in range(ntrip):
        next(it)
        next(it)
        cellpos[t, 0] = [float(x) / C.distanceBohrToAng for x in next(it).split()]
        cellpos[t, 1] = [float(x) / C.distanceBohrToAng for x in next(it).split()]
        atoms[t] = [int(x) - 1 for x in next(it).split()]
        for a in range(3):
            for b in range(3):
                for c in range(3):
                    p = next(it).split()
                    blocks[t, a, b, c] = float(p[3]) * conv
    R2, R3 = [], []
    for t in range(ntrip):
        p2, p3 = tuple(cellpos[t, 0]), tuple(cellpos[t, 1])
        if p2 not in R2:
            R2.append(p2)
        if p3 not in R3:
            R3.append(p3)
    nr2, nr3 = len(R2), len(R3)
    if nr2 != nr3:
        raise ValueError("nr2 != nr3: the reference's FC3 layout is ill-defined")
    i2 = {p: i for i, p in enumerate(R2)}
    i3 = {p: i for i, p in enumerate(R3)}
    D3 = np.zeros((nb, nb, nb, nr3, nr2))
    for t in range(ntrip):
        a1, a2, a3 = atoms[t]
        r2 = i2[tuple(cellpos[t, 0])]
        r3 = i3[tuple(cellpos[t, 1])]
        D3[3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3, 3 * a3:3 * a3 + 3, r3, r2] = blocks[t]
    w = np.ones((nr2, nat, nat))
    return FC3(D3, np.array(R2), np.array(R3), w, w.copy(), ntrip)


def read_shengbte_golden(path, nb):
    """Golden |V+|^2, |V-|^2 file: lines ``i j k Vp Vm`` (k fastest)."""
    data = np.loadtxt(path)
    vp = data[:, 3].reshape(nb, nb, nb)
    vm = data[:, 4].reshape(nb, nb, nb)
    return vp, vm
