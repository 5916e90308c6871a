"""Generate the golden fixtures of the reference's 3-phonon vertex tests.

Reads the reference's own test inputs and ShengBTE golden couplings
(test/data/444_silicon.fc, test/data/FORCE_CONSTANTS_3RD,
test/data/reference3Ph000, test/data/reference3Ph210 of mir-group/phoebe)
with this package's readers and stores them, parsed, in ``si_3ph.npz`` so the
tests can run where the reference tree is absent.  The assertions that use
them follow test/interaction3phTest.cpp:9-127 (Gamma,Gamma,Gamma; sum over the
optical manifold) and :129-350 (q-indices 10, 210, 200 on a 20^3 mesh; sum
over b1 < 2 after symmetrizeCoupling).

Usage:  python tests/golden/make_golden.py /path/to/reference
(the root of a mir-group/phoebe checkout; required)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from phoebe_b200 import readers  # noqa: E402


def main(ref):
    data = os.path.join(ref, "test", "data")
    cr, fc, diel, born = readers.read_qe_fc(os.path.join(data, "444_silicon.fc"))
    fc3 = readers.read_shengbte_fc3(os.path.join(data, "FORCE_CONSTANTS_3RD"), cr)
    nb = cr.num_bands
    vp0, vm0 = readers.read_shengbte_golden(os.path.join(data, "reference3Ph000"), nb)
    vp2, vm2 = readers.read_shengbte_golden(os.path.join(data, "reference3Ph210"), nb)
    out = os.path.join(HERE, "si_3ph.npz")
    np.savez_compressed(
        out,
        cell=cr.direct_cell, positions=cr.positions, species=cr.species,
        species_masses=cr.species_masses, fc2=fc, dielectric=diel, born=born,
        D3=fc3.D3, R2=fc3.R2, R3=fc3.R3, w2=fc3.w2, w3=fc3.w3, num_triplets=fc3.num_pairs,
        golden000_plus=vp0, golden000_mins=vm0, golden210_plus=vp2, golden210_mins=vm2,
        mesh210=np.array([20, 20, 20]), iq210=np.array([10, 210, 200]))
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
