import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and libphx.so")


@pytest.fixture(scope="session")
def si_golden():
    """Reference fixtures of test/interaction3phTest.cpp, parsed (see tests/golden/make_golden.py)."""
    from phoebe_b200.lattice import Crystal
    from phoebe_b200.synth import FC3
    z = np.load(os.path.join(GOLDEN, "si_3ph.npz"))
    cr = Crystal(z["cell"], z["positions"], z["species"], z["species_masses"])
    fc3 = FC3(z["D3"], z["R2"], z["R3"], z["w2"], z["w3"], int(z["num_triplets"]))
    return {"crystal": cr, "fc2": z["fc2"], "fc3": fc3, "z": z}


@pytest.fixture(scope="session")
def ctx():
    from phoebe_b200.core import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def diamond():
    """Diamond cell, spring FC2 and the 400-pair FC3 of the benchmark workloads."""
    from phoebe_b200 import synth
    cr = synth.diamond_crystal()
    return {"crystal": cr, "fc2": synth.diamond_fc2(cr),
            "fc3": synth.random_fc3(cr, 400, synth.SEED_BASE)}
