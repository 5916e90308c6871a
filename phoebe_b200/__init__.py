"""B200-native (sm_100a) scattering-rate path of mir-group/phoebe.

The compute runs in ``libphx.so`` (hand-written CUDA + C ABI, include/phx_abi.h);
``phoebe_b200.core`` mirrors the reference's classes over that ABI.
"""
from . import constants, lattice, synth, readers  # noqa: F401


def __getattr__(name):
    # GPU-facing classes are imported lazily so that host-only tools
    # (generators, readers) work without the CUDA library.
    if name in ("Context", "PhononH0", "BandStructure", "Interaction3Ph", "PhScatteringMatrix",
                "ws_reorder"):
        from . import core
        return getattr(core, name)
    raise AttributeError(name)
