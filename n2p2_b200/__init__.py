"""n2p2_b200: the short-range (2G) HDNNP energy/force path of n2p2 on B200.

Host API mirroring nnp::Mode / nnp::Prediction over the C ABI of
include/n2p2_b200.h; all evaluation runs in libn2p2b200.so (sm_100a).
"""
from .structure import Structure, read_structures, write_structures  # noqa: F401

__all__ = ["Structure", "read_structures", "write_structures", "Mode", "Prediction", "Batch", "Trainer",
           "InterfaceLammps"]


def __getattr__(name):
    # The GPU classes load the shared library on first use.
    if name in ("Mode", "Prediction", "Batch", "Trainer"):
        from . import mode
        return getattr(mode, name)
    if name == "InterfaceLammps":
        from . import lammps
        return lammps.InterfaceLammps
    raise AttributeError(name)
