"""admp_b200: B200-native (sm_100a) electrostatics hot path of torch-admp.

Drop-in modules with the reference's names and signatures:
    from admp_b200.pme import CoulombForceModule, setup_ewald_parameters
    from admp_b200.qeq import QEqForceModule, pgrad_optimize, matinv_optimize, qeq_solve
    from admp_b200.nblist import TorchNeighborList
    from admp_b200.electrode import PolarizableElectrode, infer, setup_from_lammps
All arithmetic runs in libadmp_b200.so (hand-written CUDA kernels); importing
a module does not need a GPU, calling one does.
"""
__version__ = "0.1.0"

from . import _lib  # noqa: F401


def native_library_path() -> str:
    return _lib.LIB_PATH
