"""Import the read-only reference (torch-admp) for fixture generation only.

The reference needs ``ase.units``, ``torchopt`` and a generated
``torch_admp._version``, none of which exist offline; these stand-ins cover
exactly what the reference uses of them (eV/Angstrom units, a forward-only
``custom_root`` decorator).  Used by ``make_golden.py`` in this directory,
never at test time and never on the GPU host.

The checkout is named by the environment variable ``TORCH_ADMP_REFERENCE``
(the directory that holds ``src/torch_admp`` and ``tests/data``).
"""
import os
import sys
import types


def reference_root() -> str:
    root = os.environ.get("TORCH_ADMP_REFERENCE")
    if not root or not os.path.isdir(os.path.join(root, "src", "torch_admp")):
        raise SystemExit("set TORCH_ADMP_REFERENCE to a torch-admp checkout (the directory holding "
                         "src/torch_admp and tests/data), e.g. TORCH_ADMP_REFERENCE=../torch-admp")
    return root


def import_reference():
    os.environ["DEVICE"] = "cpu"
    import scipy.constants as C

    ase = types.ModuleType("ase")
    units = types.ModuleType("ase.units")
    units.Ang, units.nm, units.eV = 1.0, 10.0, 1.0
    units.J = 1.0 / C.e
    units.kJ = 1000.0 * units.J
    units.mol = C.N_A
    ase.units = units
    to = types.ModuleType("torchopt")
    diff = types.ModuleType("torchopt.diff")
    imp = types.ModuleType("torchopt.diff.implicit")
    imp.custom_root = lambda *a, **k: (lambda f: f)
    diff.implicit = imp
    to.diff = diff
    ls = types.ModuleType("torchopt.linear_solve")
    ls.solve_normal_cg = lambda **k: None
    to.linear_solve = ls
    ver = types.ModuleType("torch_admp._version")
    ver.__version__ = "1.1.5"
    sys.modules.update({
        "ase": ase, "ase.units": units, "torchopt": to, "torchopt.diff": diff,
        "torchopt.diff.implicit": imp, "torchopt.linear_solve": ls, "torch_admp._version": ver,
    })
    ref_src = os.path.join(reference_root(), "src")
    if ref_src not in sys.path:
        sys.path.insert(0, ref_src)
    import torch_admp  # noqa: F401
    return torch_admp
