"""CoulombForceModule construction and setup_ewald_parameters (host-side, CPU).

The cases follow the reference's own tests (test_pme_numerical.py:404-507):
openmm and gromacs rules, no box, invalid method, gromacs without spacing,
non-orthogonal box, and the constructor's ValueErrors.  The returned kappa
and mesh sizes are compared with values the reference computed
(tests/golden/ewald_params.npz, made by make_golden.py).
"""
import math

import numpy as np
import pytest
import torch

from conftest import golden


def _setup():
    from admp_b200.pme import setup_ewald_parameters
    return setup_ewald_parameters


def test_setup_ewald_parameters_matches_reference_values():
    f = _setup()
    d = golden("ewald_params")
    rows = d["rows"]
    assert rows.shape[0] > 100
    for meth, rcut, thr, sp, lx, ly, lz, kappa, kx, ky, kz in rows:
        box = np.diag([lx, ly, lz])
        if meth == 0:
            k, *km = f(rcut, box, thr, method="openmm")
        else:
            k, *km = f(rcut, box, thr, spacing=sp, method="gromacs")
        assert k == pytest.approx(kappa, rel=1e-15, abs=0.0)
        assert [int(x) for x in km] == [int(kx), int(ky), int(kz)]


def test_setup_ewald_parameters_openmm_and_gromacs_are_reasonable():
    f = _setup()
    box = np.diag([10.0, 10.0, 10.0])
    kappa, kx, ky, kz = f(rcut=5.0, box=box, threshold=1e-5, method="openmm")
    assert kappa > 0 and min(kx, ky, kz) >= 1
    assert kappa == pytest.approx(math.sqrt(-math.log(2e-5)) / 5.0)
    kappa, kx, ky, kz = f(rcut=5.0, box=box, threshold=1e-5, spacing=1.0, method="gromacs")
    assert kappa > 0 and (kx, ky, kz) == (10, 10, 10)
    # the bisection stops where erfc(kappa rc) meets the threshold
    from scipy import special
    assert special.erfc(kappa * 5.0) == pytest.approx(1e-5, rel=1e-6)


def test_setup_ewald_parameters_accepts_a_tensor_box():
    f = _setup()
    box = torch.diag(torch.tensor([12.0, 13.0, 14.0], dtype=torch.float64))
    assert f(6.0, box, 5e-4) == f(6.0, box.numpy(), 5e-4)


def test_setup_ewald_parameters_no_box():
    assert _setup()(rcut=5.0, box=None) == (0.1, 1, 1, 1)


def test_setup_ewald_parameters_invalid_method():
    with pytest.raises(ValueError) as e:
        _setup()(rcut=5.0, box=np.diag([10.0, 10.0, 10.0]), threshold=1e-5, method="invalid")
    assert "Invalid method: invalid" in str(e.value)
    assert "Valid methods: 'openmm', 'gromacs'" in str(e.value)


def test_setup_ewald_parameters_gromacs_needs_spacing():
    with pytest.raises(AssertionError):
        _setup()(rcut=5.0, box=np.diag([10.0, 10.0, 10.0]), threshold=1e-5, method="gromacs")


def test_setup_ewald_parameters_rejects_non_orthogonal_box():
    box = np.array([[10.0, 1.0, 0.0], [0.0, 10.0, 0.0], [0.0, 0.0, 10.0]])
    with pytest.raises(AssertionError, match="Only orthogonal box"):
        _setup()(rcut=5.0, box=box, threshold=1e-5, method="openmm")


@pytest.mark.parametrize("rcut", [-1.0, 0.0])
def test_setup_ewald_parameters_invalid_rcut(rcut):
    with pytest.raises(ValueError, match=f"rcut must be positive, got {rcut}"):
        _setup()(rcut=rcut, box=np.diag([10.0, 10.0, 10.0]))


@pytest.mark.parametrize("kw,msg", [
    (dict(rcut=-1.0), "rcut must be positive, got -1.0"),
    (dict(rcut=5.0, ethresh=-1.0), "ethresh must be positive, got -1.0"),
    (dict(rcut=5.0, slab_axis=3), "slab_axis must be 0/1/2, got 3"),
    (dict(rcut=5.0, kappa=0.0), "kappa must be positive, got 0.0"),
    (dict(rcut=5.0, kmesh=[10, 0, 10]), "kmesh values must be positive, got kmesh[1] = 0"),
    (dict(rcut=5.0, spacing=[1.0, 1.0, -0.5]), "spacing values must be positive, got spacing[2] = -0.5"),
])
def test_coulomb_module_constructor_validation(kw, msg):
    from admp_b200.pme import CoulombForceModule
    with pytest.raises(ValueError) as e:
        CoulombForceModule(**kw)
    assert msg in str(e.value)


def test_coulomb_module_constructor_settings():
    from admp_b200.pme import CoulombForceModule
    m = CoulombForceModule(rcut=6.0, ethresh=5e-4)
    assert m.kappa == pytest.approx(0.438043, abs=1e-6)   # sqrt(-ln(2 ethresh)) / rcut
    m = CoulombForceModule(rcut=6.0, kspace=False)
    assert m.kappa == 0.0
    m = CoulombForceModule(rcut=6.0, kmesh=32, spacing=0.5)
    assert m.kmesh == [32, 32, 32] and m.spacing == [0.5, 0.5, 0.5]
    m = CoulombForceModule(rcut=6.0, kappa=0.3)
    assert m.kappa == 0.3
    assert m.get_rcut() == 6.0 and m.get_sel() is None
    # automatic mesh per frame: ceil(2 kappa L / (3 ethresh^0.2)) (pme.py:390-392)
    m = CoulombForceModule(rcut=6.0, ethresh=5e-4)
    box = torch.diag(torch.tensor([25.0, 31.0, 58.5], dtype=torch.float64)).unsqueeze(0)
    k = m.kappa
    assert m.kmesh_for(box) == [[math.ceil(2 * k * L / (3 * 5e-4 ** 0.2)) for L in (25.0, 31.0, 58.5)]]
    m = CoulombForceModule(rcut=6.0, spacing=1.3)
    assert m.kmesh_for(box) == [[math.ceil(L / 1.3) for L in (25.0, 31.0, 58.5)]]
