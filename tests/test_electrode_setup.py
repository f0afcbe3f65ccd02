"""Host-side electrode set-up (electrode.py:203-285 of the reference) on CPU:
masks, widths, shifted chi, constraints and finite-field groups agree with the
oracle, and the reference's refusals raise the same AttributeError (the
CONQ + finite-field case is test_electrode_conq.py's 3D bias fixture)."""
import numpy as np
import pytest
import torch

from oracle import admp_oracle as O


def _cons(spec):
    from admp_b200.electrode import LAMMPSElectrodeConstraint
    return [LAMMPSElectrodeConstraint(indices=np.arange(a, z), value=v, mode=m, eta=1.6, ffield=ff)
            for a, z, v, m, ff in spec]


@pytest.mark.parametrize("spec,symm", [
    ([(0, 108, 20.0, "conp", False), (108, 216, 0.0, "conp", False)], True),
    ([(0, 108, 20.0, "conp", True), (108, 216, 0.0, "conp", True)], False),
    ([(0, 108, -10.0, "conq", False), (108, 216, 10.0, "conq", False)], False),
    ([(0, 216, -10.0, "conq", False)], False),
])
def test_setup_from_lammps_matches_oracle(spec, symm):
    from admp_b200.electrode import setup_from_lammps
    n = 300
    got = setup_from_lammps(n, _cons(spec), symm, device="cpu")
    ref = O.setup_from_lammps(n, [dict(indices=np.arange(a, z), value=v, mode=m, eta=1.6, ffield=ff)
                                  for a, z, v, m, ff in spec], symm)
    for g, r in zip(got, ref):
        if r is None:
            assert g is None
        else:
            np.testing.assert_allclose(g.numpy().astype(float), np.asarray(r, dtype=float), rtol=0, atol=1e-15)


def test_conq_with_finite_field_is_refused():
    from admp_b200.electrode import setup_from_lammps
    with pytest.raises(AttributeError, match="ffield with conq has not been implemented yet"):
        setup_from_lammps(300, _cons([(0, 108, -10.0, "conq", True), (108, 216, 10.0, "conq", True)]), device="cpu")


def test_conq_with_symm_is_refused():
    from admp_b200.electrode import setup_from_lammps
    with pytest.raises(AttributeError, match="symm should be False for conq"):
        setup_from_lammps(300, _cons([(0, 216, 0.0, "conq", False)]), True, device="cpu")


def test_single_finite_field_group_is_refused():
    from admp_b200.electrode import setup_from_lammps
    with pytest.raises(AttributeError, match="number of ffield group should be 0 or 2"):
        setup_from_lammps(300, _cons([(0, 108, 1.0, "conp", True), (108, 216, 0.0, "conp", False)]), device="cpu")
