"""Constant-potential electrodes at the stated size of the benchmark
configuration: two fcc(111) slabs of 1,152 atoms each at 1 V and 0 V
(Gaussian width 0.5 A, total electrode charge 0), 3,000 +-1 ions in a 40 A
gap, 64 x 64 x 160 mesh, slab correction along z, rc 6 A.  Checked against
the reference's own infer(method="lbfgs") on the same system
(tests/golden/electrode_cfg3.npz; the oracle is pinned to it in
test_oracle.py)."""
import numpy as np
import pytest
import torch

from conftest import golden
from _gpu_helpers import T, rel

pytestmark = pytest.mark.gpu


def _run(cuda, dtype, eps, method="lbfgs"):
    from admp_b200 import synthetic
    from admp_b200.electrode import LAMMPSElectrodeConstraint, PolarizableElectrode, infer, setup_from_lammps
    from admp_b200.nblist import TorchNeighborList
    d = golden("electrode_cfg3")
    pos_np, box_np, q_np, top, bot = synthetic.electrode_system(1024)
    assert np.array_equal(pos_np, d["pos"])
    rc = float(d["rcut"])
    calc = PolarizableElectrode(rcut=rc, ethresh=float(d["ethresh"]), kmesh=d["kmesh"].tolist(), slab_corr=True,
                                eps=eps, ls_eps=eps, max_iter=1000)
    pos = T(pos_np, cuda, dtype, grad=True)
    box = T(box_np, cuda, dtype)
    charges = T(q_np, cuda, dtype)
    nb = TorchNeighborList(rc)
    pairs = nb(pos, box)
    cons = [LAMMPSElectrodeConstraint(indices=np.arange(int(a), int(z)), value=float(v), mode="conp",
                                      eta=float(d["lammps_eta"])) for a, z, v, _ in d["cons"]]
    data = setup_from_lammps(len(q_np), cons, True, device=cuda, dtype=dtype)
    E, F, q = infer(calc, pos, box, charges, pairs, nb.get_ds(), nb.get_buffer_scales(), *data, method=method)
    torch.cuda.synchronize()
    mask = data[0].cpu().numpy()
    return d, float(E), F.detach().double().cpu().numpy(), q.detach().double().cpu().numpy(), mask, calc


def test_electrode_cfg3_fp64_matches_reference(cuda):
    d, E, F, q, mask, calc = _run(cuda, torch.float64, 1e-10)
    assert calc.submodels["coulomb"]._kmesh.tolist() == [64, 64, 160]
    assert abs(E - float(d["E"])) / abs(float(d["E"])) < 1e-8
    assert rel(F, d["forces"]) < 1e-6
    # the reference's LBFGS stops at ||P grad||/N < 1e-8, which leaves ~5e-7 e in its charges
    assert np.abs(q - d["q_ref"]).max() / np.abs(d["q_ref"]).max() < 2e-6
    assert abs(q[mask].sum()) < 1e-9
    assert np.array_equal(q[~mask], d["q_in"][~mask])


def test_electrode_cfg3_fp32_within_stated_error(cuda):
    """FP32 bulk arithmetic (FP64 solve reductions): max relative force error
    1e-4 and max charge error 1e-5 e against the FP64 reference."""
    d, E, F, q, mask, calc = _run(cuda, torch.float32, 1e-7)
    assert rel(F, d["forces"]) < 1e-4
    assert np.abs(q - d["q_ref"]).max() < 1e-5
    assert abs(E - float(d["E"])) / abs(float(d["E"])) < 1e-5


def test_electrode_cfg3_dense_kkt_matches_reference(cuda):
    """method="matinv": the 2,304 x 2,304 electrode Hessian from batched
    Hessian-vector products (64 unit vectors per call) and the dense KKT solve
    give the reference's charges and forces as well."""
    d, E, F, q, mask, calc = _run(cuda, torch.float64, 1e-10, method="matinv")
    assert abs(E - float(d["E"])) / abs(float(d["E"])) < 1e-8
    assert rel(F, d["forces"]) < 1e-6
    assert np.abs(q - d["q_ref"]).max() / np.abs(d["q_ref"]).max() < 2e-6
    assert abs(q[mask].sum()) < 1e-9
