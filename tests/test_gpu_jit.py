"""Scripted modules give the energies and charge gradients of the eager ones
(the reference's test_jit.py: 100 atoms in a 10 Angstrom box, rc 4,
ethresh 1e-5; open and periodic boundaries, slab corrections along x / y / z,
Gaussian damping, site energy, QEq) and match the oracle."""
import io

import numpy as np
import pytest
import torch

from oracle import admp_oracle as O

pytestmark = pytest.mark.gpu

RCUT, ETHRESH, L_BOX, N = 4.0, 1e-5, 10.0, 100


def _inputs(dev, periodic):
    from admp_b200.nblist import TorchNeighborList
    rng = np.random.default_rng(1024)
    pos_np = rng.random((N, 3)) * L_BOX
    q_np = rng.uniform(-1.0, 1.0, N)
    q_np -= q_np.mean()
    pos = torch.tensor(pos_np, device=dev, requires_grad=True)
    box = torch.tensor(np.diag([L_BOX] * 3), device=dev) if periodic else None
    q = torch.tensor(q_np, device=dev, requires_grad=True)
    nb = TorchNeighborList(cutoff=RCUT)
    pairs = nb(pos, box)
    params = {"charge": q, "eta": torch.ones(N, device=dev, dtype=torch.float64),
              "chi": torch.ones(N, device=dev, dtype=torch.float64),
              "hardness": torch.zeros(N, device=dev, dtype=torch.float64)}
    return pos, box, pairs, nb.get_ds(), nb.get_buffer_scales(), params, pos_np, q_np


def _cases():
    from admp_b200.pme import CoulombForceModule
    from admp_b200.qeq import GaussianDampingForceModule, QEqForceModule, SiteForceModule
    return {
        "obc": (False, lambda: CoulombForceModule(rcut=RCUT, ethresh=ETHRESH)),
        "pbc": (True, lambda: CoulombForceModule(rcut=RCUT, ethresh=ETHRESH)),
        "slab_x": (True, lambda: CoulombForceModule(rcut=RCUT, ethresh=ETHRESH, slab_corr=True, slab_axis=0)),
        "slab_y": (True, lambda: CoulombForceModule(rcut=RCUT, ethresh=ETHRESH, slab_corr=True, slab_axis=1)),
        "slab_z": (True, lambda: CoulombForceModule(rcut=RCUT, ethresh=ETHRESH, slab_corr=True, slab_axis=2)),
        "damping": (True, lambda: GaussianDampingForceModule()),
        "site": (True, lambda: SiteForceModule()),
        "qeq": (True, lambda: QEqForceModule(rcut=RCUT, ethresh=ETHRESH)),
    }


@pytest.mark.parametrize("case", list(_cases()))
def test_scripted_equals_eager(cuda, case):
    periodic, make = _cases()[case]
    pos, box, pairs, ds, bs, params, _, _ = _inputs(cuda, periodic)
    m = make()
    sm = torch.jit.script(make())
    buf = io.BytesIO()
    torch.jit.save(sm, buf)
    buf.seek(0)
    lm = torch.jit.load(buf)
    outs = []
    for mod in (m, sm, lm):
        E = mod(pos, box, pairs, ds, bs, params)
        gq, gr = torch.autograd.grad(E.sum(), [params["charge"], pos], allow_unused=True, retain_graph=True)
        outs.append((E.item(), gq, gr))
    for E, gq, gr in outs[1:]:
        assert E == pytest.approx(outs[0][0], rel=1e-12, abs=1e-12)
        assert torch.allclose(gq, outs[0][1], rtol=1e-12, atol=1e-12)
        if gr is not None:
            assert torch.allclose(gr, outs[0][2], rtol=1e-12, atol=1e-12)


def test_scripted_pbc_matches_oracle(cuda):
    from admp_b200.pme import CoulombForceModule
    pos, box, pairs, ds, bs, params, pos_np, q_np = _inputs(cuda, True)
    sm = torch.jit.script(CoulombForceModule(rcut=RCUT, ethresh=ETHRESH))
    E = sm(pos, box, pairs, ds, bs, params)
    F = -torch.autograd.grad(E.sum(), pos)[0]
    box_np = np.diag([L_BOX] * 3)
    pr = O.nblist_pbc(pos_np, box_np, RCUT)
    ref = O.coulomb_forces(pos_np, box_np, pr, O.pair_buffer_scales(pr), q_np, rcut=RCUT, ethresh=ETHRESH)
    assert abs(E.item() - ref["E"]) / abs(ref["E"]) < 1e-9
    assert np.abs(F.cpu().numpy() - ref["forces"]).max() / np.abs(ref["forces"]).max() < 1e-8
    assert sm._kmesh.tolist() == list(O.auto_kmesh(box_np, O.ewald_kappa(RCUT, ETHRESH), ETHRESH))


def test_scripted_qeq_func_energy_and_optimality(cuda):
    from admp_b200.qeq import QEqForceModule
    from admp_b200.utils import vector_projection_coeff_matrix
    pos, box, pairs, ds, bs, params, _, _ = _inputs(cuda, True)
    m = QEqForceModule(rcut=RCUT, ethresh=ETHRESH)
    sm = torch.jit.script(QEqForceModule(rcut=RCUT, ethresh=ETHRESH))
    args = (params["charge"], pos, box, params["chi"], params["hardness"] + 1.0, params["eta"], pairs, ds, bs)
    assert sm.func_energy(*args).item() == pytest.approx(m.func_energy(*args).item(), rel=1e-12)
    C = torch.ones(1, N, dtype=torch.float64, device=cuda)
    coeff = vector_projection_coeff_matrix(C)
    a = sm.optimality(*args, C, coeff).item()
    b = m.optimality(*args, C, coeff).item()
    assert a == pytest.approx(b, rel=1e-10)
