"""PME energy / forces / box gradient / dE/dds / dE/dq on the B200 against the
golden vectors produced by the reference (FP64: 1e-6 relative or better;
FP32: 1e-4 relative force error, the bar of the FP32 bulk path)."""
import numpy as np
import pytest
import torch

from conftest import golden
from _gpu_helpers import T, rel

pytestmark = pytest.mark.gpu

PME_CASES = ["pme_small", "pme_cfg1", "pme_triclinic", "pme_kspace", "pme_slab"]


def module_for(d):
    from admp_b200.pme import CoulombForceModule
    km = None if np.all(d["kmesh_arg"] < 0) else d["kmesh_arg"].tolist()
    sp = None if np.all(d["spacing_arg"] < 0) else float(d["spacing_arg"])
    kappa = float(d["kappa"]) if sp is not None else None
    return CoulombForceModule(rcut=float(d["rcut"]), ethresh=float(d["ethresh"]), kmesh=km, spacing=sp, kappa=kappa,
                              rspace=bool(d["rspace"]), kspace=bool(d["kspace"]), slab_corr=bool(d["slab"]),
                              slab_axis=int(d["axis"]))


def run_case(d, dev, dtype=torch.float64):
    from admp_b200.nblist import TorchNeighborList
    pos = T(d["pos"], dev, dtype, grad=True)
    box = T(d["box"], dev, dtype, grad=True)
    q = T(d["q"], dev, dtype)
    nb = TorchNeighborList(float(d["rcut"]))
    pairs = nb(pos, box)
    m = module_for(d)
    E = m(pos, box, pairs, nb.get_ds(), nb.get_buffer_scales(), {"charge": q})
    gp, gb = torch.autograd.grad(E.sum(), [pos, box])
    return m, pairs, E, -gp, gb


@pytest.mark.parametrize("name", PME_CASES)
def test_pme_fp64_matches_reference(cuda, name):
    d = golden(name)
    m, pairs, E, F, gb = run_case(d, cuda)
    assert pairs.shape[0] == int(d["n_pairs"])
    assert m._kmesh.tolist() == d["kmesh"].tolist()
    assert rel(E, d["E"]) < 1e-9
    assert rel(F, d["forces"]) < 1e-8
    assert rel(gb, d["box_grad"]) < 1e-8
    if bool(d["rspace"]):
        assert rel(m.real_energy, d["E_real"]) < 1e-10
    if bool(d["kspace"]):
        assert rel(m.reciprocal_energy, d["E_recip"]) < 1e-10
        assert rel(m.self_energy, d["E_self"]) < 1e-12
    if bool(d["slab"]):
        assert rel(m.slab_corr_energy, d["E_slab"]) < 1e-10


@pytest.mark.parametrize("name", ["pme_small", "pme_triclinic", "pme_slab"])
def test_pme_grad_wrt_caller_ds_and_q(cuda, name):
    """Drop-in contract: gradients flow to the caller's ds and to the charges."""
    d = golden(name)
    m = module_for(d)
    pos = T(d["pos"], cuda)
    ds = T(d["ds"], cuda, grad=True)
    q = T(d["q"], cuda, grad=True)
    pairs = torch.tensor(d["pairs"], device=cuda)
    bs = torch.tensor(d["bs"], device=cuda)
    E = m(pos, T(d["box"], cuda), pairs, ds, bs, {"charge": q})
    gds, gq = torch.autograd.grad(E.sum(), [ds, q])
    assert rel(E, d["E"]) < 1e-9
    assert rel(gds, d["dE_dds"]) < 1e-9
    assert rel(gq, d["dE_dq"]) < 1e-9


def test_pme_fp32_force_error(cuda):
    d = golden("pme_cfg1")
    _, _, E, F, gb = run_case(d, cuda, torch.float32)
    ref = d["forces"]
    err = np.abs(F.detach().cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 1e-4, err
    assert rel(E, d["E"]) < 1e-5


def test_pme_multiframe_batch(cuda):
    """nframes > 1 with different boxes and meshes goes through one batched launch."""
    from admp_b200.pme import CoulombForceModule
    from oracle import admp_oracle as O
    rng = np.random.default_rng(5)
    nf, n = 3, 120
    pos = np.stack([rng.random((n, 3)) * 14.0 for _ in range(nf)])
    boxes = np.stack([np.diag([14.0, 14.0, 14.0]), np.diag([14.5, 14.0, 15.0]), np.diag([14.0, 16.0, 14.0])])
    q = rng.uniform(-1, 1, (nf, n))
    pairs = [O.nblist_pbc(pos[f], boxes[f], 5.0) for f in range(nf)]
    P = max(len(p) for p in pairs)
    pp = np.zeros((nf, P, 2), np.int64)
    bs = np.zeros((nf, P))
    ds = np.ones((nf, P))
    for f in range(nf):
        k = len(pairs[f])
        pp[f, :k] = pairs[f]
        bs[f, :k] = O.pair_buffer_scales(pairs[f])
        ds[f, :k] = O.pairs_ds(pos[f], pairs[f], boxes[f])
    m = CoulombForceModule(rcut=5.0, ethresh=1e-5)
    E = m(T(pos, cuda), T(boxes, cuda), torch.tensor(pp, device=cuda), T(ds, cuda), T(bs, cuda),
          {"charge": T(q, cuda)})
    for f in range(nf):
        o = O.coulomb(pos[f], boxes[f], pp[f], ds[f], bs[f], q[f], rcut=5.0, ethresh=1e-5)
        assert rel(E[f], o["E"]) < 1e-9


def test_obc_lammps(cuda):
    from admp_b200.nblist import TorchNeighborList
    from admp_b200.pme import CoulombForceModule
    d = golden("obc")
    pos = T(d["pos"], cuda, grad=True)
    nb = TorchNeighborList(4.0)
    pairs = nb(pos, None)
    assert pairs.shape[0] == d["pairs"].shape[0]
    m = CoulombForceModule(rcut=5.0, ethresh=1e-5)
    E = m(pos, None, pairs, nb.get_ds(), nb.get_buffer_scales(), {"charge": T(d["q"], cuda)})
    F = -torch.autograd.grad(E.sum(), pos)[0]
    np.testing.assert_allclose(E.detach().cpu().numpy(), [float(d["E_lammps"])], atol=1e-6, rtol=1e-6)
    np.testing.assert_allclose(F.cpu().numpy(), d["F_lammps"], atol=1e-6, rtol=1e-6)
    assert rel(F, d["forces"]) < 1e-10


def test_slab_corr_lammps(cuda):
    from admp_b200.nblist import TorchNeighborList
    from admp_b200.pme import CoulombForceModule
    d = golden("slab_lammps")
    pos = T(d["pos"], cuda, grad=True)
    box = T(d["box"], cuda)
    nb = TorchNeighborList(4.0)
    pairs = nb(pos, box)
    m = CoulombForceModule(rcut=4.0, ethresh=1e-3, kspace=False, rspace=False, slab_corr=True, slab_axis=2)
    E = m(pos, box, pairs, nb.get_ds(), nb.get_buffer_scales(), {"charge": T(d["q"], cuda)})
    F = -torch.autograd.grad(E.sum(), pos)[0]
    np.testing.assert_allclose(E.detach().cpu().numpy(), [float(d["E_lammps"])], atol=1e-6, rtol=1e-6)
    np.testing.assert_allclose(F.cpu().numpy(), d["F_lammps"], atol=1e-6, rtol=1e-6)


def test_damping_and_site(cuda):
    from admp_b200.qeq import GaussianDampingForceModule, SiteForceModule
    d = golden("damping_site")
    pos = T(d["pos"], cuda)
    box = T(d["box"], cuda)
    ds = T(d["ds"], cuda, grad=True)
    q = T(d["q"], cuda, grad=True)
    eta = T(d["eta"], cuda, grad=True)
    chi = T(d["chi"], cuda, grad=True)
    hd = T(d["hardness"], cuda, grad=True)
    pairs = torch.tensor(d["pairs"], device=cuda)
    bs = torch.tensor(d["bs"], device=cuda)
    Ed = GaussianDampingForceModule()(pos, box, pairs, ds, bs, {"charge": q, "eta": eta})
    gds, gq, ge = torch.autograd.grad(Ed.sum(), [ds, q, eta])
    assert rel(Ed, d["E_damp"]) < 1e-12
    assert rel(gq, d["dq_damp"]) < 1e-12
    ok = np.isfinite(d["deta_damp"])
    assert rel(ge.cpu().numpy()[ok], d["deta_damp"][ok]) < 1e-10
    Es = SiteForceModule()(pos, box, pairs, ds, bs, {"charge": q, "chi": chi, "hardness": hd})
    gsq, gc, gh = torch.autograd.grad(Es.sum(), [q, chi, hd])
    assert rel(Es, d["E_site"]) < 1e-13
    assert rel(gsq, d["dq_site"]) < 1e-13 and rel(gc, d["dchi"]) < 1e-13 and rel(gh, d["dhard"]) < 1e-13


def test_bad_pair_index_raises(cuda):
    from admp_b200.pme import CoulombForceModule
    m = CoulombForceModule(rcut=5.0, ethresh=1e-5, kmesh=8)
    pos = torch.rand(10, 3, dtype=torch.float64, device=cuda) * 10
    pairs = torch.tensor([[0, 1], [1, 12]], device=cuda)
    with pytest.raises(IndexError):
        m(pos, torch.eye(3, dtype=torch.float64, device=cuda) * 10, pairs,
          torch.ones(2, dtype=torch.float64, device=cuda), torch.ones(2, dtype=torch.float64, device=cuda),
          {"charge": torch.zeros(10, dtype=torch.float64, device=cuda)})


@pytest.mark.parametrize("name", ["pme_small", "pme_triclinic", "pme_slab"])
def test_autograd_matches_finite_differences(cuda, name):
    """dE/dpositions and dE/dbox from the hand-written gradients against central
    finite differences of the energy (the reference's test_autodiff.py check,
    step 1e-5), with ds recomputed from the displaced positions / box and the
    pair list held fixed."""
    from admp_b200.nblist import TorchNeighborList
    d = golden(name)
    m = module_for(d)
    pos0 = T(d["pos"], cuda)
    box0 = T(d["box"], cuda)
    q = T(d["q"], cuda)
    pairs = TorchNeighborList(float(d["rcut"]))(pos0, box0)
    bs = (pairs[:, 0] < pairs[:, 1]).to(torch.float64)

    def energy(pos, box):
        ds = TorchNeighborList.pairs_ds(pos, pairs, box)
        return m(pos, box, pairs, ds, bs, {"charge": q}).sum()

    pos = pos0.clone().requires_grad_(True)
    box = box0.clone().requires_grad_(True)
    gp, gb = torch.autograd.grad(energy(pos, box), [pos, box])
    rng = np.random.default_rng(7)
    h = 1e-5
    with torch.no_grad():
        for k in rng.choice(pos0.numel(), 6, replace=False):
            e = torch.zeros_like(pos0).reshape(-1)
            e[k] = h
            e = e.reshape(pos0.shape)
            fd = (energy(pos0 + e, box0) - energy(pos0 - e, box0)).item() / (2 * h)
            assert fd == pytest.approx(gp.reshape(-1)[k].item(), rel=1e-5, abs=1e-6)
        for k in range(9):
            e = torch.zeros(9, dtype=torch.float64, device=cuda)
            e[k] = h
            e = e.reshape(3, 3)
            fd = (energy(pos0, box0 + e) - energy(pos0, box0 - e)).item() / (2 * h)
            assert fd == pytest.approx(gb.reshape(-1)[k].item(), rel=1e-5, abs=1e-6)
