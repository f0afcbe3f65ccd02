"""QEq charge solve on the B200 (matrix-free projected CG) against the
reference's matinv / quadratic solutions, Hessian identity and the implicit
adjoint against central finite differences."""
import numpy as np
import pytest
import torch

from conftest import golden
from _gpu_helpers import T, rel

pytestmark = pytest.mark.gpu


def setup(d, dev, kmesh=None, dtype=torch.float64, eps=1e-8, max_iter=500):
    from admp_b200.nblist import TorchNeighborList
    from admp_b200.qeq import QEqForceModule
    m = QEqForceModule(float(d["rcut"]), float(d["ethresh"]), kmesh=kmesh, eps=eps, max_iter=max_iter)
    pos = T(d["pos"], dev, dtype, grad=True)
    box = T(d["box"], dev, dtype)
    pairs = torch.tensor(d["pairs"], device=dev)
    # distances connected to positions, as the reference's nblist returns them
    ds = TorchNeighborList.pairs_ds(pos, pairs, box)
    bs = torch.tensor(d["bs"], device=dev)
    n = pos.shape[0]
    C = torch.ones(1, n, dtype=dtype, device=dev)
    b = torch.zeros(1, dtype=dtype, device=dev)
    return m, pos, box, pairs, ds, bs, T(d["chi"], dev, dtype), T(d["hardness"], dev, dtype), T(d["eta"], dev, dtype), C, b


@pytest.mark.parametrize("name,kmesh", [("qeq_small", None), ("qeq_water_small", 20)])
def test_qeq_cg_matches_reference(cuda, name, kmesh):
    from admp_b200.qeq import pgrad_optimize
    d = golden(name)
    m, pos, box, pairs, ds, bs, chi, hd, eta, C, b = setup(d, cuda, kmesh)
    E, q = pgrad_optimize(m, None, pos, box, chi, hd, eta, pairs, ds, bs, C, b, method="quadratic")
    assert m.converge_iter >= 0
    assert np.abs(q.detach().cpu().numpy() - d["q_matinv"]).max() < 1e-7
    assert rel(E, d["E_matinv"]) < 1e-8
    F = -torch.autograd.grad(E.sum(), pos)[0]
    assert np.abs(F.cpu().numpy() - d["F_matinv"]).max() < 5e-6


def test_qeq_eps_criterion_and_iterations(cuda):
    """Stopping rule ||P grad|| / N < eps as in the reference (eps=1e-6)."""
    from admp_b200.qeq import pgrad_optimize
    from admp_b200.utils import calc_pgrads, vector_projection_coeff_matrix
    d = golden("qeq_water_small")
    m, pos, box, pairs, ds, bs, chi, hd, eta, C, b = setup(d, cuda, 20, eps=1e-6, max_iter=100)
    E, q = pgrad_optimize(m, torch.zeros(pos.shape[0], dtype=torch.float64, device=cuda), pos, box, chi, hd, eta,
                          pairs, ds, bs, C, b, reinit_q=True, method="lbfgs")
    assert 0 <= m.converge_iter <= 100
    pg = calc_pgrads(E, q, C, vector_projection_coeff_matrix(C))
    assert (pg.norm() / q.shape[0]).item() < 1e-6 * 1.01
    assert abs(q.sum().item()) < 1e-10


def test_qeq_matinv_matches_reference(cuda):
    from admp_b200.qeq import matinv_optimize
    d = golden("qeq_water_small")
    m, pos, box, pairs, ds, bs, chi, hd, eta, C, b = setup(d, cuda, 20)
    E, q = matinv_optimize(m, pos, box, chi, hd, eta, pairs, ds, bs, C, b)
    assert np.abs(q.detach().cpu().numpy() - d["q_matinv"]).max() < 1e-10
    assert rel(E, d["E_matinv"]) < 1e-10


def test_hessian_identity(cuda):
    """1/2 q^T H q = E_coulomb + E_damping (reference test_qeq_numerical.py:331-369)."""
    d = golden("qeq_water_small")
    m, pos, box, pairs, ds, bs, chi, hd, eta, C, b = setup(d, cuda, 20)
    zero = torch.zeros_like(chi)
    H = m.calc_hessian(pos, box, chi, zero, eta, pairs, ds, bs)
    rng = np.random.default_rng(0)
    q = T(rng.uniform(-1, 1, pos.shape[0]), cuda)
    e1 = m.submodels["coulomb"](pos, box, pairs, ds, bs, {"charge": q})
    e2 = m.submodels["damping"](pos, box, pairs, ds, bs, {"charge": q, "eta": eta})
    assert rel(0.5 * q @ H @ q, (e1 + e2).sum()) < 1e-10
    assert rel(H, H.T) < 1e-12


def test_qeq_cfg2_water_fp64_and_fp32(cuda):
    """1,000 waters, 48^3 mesh.  FP64 against the reference's charges (which are
    converged to ||P grad|| / N < 1e-7); the FP32 bulk path against FP64 within
    1e-5 e charge and 1e-4 relative force error."""
    from admp_b200.nblist import TorchNeighborList
    from admp_b200.qeq import QEqForceModule, pgrad_optimize
    d = golden("qeq_water_cfg2")
    out = {}
    for dtype in (torch.float64, torch.float32):
        m = QEqForceModule(6.0, 5e-4, kmesh=48, eps=1e-9 if dtype == torch.float64 else 1e-7, max_iter=300)
        pos = T(d["pos"], cuda, dtype, grad=True)
        box = T(d["box"], cuda, dtype)
        nb = TorchNeighborList(6.0)
        pairs = nb(pos, box)
        n = pos.shape[0]
        C = torch.ones(1, n, dtype=dtype, device=cuda)
        E, q = pgrad_optimize(m, None, pos, box, T(d["chi"], cuda, dtype), T(d["hardness"], cuda, dtype),
                              T(d["eta"], cuda, dtype), pairs, nb.get_ds(), nb.get_buffer_scales(), C,
                              torch.zeros(1, dtype=dtype, device=cuda), method="quadratic")
        assert m.converge_iter >= 0
        F = -torch.autograd.grad(E.sum(), pos)[0].double().cpu().numpy()
        out[dtype] = (q.detach().double().cpu().numpy(), F, float(E.sum()))
    q64, F64, E64 = out[torch.float64]
    fscale = np.abs(d["F_quadratic"]).max()
    assert np.abs(q64 - d["q_quadratic"]).max() < 1e-6
    assert np.abs(F64 - d["F_quadratic"]).max() / fscale < 5e-5
    assert abs(E64 - float(d["E_quadratic"][0])) / abs(float(d["E_quadratic"][0])) < 1e-6
    q32, F32, E32 = out[torch.float32]
    assert np.abs(q32 - q64).max() < 1e-5
    assert np.abs(F32 - F64).max() / np.abs(F64).max() < 1e-4


def test_implicit_adjoint_vs_finite_differences(cuda):
    """d(w . q*)/d theta through the adjoint CG vs central differences (step 1e-4)."""
    from admp_b200.nblist import TorchNeighborList
    from admp_b200.qeq import QEqForceModule, qeq_solve
    d = golden("qeq_water_small")
    m = QEqForceModule(6.0, 5e-4, kmesh=20, eps=1e-10, max_iter=500)
    n = d["pos"].shape[0]
    rng = np.random.default_rng(1)
    w = T(rng.normal(size=n), cuda)
    C = torch.ones(1, n, dtype=torch.float64, device=cuda)

    def loss(pos_np, chi_np, eta_np, hd_np, grad=False):
        pos = T(pos_np, cuda, grad=grad)
        box = T(d["box"], cuda)
        chi = T(chi_np, cuda, grad=grad)
        eta = T(eta_np, cuda, grad=grad)
        hd = T(hd_np, cuda, grad=grad)
        nb = TorchNeighborList(6.0)
        pairs = nb(pos, box)
        q = qeq_solve(m, pos, box, chi, hd, eta, pairs, nb.get_ds(), nb.get_buffer_scales(), C)
        return (w * q).sum(), (pos, chi, eta, hd)

    L0, (pos, chi, eta, hd) = loss(d["pos"], d["chi"], d["eta"], d["hardness"], grad=True)
    gpos, gchi, geta, ghd = torch.autograd.grad(L0, [pos, chi, eta, hd])
    h = 1e-4
    for arr_name, g in [("chi", gchi), ("eta", geta), ("hardness", ghd), ("pos", gpos)]:
        for k in [0, 5, 17]:
            base = {"pos": d["pos"].copy(), "chi": d["chi"].copy(), "eta": d["eta"].copy(),
                    "hardness": d["hardness"].copy()}
            idx = (k, 1) if arr_name == "pos" else k
            base[arr_name][idx] += h
            lp = loss(base["pos"], base["chi"], base["eta"], base["hardness"])[0].item()
            base[arr_name][idx] -= 2 * h
            lm = loss(base["pos"], base["chi"], base["eta"], base["hardness"])[0].item()
            fd = (lp - lm) / (2 * h)
            an = g[idx].item()
            assert abs(fd - an) < 1e-6 + 1e-4 * abs(fd), (arr_name, k, fd, an)


@pytest.mark.parametrize("groups", [2, 3])
def test_qeq_cg_group_constraints_match_kkt(cuda, groups):
    """Several constraint rows that are not the all-ones row (charge of each of
    `groups` atom groups fixed): the projected CG and the dense KKT solve give
    the same charges, and every group carries its prescribed charge."""
    from admp_b200.qeq import matinv_optimize, pgrad_optimize
    d = golden("qeq_water_small")
    m, pos, box, pairs, ds, bs, chi, hd, eta, _, _ = setup(d, cuda, 20, eps=1e-10, max_iter=2000)
    n = pos.shape[0]
    edges = np.linspace(0, n, groups + 1).astype(int)
    C = torch.zeros(groups, n, dtype=torch.float64, device=cuda)
    for g in range(groups):
        C[g, edges[g]:edges[g + 1]] = 1.0
    b = torch.tensor(np.linspace(-1.5, 1.0, groups), dtype=torch.float64, device=cuda)
    _, q_cg = pgrad_optimize(m, torch.zeros(n, dtype=torch.float64, device=cuda), pos, box, chi, hd, eta, pairs, ds,
                             bs, C, b, method="quadratic", reinit_q=True)
    _, q_kkt = matinv_optimize(m, pos, box, chi, hd, eta, pairs, ds, bs, C, b)
    np.testing.assert_allclose((C @ q_cg.detach()).cpu().numpy(), b.cpu().numpy(), atol=1e-9)
    assert (q_cg.detach() - q_kkt.detach()).abs().max().item() < 1e-7
