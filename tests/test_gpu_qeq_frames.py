"""The differentiation batch: jittered frames of the 1,000-water QEq system
(3,000 atoms, 31 A box, 48^3 mesh, rc 6) solved together
(admp_qeq_solve_frames), with energy gradients w.r.t. positions, box, chi,
hardness and eta through the hand-written backward passes and the implicit
adjoint of the charge solve (one second batched CG).

Checked against the reference's autograd gradients (tests/golden/qeq_cfg4.npz:
the reference evaluates E at its detached optimum, so its autograd gradient
is the total derivative), against autograd through the reference's dense
KKT solve for dq/dchi (tests/golden/qeq_dq_dchi.npz), and against central
finite differences (step 1e-4) of a charge-dependent loss, which is what
exercises the adjoint (energy gradients do not: at the constrained minimum
the charge response drops out)."""
import numpy as np
import pytest
import torch

from conftest import golden
from _gpu_helpers import T, rel

pytestmark = pytest.mark.gpu

RC, ETHRESH, KMESH = 6.0, 5e-4, 48


def _module(tol, max_iter=2000):
    from admp_b200.qeq import QEqForceModule
    return QEqForceModule(RC, ETHRESH, kmesh=KMESH, eps=tol, max_iter=max_iter)


def _frames(cuda, nf, dtype, seed=1024):
    from admp_b200 import synthetic
    pos, box, chi, hard, eta, elem = synthetic.water_frames(nf, seed)
    return (T(pos, cuda, dtype, grad=True), T(box, cuda, dtype, grad=True), T(chi, cuda, dtype, grad=True),
            T(hard, cuda, dtype, grad=True), T(eta, cuda, dtype, grad=True), elem)


def _energy(module, pos, box, chi, hard, eta, pairs, ds, bs, tol):
    """Per-frame QEq energy at the batched, differentiable optimum."""
    from admp_b200.qeq import qeq_solve_frames
    nf, n = pos.shape[0], pos.shape[1]
    C = torch.ones(1, n, dtype=pos.dtype, device=pos.device)
    q = qeq_solve_frames(module, pos, box, chi, hard, eta, pairs, ds, bs, C, tol=tol)
    params = {"charge": q, "chi": chi.expand(nf, n), "hardness": hard.expand(nf, n), "eta": eta.expand(nf, n)}
    return module(pos, box, pairs, ds, bs, params), q


def test_frames_solve_equals_single_frame_solves(cuda):
    """Three frames in one batched CG give each frame's single-frame charges."""
    from admp_b200.nblist import TorchNeighborList, frame_pair_lists
    from admp_b200.qeq import pgrad_optimize, qeq_solve_frames
    pos, box, chi, hard, eta, _ = _frames(cuda, 3, torch.float64)
    m = _module(1e-11)
    pairs, ds, bs = frame_pair_lists(pos, box, RC)
    n = pos.shape[1]
    C = torch.ones(1, n, dtype=torch.float64, device=cuda)
    q = qeq_solve_frames(m, pos, box, chi, hard, eta, pairs, ds, bs, C).detach()
    assert len(m.frame_iters) == 3 and max(m.frame_residuals) < 1e-11
    for f in range(3):
        nb = TorchNeighborList(RC)
        pr = nb(pos[f], box[f])
        _, qs = pgrad_optimize(m, None, pos[f], box[f], chi, hard, eta, pr, nb.get_ds(), nb.get_buffer_scales(), C,
                               torch.zeros(1, dtype=torch.float64, device=cuda), method="quadratic")
        assert np.abs((q[f] - qs.detach()).cpu().numpy()).max() < 1e-9
        assert abs(float(q[f].sum())) < 1e-10


def test_cfg4_energy_gradients_match_reference_autograd(cuda):
    """Frames 0 and 1: energy and its gradients w.r.t. positions, box, chi,
    hardness and eta (per atom) against the reference's autograd."""
    from admp_b200.nblist import frame_pair_lists
    d = golden("qeq_cfg4")
    pos, box, chi, hard, eta, _ = _frames(cuda, 2, torch.float64)
    assert np.array_equal(pos.detach().cpu().numpy(), d["pos"])
    m = _module(1e-11)
    pairs, ds, bs = frame_pair_lists(pos, box, RC)
    E, q = _energy(m, pos, box, chi, hard, eta, pairs, ds, bs, 1e-11)
    gpos, gbox, gchi, ghard, geta = torch.autograd.grad(E.sum(), [pos, box, chi, hard, eta])
    # per-frame gradients of the shared parameters: one frame at a time
    for f in range(2):
        assert abs(float(E[f]) - float(d[f"E_{f}"][0])) / abs(float(d[f"E_{f}"][0])) < 1e-9
        assert np.abs(q[f].detach().cpu().numpy() - d[f"q_{f}"]).max() < 1e-6
        assert rel(gpos[f], d[f"dpos_{f}"]) < 1e-6
        assert rel(gbox[f], d[f"dbox_{f}"]) < 1e-6
    for name, g in (("dchi", gchi), ("dhard", ghard), ("deta", geta)):
        assert rel(g, d[f"{name}_0"] + d[f"{name}_1"]) < 1e-6, name


def _fixed_pair_ds(pos, box, pairs):
    """Distances of a fixed pair list (so finite differences see no pair
    entering or leaving the cutoff)."""
    from admp_b200.nblist import TorchNeighborList
    return torch.stack([TorchNeighborList.pairs_ds(pos[f], pairs[f], box[f], True) for f in range(pos.shape[0])])


def test_cfg4_adjoint_matches_finite_differences(cuda):
    """dL/dtheta of the charge-dependent loss L = sum_i w_i q_i (which needs
    the adjoint) against central differences with step 1e-4: positions, box
    (diagonal and off-diagonal entries), and per-element chi, hardness, eta."""
    from admp_b200.nblist import frame_pair_lists
    from admp_b200.qeq import qeq_solve_frames
    pos, box, chi, hard, eta, elem = _frames(cuda, 1, torch.float64)
    m = _module(1e-13)
    pairs, _, bs = frame_pair_lists(pos, box, RC)
    pairs, bs = pairs.detach(), bs.detach()
    n = pos.shape[1]
    C = torch.ones(1, n, dtype=torch.float64, device=cuda)
    w = torch.tensor(np.random.default_rng(7).normal(size=n), dtype=torch.float64, device=cuda)

    def loss(p, b, c, h, e):
        q = qeq_solve_frames(m, p, b, c, h, e, pairs, _fixed_pair_ds(p, b, pairs), bs, C, tol=1e-13)
        return (q[0] * w).sum()

    L0 = loss(pos, box, chi, hard, eta)
    gpos, gbox, gchi, ghard, geta = torch.autograd.grad(L0, [pos, box, chi, hard, eta])
    h = 1e-4
    O = torch.tensor(elem == "O", device=cuda)
    checks = []
    with torch.no_grad():
        for (a, k) in [(0, 0), (17, 1), (1500, 2), (2999, 0)]:
            dp = torch.zeros_like(pos)
            dp[0, a, k] = h
            fd = (loss(pos + dp, box, chi, hard, eta) - loss(pos - dp, box, chi, hard, eta)) / (2 * h)
            checks.append(("pos", float(gpos[0, a, k]), float(fd)))
        for (i, j) in [(0, 0), (1, 1), (2, 2), (0, 1), (2, 0)]:
            db = torch.zeros_like(box)
            db[0, i, j] = h
            fd = (loss(pos, box + db, chi, hard, eta) - loss(pos, box - db, chi, hard, eta)) / (2 * h)
            checks.append(("box", float(gbox[0, i, j]), float(fd)))
        for name, g, k in (("chi", gchi, 2), ("hardness", ghard, 3), ("eta", geta, 4)):
            for sel in (O, ~O):
                args = [pos, box, chi, hard, eta]
                dv = torch.where(sel, torch.full_like(chi, h), torch.zeros_like(chi))
                up, dn = list(args), list(args)
                up[k] = args[k] + dv
                dn[k] = args[k] - dv
                fd = (loss(*up) - loss(*dn)) / (2 * h)
                checks.append((name, float(g[sel].sum()), float(fd)))
    for name, an, fd in checks:
        assert abs(an - fd) <= 1e-5 * max(abs(fd), 1e-2), (name, an, fd)


def test_dq_dchi_matches_reference_dense_solve(cuda):
    """dL/dchi for L = sum_i w_i q_i against autograd through the reference's
    dense KKT solve (192 atoms)."""
    from admp_b200.nblist import frame_pair_lists
    from admp_b200.qeq import QEqForceModule, qeq_solve_frames
    d = golden("qeq_dq_dchi")
    pos = T(d["pos"][None], cuda)
    box = T(d["box"][None], cuda)
    chi = T(d["chi"], cuda, grad=True)
    m = QEqForceModule(float(d["rcut"]), float(d["ethresh"]), kmesh=int(d["kmesh"]), eps=1e-13, max_iter=2000)
    pairs, ds, bs = frame_pair_lists(pos, box, float(d["rcut"]))
    n = pos.shape[1]
    q = qeq_solve_frames(m, pos, box, chi, T(d["hardness"], cuda), T(d["eta"], cuda), pairs, ds, bs,
                         torch.ones(1, n, dtype=torch.float64, device=cuda))
    assert np.abs(q[0].detach().cpu().numpy() - d["q"]).max() < 1e-10
    (g,) = torch.autograd.grad((q[0] * T(d["w"], cuda)).sum(), [chi])
    assert rel(g, d["dL_dchi"]) < 1e-8


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_cfg4_batch_of_64_frames(cuda, dtype):
    """All 64 frames in one batched solve + adjoint: frames 0 and 1 reproduce
    the reference's gradients (FP64 to 1e-6; FP32 bulk arithmetic to 1e-4
    relative force and 1e-5 e), and every frame converges."""
    import time
    from admp_b200.nblist import frame_pair_lists
    d = golden("qeq_cfg4")
    tol = 1e-10 if dtype == torch.float64 else 1e-7
    pos, box, chi, hard, eta, _ = _frames(cuda, 64, dtype)
    m = _module(tol)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pairs, ds, bs = frame_pair_lists(pos, box, RC)
    E, q = _energy(m, pos, box, chi, hard, eta, pairs, ds, bs, tol)
    gpos, gbox = torch.autograd.grad(E.sum(), [pos, box])
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert len(m.frame_iters) == 64 and max(m.frame_residuals) < tol
    ftol, qtol = (1e-6, 1e-6) if dtype == torch.float64 else (1e-4, 1e-5)
    for f in range(2):
        assert rel(gpos[f].double(), d[f"dpos_{f}"]) < ftol
        assert rel(gbox[f].double(), d[f"dbox_{f}"]) < ftol * 10
        assert np.abs(q[f].detach().double().cpu().numpy() - d[f"q_{f}"]).max() < qtol
    print(f"64 frames x 3000 atoms ({dtype}): neighbour lists + solve + energy + gradients {dt * 1e3:.1f} ms")
