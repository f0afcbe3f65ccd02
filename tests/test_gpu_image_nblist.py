"""Neighbour list over periodic images on the B200 (dp_nblist / vesin_nblist,
nblist.py:33-138) against the oracle's image enumeration: pair sets with
image shifts, distances, the per-atom nnei cut, distance gradients, and the
Ewald energy with a real-space cutoff above half the box."""
import numpy as np
import pytest
import torch

from _gpu_helpers import T, rel
from oracle import admp_oracle as O

pytestmark = pytest.mark.gpu


def _keyed(pairs, shifts):
    return {(int(p[0]), int(p[1]), *map(int, s)) for p, s in zip(pairs, shifts)}


def test_dp_nblist_reference_config(cuda):
    """The reference's own consistency case: 100 atoms, 10 A box, rc 6 > L/2, nnei 150."""
    from admp_b200 import nblist
    rng = np.random.default_rng(20240601)
    pos = rng.random((100, 3)) * 10.0
    box = np.diag([10.0, 10.0, 10.0])
    pairs, ds, bs = nblist.dp_nblist(T(pos, cuda), T(box, cuda), 150, 6.0)
    op, osh, ods, obs = O.image_nblist(pos, box, 6.0, 150)
    assert pairs.shape == (len(op), 2) and ds.shape == (len(op),)
    assert pairs.dtype == torch.long and bs.dtype == torch.get_default_dtype()
    assert torch.equal(nblist.sort_pairs(pairs).cpu(), nblist.sort_pairs(torch.from_numpy(op)))
    assert rel(torch.sort(ds)[0], np.sort(ods)) < 1e-14
    assert np.array_equal(bs.cpu().numpy(), obs)
    # the reference test: dp_nblist and vesin_nblist agree (no self images at rc < L)
    p2, ds2, bs2 = nblist.vesin_nblist(T(pos, cuda), T(box, cuda), 6.0)
    assert torch.equal(nblist.sort_pairs(pairs), nblist.sort_pairs(p2))
    assert torch.equal(torch.sort(ds)[0], torch.sort(ds2)[0])
    assert bool((bs2 == 1).all())


@pytest.mark.parametrize("rc", [7.5, 13.0])
def test_image_pairs_shifts_triclinic(cuda, rc):
    from admp_b200.ops import image_neighbor_pairs
    rng = np.random.default_rng(31)
    box = np.array([[10.0, 0.0, 0.0], [2.0, 9.0, 0.0], [-1.0, 1.5, 11.0]])
    pos = rng.random((60, 3)) @ box + rng.normal(0, 3.0, (60, 3))
    pairs, shifts, n_ij, ntr = image_neighbor_pairs(T(pos, cuda), T(box, cuda), rc, -1)
    op, osh, ods, obs = O.image_nblist(pos, box, rc, -1)
    assert ntr == 0 and n_ij == int((obs == 1.0).sum())
    p, s = pairs.cpu().numpy(), shifts.cpu().numpy()
    assert _keyed(p[:n_ij], s[:n_ij]) == _keyed(op[:n_ij], osh[:n_ij])
    assert _keyed(p[n_ij:], s[n_ij:]) == _keyed(op[n_ij:], osh[n_ij:])
    if rc > 11.0:
        assert len(p) > n_ij
    # i-major order inside each block
    assert np.all(np.diff(p[:n_ij, 0]) >= 0) and np.all(np.diff(p[n_ij:, 0]) >= 0)


def test_image_nnei_cut_matches_oracle(cuda):
    from admp_b200.ops import image_neighbor_pairs
    rng = np.random.default_rng(5)
    box = np.eye(3) * 8.0
    pos = rng.random((50, 3)) * 8.0
    for nnei in (0, 1, 20, 80):
        pairs, shifts, n_ij, ntr = image_neighbor_pairs(T(pos, cuda), T(box, cuda), 7.0, nnei)
        op, osh, ods, obs = O.image_nblist(pos, box, 7.0, nnei)
        assert _keyed(pairs.cpu().numpy(), shifts.cpu().numpy()) == _keyed(op, osh)
        assert ntr == 50 if nnei <= 20 else ntr >= 0


def test_image_ds_gradients(cuda):
    from admp_b200 import nblist
    from admp_b200.ops import image_neighbor_pairs
    rng = np.random.default_rng(8)
    box = np.array([[9.0, 0.0, 0.0], [1.0, 8.5, 0.0], [0.5, -1.0, 9.5]])
    pos = rng.random((40, 3)) @ box
    p = T(pos, cuda, grad=True)
    b = T(box, cuda, grad=True)
    pairs, ds, bs = nblist.dp_nblist(p, b, 500, 10.0)
    pr, sh, _, _ = image_neighbor_pairs(T(pos, cuda), T(box, cuda), 10.0, 500)
    assert torch.equal(pr, pairs)
    w = torch.linspace(0.5, 1.5, ds.shape[0], dtype=torch.float64, device=cuda)
    gp, gb = torch.autograd.grad((ds * w * bs).sum(), [p, b])
    P, S = pairs.cpu().numpy(), sh.cpu().numpy()
    dr = pos[P[:, 1]] - pos[P[:, 0]] + S @ box
    d = np.linalg.norm(dr, axis=1)
    assert rel(ds, d) < 1e-14
    g = (w * bs).cpu().numpy()[:, None] * dr / d[:, None]
    ref_gp = np.zeros_like(pos)
    np.add.at(ref_gp, P[:, 1], g)
    np.add.at(ref_gp, P[:, 0], -g)
    ref_gb = S.T.astype(float) @ g
    assert rel(gp, ref_gp) < 1e-12
    assert rel(gb, ref_gb) < 1e-12


def test_image_open_boundary_and_empty(cuda):
    from admp_b200 import nblist
    rng = np.random.default_rng(2)
    pos = rng.random((40, 3)) * 12.0
    pairs, ds, bs = nblist.dp_nblist(T(pos, cuda), None, 100, 5.0)
    op, _, ods, _ = O.image_nblist(pos, None, 5.0, -1)
    assert set(map(tuple, pairs.cpu().numpy())) == set(map(tuple, op))
    assert rel(torch.sort(ds)[0], np.sort(ods)) < 1e-14
    pairs, ds, bs = nblist.dp_nblist(T(np.zeros((0, 3)), cuda), T(np.eye(3) * 5, cuda), 10, 3.0)
    assert pairs.shape == (0, 2) and ds.shape == (0,)
    pairs, ds, bs = nblist.dp_nblist(T(np.array([[1.0, 2.0, 3.0]]), cuda), T(np.eye(3) * 4, cuda), 10, 4.5)
    # a lone atom in a 4 A box sees its 6 face images at 4 A
    assert pairs.shape == (6, 2) and bool((pairs == 0).all()) and bool((bs == 0.5).all())
    assert rel(ds, np.full(6, 4.0)) < 1e-14


def test_image_fp32(cuda):
    from admp_b200.ops import image_neighbor_pairs
    rng = np.random.default_rng(9)
    box = np.eye(3) * 9.0
    pos = (rng.random((80, 3)) * 9.0).astype(np.float32).astype(np.float64)
    pairs, shifts, n_ij, _ = image_neighbor_pairs(T(pos, cuda, torch.float32), T(box, cuda, torch.float32), 8.0, -1)
    op, osh, _, _ = O.image_nblist(pos, box, 8.0, -1)
    got, ref = _keyed(pairs.cpu().numpy(), shifts.cpu().numpy()), _keyed(op, osh)
    assert len(got ^ ref) <= 4


def test_ewald_energy_with_cutoff_above_half_box(cuda):
    """The Ewald energy does not depend on the real/reciprocal split: a
    cutoff of 9 A in a 10 A box (dp_nblist pairs, self images included) must
    give the energy and forces of the usual rc < L/2 set-up."""
    from admp_b200 import nblist
    from admp_b200.nblist import TorchNeighborList
    from admp_b200.pme import CoulombForceModule
    rng = np.random.default_rng(17)
    n = 64
    box = np.diag([10.0, 10.0, 10.0])
    pos = rng.random((n, 3)) * 10.0
    q = rng.normal(0, 1, n)
    q -= q.mean()

    def run(rc, pairs_fn):
        p = T(pos, cuda, grad=True)
        b = T(box, cuda)
        pairs, ds, bs = pairs_fn(p, b, rc)
        m = CoulombForceModule(rcut=rc, ethresh=1e-7)
        e = m(p, b, pairs, ds, bs, {"charge": T(q, cuda)})
        f = -torch.autograd.grad(e, p)[0]
        return float(e.detach()), f

    def cell_list(p, b, rc):
        nb = TorchNeighborList(rc)
        pairs = nb(p, b)
        return pairs, nb.get_ds(), nb.get_buffer_scales()

    e1, f1 = run(4.9, cell_list)
    e2, f2 = run(9.0, lambda p, b, rc: nblist.dp_nblist(p, b, 4000, rc))
    assert abs(e2 - e1) / abs(e1) < 2e-6
    assert rel(f2, f1) < 2e-5


def test_vesin_half_list_with_self_images(cuda):
    """rc above the box length: vesin_nblist keeps one of each +-n self-image
    couple with scale 1, dp_nblist both with scale 1/2; their pair energies agree."""
    from admp_b200 import nblist
    from admp_b200.ops import image_neighbor_pairs
    rng = np.random.default_rng(13)
    box = np.array([[7.0, 0.0, 0.0], [1.0, 7.5, 0.0], [0.5, -0.5, 8.0]])
    pos = rng.random((30, 3)) @ box
    rc = 9.0
    p_dp, ds_dp, bs_dp = nblist.dp_nblist(T(pos, cuda), T(box, cuda), 10000, rc)
    p_v, ds_v, bs_v = nblist.vesin_nblist(T(pos, cuda), T(box, cuda), rc)
    pr, sh, n_ij, _ = image_neighbor_pairs(T(pos, cuda), T(box, cuda), rc, -1)
    n_self = pr.shape[0] - n_ij
    assert n_self > 0 and n_self % 2 == 0
    assert p_v.shape[0] == n_ij + n_self // 2 and bool((bs_v == 1).all())
    # kept self images: first non-zero shift component positive
    s = sh[n_ij:].cpu().numpy()
    first = np.where(s[:, 0] != 0, s[:, 0], np.where(s[:, 1] != 0, s[:, 1], s[:, 2]))
    assert (first > 0).sum() == n_self // 2
    # any pair function summed with the buffer scales is the same over both lists
    q = rng.normal(size=30)
    qt = T(q, cuda)

    def pair_sum(p, ds, bs):
        return float((qt[p[:, 0]] * qt[p[:, 1]] * torch.erfc(0.3 * ds) / ds * bs.to(ds.dtype)).sum())

    a, b = pair_sum(p_dp, ds_dp, bs_dp), pair_sum(p_v, ds_v, bs_v)
    assert abs(a - b) <= 1e-12 * max(1.0, abs(a))
