"""Cell-list neighbour list on the B200 vs the reference's pair sets, ds and
ds-gradients (golden nblist.npz), plus edge cases."""
import numpy as np
import pytest
import torch

from conftest import golden
from _gpu_helpers import T, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["cubic", "tric"])
def test_nblist_pairs_ds_grads(cuda, tag):
    from admp_b200.nblist import TorchNeighborList
    d = golden("nblist")
    pos = T(d[tag + "_pos"], cuda, grad=True)
    box = T(d[tag + "_box"], cuda, grad=True)
    nb = TorchNeighborList(6.0)
    pairs = nb(pos, box)
    p = pairs.cpu().numpy()
    ref = d[tag + "_pairs"]
    assert p.shape == ref.shape
    assert set(map(tuple, p)) == set(map(tuple, ref))
    # output sorted by (i, j)
    key = p[:, 0] * 100000 + p[:, 1]
    assert np.all(np.diff(key) > 0)
    assert np.array_equal(nb.get_buffer_scales().cpu().numpy(), (p[:, 0] < p[:, 1]).astype(np.int64))
    order = {tuple(x): i for i, x in enumerate(ref)}
    idx = np.array([order[tuple(x)] for x in p])
    assert rel(nb.get_ds(), d[tag + "_ds"][idx]) < 1e-14
    w = T(np.linspace(0.5, 1.5, len(ref))[idx], cuda)
    gp, gb = torch.autograd.grad((nb.get_ds() * w).sum(), [pos, box])
    assert rel(gp, d[tag + "_gpos"]) < 1e-12
    assert rel(gb, d[tag + "_gbox"]) < 1e-12


def test_nblist_cutoff_too_large(cuda):
    from admp_b200.nblist import TorchNeighborList
    pos = torch.rand(20, 3, dtype=torch.float64, device=cuda) * 8
    with pytest.raises(AssertionError, match="larger than half the minimum height"):
        TorchNeighborList(5.0)(pos, torch.eye(3, dtype=torch.float64, device=cuda) * 8)


def test_nblist_small_box_two_cells(cuda):
    """rc between L/3 and L/2: two cells per dimension, no double counting."""
    from admp_b200.nblist import TorchNeighborList
    from oracle import admp_oracle as O
    rng = np.random.default_rng(3)
    L = 12.6
    pos = rng.random((200, 3)) * L
    nb = TorchNeighborList(6.0)
    pairs = nb(T(pos, cuda), T(np.diag([L] * 3), cuda)).cpu().numpy()
    ref = O.nblist_pbc(pos, np.diag([L] * 3), 6.0)
    assert set(map(tuple, pairs)) == set(map(tuple, ref)) and len(pairs) == len(ref)


def test_nblist_empty_and_single(cuda):
    from admp_b200.nblist import TorchNeighborList
    nb = TorchNeighborList(3.0)
    pairs = nb(torch.zeros(1, 3, dtype=torch.float64, device=cuda), torch.eye(3, dtype=torch.float64, device=cuda) * 10)
    assert pairs.shape == (0, 2)
    pairs = nb(T([[0.0, 0, 0], [20.0, 20, 20]], cuda), None)
    assert pairs.shape == (0, 2)


def test_nblist_obc_matches_oracle(cuda):
    from admp_b200.nblist import TorchNeighborList
    from oracle import admp_oracle as O
    d = golden("obc")
    pairs = TorchNeighborList(4.0)(T(d["pos"], cuda), None).cpu().numpy()
    assert set(map(tuple, pairs)) == set(map(tuple, d["pairs"]))


def test_nblist_fp32(cuda):
    from admp_b200.nblist import TorchNeighborList
    d = golden("nblist")
    nb = TorchNeighborList(6.0)
    pairs = nb(T(d["cubic_pos"], cuda, torch.float32), T(d["cubic_box"], cuda, torch.float32)).cpu().numpy()
    ref = set(map(tuple, d["cubic_pairs"]))
    got = set(map(tuple, pairs))
    # float32 input may flip pairs within ~1e-6 A of the cutoff
    assert len(ref ^ got) <= 4
