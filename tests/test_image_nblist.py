"""Neighbour list over periodic images (dp_nblist, nblist.py:33-93) -- CPU side.

The oracle's image enumeration is pinned on the golden TorchNeighborList
pairs (made by running the reference): for rc <= L/2 each pair has a single
image, so dp_nblist's i < j set equals the reference's half list.  For
rc > L/2 it is checked against a wider enumeration, against the per-atom
nnei cut, and the Python entry point's argument checks run without a GPU.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import admp_oracle as O


@pytest.mark.parametrize("tag", ["cubic", "tric"])
def test_image_oracle_matches_reference_half_list(tag):
    d = golden("nblist")
    pos, box = d[tag + "_pos"], d[tag + "_box"]
    pairs, shifts, ds, bs = O.image_nblist(pos, box, 6.0, -1)
    ref = d[tag + "_pairs"]
    half = ref[:, 0] < ref[:, 1]
    assert set(map(tuple, pairs)) == set(map(tuple, ref[half]))
    assert len(pairs) == half.sum() and np.all(bs == 1.0)
    order = {tuple(p): i for i, p in enumerate(ref)}
    idx = np.array([order[tuple(p)] for p in pairs])
    assert np.abs(ds - d[tag + "_ds"][idx]).max() < 1e-12
    assert np.abs(np.linalg.norm(pos[pairs[:, 1]] - pos[pairs[:, 0]] + shifts @ box, axis=1) - ds).max() < 1e-12


def _brute(pos, box, rc, extra=2):
    """All (i <= j, n) with r <= rc over a generously wide image range."""
    binv = np.linalg.inv(box)
    V = abs(np.linalg.det(box))
    h = np.array([V / np.linalg.norm(np.cross(box[(d + 1) % 3], box[(d + 2) % 3])) for d in range(3)])
    k = np.floor(pos @ binv)
    m = np.ceil(rc / h).astype(int) + int(np.abs(k).max()) + extra
    rng = [np.arange(-m[d], m[d] + 1) for d in range(3)]
    imgs = np.stack(np.meshgrid(*rng, indexing="ij"), -1).reshape(-1, 3)
    out = set()
    n = len(pos)
    for i in range(n):
        for j in range(i, n):
            r = np.linalg.norm(pos[j] - pos[i] + imgs @ box, axis=1)
            for a in np.nonzero(r <= rc)[0]:
                if j == i and not imgs[a].any():
                    continue
                out.add((i, j, *imgs[a]))
    return out


@pytest.mark.parametrize("rc", [6.0, 11.0, 17.0])
def test_image_oracle_large_cutoff_complete(rc):
    rng = np.random.default_rng(11)
    box = np.array([[10.0, 0.0, 0.0], [2.0, 9.0, 0.0], [-1.0, 1.5, 11.0]])
    pos = rng.random((12, 3)) @ box + rng.normal(0, 3.0, (12, 3))   # some atoms outside the cell
    pairs, shifts, ds, bs = O.image_nblist(pos, box, rc, -1)
    got = {(int(p[0]), int(p[1]), *map(int, s)) for p, s in zip(pairs, shifts)}
    assert got == _brute(pos, box, rc)
    nij = int((bs == 1.0).sum())
    assert np.all(pairs[:nij, 0] < pairs[:nij, 1]) and np.all(pairs[nij:, 0] == pairs[nij:, 1])
    assert np.all(bs[nij:] == 0.5)
    if rc > 10.0:
        assert len(pairs) > nij                          # self images present
        # self images come in +n / -n couples
        si = {(int(p[0]), *map(int, s)) for p, s in zip(pairs[nij:], shifts[nij:])}
        assert all((t[0], -t[1], -t[2], -t[3]) in si for t in si)


def test_image_oracle_nnei_cut():
    rng = np.random.default_rng(5)
    box = np.eye(3) * 8.0
    pos = rng.random((30, 3)) * 8.0
    full = O.image_nblist(pos, box, 7.0, -1)
    cut = O.image_nblist(pos, box, 7.0, 20)
    fs = {(int(p[0]), int(p[1]), *map(int, s)) for p, s in zip(full[0], full[1])}
    cs = {(int(p[0]), int(p[1]), *map(int, s)) for p, s in zip(cut[0], cut[1])}
    assert cs < fs
    # per atom i: the kept i -> (j >= i) entries are exactly those within the
    # distance of i's 20th nearest image (over all j)
    for i in range(30):
        df = pos[None, :, :] - pos[i] + (np.stack(np.meshgrid(*[np.arange(-2, 3)] * 3, indexing="ij"), -1)
                                         .reshape(-1, 1, 3) @ box)
        r = np.linalg.norm(df, axis=-1).ravel()
        r = np.sort(r[(r > 0) & (r <= 7.0)])
        th = r[19] * (1 + 1e-12)   # the 20th distance, computed another way
        want = {t for t in fs if t[0] == i and
                np.linalg.norm(pos[t[1]] - pos[i] + np.array(t[2:]) @ box) <= th}
        assert {t for t in cs if t[0] == i} == want


def test_image_oracle_open_boundary():
    rng = np.random.default_rng(2)
    pos = rng.random((40, 3)) * 12.0
    pairs, shifts, ds, bs = O.image_nblist(pos, None, 5.0, -1)
    full = O.nblist_obc(pos, 5.0)
    assert set(map(tuple, pairs)) == {tuple(p) for p in full if p[0] < p[1]}
    assert not shifts.any() and np.all(bs == 1.0)


def test_dp_nblist_rejects_bad_cutoff_without_gpu():
    import torch
    from admp_b200 import nblist
    pos = torch.rand(5, 3, dtype=torch.float64)
    box = torch.eye(3, dtype=torch.float64) * 5
    for rc in (-1.0, 0.0):
        with pytest.raises(ValueError, match=f"rcut must be positive, got {rc}"):
            nblist.dp_nblist(pos, box, 10, rcut=rc)
        with pytest.raises(ValueError, match=f"rcut must be positive, got {rc}"):
            nblist.vesin_nblist(pos, box, rcut=rc)


def test_sort_pairs():
    import torch
    from admp_b200.nblist import sort_pairs
    p = torch.tensor([[3, 1], [0, 5], [3, 0], [0, 2], [1, 1]])
    assert sort_pairs(p).tolist() == [[0, 2], [0, 5], [1, 1], [3, 0], [3, 1]]
