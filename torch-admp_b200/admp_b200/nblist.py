"""Neighbour lists on the GPU.

TorchNeighborList (nblist.py:268-617, check_cutoff :620-660) on a cell list:
``forward(positions, box)`` returns the full pair list (both orders, sorted by
(i, j)) and stores ``pairs``, ``buffer_scales`` (1 if i < j) and ``ds``; ``ds``
is differentiable with respect to positions and box (hand-written backward),
as in the reference, so forces can flow through the caller's distances.

dp_nblist / vesin_nblist (nblist.py:33-138) for cutoffs above half the box:
one pair per periodic image within the cutoff, built by the image kernels,
with distances differentiable through the stored image shifts.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import _lib as L
from .ops import ImagePairDistanceFn, PairDistanceFn, image_neighbor_pairs, neighbor_pairs


def check_cutoff(box: torch.Tensor, cutoff: float) -> None:
    """Assert rc <= half the minimum box height (nblist.py:620-660)."""
    b = box.detach().to("cpu", torch.float64)
    a1, a2, a3 = b[0], b[1], b[2]
    normals = torch.stack([torch.cross(a2, a3, dim=-1), torch.cross(a3, a1, dim=-1), torch.cross(a1, a2, dim=-1)])
    unit = normals / torch.norm(normals, dim=1, keepdim=True)
    heights = torch.abs(torch.einsum("ij,ij->i", b, unit))
    mh = torch.min(heights) / 2
    assert cutoff <= mh, (f"Cutoff {cutoff} is larger than half the minimum height {mh} of the box. "
                          "This may lead to unphysical results.")


class TorchNeighborList(torch.nn.Module):
    def __init__(self, cutoff: float) -> None:
        super().__init__()
        self.cutoff = cutoff
        self.pairs = torch.empty(1, dtype=torch.long)
        self.buffer_scales = torch.empty(1, dtype=torch.long)
        self.ds = torch.empty(1)

    def forward(self, positions: torch.Tensor, box: Optional[torch.Tensor] = None) -> torch.Tensor:
        L.require_cuda(positions, "positions")
        pos_c = positions.detach().contiguous()
        box_c = box.detach().to(positions.dtype).contiguous() if box is not None else None
        try:
            pairs, bs = neighbor_pairs(pos_c, box_c, self.cutoff)
        except AssertionError:
            check_cutoff(box, self.cutoff)
            raise
        self.pairs = pairs
        self.buffer_scales = bs
        self.ds = self.pairs_ds(positions, pairs, box, box is not None)
        return pairs

    @staticmethod
    def pairs_buffer_scales(pairs: torch.Tensor) -> torch.Tensor:
        return (pairs[:, 0] < pairs[:, 1]).to(torch.long)

    @staticmethod
    def pairs_ds(positions: torch.Tensor, pairs: torch.Tensor, box: Optional[torch.Tensor] = None,
                 pbc_flag: bool = True) -> torch.Tensor:
        pos = positions.contiguous()
        b = box.to(positions.dtype).contiguous() if (pbc_flag and box is not None) else None
        if pbc_flag:
            assert b is not None, "Box should be provided for periodic system."
        return PairDistanceFn.apply(pos, b, pairs.to(torch.long).contiguous())

    def set_pairs(self, pairs):
        self.pairs = pairs

    def set_buffer_scales(self, buffer_scales):
        self.buffer_scales = buffer_scales

    def set_ds(self, ds):
        self.ds = ds

    def get_pairs(self):
        return self.pairs

    def get_buffer_scales(self):
        return self.buffer_scales

    def get_ds(self):
        return self.ds


def _image_list(positions: torch.Tensor, box: Optional[torch.Tensor], rcut: float, nnei: int):
    if rcut <= 0.0:
        raise ValueError(f"rcut must be positive, got {rcut}")
    L.require_cuda(positions, "positions")
    pos = positions.reshape(-1, 3)
    b = box.reshape(3, 3).to(pos.dtype) if box is not None else None
    pairs, shifts, n_ij, _ = image_neighbor_pairs(pos.detach().contiguous(),
                                                  b.detach().contiguous() if b is not None else None,
                                                  float(rcut), int(nnei))
    ds = ImagePairDistanceFn.apply(pos.contiguous(), b.contiguous() if b is not None else None, pairs, shifts)
    return pairs, shifts, ds, n_ij


def dp_nblist(positions: torch.Tensor, box: Optional[torch.Tensor], nnei: int, rcut: float):
    """Pairs over periodic images (nblist.py:33-93): returns (pairs, ds, buffer_scales).

    pairs holds every image (i, j) with i < j and r <= rcut (buffer scale 1),
    followed by every self image (i, i) of an atom (scale 1/2); each atom
    keeps its ``nnei`` nearest images, the ``sel`` cut of the per-atom list
    dp_nblist is built from (atoms with a tie at the nnei-th distance keep all
    tied images).  ds is differentiable in positions and box.  Within each
    block pairs are ordered by (i, j, image) rather than by distance.
    """
    pairs, _shifts, ds, n_ij = _image_list(positions, box, rcut, nnei)
    buffer_scales = torch.ones(pairs.shape[0], device=pairs.device)
    buffer_scales[n_ij:] = 0.5
    return pairs, ds, buffer_scales


def vesin_nblist(positions: torch.Tensor, box: torch.Tensor, rcut: float):
    """Half list over periodic images (nblist.py:96-138): returns (pairs, ds, buffer_scales).

    Same image pairs as dp_nblist, but each self image is kept once (of the
    two opposite shifts n and -n, the one whose first non-zero component is
    positive) and every buffer scale is 1 -- the half-list convention.
    """
    pairs, shifts, ds, n_ij = _image_list(positions, box, rcut, -1)
    if pairs.shape[0] > n_ij:
        s = shifts[n_ij:].to(torch.long)
        first = torch.where(s[:, 0] != 0, s[:, 0], torch.where(s[:, 1] != 0, s[:, 1], s[:, 2]))
        keep = torch.cat([torch.ones(n_ij, dtype=torch.bool, device=pairs.device), first > 0])
        pairs, ds = pairs[keep], ds[keep]
    return pairs, ds, torch.ones_like(ds)


def sort_pairs(pairs: torch.Tensor) -> torch.Tensor:
    """Rows sorted by (first, second) index (nblist.py:243-264)."""
    idx = torch.argsort(pairs[:, 1])
    pairs = pairs[idx]
    idx = torch.argsort(pairs[:, 0], stable=True)
    return pairs[idx]


def frame_pair_lists(positions: torch.Tensor, box: torch.Tensor, cutoff: float):
    """Neighbour lists of nf frames stacked for the multi-frame calls:
    pairs [nf, P, 2] (frame-local indices), ds [nf, P] (differentiable with
    respect to positions [nf, N, 3] and box [nf, 3, 3]) and buffer_scales
    [nf, P], with P the longest frame's list; the rows past a frame's own
    pairs hold (0, 0) with distance 1 and scale 0, which every kernel skips."""
    nf = positions.shape[0]
    lists = []
    for f in range(nf):
        nb = TorchNeighborList(cutoff)
        pr = nb(positions[f], box[f])
        lists.append((pr, nb.get_ds(), nb.get_buffer_scales()))
    P = max(int(p.shape[0]) for p, _, _ in lists)
    pairs, ds, bs = [], [], []
    for pr, d, s in lists:
        pad = P - int(pr.shape[0])
        pairs.append(torch.cat([pr, pr.new_zeros(pad, 2)]))
        ds.append(torch.cat([d, d.new_ones(pad)]))
        bs.append(torch.cat([s, s.new_zeros(pad)]))
    return torch.stack(pairs), torch.stack(ds), torch.stack(bs)
