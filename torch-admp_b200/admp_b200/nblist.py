"""TorchNeighborList on the GPU cell list (nblist.py:268-617, check_cutoff :620-660).

``forward(positions, box)`` returns the full pair list (both orders, sorted by
(i, j)) and stores ``pairs``, ``buffer_scales`` (1 if i < j) and ``ds``; ``ds``
is differentiable with respect to positions and box (hand-written backward),
as in the reference, so forces can flow through the caller's distances.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import _lib as L
from .ops import PairDistanceFn, neighbor_pairs


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
