"""BaseForceModule: the drop-in boundary (base_force.py:18-339 of the reference).

Same forward signature, same shape standardisation to (nframes, ...) and the
same ValueError messages; units are converted exactly as in the reference
(positions, box and ds times length_coeff, energy divided by energy_coeff).
forward and the subclasses' _forward_impl are TorchScript code: the modules
compile with torch.jit.script (their kernels are torch.ops.admp_b200.*).
"""

from abc import ABC, abstractmethod
from typing import Dict, Optional, Tuple

import torch

from .utils import TorchConstants


class BaseForceModule(torch.nn.Module, ABC):
    def __init__(self, units_dict: Optional[Dict] = None) -> None:
        torch.nn.Module.__init__(self)
        self.const_lib = TorchConstants(units_dict)

    def forward(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor, ds: torch.Tensor,
                buffer_scales: torch.Tensor, params: Dict[str, torch.Tensor]) -> torch.Tensor:
        _positions, _box, _pairs, _ds, _buffer_scales = self.standardize_input_tensor(
            positions, box, pairs, ds, buffer_scales)
        nf = _positions.size(0)
        _params: Dict[str, torch.Tensor] = {}
        for k, v in params.items():
            _params[k] = v.reshape(nf, -1)
        lc = self.const_lib.length_coeff
        ec = self.const_lib.energy_coeff
        if lc != 1.0:
            _positions = _positions * lc
            _ds = _ds * lc
            if _box is not None:
                _box = _box * lc
        energy = self._forward_impl(_positions, _box, _pairs, _ds, _buffer_scales, _params)
        if ec != 1.0:
            energy = energy / ec
        return energy

    @abstractmethod
    def _forward_impl(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor,
                      ds: torch.Tensor, buffer_scales: torch.Tensor,
                      params: Dict[str, torch.Tensor]) -> torch.Tensor:
        """Energy of standardised (nframes, ...) inputs."""

    def standardize_input_tensor(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor,
                                 ds: torch.Tensor, buffer_scales: torch.Tensor
                                 ) -> Tuple[torch.Tensor, Optional[torch.Tensor], torch.Tensor, torch.Tensor,
                                            torch.Tensor]:
        """Shape checks with the reference's messages (base_force.py:175-339)."""
        nframes = 1
        if positions.dim() == 3:
            if positions.size(2) != 3:
                raise ValueError(f"positions must have shape (nframes, natoms, 3), got {positions.shape}")
            nframes = positions.size(0)
        elif positions.dim() == 2:
            if positions.size(1) != 3:
                raise ValueError(f"positions must have shape (natoms, 3), got {positions.shape}")
            positions = positions.unsqueeze(0)
        else:
            raise ValueError(f"positions must be 2D or 3D tensor, got {positions.dim()}D")

        if box is not None:
            if box.dim() == 3:
                if box.size(1) != 3 or box.size(2) != 3:
                    raise ValueError(f"box must have shape (nframes, 3, 3), got {box.shape}")
                if box.size(0) != nframes:
                    raise ValueError(f"box is expected to have {nframes} frame(s), got {box.size(0)}")
            elif box.dim() == 2:
                if box.size(0) != 3 or box.size(1) != 3:
                    raise ValueError(f"box must have shape (3, 3), got {box.shape}")
                if nframes != 1:
                    raise ValueError(f"box must include a frame dimension when positions has {nframes} frames")
                box = box.unsqueeze(0)
            else:
                raise ValueError(f"box must be 2D or 3D tensor, got {box.dim()}D")

        if pairs.dim() == 3:
            if pairs.size(2) != 2:
                raise ValueError(f"pairs must have shape (nframes, n_pairs, 2), got {pairs.shape}")
            if pairs.size(0) != nframes:
                raise ValueError(f"pairs is expected to have {nframes} frame(s), got {pairs.size(0)}")
        elif pairs.dim() == 2:
            if pairs.size(1) != 2:
                raise ValueError(f"pairs must have shape (n_pairs, 2), got {pairs.shape}")
            if nframes != 1:
                raise ValueError(f"pairs must include a frame dimension when positions has {nframes} frames")
            pairs = pairs.unsqueeze(0)
        else:
            raise ValueError(f"pairs must be 2D or 3D tensor, got {pairs.dim()}D")
        n_pairs = pairs.size(-2)

        if ds.dim() == 2:
            if ds.size(0) != nframes:
                raise ValueError(f"ds is expected to have {nframes} frame(s), got {ds.size(0)}")
            if ds.size(1) != n_pairs:
                raise ValueError(f"ds is expected to have {n_pairs} pairs(s), got {ds.size(1)}")
        elif ds.dim() == 1:
            if ds.size(0) != n_pairs:
                raise ValueError(f"ds is expected to have {n_pairs} pairs(s), got {ds.size(0)}")
            if nframes != 1:
                raise ValueError(f"ds must include a frame dimension when positions has {nframes} frames")
            ds = ds.unsqueeze(0)
        else:
            raise ValueError(f"ds must be 1D or 2D tensor, got {ds.dim()}D")

        if buffer_scales.dim() == 2:
            if buffer_scales.size(0) != nframes:
                raise ValueError(
                    f"buffer_scales is expected to have {nframes} frame(s), got {buffer_scales.size(0)}")
            if buffer_scales.size(1) != n_pairs:
                raise ValueError(
                    f"buffer_scales is expected to have {n_pairs} pairs(s), got {buffer_scales.size(1)}")
        elif buffer_scales.dim() == 1:
            if buffer_scales.size(0) != n_pairs:
                raise ValueError(
                    f"buffer_scales is expected to have {n_pairs} pairs(s), got {buffer_scales.size(0)}")
            if nframes != 1:
                raise ValueError(
                    f"buffer_scales must include a frame dimension when positions has {nframes} frames")
            buffer_scales = buffer_scales.unsqueeze(0)
        else:
            raise ValueError(f"buffer_scales must be 1D or 2D tensor, got {buffer_scales.dim()}D")
        return positions, box, pairs, ds, buffer_scales


def prep_float(t: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
    """Contiguous tensor of the compute dtype (autograd-preserving)."""
    if t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()
