"""CoulombForceModule on B200 kernels (drop-in for torch_admp.pme, pme.py:24-683).

Constructor arguments, validation messages, energy components
(``real_energy`` ... ``slab_corr_energy``), ``_kmesh``, ``kappa``,
``get_rcut`` / ``get_sel`` and ``setup_ewald_parameters`` follow the
reference.  The energy and every gradient come from the CUDA library.
"""

import math
from typing import Dict, List, Optional, Tuple, Union

import numpy as np
import torch
from scipy import special

from . import _lib as L
from .base_force import BaseForceModule, prep_float

L.load_torch_ops()  # torch.ops.admp_b200.* used by the forward passes


def _auto_kmesh(box_cpu: torch.Tensor, kappa: float, ethresh: float, kmesh, spacing) -> List[List[int]]:
    """Mesh per frame: explicit kmesh, ceil(L/spacing) or ceil(2 kappa L / (3 ethresh^0.2)) -- pme.py:380-392."""
    nf = box_cpu.shape[0]
    if kmesh is not None:
        return [list(int(k) for k in kmesh)] * nf
    diag = torch.diagonal(box_cpu, dim1=1, dim2=2)
    if spacing is not None:
        sp = torch.as_tensor(spacing, dtype=diag.dtype)
        km = torch.ceil(diag / sp).to(torch.long)
    else:
        km = torch.ceil(2 * kappa * diag / (3.0 * ethresh ** (1.0 / 5.0))).to(torch.long)
    return km.tolist()


class CoulombForceModule(BaseForceModule):
    """Coulomb energy with PME (pme.py:24-561)."""

    # TorchScript attribute types (the mesh / spacing settings as lists, empty = automatic)
    _kmesh_fixed: List[int]
    _spacing_list: List[float]

    def __init__(self, rcut: float, ethresh: float = 1e-5, kspace: bool = True, rspace: bool = True,
                 slab_corr: bool = False, slab_axis: int = 2, units_dict: Optional[Dict] = None,
                 sel: Optional[list] = None, kappa: Optional[float] = None,
                 spacing: Union[List[float], float, None] = None, kmesh: Union[List[int], int, None] = None) -> None:
        BaseForceModule.__init__(self, units_dict)
        if rcut <= 0.0:
            raise ValueError(f"rcut must be positive, got {rcut}")
        if ethresh <= 0.0:
            raise ValueError(f"ethresh must be positive, got {ethresh}")
        if slab_axis not in (0, 1, 2):
            raise ValueError(f"slab_axis must be 0/1/2, got {slab_axis}")
        self.kspace_flag = kspace
        if kappa is not None:
            if kappa <= 0.0:
                raise ValueError(f"kappa must be positive, got {kappa}")
            self.kappa = kappa
        elif self.kspace_flag:
            self.kappa = math.sqrt(-math.log(2 * ethresh)) / rcut / self.const_lib.length_coeff
        else:
            self.kappa = 0.0
        self.ethresh = ethresh
        if kmesh is not None:
            if isinstance(kmesh, int):
                kmesh = [kmesh, kmesh, kmesh]
            for i, k in enumerate(kmesh):
                if k <= 0:
                    raise ValueError(f"kmesh values must be positive, got kmesh[{i}] = {k}")
            self.kmesh = [int(k) for k in kmesh]
        else:
            self.kmesh = None
        self._kmesh = torch.zeros(3, dtype=torch.long)
        if spacing is not None:
            if isinstance(spacing, float):
                spacing = [spacing, spacing, spacing]
            for i, s in enumerate(spacing):
                if s <= 0:
                    raise ValueError(f"spacing values must be positive, got spacing[{i}] = {s}")
            self.spacing = [float(s) for s in spacing]
        else:
            self.spacing = None
        self._kmesh_fixed = list(self.kmesh) if self.kmesh is not None else []
        self._spacing_list = list(self.spacing) if self.spacing is not None else []
        self.kappa = float(self.kappa)
        self.ethresh = float(ethresh)
        self.rspace_flag = rspace
        self.slab_corr_flag = slab_corr
        self.slab_axis = slab_axis
        z = torch.zeros(1, dtype=torch.float64)
        self.real_energy = z
        self.reciprocal_energy = z
        self.self_energy = z
        self.non_neutral_energy = z
        self.slab_corr_energy = z
        self.pme_order = 6
        self.rcut = rcut
        self.sel = sel

    def get_rcut(self) -> float:
        return self.rcut

    def get_sel(self) -> Optional[list]:
        return self.sel

    def kmesh_for(self, box: torch.Tensor) -> List[List[int]]:
        """Mesh sizes used for each frame of ``box`` (nf, 3, 3)."""
        if self.kmesh is not None:
            return [list(self.kmesh)] * box.shape[0]
        return _auto_kmesh(box.detach().to("cpu", torch.float64), self.kappa, self.ethresh, None, self.spacing)

    def _forward_impl(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor,
                      ds: torch.Tensor, buffer_scales: torch.Tensor,
                      params: Dict[str, torch.Tensor]) -> torch.Tensor:
        nf, na = positions.size(0), positions.size(1)
        if not positions.is_cuda:
            raise ValueError("admp_b200 runs on CUDA tensors (there is no CPU path); positions are on "
                             + str(positions.device))
        dt = positions.dtype
        charges = params["charge"].reshape(nf, na).to(dt)
        bs = buffer_scales.to(dt)
        dsc = ds.to(dt)
        ke = self.const_lib.dielectric
        if box is None:
            return torch.ops.admp_b200.coulomb_obc(pairs, dsc, bs, charges, ke)
        out = torch.ops.admp_b200.coulomb_pbc(positions.to(dt), box.to(dt), pairs, dsc, bs, charges, self.kappa,
                                              self._kmesh_fixed, self._spacing_list, self.ethresh, ke,
                                              self.rspace_flag, self.kspace_flag, self.slab_corr_flag,
                                              self.slab_axis)
        c = out[1].to(dt)
        if self.kspace_flag:
            self._kmesh = out[2][-1]
            self.reciprocal_energy = c[:, 1]
            self.self_energy = c[:, 2]
            self.non_neutral_energy = c[:, 3]
        if self.rspace_flag:
            self.real_energy = c[:, 0]
        if self.slab_corr_flag:
            self.slab_corr_energy = c[:, 4]
        return out[0]


def setup_ewald_parameters(rcut: float, box=None, threshold: float = 1e-5, spacing: Optional[float] = None,
                           method: str = "openmm") -> Tuple[float, int, int, int]:
    """kappa and mesh sizes -- pme.py:564-658 (host-side scalar arithmetic)."""
    if rcut <= 0.0:
        raise ValueError(f"rcut must be positive, got {rcut}")
    if box is None:
        return 0.1, 1, 1, 1
    if isinstance(box, torch.Tensor):
        box = box.detach().cpu().numpy()
    box = np.asarray(box)
    assert np.inner(box[0], box[1]) == 0.0, "Only orthogonal box is supported currently."
    assert np.inner(box[0], box[2]) == 0.0, "Only orthogonal box is supported currently."
    assert np.inner(box[1], box[2]) == 0.0, "Only orthogonal box is supported currently."
    if method == "openmm":
        kappa = np.sqrt(-np.log(2 * threshold)) / rcut
        kx = np.ceil(2 * kappa * box[0, 0] / (3.0 * threshold ** (1.0 / 5.0))).astype(int)
        ky = np.ceil(2 * kappa * box[1, 1] / (3.0 * threshold ** (1.0 / 5.0))).astype(int)
        kz = np.ceil(2 * kappa * box[2, 2] / (3.0 * threshold ** (1.0 / 5.0))).astype(int)
    elif method == "gromacs":
        assert spacing is not None, "Spacing must be provided for gromacs method."
        kappa = 5.0
        i = 0
        while special.erfc(kappa * rcut) > threshold:
            i += 1
            kappa *= 2
        n = i + 60
        low, high = 0.0, kappa
        for _ in range(n):
            kappa = (low + high) / 2
            if special.erfc(kappa * rcut) > threshold:
                low = kappa
            else:
                high = kappa
        kx = np.ceil(box[0, 0] / spacing).astype(int)
        ky = np.ceil(box[1, 1] / spacing).astype(int)
        kz = np.ceil(box[2, 2] / spacing).astype(int)
    else:
        raise ValueError(f"Invalid method: {method}." "Valid methods: 'openmm', 'gromacs'")
    return kappa, kx, ky, kz
