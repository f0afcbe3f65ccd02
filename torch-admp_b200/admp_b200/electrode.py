"""Constant-potential / constant-charge electrodes on B200 kernels
(drop-in for torch_admp.electrode, electrode.py:21-560).

The electrode sub-problem is solved by the GPU projected CG (or the dense KKT
path for method="matinv"); the electrode potential (the b-vector) and the
final energy and forces come from the same CUDA energy kernels through
autograd, as in the reference.
"""
from __future__ import annotations

from typing import List, Optional, Tuple, Union

import numpy as np
import torch

from .qeq import QEqForceModule, matinv_optimize, pgrad_optimize
from .utils import calc_grads


class PolarizableElectrode(QEqForceModule):
    """Polarizable electrode model (electrode.py:21-133)."""

    def __init__(self, rcut: float, ethresh: float = 1e-5, **kwargs) -> None:
        super().__init__(rcut, ethresh, **kwargs)

    def calc_coulomb_potential(self, electrode_mask, positions, box, eta, charges, pairs, ds, buffer_scales):
        """dE/dq with electrode charges zeroed (electrode.py:49-84)."""
        if electrode_mask is None:
            modified = charges.detach().clone()
        else:
            modified = torch.where(electrode_mask == 0, charges.detach(), torch.zeros_like(charges))
        modified.requires_grad_(True)
        energy = self.forward(positions, box, pairs, ds, buffer_scales,
                              {"charge": modified, "eta": eta, "hardness": torch.zeros_like(eta),
                               "chi": torch.zeros_like(eta)})
        assert energy.size(0) == 1
        return calc_grads(energy[0], modified), energy

    def coulomb_calculator(self, positions, box, charges, eta, pairs, ds, buffer_scales, efield=None):
        """Energy and forces of the full system (electrode.py:87-133)."""
        _energy = self.forward(positions, box, pairs, ds, buffer_scales,
                               {"charge": charges, "eta": eta, "hardness": torch.zeros_like(eta),
                                "chi": torch.zeros_like(eta)})
        assert _energy.size(0) == 1
        energy = _energy[0]
        if not positions.requires_grad:
            raise ValueError("positions must require grad to compute forces; call positions.requires_grad_(True)")
        forces = -calc_grads(energy, positions)
        if efield is not None:
            ef = torch.zeros(3, dtype=positions.dtype, device=positions.device)
            ef[self.slab_axis] = efield[self.slab_axis]
            forces = forces + charges.unsqueeze(1) * ef
            energy = energy + torch.sum(ef.reshape(1, 3) * charges.unsqueeze(1) * positions)
        return energy, forces


class LAMMPSElectrodeConstraint:
    """LAMMPS-style electrode constraint (electrode.py:136-200)."""

    def __init__(self, indices: Union[List[int], np.ndarray], mode: str, value: float, eta: float,
                 chi: float = 0.0, hardness: float = 0.0, ffield: bool = False) -> None:
        self.indices = np.array(indices, dtype=int)
        assert self.indices.ndim == 1
        self.mode = mode
        assert mode in ["conp", "conq"], f"mode {mode} not supported"
        self.value = value
        self.eta = eta
        self.hardness = hardness
        self.chi = chi
        self.ffield = ffield


def setup_from_lammps(n_atoms: int, constraint_list: List[LAMMPSElectrodeConstraint], symm: bool = False,
                      device: Union[str, torch.device] = "cuda", dtype: torch.dtype = torch.float64):
    """Electrode masks, widths and constraints from LAMMPS-like definitions (electrode.py:203-285)."""
    mask = np.zeros(n_atoms, dtype=bool)
    eta = np.zeros(n_atoms)
    chi = np.zeros(n_atoms)
    hardness = np.zeros(n_atoms)
    cmat, cval, ffm, ffp = [], [], [], []
    for c in constraint_list:
        mask[c.indices] = True
        eta[c.indices] = 1 / c.eta * np.sqrt(2) / 2.0
        chi[c.indices] = c.chi
        hardness[c.indices] = c.hardness
        if c.mode == "conq":
            if symm:
                raise AttributeError("symm should be False for conq, user can implement symm by conq")
            if c.ffield:
                raise AttributeError("ffield with conq has not been implemented yet")
            row = np.zeros((1, n_atoms))
            row[0, c.indices] = 1.0
            cmat.append(row)
            cval.append(c.value)
        if c.mode == "conp":
            chi[c.indices] -= c.value
        if c.ffield:
            row = np.zeros((1, n_atoms))
            row[0, c.indices] = 1.0
            ffm.append(row)
            ffp.append(c.value)
    if len(ffm) == 0:
        ff_mask, ff_pot = None, None
    elif len(ffm) == 2:
        ff_mask = torch.tensor(np.concatenate(ffm, axis=0), dtype=torch.bool, device=device)
        ff_pot = torch.tensor(np.array(ffp), dtype=dtype, device=device)
    else:
        raise AttributeError("number of ffield group should be 0 or 2")
    if symm:
        cmat.append(np.ones((1, n_atoms)))
        cval.append(0.0)
    if cmat:
        C = torch.tensor(np.concatenate(cmat, axis=0)[:, mask], dtype=dtype, device=device)
        b = torch.tensor(np.array(cval), dtype=dtype, device=device)
    else:
        C = torch.zeros((0, int(mask.sum())), dtype=dtype, device=device)
        b = torch.zeros(0, dtype=dtype, device=device)
    t = lambda a: torch.tensor(a, dtype=dtype, device=device)  # noqa: E731
    return (torch.tensor(mask, device=device), t(eta), t(chi), t(hardness), C, b, ff_mask, ff_pot)


def finite_field_add_chi(positions, box, ffield_electrode_mask, ffield_potential, slab_axis: int = 2):
    """Finite-field potential on the electrode atoms (electrode.py:288-336)."""
    assert positions.dim() == 2 and box.dim() == 2
    assert ffield_potential.dim() == 1 and ffield_electrode_mask.dim() == 2
    assert ffield_electrode_mask.shape[0] == 2 and positions.shape[1] == 3
    assert ffield_electrode_mask.shape[1] == positions.shape[0]
    assert ffield_potential.shape[0] == 2
    first, second = ffield_electrode_mask[0], ffield_electrode_mask[1]
    drop = ffield_potential[0] - ffield_potential[1]
    mx0 = torch.max(positions[first, slab_axis])
    mx1 = torch.max(positions[second, slab_axis])
    lz = box[slab_axis][slab_axis]
    z = positions[:, slab_axis] / lz
    if mx0 > mx1:
        offset, efield = z, -drop / lz
    else:
        offset, efield = -z, drop / lz
    potential = drop * offset
    return potential[first | second], efield


def infer(calculator: PolarizableElectrode, positions, box, charges, pairs, ds, buffer_scales, electrode_mask, eta,
          chi, hardness, constraint_matrix, constraint_vals, ffield_electrode_mask, ffield_potential,
          method: str = "lbfgs"):
    """Electrode charge solve, then energy and forces (electrode.py:339-453)."""
    _pos, _box, _pairs, _ds, _bs = calculator.standardize_input_tensor(positions, box, pairs, ds, buffer_scales)
    assert _pos.shape[0] == 1
    assert _box is not None
    _q, efield = charge_optimization(calculator, _pos[0], _box[0], charges, _pairs[0], _ds[0], _bs[0], electrode_mask,
                                     eta, chi, hardness, constraint_matrix, constraint_vals, ffield_electrode_mask,
                                     ffield_potential, method)
    q_opt = charges.detach().clone()
    q_opt[electrode_mask] = _q.detach().to(q_opt.dtype)
    energy, forces = calculator.coulomb_calculator(positions=positions, box=box, charges=q_opt, eta=eta, pairs=pairs,
                                                   ds=ds, buffer_scales=buffer_scales, efield=efield)
    return energy, forces, q_opt


def charge_optimization(calculator: PolarizableElectrode, positions, box, charges, pairs, ds, buffer_scales,
                        electrode_mask, eta, chi, hardness, constraint_matrix, constraint_vals,
                        ffield_electrode_mask, ffield_potential, method: str = "lbfgs"):
    """QEq on the electrode sub-system (electrode.py:456-560)."""
    device, dtype = positions.device, positions.dtype
    if electrode_mask.sum() == 0:
        return charges[electrode_mask], None
    if ffield_electrode_mask is not None and calculator.slab_corr:
        raise ValueError("Slab correction and finite field cannot be used together.")
    chi_elec, _ = calculator.calc_coulomb_potential(electrode_mask, positions, box, eta, charges, pairs, ds,
                                                    buffer_scales)
    chi_t = (chi + chi_elec.detach())[electrode_mask]
    efield = None
    if ffield_electrode_mask is not None:
        chi_ff, _ef = finite_field_add_chi(positions.detach(), box.detach(), ffield_electrode_mask, ffield_potential,
                                           calculator.slab_axis)
        chi_t = chi_t + chi_ff
        efield = torch.zeros(3, dtype=dtype, device=device)
        efield[calculator.slab_axis] = _ef
    pair_mask = electrode_mask[pairs[:, 0]] & electrode_mask[pairs[:, 1]]
    idx = torch.nonzero(electrode_mask).reshape(-1)
    mapping = torch.zeros(electrode_mask.size(0), dtype=torch.long, device=device)
    mapping[idx] = torch.arange(idx.numel(), device=device, dtype=torch.long)
    sub_pairs = torch.stack([mapping[pairs[pair_mask][:, 0]], mapping[pairs[pair_mask][:, 1]]], dim=1)
    kw = dict(module=calculator, positions=positions.detach()[electrode_mask], box=box.detach(), chi=chi_t,
              hardness=hardness[electrode_mask], eta=eta[electrode_mask], pairs=sub_pairs,
              ds=ds.detach()[pair_mask], buffer_scales=buffer_scales[pair_mask],
              constraint_matrix=constraint_matrix if constraint_matrix is not None and constraint_matrix.shape[0] > 0
              else None,
              constraint_vals=constraint_vals if constraint_matrix is not None and constraint_matrix.shape[0] > 0
              else None)
    if method == "matinv":
        _e, q = matinv_optimize(**kw)
    else:
        _e, q = pgrad_optimize(q0=charges.detach()[electrode_mask].reshape(-1), method=method, reinit_q=True, **kw)
    return q, efield
