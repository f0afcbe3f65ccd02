"""Constants, units and small helpers (mirrors torch_admp.utils, utils.py:21-283).

Unit handling follows the reference: inputs in the user's length/energy
units are converted to Angstrom / eV (ASE conventions, CODATA 2014 values as
used by ``ase.units``) before the kernels run.
"""

from typing import Dict, List, Optional

import numpy as np
import torch
from scipy import constants as _C

# vacuum permittivity in e^2 / (eV * Angstrom) and k_e = 1/(4 pi eps0)  (utils.py:265-278)
EPSILON = _C.epsilon_0 / _C.elementary_charge * _C.angstrom
DIELECTRIC = 1.0 / (4.0 * np.pi * EPSILON)

# ASE unit table (ase/units.py, CODATA 2014) for the units the reference accepts
_CODATA2014_e = 1.6021766208e-19
_CODATA2014_NA = 6.022140857e23
_ASE_UNITS = {
    "Ang": 1.0, "Angstrom": 1.0, "nm": 10.0, "Bohr": 0.52917721067, "m": 1e10,
    "eV": 1.0, "J": 1.0 / _CODATA2014_e, "kJ": 1000.0 / _CODATA2014_e, "kcal": 4184.0 / _CODATA2014_e,
    "Hartree": 27.211386024367243, "Ry": 13.605693012183622, "mol": _CODATA2014_NA,
}


class TorchConstants(torch.nn.Module):
    """Unit coefficients and constants -- utils.py:213-283."""

    def __init__(self, units_dict: Optional[Dict] = None):
        super().__init__()
        self.pi = float(np.pi)
        self.sqrt_pi = float(np.sqrt(np.pi))
        units_dict = units_dict or {}
        user_energy = units_dict.get("energy", "eV")
        user_length = units_dict.get("length", "Ang")
        if user_length not in _ASE_UNITS:
            raise ValueError(f"Unknown length unit: {user_length}")
        if user_energy == "kJ/mol":
            energy_coeff = _ASE_UNITS["kJ"] / _ASE_UNITS["mol"]
        elif user_energy in _ASE_UNITS:
            energy_coeff = _ASE_UNITS[user_energy]
        else:
            raise ValueError(f"Unknown energy unit: {user_energy}")
        self.length_coeff = float(_ASE_UNITS[user_length])
        self.energy_coeff = float(energy_coeff)
        self.epsilon = float(EPSILON)
        self.dielectric = float(DIELECTRIC)


def safe_inverse(x: torch.Tensor, threshold: float = 1e-8) -> torch.Tensor:
    """1/x where |x| > threshold else 0 -- utils.py:66-82."""
    return torch.where(x.abs() > threshold, 1 / x, torch.zeros_like(x))


def pair_buffer_scales(pairs: torch.Tensor) -> torch.Tensor:
    """1 if i < j else 0 -- utils.py:21-41."""
    return (pairs[:, 0] < pairs[:, 1]).to(torch.long)


def vector_projection_coeff_matrix(constraint_matrix: torch.Tensor) -> torch.Tensor:
    """C^T (C C^T)^-1 -- utils.py:152-172."""
    ct = constraint_matrix.transpose(0, 1)
    return ct @ torch.inverse(constraint_matrix @ ct)


def vector_projection(vector_in: torch.Tensor, constraint_matrix: torch.Tensor,
                      constraint_vector: Optional[torch.Tensor] = None) -> torch.Tensor:
    """x + C^T (C C^T)^-1 (b - C x) -- utils.py:175-210."""
    if constraint_vector is None:
        constraint_vector = torch.zeros(constraint_matrix.shape[0], device=vector_in.device,
                                        dtype=vector_in.dtype)
    coeff = vector_projection_coeff_matrix(constraint_matrix)
    residual = constraint_vector.reshape(-1, 1) - constraint_matrix @ vector_in.reshape(-1, 1)
    return (vector_in.reshape(-1, 1) + coeff @ residual).reshape(-1)


def calc_grads(t_out: torch.Tensor, t_in: torch.Tensor) -> torch.Tensor:
    """d(sum t_out)/d t_in -- utils.py:85-112."""
    assert t_in.requires_grad, "Input tensor requires grad"
    grad_outputs: List[Optional[torch.Tensor]] = [torch.ones_like(t_out)]
    g = torch.autograd.grad([t_out], [t_in], grad_outputs=grad_outputs, retain_graph=True)[0]
    assert g is not None
    return g


def calc_pgrads(t_out: torch.Tensor, t_in: torch.Tensor, constraint_matrix: torch.Tensor,
                coeff_matrix: torch.Tensor) -> torch.Tensor:
    """Projected gradient -- utils.py:116-149."""
    g = calc_grads(t_out, t_in).reshape(-1, 1)
    residual = -constraint_matrix @ g
    return (g + coeff_matrix @ residual).reshape(-1)
