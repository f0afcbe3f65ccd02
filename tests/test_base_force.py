"""BaseForceModule boundary on CPU (the reference's test_base_force.py cases,
restated): shape standardisation of single and batched inputs, a ValueError
for every malformed input, forward with and without a box, unit handling."""
from typing import Dict, Optional

import numpy as np
import pytest
import torch

from admp_b200.base_force import BaseForceModule

F64 = torch.float64


class _Probe(BaseForceModule):
    """Minimal subclass: energy = sum of the (unit-converted) positions and ds."""

    def _forward_impl(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor,
                      ds: torch.Tensor, buffer_scales: torch.Tensor, params: Dict[str, torch.Tensor]) -> torch.Tensor:
        return positions.sum(dim=(1, 2)) + ds.sum(dim=1)


def _single(rng, n=10, p=20):
    return (torch.tensor(rng.random((n, 3)), dtype=F64), torch.eye(3, dtype=F64),
            torch.tensor(rng.integers(0, n, (p, 2))), torch.tensor(rng.normal(size=p), dtype=F64),
            torch.ones(p, dtype=F64))


def _batched(rng, nf=5, n=10, p=20):
    return (torch.tensor(rng.random((nf, n, 3)), dtype=F64), torch.eye(3, dtype=F64).repeat(nf, 1, 1),
            torch.tensor(rng.integers(0, n, (nf, p, 2))), torch.tensor(rng.normal(size=(nf, p)), dtype=F64),
            torch.ones(nf, p, dtype=F64))


def test_standardize_single_and_batched():
    rng = np.random.default_rng(1024)
    m = _Probe()
    pos, box, pairs, ds, bs = m.standardize_input_tensor(*_single(rng))
    assert pos.shape == (1, 10, 3) and box.shape == (1, 3, 3) and pairs.shape == (1, 20, 2)
    assert ds.shape == (1, 20) and bs.shape == (1, 20)
    pos, box, pairs, ds, bs = m.standardize_input_tensor(*_batched(rng))
    assert pos.shape == (5, 10, 3) and box.shape == (5, 3, 3) and ds.shape == (5, 20)


def _bad_cases(rng):
    s, b = _single(rng), _batched(rng)
    return {
        "positions 2 columns": (s[0][:, :2],) + s[1:],
        "positions 3D wrong last dim": (torch.zeros(5, 10, 2, dtype=F64),) + b[1:],
        "positions 4D": (torch.zeros(1, 5, 10, 3, dtype=F64),) + b[1:],
        "box 3D wrong shape": (b[0], torch.zeros(5, 3, 2, dtype=F64)) + b[2:],
        "box frame mismatch": (b[0], torch.eye(3, dtype=F64).repeat(4, 1, 1)) + b[2:],
        "box 2D wrong shape": (s[0], torch.zeros(3, 2, dtype=F64)) + s[2:],
        "box 2D with frames": (b[0], torch.eye(3, dtype=F64)) + b[2:],
        "box 1D": (s[0], torch.ones(3, dtype=F64)) + s[2:],
        "pairs 3D wrong last dim": b[:2] + (torch.zeros(5, 20, 3, dtype=torch.long),) + b[3:],
        "pairs frame mismatch": b[:2] + (b[2][:4],) + b[3:],
        "pairs 2D with frames": b[:2] + (s[2],) + b[3:],
        "pairs 1D": s[:2] + (torch.zeros(20, dtype=torch.long),) + s[3:],
        "ds frame mismatch": b[:3] + (b[3][:4],) + b[4:],
        "ds pair mismatch": b[:3] + (b[3][:, :19],) + b[4:],
        "ds 1D with frames": b[:3] + (s[3],) + b[4:],
        "ds 3D": s[:3] + (s[3].reshape(1, 1, -1),) + s[4:],
        "buffer_scales frame mismatch": b[:4] + (b[4][:4],),
        "buffer_scales pair mismatch": b[:4] + (b[4][:, :19],),
        "buffer_scales 1D with frames": b[:4] + (s[4],),
        "buffer_scales 3D": s[:4] + (s[4].reshape(1, 1, -1),),
        "ds 1D pair mismatch": s[:3] + (s[3][:19],) + s[4:],
        "buffer_scales 1D pair mismatch": s[:4] + (s[4][:19],),
    }


@pytest.mark.parametrize("case", list(_bad_cases(np.random.default_rng(0))))
def test_malformed_inputs_raise_value_error(case):
    args = _bad_cases(np.random.default_rng(1024))[case]
    with pytest.raises(ValueError):
        _Probe().standardize_input_tensor(*args)


def test_forward_with_and_without_box_and_units():
    rng = np.random.default_rng(1024)
    pos, box, pairs, ds, bs = _single(rng)
    params = {"charge": torch.tensor(rng.normal(size=10), dtype=F64)}
    e = _Probe()(pos, box, pairs, ds, bs, params)
    assert torch.allclose(e, (pos.sum() + ds.sum()).reshape(1))
    assert torch.allclose(_Probe()(pos, None, pairs, ds, bs, params), e)
    # positions / ds in nm are multiplied by 10 before the energy; the energy in kJ/mol is divided by eV -> kJ/mol
    m = _Probe(units_dict={"length": "nm", "energy": "kJ/mol"})
    assert m.const_lib.length_coeff == 10.0
    ec = m.const_lib.energy_coeff
    assert ec == pytest.approx(1.0 / 96.485, rel=1e-3)
    assert torch.allclose(m(pos, box, pairs, ds, bs, params), 10.0 * e / ec)


def test_unknown_units_raise():
    with pytest.raises(ValueError, match="Unknown length unit"):
        _Probe(units_dict={"length": "furlong"})
    with pytest.raises(ValueError, match="Unknown energy unit"):
        _Probe(units_dict={"energy": "erg"})
