"""Reciprocal PME energy and forces for every mesh length from 17 to 80 on each
axis, against the oracle's NumPy FFT (pme.py:351-446, recip.py:146-308).

The reference's automatic mesh rule (pme.py:390-392) produces any length in
this range, so every radix path of the shared-memory FFT runs here: powers of
two, radix 3 / 5 stages, the folded odd-prime stages on their own (17, 79) and
after other stages (74 = 2 * 37, 77 = 7 * 11, 49 = 7 * 7).  All 64 systems go
through one batched call, each with its own mesh, so the per-system packing of
meshes and spectra is exercised as well.  Tolerances: FP64 1e-10 relative
energy / 1e-9 relative force; FP32 1e-5 / 1e-4."""
import numpy as np
import pytest
import torch

from oracle import admp_oracle as O

pytestmark = pytest.mark.gpu

LENGTHS = list(range(17, 81))
N_ATOMS = 48
KAPPA = 0.3


def _cases():
    rng = np.random.default_rng(2024)
    nl = len(LENGTHS)
    kmesh = [(LENGTHS[i], LENGTHS[(i + 21) % nl], LENGTHS[(i + 43) % nl]) for i in range(nl)]
    pos, box, q = [], [], []
    for _ in range(nl):
        b = np.diag(rng.uniform(16.0, 24.0, 3))
        b[1, 0], b[2, 0], b[2, 1] = rng.uniform(-2.0, 2.0, 3)   # triclinic, lower triangular
        frac = rng.uniform(0.0, 1.0, (N_ATOMS, 3))
        c = rng.normal(size=N_ATOMS)
        box.append(b)
        pos.append(frac @ b)
        q.append(c - c.mean())
    return kmesh, np.stack(pos), np.stack(box), np.stack(q)


@pytest.fixture(scope="module")
def sweep():
    kmesh, pos, box, q = _cases()
    ref = [O.pme_recip(pos[f], box[f], q[f], KAPPA, kmesh[f]) for f in range(len(kmesh))]
    return kmesh, pos, box, q, ref


@pytest.mark.parametrize("dtype,etol,ftol", [(torch.float64, 1e-10, 1e-9), (torch.float32, 1e-5, 1e-4)])
def test_recip_every_mesh_length(cuda, sweep, dtype, etol, ftol):
    from admp_b200 import ops
    kmesh, pos, box, q, ref = sweep
    nf = len(kmesh)
    tp = torch.tensor(pos, dtype=dtype, device=cuda)
    tb = torch.tensor(box, dtype=dtype, device=cuda)
    tq = torch.tensor(q, dtype=dtype, device=cuda)
    pairs = torch.zeros(nf, 0, 2, dtype=torch.int64, device=cuda)
    ds = torch.zeros(nf, 0, dtype=dtype, device=cuda)
    bs = torch.zeros(nf, 0, dtype=dtype, device=cuda)
    _, comps, g = ops.coulomb_pbc(tp, tb, pairs, ds, bs, tq, KAPPA, kmesh, float(O.DIELECTRIC), rspace=False,
                                  kspace=True, slab=False, axis=2, need_grad=True)
    E = comps[:, 1].cpu().numpy()
    dpos = g["pos"].double().cpu().numpy()
    bad = []
    for f in range(nf):
        e_err = abs(E[f] - ref[f]["E"]) / abs(ref[f]["E"])
        f_err = np.abs(dpos[f] - ref[f]["dpos"]).max() / np.abs(ref[f]["dpos"]).max()
        if not (e_err < etol and f_err < ftol):
            bad.append((kmesh[f], e_err, f_err))
    assert not bad, bad
