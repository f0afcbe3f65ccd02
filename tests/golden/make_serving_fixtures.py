"""Oracle fixtures for large serving requests (5,000-20,000 atoms) whose
automatic meshes have large prime factors: K = 59, 73, 79 (prime) for PME
requests and K = 67, 71 (prime), 74 = 2 x 37 for QEq waters.

Run from the repository root:  ``python tests/golden/make_serving_fixtures.py``
(CPU only; it runs the NumPy oracle, which tests/test_oracle.py pins to the
reference's own outputs).  The requests are rebuilt from their seeds at test
time, so each case stores only checks that do not grow with the system:
the energy, the forces (and QEq charges) of 256 seeded sample atoms, and
four seeded random projections of the whole force (and charge) vector.
"""
from __future__ import annotations

import math
import os
import sys
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
for p in (REPO, os.path.join(REPO, "torch-admp_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

RC, ETHRESH = 6.0, 5e-4
# (kind, atoms or molecules, seed): meshes 79, 73, 59 (PME) and 74, 71, 67 (QEq)
CASES = [("pme", 19990, 11), ("pme", 16000, 12), ("pme", 8400, 13),
         ("qeq", 5546, 14), ("qeq", 4906, 15), ("qeq", 4117, 16)]
NSAMPLE, NPROJ = 256, 4


def request(kind, n, seed):
    """The request of one case: PME with n balanced +-1 charges, or QEq on n
    waters, cubic box at 0.1 atoms per cubic Angstrom (as serving_stream)."""
    from admp_b200 import synthetic
    if kind == "pme":
        L = (n / 0.1) ** (1.0 / 3.0)
        pos, box, q = synthetic.random_charges_system(n, L, seed, balanced=True)
        return synthetic.Request(seed, "pme", 0.0, pos, box, charges=q)
    L = (3 * n / 0.1) ** (1.0 / 3.0)
    pos, box, chi, hard, eta, _ = synthetic.water_system(n, L, seed)
    return synthetic.Request(seed, "qeq", 0.0, pos, box, chi=chi, hardness=hard, eta=eta)


def checks(n_atoms, seed):
    """Sample atom indices and projection vectors of a case."""
    rng = np.random.default_rng(seed + 1000)
    idx = np.sort(rng.choice(n_atoms, NSAMPLE, replace=False))
    wf = rng.normal(size=(NPROJ, n_atoms, 3))
    wq = rng.normal(size=(NPROJ, n_atoms))
    return idx, wf, wq


def run_case(case):
    from oracle import admp_oracle as O
    kind, n, seed = case
    r = request(kind, n, seed)
    pos, box = r.pos, r.box
    kappa = O.ewald_kappa(RC, ETHRESH)
    km = O.auto_kmesh(box, kappa, ETHRESH)
    t0 = time.time()
    pairs = O.nblist_pbc_cells(pos, box, RC)
    bs = O.pair_buffer_scales(pairs)
    if kind == "pme":
        q = r.charges
        o = O.coulomb_forces(pos, box, pairs, bs, q, rcut=RC, ethresh=ETHRESH)
        E, F = o["E"], o["forces"]
    else:
        N = pos.shape[0]
        ds = O.pairs_ds(pos, pairs, box)
        s = O.QEqSystem(pos, box, r.chi, r.hardness, r.eta, pairs, ds, bs, rcut=RC, ethresh=ETHRESH)
        q, it = O.solve_linear_cg(s, np.zeros(N), np.ones((1, N)), np.zeros(1), tol=1e-11)
        E, _ = s.energy_grad(q)
        # forces at the solved charges: Coulomb (PME) + damping through the distances
        o = O.coulomb_forces(pos, box, pairs, bs, q, rcut=RC, ethresh=ETHRESH)
        Ed, dds, _, _ = O.damping(q, r.eta, pairs, ds, bs)
        dpd, _ = O.ds_backward(pos, box, pairs, dds)
        F = o["forces"] - dpd
    idx, wf, wq = checks(pos.shape[0], seed)
    out = dict(kind=kind, n=n, seed=seed, natoms=pos.shape[0], kmesh=np.asarray(km), E=E, idx=idx, F_sample=F[idx],
               F_proj=np.einsum("kij,ij->k", wf, F), q_sample=q[idx], q_proj=wq @ q)
    print(f"{kind} n={n} atoms={pos.shape[0]} kmesh={list(km)} E={E:.6f} {time.time() - t0:.1f}s", flush=True)
    return out


def main():
    with ProcessPoolExecutor(max_workers=min(len(CASES), os.cpu_count() or 1)) as ex:
        outs = list(ex.map(run_case, CASES))
    arrays = {}
    for k, o in enumerate(outs):
        for key, v in o.items():
            arrays[f"c{k}_{key}"] = np.asarray(v)
    path = os.path.join(HERE, "serving_large.npz")
    np.savez_compressed(path, ncases=len(CASES), **arrays)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.1f} KB)")


if __name__ == "__main__":
    main()
