"""Large serving requests against the oracle: 8,400-20,000 atoms on the
reference's automatic meshes K = 59, 73, 79 (prime, PME requests) and
K = 67, 71 (prime), 74 = 2 x 37 (QEq waters), so every prime-length FFT
stage of those sizes runs.  The oracle's energies, sampled forces / charges
and random projections of the whole vectors are in
tests/golden/serving_large.npz (make_serving_fixtures.py)."""
import os
import sys

import numpy as np
import pytest
import torch

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def _cases():
    from make_serving_fixtures import CASES, checks, request
    d = golden("serving_large")
    out = []
    for k, (kind, n, seed) in enumerate(CASES):
        ref = {key: d[f"c{k}_{key}"] for key in ("E", "idx", "F_sample", "F_proj", "q_sample", "q_proj", "kmesh",
                                                 "natoms")}
        out.append((request(kind, n, seed), ref, checks(int(ref["natoms"]), seed)))
    return out


@pytest.fixture(scope="module")
def large_cases():
    return _cases()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_large_requests_match_oracle(cuda, large_cases, dtype):
    from admp_b200.serving import ServingEngine, auto_kmesh
    reqs = [c[0] for c in large_cases]
    fp64 = dtype == torch.float64
    eng = ServingEngine(dtype=dtype, max_atoms=200_000, max_slots=16, mesh_budget=4_000_000,
                        tol=1e-11 if fp64 else 1e-7, max_iter=1000)
    res = {r.rid: r for r in eng.run(reqs, arrivals=False)}
    torch.cuda.synchronize()
    for req, ref, (idx, wf, wq) in large_cases:
        assert auto_kmesh(np.diagonal(req.box), eng.kappa, eng.ethresh) == ref["kmesh"].tolist()
        out = res[req.rid]
        assert out.status == 0
        F = np.asarray(out.forces, dtype=np.float64)
        fs = F[ref["idx"]]
        fscale = np.abs(ref["F_sample"]).max()
        ferr = np.abs(fs - ref["F_sample"]).max() / fscale
        perr = np.abs(np.einsum("kij,ij->k", wf, F) - ref["F_proj"]).max() / np.abs(ref["F_proj"]).max()
        eerr = abs(out.energy - float(ref["E"])) / abs(float(ref["E"]))
        if fp64:
            assert eerr < 1e-9 and ferr < 1e-8 and perr < 1e-8, (req.kind, req.natoms, eerr, ferr, perr)
        else:
            assert eerr < 1e-5 and ferr < 1e-4 and perr < 1e-4, (req.kind, req.natoms, eerr, ferr, perr)
        if req.kind == "qeq":
            q = np.asarray(out.charges, dtype=np.float64)
            qerr = np.abs(q[ref["idx"]] - ref["q_sample"]).max()
            qperr = np.abs(wq @ q - ref["q_proj"]).max()
            qtol = 1e-8 if fp64 else 1e-5
            assert qerr < qtol and qperr < qtol * np.sqrt(q.size), (req.natoms, qerr, qperr)
            assert abs(q.sum()) < (1e-9 if fp64 else 1e-4)
