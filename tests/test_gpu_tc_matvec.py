"""The FP32 CG matvec's mesh passes on the tensor cores (x, y and z passes as
tcgen05 products, 3xTF32) for every mesh length 17-79 on every axis: the QEq
Hessian-vector product of admp_qeq_hvp_frames in FP32 (which takes that
path) against the same call in FP64 (the shared-memory FFT, pinned to the
oracle by the PME and QEq parity tests).  63 frames of 48 atoms, each with
its own mesh, in one batched call; reciprocal and self terms only
(flags = ADMP_QEQ_KSPACE).  Tolerance: 2e-5 relative to the largest entry."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LENGTHS = list(range(17, 80))
N_ATOMS = 48


def _run(cuda, dtype, kmesh, pos, box, p):
    from admp_b200 import _lib as L
    lib = L.load()
    nf = len(kmesh)
    kp, _keep = L.int3([k for km in kmesh for k in km])
    tp = torch.tensor(pos, dtype=dtype, device=cuda)
    tb = torch.tensor(box, dtype=dtype, device=cuda)
    hard = torch.full((nf, N_ATOMS), 5.0, dtype=dtype, device=cuda)
    eta = torch.full((nf, N_ATOMS), 1.2, dtype=dtype, device=cuda)
    vec = torch.tensor(p, dtype=dtype, device=cuda)
    out = torch.zeros_like(vec)
    nbytes = lib.admp_qeq_frames_workspace_size(L.dtype_code(dtype), nf, N_ATOMS, 0, kp, 0)
    assert nbytes > 0
    ws = L.workspace(nbytes, cuda)
    L.check(lib.admp_qeq_hvp_frames(L.dtype_code(dtype), L.QEQ_KSPACE, nf, N_ATOMS, kp, L.ptr(tp), L.ptr(tb), 0,
                                    None, None, None, L.ptr(hard), L.ptr(eta), 0.3, 138.935456, L.ptr(vec),
                                    L.ptr(out), L.ptr(ws), nbytes, L.stream_of(cuda)), "hvp")
    torch.cuda.synchronize()
    return out.double().cpu().numpy()


def test_tc_matvec_every_mesh_length(cuda):
    rng = np.random.default_rng(77)
    nl = len(LENGTHS)
    kmesh = [(LENGTHS[i], LENGTHS[(i + 21) % nl], LENGTHS[(i + 42) % nl]) for i in range(nl)]
    box = np.stack([np.diag(rng.uniform(18.0, 24.0, 3)) for _ in range(nl)])
    pos = np.stack([rng.uniform(0.0, 1.0, (N_ATOMS, 3)) @ box[f] for f in range(nl)])
    p = rng.normal(size=(nl, N_ATOMS))
    h32 = _run(cuda, torch.float32, kmesh, pos, box, p)
    h64 = _run(cuda, torch.float64, kmesh, pos, box, p)
    bad = []
    for f in range(nl):
        err = np.abs(h32[f] - h64[f]).max() / np.abs(h64[f]).max()
        if not err < 2e-5:
            bad.append((kmesh[f], err))
    assert not bad, bad
