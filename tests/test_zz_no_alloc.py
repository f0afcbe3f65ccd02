"""admp_pme_recip_noalloc against admp_pme_recip, through the C ABI.

The no-allocation variant serves callers that cannot allocate device memory
when they call the library (for example a plugin inside an MD engine that
owns all device memory, or a step loop that must not trigger cudaMalloc's
device-wide synchronisation); it keeps its scratch in a fixed array inside
the library.  Two calls in a row must both reproduce the workspace-based
entry point, which also shows that leftovers of the first call in the shared
array do not leak into the second.  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _inputs(dev, dtype, n=300, L=18.0, nf=2, seed=3):
    rng = np.random.default_rng(seed)
    pos = torch.tensor(rng.random((nf, n, 3)) * L, dtype=dtype, device=dev)
    box = torch.tensor(np.stack([np.diag([L, L, L]), np.diag([L, L * 1.05, L * 0.95])]), dtype=dtype, device=dev)
    q = rng.uniform(-1, 1, (nf, n))
    q -= q.mean(axis=1, keepdims=True)
    return pos, box, torch.tensor(q, dtype=dtype, device=dev)


def _call(lib, fn, dt, pos, box, q, kmesh, with_ws):
    from admp_b200 import _lib as L
    nf, n = q.shape
    km = (ctypes.c_int * (3 * nf))(*[k for row in kmesh for k in row])
    kp = ctypes.cast(km, ctypes.POINTER(ctypes.c_int))
    e = torch.zeros(nf, dtype=torch.float64, device=q.device)
    gp = torch.zeros_like(pos)
    gq = torch.zeros_like(q)
    gb = torch.zeros_like(box)
    st = torch.cuda.current_stream().cuda_stream
    args = [dt, nf, n, kp, pos.data_ptr(), box.data_ptr(), q.data_ptr(), 0.45, 14.399645, e.data_ptr(),
            gp.data_ptr(), gq.data_ptr(), gb.data_ptr()]
    if with_ws:
        nbytes = lib.admp_pme_recip_workspace_size(dt, nf, kp)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=q.device)
        status = fn(*args, ws.data_ptr(), nbytes, st)
    else:
        status = fn(*args, st)
    assert status == L.OK, lib.admp_last_error_message()
    torch.cuda.synchronize()
    return e, gp, gq, gb


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 2e-5)])
def test_noalloc_matches_workspace_entry_point_twice(cuda, dtype, tol):
    from admp_b200 import _lib as L
    lib = L.load()
    dt = L.dtype_code(dtype)
    kmesh = [[24, 24, 24], [24, 25, 23]]
    pos, box, q = _inputs(cuda, dtype)
    ref = _call(lib, lib.admp_pme_recip, dt, pos, box, q, kmesh, True)
    for _ in range(2):  # two calls in a row share the static scratch array
        out = _call(lib, lib.admp_pme_recip_noalloc, dt, pos, box, q, kmesh, False)
        for a, b in zip(out, ref):
            err = (a - b).abs().max().item() / max(b.abs().max().item(), 1e-30)
            assert err < tol, err


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 2e-5)])
def test_noalloc_smaller_mesh_after_larger_one(cuda, dtype, tol):
    """A call with a different, smaller mesh layout right after the two-frame
    call: whatever the previous call left in the shared array must not leak
    into it (compared with the workspace entry point on a fresh workspace)."""
    from admp_b200 import _lib as L
    lib = L.load()
    dt = L.dtype_code(dtype)
    pos, box, q = _inputs(cuda, dtype)
    _call(lib, lib.admp_pme_recip_noalloc, dt, pos, box, q, [[24, 24, 24], [24, 25, 23]], False)
    p1, b1, q1 = _inputs(cuda, dtype, n=200, L=15.0, nf=1, seed=5)
    kmesh = [[18, 17, 20]]
    ref = _call(lib, lib.admp_pme_recip, dt, p1, b1, q1, kmesh, True)
    out = _call(lib, lib.admp_pme_recip_noalloc, dt, p1, b1, q1, kmesh, False)
    for a, b in zip(out, ref):
        err = (a - b).abs().max().item() / max(b.abs().max().item(), 1e-30)
        assert err < tol, err


def test_noalloc_rejects_scratch_beyond_its_limit(cuda):
    from admp_b200 import _lib as L
    lib = L.load()
    cap = lib.admp_pme_recip_noalloc_max_scratch()
    assert cap == 16 << 20
    kmesh = [[160, 160, 160]]  # about 66 MB of FP64 scratch: refused on the host, nothing launched
    km = (ctypes.c_int * 3)(*kmesh[0])
    kp = ctypes.cast(km, ctypes.POINTER(ctypes.c_int))
    assert lib.admp_pme_recip_workspace_size(L.F64, 1, kp) > cap
    pos, box, q = _inputs(cuda, torch.float64, nf=1)
    e = torch.zeros(1, dtype=torch.float64, device=cuda)
    status = lib.admp_pme_recip_noalloc(L.F64, 1, q.shape[1], kp, pos.data_ptr(), box.data_ptr(), q.data_ptr(),
                                        0.45, 14.4, e.data_ptr(), None, None, None,
                                        torch.cuda.current_stream().cuda_stream)
    assert status == L.WORKSPACE
    assert b"fixed" in lib.admp_last_error_message()
