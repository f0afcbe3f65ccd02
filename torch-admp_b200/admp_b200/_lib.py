"""ctypes binding of libadmp_b200.so (the C ABI declared in include/admp_b200.h).

The library is the product: there is no Python or PyTorch fallback.  Loading
fails with an ImportError that says how to build it when the shared object
is missing, and every call raises when its status is not ADMP_OK.
"""
from __future__ import annotations

import ctypes
import os
import warnings

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libadmp_b200.so")
TORCH_OPS_PATH = os.path.join(_HERE, "_torch_ops.so")
_torch_ops_loaded = False


def load_torch_ops() -> None:
    """Register torch.ops.admp_b200.* (the TorchScript-visible operators over the
    C ABI, csrc/torch_ops.cpp) once.  Raises ImportError if it is not built."""
    global _torch_ops_loaded
    if _torch_ops_loaded:
        return
    if not os.path.exists(TORCH_OPS_PATH):
        raise ImportError(
            f"admp_b200 torch operators not found at {TORCH_OPS_PATH}; build them with "
            "`python torch-admp_b200/build.py`.  There is no CPU fallback.")
    torch.ops.load_library(TORCH_OPS_PATH)
    _torch_ops_loaded = True

OK, BAD_ARG, CUTOFF, NOT_CONVERGED, WORKSPACE, CUDA, BAD_INDEX, CAPACITY, NONFINITE, MESH = range(10)
F64, F32 = 0, 1
PAIR_EWALD, PAIR_OBC, PAIR_DAMPING = 0, 1, 2
TERM_SELF, TERM_NON_NEUTRAL, TERM_SLAB, TERM_DAMP_SELF, TERM_SITE = 1, 2, 4, 8, 16
QEQ_KSPACE, QEQ_RSPACE, QEQ_DAMPING, QEQ_SLAB, QEQ_PROJECT_Q0 = 1, 2, 4, 8, 16

EXPORTS = [
    "admp_abi_version", "admp_status_string", "admp_last_error_message", "admp_set_sync_checks",
    "admp_check_errors", "admp_pme_recip_workspace_size", "admp_pme_recip", "admp_pair_energy",
    "admp_atom_terms", "admp_pair_distances", "admp_pair_distances_backward", "admp_nblist_workspace_size",
    "admp_nblist_count", "admp_nblist_fill", "admp_qeq_workspace_size", "admp_qeq_solve", "admp_qeq_hvp",
    "admp_qeq_frames_workspace_size", "admp_qeq_solve_frames", "admp_qeq_hvp_frames",
    "admp_launch_count", "admp_profile_enable", "admp_profile_read", "admp_serve_slot_state_bytes",
    "admp_serve_sys_scratch_bytes", "admp_serve_cells_needed", "admp_serve_neighbors", "admp_serve_energy_forces",
    "admp_serve_qeq_init", "admp_serve_qeq_iterate", "admp_serve_qeq_finish", "admp_pme_recip_noalloc_max_scratch",
    "admp_pme_recip_noalloc", "admp_image_nblist_workspace_size", "admp_image_nblist_count",
    "admp_image_nblist_fill", "admp_image_pair_distances", "admp_image_pair_distances_backward",
]
PROFILE_KERNELS = ["spread", "fft_z_fwd", "fft_y_fwd", "fft_x_green", "fft_y_inv", "fft_z_inv", "gather", "pair_ef",
                   "csr_spmv", "neighbors", "cg_vector", "tc_z_fwd", "tc_y_fwd", "tc_x", "tc_y_inv", "tc_z_inv"]

_vp, _i, _ll, _d, _sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_size_t
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)
_dp = ctypes.POINTER(ctypes.c_double)

_SIGS = {
    "admp_abi_version": (_i, []),
    "admp_status_string": (ctypes.c_char_p, [_i]),
    "admp_last_error_message": (ctypes.c_char_p, []),
    "admp_set_sync_checks": (None, [_i]),
    "admp_check_errors": (_i, [_vp]),
    "admp_pme_recip_workspace_size": (_sz, [_i, _i, _ip]),
    "admp_pme_recip": (_i, [_i, _i, _i, _ip, _vp, _vp, _vp, _d, _d, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "admp_pair_energy": (_i, [_i, _i, _i, _i, _ll, _vp, _vp, _vp, _vp, _vp, _d, _d, _vp, _vp, _vp, _vp, _vp]),
    "admp_atom_terms": (_i, [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp,
                             _vp, _vp, _vp]),
    "admp_pair_distances": (_i, [_i, _i, _i, _ll, _vp, _vp, _vp, _vp, _vp]),
    "admp_pair_distances_backward": (_i, [_i, _i, _i, _ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "admp_nblist_workspace_size": (_sz, [_i]),
    "admp_nblist_count": (_i, [_i, _i, _i, _vp, _vp, _d, _vp, _sz, _llp, _vp]),
    "admp_nblist_fill": (_i, [_i, _i, _i, _vp, _vp, _d, _vp, _sz, _vp, _vp, _ll, _vp]),
    "admp_qeq_workspace_size": (_sz, [_i, _i, _ll, _ip, _i]),
    "admp_qeq_solve": (_i, [_i, _i, _i, _ip, _vp, _vp, _ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _i, _vp,
                            _dp, _vp, _d, _i, _ip, _dp, _vp, _sz, _vp]),
    "admp_qeq_frames_workspace_size": (_sz, [_i, _i, _i, _ll, _ip, _i]),
    "admp_qeq_solve_frames": (_i, [_i, _i, _i, _i, _ip, _vp, _vp, _ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d,
                                   _i, _vp, _dp, _vp, _d, _i, _ip, _dp, _vp, _sz, _vp]),
    "admp_qeq_hvp_frames": (_i, [_i, _i, _i, _i, _ip, _vp, _vp, _ll, _vp, _vp, _vp, _vp, _vp, _d, _d, _vp, _vp,
                                 _vp, _sz, _vp]),
    "admp_qeq_hvp": (_i, [_i, _i, _i, _ip, _vp, _vp, _ll, _vp, _vp, _vp, _vp, _vp, _d, _d, _vp, _vp, _vp, _sz,
                          _vp]),
    "admp_launch_count": (_ll, []),
    "admp_pme_recip_noalloc_max_scratch": (_sz, []),
    "admp_pme_recip_noalloc": (_i, [_i, _i, _i, _ip, _vp, _vp, _vp, _d, _d, _vp, _vp, _vp, _vp, _vp]),
    "admp_image_nblist_workspace_size": (_sz, [_i]),
    "admp_image_nblist_count": (_i, [_i, _i, _i, _vp, _vp, _d, _i, _vp, _sz, _llp, _llp, _ip, _vp]),
    "admp_image_nblist_fill": (_i, [_i, _i, _i, _vp, _vp, _d, _vp, _sz, _vp, _vp, _ll, _vp]),
    "admp_image_pair_distances": (_i, [_i, _i, _ll, _vp, _vp, _vp, _vp, _vp, _vp]),
    "admp_image_pair_distances_backward": (_i, [_i, _i, _ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "admp_profile_enable": (_i, [_i]),
    "admp_profile_read": (_i, [_dp, _llp, _dp, _i]),
}

_lib = None


def load():
    """Load the shared library (once).  Raises ImportError if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"admp_b200 native library not found at {LIB_PATH}; build it with "
            "`python torch-admp_b200/build.py` (nvcc, sm_100a).  There is no CPU fallback.")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class NotConvergedWarning(UserWarning):
    pass


class AdmpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


def check(status: int, what: str = "") -> None:
    if status == OK:
        return
    lib = load()
    msg = lib.admp_last_error_message().decode(errors="replace")
    text = f"{what}: {msg}" if what else msg
    if status == BAD_ARG or status == MESH:
        raise ValueError(text)
    if status == CUTOFF:
        raise AssertionError(msg)
    if status == BAD_INDEX:
        raise IndexError(text)
    raise AdmpError(status, f"{text} [{lib.admp_status_string(status).decode()}]")


def ptr(t) -> int | None:
    """Device pointer of a tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_of(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def dtype_code(dt: torch.dtype) -> int:
    if dt == torch.float64:
        return F64
    if dt == torch.float32:
        return F32
    raise TypeError(f"admp_b200 supports float64 and float32 tensors, got {dt}")


def require_cuda(t: torch.Tensor, name: str = "tensor") -> None:
    if not t.is_cuda:
        raise RuntimeError(
            f"admp_b200: {name} is on {t.device}; the B200 kernels need CUDA tensors "
            "(there is no CPU fallback).")


def launch_count() -> int:
    return int(load().admp_launch_count())


def profile_enable(capacity: int) -> None:
    check(load().admp_profile_enable(int(capacity)), "profile enable")


def profile_read() -> dict:
    n = len(PROFILE_KERNELS)
    ms = (ctypes.c_double * n)()
    cnt = (ctypes.c_longlong * n)()
    by = (ctypes.c_double * n)()
    check(load().admp_profile_read(ms, cnt, by, n), "profile read")
    return {k: {"ms": ms[i], "launches": cnt[i], "bytes": by[i]} for i, k in enumerate(PROFILE_KERNELS)}


def workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def int3(vals):
    arr = (ctypes.c_int * len(vals))(*[int(v) for v in vals])
    return ctypes.cast(arr, _ip), arr


def warn_not_converged(msg: str) -> None:
    warnings.warn(msg, NotConvergedWarning, stacklevel=3)
