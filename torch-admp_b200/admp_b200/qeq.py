"""QEq on B200 kernels (drop-in for torch_admp.qeq, qeq.py:33-1670).

The charge solve runs as a matrix-free projected conjugate gradient on the
GPU (admp_qeq_solve) for every ``method`` the reference accepts ("lbfgs",
"quadratic"): E(q) is quadratic, so all of them reach the same minimiser,
stopped by the reference's criterion ||P grad||_2 / N < eps (qeq.py:1516).
``matinv`` builds the dense Hessian column by column from GPU
Hessian-vector products and solves the KKT system (qeq.py:1530-1617).

``qeq_solve`` additionally returns charges that are differentiable with
respect to positions, box, chi, hardness, eta and a right-hand-side shift
through the implicit function theorem: the backward runs a second CG with the
same operator (the adjoint) and contracts it with mixed second derivatives
obtained from the energy kernels (polarisation identity).
"""

import ctypes
from typing import Dict, List, Optional, Tuple, Union

import torch

from . import _lib as L
from .base_force import BaseForceModule, prep_float
from .ops import DampingFn, SiteFn, coulomb_pbc, damping_raw
from .pme import CoulombForceModule
from .utils import calc_pgrads, vector_projection, vector_projection_coeff_matrix

L.load_torch_ops()  # torch.ops.admp_b200.* used by the forward passes


class GaussianDampingForceModule(BaseForceModule):
    """Gaussian short-range damping (qeq.py:33-129)."""

    def __init__(self, units_dict: Optional[Dict] = None) -> None:
        BaseForceModule.__init__(self, units_dict)

    def _forward_impl(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor,
                      ds: torch.Tensor, buffer_scales: torch.Tensor,
                      params: Dict[str, torch.Tensor]) -> torch.Tensor:
        nf, na = positions.size(0), positions.size(1)
        dt = positions.dtype
        q = params["charge"].reshape(nf, na).to(dt)
        eta = (params["eta"].reshape(nf, na) * self.const_lib.length_coeff).to(dt)
        return torch.ops.admp_b200.damping(ds.to(dt), q, eta, pairs, buffer_scales.to(dt), self.const_lib.dielectric)


class SiteForceModule(BaseForceModule):
    """Chemical site energy chi q + hardness q^2 (qeq.py:132-209)."""

    def __init__(self, units_dict: Optional[Dict] = None) -> None:
        BaseForceModule.__init__(self, units_dict)

    def _forward_impl(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor,
                      ds: torch.Tensor, buffer_scales: torch.Tensor,
                      params: Dict[str, torch.Tensor]) -> torch.Tensor:
        nf, na = positions.size(0), positions.size(1)
        dt = positions.dtype
        ec = self.const_lib.energy_coeff
        chi = (params["chi"].reshape(nf, na) * ec).to(dt)
        hard = (params["hardness"].reshape(nf, na) * ec).to(dt)
        q = params["charge"].reshape(nf, na).to(dt)
        return torch.ops.admp_b200.site(q, chi, hard)


class QEqForceModule(BaseForceModule):
    """Charge equilibration model (qeq.py:212-1114)."""

    def __init__(self, rcut: float, ethresh: float = 1e-5, kspace: bool = True, rspace: bool = True,
                 slab_corr: bool = False, slab_axis: int = 2, max_iter: int = 20, ls_eps: float = 1e-4,
                 eps: float = 1e-4, units_dict: Optional[Dict] = None, damping: bool = True,
                 sel: Optional[list] = None, kappa: Optional[float] = None,
                 spacing: Union[List[float], float, None] = None, kmesh: Union[List[int], int, None] = None) -> None:
        BaseForceModule.__init__(self, units_dict)
        models: Dict[str, BaseForceModule] = {
            "site": SiteForceModule(units_dict=units_dict),
            "coulomb": CoulombForceModule(rcut=rcut, ethresh=ethresh, kspace=kspace, rspace=rspace,
                                          slab_corr=slab_corr, slab_axis=slab_axis, units_dict=units_dict,
                                          kappa=kappa, spacing=spacing, kmesh=kmesh),
        }
        if damping:
            models["damping"] = GaussianDampingForceModule(units_dict=units_dict)
        self.submodels = torch.nn.ModuleDict(models)
        self.rcut = rcut
        self.max_iter = max_iter
        self.ls_eps = ls_eps
        self.eps = eps
        self.converge_iter: int = -1
        self.sel = sel
        self.slab_axis = slab_axis
        self.slab_corr = slab_corr
        self.last_residual = float("nan")

    def get_rcut(self) -> float:
        return self.rcut

    def get_sel(self):
        return self.sel

    def _forward_impl(self, positions: torch.Tensor, box: Optional[torch.Tensor], pairs: torch.Tensor,
                      ds: torch.Tensor, buffer_scales: torch.Tensor,
                      params: Dict[str, torch.Tensor]) -> torch.Tensor:
        energy = torch.zeros(positions.size(0), device=positions.device, dtype=positions.dtype)
        for model in self.submodels.values():
            energy = energy + model(positions, box, pairs, ds, buffer_scales, params)
        return energy

    @torch.jit.export
    def func_energy(self, charges: torch.Tensor, positions: torch.Tensor, box: Optional[torch.Tensor],
                    chi: torch.Tensor, hardness: torch.Tensor, eta: torch.Tensor, pairs: torch.Tensor,
                    ds: torch.Tensor, buffer_scales: torch.Tensor) -> torch.Tensor:
        """Total QEq energy (qeq.py:408-458)."""
        params: Dict[str, torch.Tensor] = {"charge": charges, "chi": chi, "hardness": hardness, "eta": eta}
        energy = torch.zeros(1, device=positions.device, dtype=positions.dtype)
        for model in self.submodels.values():
            energy = energy + model(positions, box, pairs, ds, buffer_scales, params)
        return energy

    @torch.jit.export
    def optimality(self, charges: torch.Tensor, positions: torch.Tensor, box: Optional[torch.Tensor],
                   chi: torch.Tensor, hardness: torch.Tensor, eta: torch.Tensor, pairs: torch.Tensor,
                   ds: torch.Tensor, buffer_scales: torch.Tensor, constraint_matrix: torch.Tensor,
                   coeff_matrix: torch.Tensor) -> torch.Tensor:
        """Normalised projected gradient ||P dE/dq|| / N, ~0 at the optimal charges (qeq.py:714-764)."""
        energy = self.func_energy(charges, positions, box, chi, hardness, eta, pairs, ds, buffer_scales)
        pgrads = calc_pgrads(energy, charges, constraint_matrix, coeff_matrix)
        return torch.norm(pgrads) / charges.shape[0]

    # -- solver plumbing -------------------------------------------------
    def _flags(self) -> int:
        c = self.submodels["coulomb"]
        f = 0
        if c.kspace_flag:
            f |= L.QEQ_KSPACE
        if c.rspace_flag:
            f |= L.QEQ_RSPACE
        if "damping" in self.submodels:
            f |= L.QEQ_DAMPING
        if c.slab_corr_flag:
            f |= L.QEQ_SLAB | (int(c.slab_axis) << 8)
        return f

    def _solve(self, q0, positions, box, chi, hardness, eta, pairs, ds, buffer_scales, constraint_matrix,
               constraint_vals, project_q0: bool, tol: float, max_iter: int, shift=None):
        """Run the GPU CG; returns (q, iterations, residual, status)."""
        return _qeq_solve_raw(self, q0, positions, box, chi, hardness, eta, pairs, ds, buffer_scales,
                              constraint_matrix, constraint_vals, project_q0, tol, max_iter, shift)

    def calc_hessian(self, positions, box, chi, hardness, eta, pairs, ds, buffer_scales):
        """Dense Hessian d2E/dq2 from GPU Hessian-vector products (qeq.py:460-515)."""
        return _hessian(self, positions, box, hardness, eta, pairs, ds, buffer_scales)

    def solve_matrix_inversion(self, positions, box, chi, hardness, eta, pairs, ds, buffer_scales,
                               constraint_matrix, constraint_vals, check_hessian: bool = False):
        """KKT solve with the dense Hessian (qeq.py:517-607)."""
        hessian = self.calc_hessian(positions, box, chi, hardness, eta, pairs, ds, buffer_scales)
        q = _kkt(hessian, chi, constraint_matrix, constraint_vals)
        q_opt = q.detach().clone().requires_grad_(True)
        energy = self.func_energy(q_opt, positions, box, chi, hardness, eta, pairs, ds, buffer_scales)
        fermi = torch.mean(chi + hessian @ q)
        return energy, q, torch.diag(hessian), fermi

    def solve_pgrad(self, q0, positions, box, chi, hardness, eta, pairs, ds, buffer_scales, constraint_matrix,
                    constraint_vals, coeff_matrix=None, reinit_q: bool = False, method: str = "lbfgs"):
        """Projected-gradient solve (qeq.py:609-712) -> (energy, q_opt)."""
        if method not in ("lbfgs", "quadratic", "cg"):
            raise ValueError(f"Method {method} is not supported.")
        n = positions.shape[0]
        if q0 is None:
            q0 = torch.rand(n, device=positions.device, dtype=positions.dtype)
            reinit_q = True
        assert q0.shape[0] == n
        q, iters, resid, status = self._solve(q0.reshape(-1), positions, box, chi, hardness, eta, pairs, ds,
                                              buffer_scales, constraint_matrix, constraint_vals, reinit_q,
                                              self.eps, self.max_iter)
        self.converge_iter = iters if status == L.OK else -1
        self.last_residual = resid
        q_opt = q.detach().clone().requires_grad_(True)
        energy = self.func_energy(q_opt, positions, box, chi, hardness, eta, pairs, ds, buffer_scales)
        return energy, q_opt


def _kkt(hessian, chi, C, b):
    n = hessian.shape[0]
    if C is None:
        return torch.linalg.solve(hessian, -chi.reshape(-1, 1)).reshape(-1)
    m = C.shape[0]
    A = torch.cat([torch.cat([hessian, C.T.to(hessian.dtype)], 1),
                   torch.cat([C.to(hessian.dtype), torch.zeros(m, m, device=hessian.device, dtype=hessian.dtype)], 1)], 0)
    rhs = torch.cat([-chi.reshape(-1).to(hessian.dtype), b.reshape(-1).to(hessian.dtype)])
    return torch.linalg.solve(A, rhs.reshape(-1, 1)).reshape(-1)[:n]


def _std_inputs(module, positions, box, pairs, ds, buffer_scales, *vecs):
    dt = positions.dtype
    L.require_cuda(positions, "positions")
    lc = module.const_lib.length_coeff
    pos = prep_float(positions.detach() * lc, dt)
    bx = prep_float(box.detach() * lc, dt)
    pr = pairs.to(torch.long).contiguous()
    dsc = prep_float(ds.detach() * lc, dt)
    bsc = prep_float(buffer_scales, dt)
    out = [None if v is None else prep_float(v.detach().reshape(-1), dt) for v in vecs]
    return pos, bx, pr, dsc, bsc, out


def _kmesh_of(module, box):
    c = module.submodels["coulomb"]
    if not c.kspace_flag:
        return [1, 1, 1]
    km = c.kmesh_for(box.reshape(1, 3, 3))[0]
    c._kmesh = torch.tensor(km, dtype=torch.long)
    return km


def _qeq_solve_raw(module, q0, positions, box, chi, hardness, eta, pairs, ds, buffer_scales, C, b, project_q0,
                   tol, max_iter, shift=None):
    lib = L.load()
    if box is None:
        raise ValueError("admp_b200 QEq solve needs a periodic box")
    ec = module.const_lib.energy_coeff
    pos, bx, pr, dsc, bsc, (chi_c, hard_c, eta_c, sh, qv) = _std_inputs(
        module, positions, box, pairs, ds, buffer_scales, chi * ec, hardness * ec,
        eta * module.const_lib.length_coeff if eta is not None else None, shift, q0)
    n = pos.shape[0]
    dt = pos.dtype
    dev = pos.device
    if eta_c is None:
        eta_c = torch.zeros(n, dtype=dt, device=dev)
    flags = module._flags()
    if project_q0:
        flags |= L.QEQ_PROJECT_Q0
    c = module.submodels["coulomb"]
    km = _kmesh_of(module, bx)
    kp, _keep = L.int3(km)
    P = pr.shape[0]
    nc = 0 if C is None else int(C.shape[0])
    Cc = prep_float(C.detach().reshape(nc, n), dt) if nc else None
    bvals = (ctypes.c_double * max(nc, 1))(*([float(v) for v in b.detach().reshape(-1).tolist()] if nc else [0.0]))
    nbytes = lib.admp_qeq_workspace_size(L.dtype_code(dt), n, P, kp if c.kspace_flag else None, nc)
    ws = L.workspace(nbytes, dev)
    q = qv.clone()
    iters = ctypes.c_int(0)
    resid = ctypes.c_double(0.0)
    st = lib.admp_qeq_solve(L.dtype_code(dt), flags, n, kp, L.ptr(pos), L.ptr(bx), P, L.ptr(pr), L.ptr(dsc),
                            L.ptr(bsc), L.ptr(chi_c), L.ptr(hard_c), L.ptr(eta_c), L.ptr(sh), float(c.kappa) or 1.0,
                            module.const_lib.dielectric, nc, L.ptr(Cc), bvals, L.ptr(q), float(tol), int(max_iter),
                            ctypes.byref(iters), ctypes.byref(resid), L.ptr(ws), nbytes, L.stream_of(dev))
    if st == L.NOT_CONVERGED:
        L.warn_not_converged(lib.admp_last_error_message().decode())
    elif st != L.OK:
        L.check(st, "QEq solve")
    return q, int(iters.value), float(resid.value), st


def _hessian(module, positions, box, hardness, eta, pairs, ds, buffer_scales, max_cols: int = 64,
             max_pair_rows: int = 16_000_000):
    """Dense d2E/dq2 from batched GPU Hessian-vector products: columns in
    chunks, each chunk one admp_qeq_hvp_frames call on unit vectors (the
    geometry repeated per column), with one workspace for all chunks."""
    lib = L.load()
    ec = module.const_lib.energy_coeff
    pos, bx, pr, dsc, bsc, (hard_c, eta_c) = _std_inputs(
        module, positions, box, pairs, ds, buffer_scales, hardness * ec,
        eta * module.const_lib.length_coeff if eta is not None else None)
    n = pos.shape[0]
    dt, dev = pos.dtype, pos.device
    if eta_c is None:
        eta_c = torch.zeros(n, dtype=dt, device=dev)
    P = int(pr.shape[0])
    nv = max(1, min(max_cols, n, max_pair_rows // max(P, 1)))
    c = module.submodels["coulomb"]
    km = _kmesh_of(module, bx)
    flags = module._flags()
    kp, _keep = L.int3(km * nv)
    nbytes = lib.admp_qeq_frames_workspace_size(L.dtype_code(dt), nv, n, P * nv, kp if c.kspace_flag else None, 0)
    if nbytes == 0:
        L.check(L.BAD_ARG, "QEq Hessian workspace")
    ws = L.workspace(nbytes, dev)
    offs = (torch.arange(nv, device=dev, dtype=torch.long) * n).view(nv, 1, 1)
    pos_r = pos.reshape(1, n, 3).expand(nv, n, 3).contiguous()
    box_r = bx.reshape(1, 3, 3).expand(nv, 3, 3).contiguous()
    pr_r = (pr.reshape(1, P, 2) + offs).reshape(-1, 2).contiguous()
    ds_r = dsc.reshape(1, P).expand(nv, P).contiguous()
    bs_r = bsc.reshape(1, P).expand(nv, P).contiguous()
    hard_r = hard_c.reshape(1, n).expand(nv, n).contiguous()
    eta_r = eta_c.reshape(1, n).expand(nv, n).contiguous()
    H = torch.empty(n, n, dtype=dt, device=dev)
    E = torch.zeros(nv, n, dtype=dt, device=dev)
    out = torch.empty(nv, n, dtype=dt, device=dev)
    for k0 in range(0, n, nv):
        m = min(nv, n - k0)
        E.zero_()
        E[torch.arange(m, device=dev), torch.arange(k0, k0 + m, device=dev)] = 1.0
        L.check(lib.admp_qeq_hvp_frames(L.dtype_code(dt), flags, m, n, kp, L.ptr(pos_r), L.ptr(box_r), P * m,
                                        L.ptr(pr_r), L.ptr(ds_r), L.ptr(bs_r), L.ptr(hard_r), L.ptr(eta_r),
                                        float(c.kappa) or 1.0, module.const_lib.dielectric, L.ptr(E), L.ptr(out),
                                        L.ptr(ws), nbytes, L.stream_of(dev)), "QEq Hessian-vector products")
        H[:, k0:k0 + m] = out[:m].T
    return 0.5 * (H + H.T)


def pgrad_optimize(module: QEqForceModule, q0, positions, box, chi, hardness, eta, pairs, ds, buffer_scales,
                   constraint_matrix, constraint_vals, coeff_matrix=None, reinit_q: bool = False,
                   method: str = "lbfgs", **kwargs):
    """qeq.py:1117-1270 -> (energy, q_opt) with module.converge_iter set."""
    if method not in ("lbfgs", "quadratic", "cg"):
        raise ValueError(f"Method {method} is not supported.")
    n = positions.shape[0]
    if q0 is None:
        q0 = torch.rand(n, device=positions.device, dtype=positions.dtype)
        reinit_q = True
    assert q0.shape[0] == n
    q, iters, resid, status = module._solve(q0.reshape(-1), positions, box, chi, hardness, eta, pairs, ds,
                                            buffer_scales, constraint_matrix, constraint_vals, reinit_q, module.eps,
                                            module.max_iter)
    module.converge_iter = iters if status == L.OK else -1
    module.last_residual = resid
    q_opt = q.detach().clone().requires_grad_(True)
    energy = module.func_energy(q_opt, positions, box, chi, hardness, eta, pairs, ds, buffer_scales)
    return energy, q_opt


def matinv_optimize(module: QEqForceModule, positions, box, chi, hardness, eta, pairs, ds, buffer_scales,
                    constraint_matrix, constraint_vals, **kwargs):
    """qeq.py:1530-1617 -> (energy, q_opt)."""
    hessian = _hessian(module, positions, box, hardness, eta, pairs, ds, buffer_scales)
    q = _kkt(hessian, chi.detach() * module.const_lib.energy_coeff, constraint_matrix, constraint_vals)
    q_opt = q.detach().clone().requires_grad_(True)
    energy = module.func_energy(q_opt, positions, box, chi, hardness, eta, pairs, ds, buffer_scales)
    return energy, q_opt


def calc_hessian(func_energy, positions, box, chi, hardness, eta, pairs, ds, buffer_scales):
    """Module-level Hessian helper (qeq.py:1620-1670); needs the bound QEqForceModule."""
    module = getattr(func_energy, "__self__", None)
    if not isinstance(module, QEqForceModule):
        raise TypeError("calc_hessian expects a QEqForceModule.func_energy bound method")
    return _hessian(module, positions, box, hardness, eta, pairs, ds, buffer_scales)


# ---------------------------------------------------------------------------
# differentiable solve (implicit adjoint)
# ---------------------------------------------------------------------------
def _quadratic_part_grads(module, pos, bx, pr, dsc, bsc, q, eta_c):
    """Gradients of E_J(q) = Coulomb + damping (the part quadratic in q) w.r.t. pos, box, ds, eta."""
    c = module.submodels["coulomb"]
    km = _kmesh_of(module, bx)
    qf = q.reshape(1, -1).contiguous()
    _, _, g = coulomb_pbc(pos.reshape(1, -1, 3), bx.reshape(1, 3, 3), pr.reshape(1, -1, 2), dsc.reshape(1, -1),
                          bsc.reshape(1, -1), qf, float(c.kappa), [km], module.const_lib.dielectric, c.rspace_flag,
                          c.kspace_flag, c.slab_corr_flag, c.slab_axis, True)
    out = {"pos": g["pos"][0], "box": g["box"][0], "ds": g["ds"][0], "eta": torch.zeros_like(qf[0])}
    if "damping" in module.submodels:
        _, gds, _, geta = damping_raw(dsc.reshape(1, -1), qf, eta_c.reshape(1, -1), pr.reshape(1, -1, 2),
                                      bsc.reshape(1, -1), module.const_lib.dielectric, True)
        out["ds"] = out["ds"] + gds[0]
        out["eta"] = geta[0]
    return out


class QEqSolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, box, chi, hardness, eta, ds, shift, module, pairs, buffer_scales, C, b, q0, tol,
                max_iter):
        q, iters, resid, status = _qeq_solve_raw(module, q0, positions, box, chi, hardness, eta, pairs, ds,
                                                 buffer_scales, C, b, True, tol, max_iter, shift)
        module.converge_iter = iters if status == L.OK else -1
        module.last_residual = resid
        ctx.module = module
        ctx.tol = tol
        ctx.max_iter = max_iter
        ctx.save_for_backward(positions, box, chi, hardness, eta, ds, pairs, buffer_scales,
                              C if C is not None else torch.empty(0), q)
        ctx.has_C = C is not None
        return q

    @staticmethod
    def backward(ctx, gq):
        positions, box, chi, hardness, eta, ds, pairs, bs, C, q = ctx.saved_tensors
        module = ctx.module
        Cm = C if ctx.has_C else None
        n = q.shape[0]
        zero_b = torch.zeros(Cm.shape[0], dtype=q.dtype, device=q.device) if Cm is not None else None
        # adjoint: min 1/2 l^T H l - gq^T l  s.t. C l = 0  ->  l = Z (Z^T H Z)^-1 Z^T gq
        lam, _, _, _ = _qeq_solve_raw(module, torch.zeros_like(q), positions, box, -gq.detach(), hardness, eta,
                                      pairs, ds, bs, Cm, zero_b, True, min(ctx.tol, 1e-8), max(ctx.max_iter, 200))
        out = [None] * 15
        ec = module.const_lib.energy_coeff
        if ctx.needs_input_grad[2]:
            out[2] = -lam
        if ctx.needs_input_grad[6]:
            out[6] = -lam / ec
        if ctx.needs_input_grad[3]:
            out[3] = -2.0 * q * lam
        if any(ctx.needs_input_grad[i] for i in (0, 1, 4, 5)):
            pos, bx, pr, dsc, bsc, (eta_c,) = _std_inputs(module, positions, box, pairs, ds, bs,
                                                           eta * module.const_lib.length_coeff)
            gp = _quadratic_part_grads(module, pos, bx, pr, dsc, bsc, q + lam, eta_c)
            gm = _quadratic_part_grads(module, pos, bx, pr, dsc, bsc, q - lam, eta_c)
            lc = module.const_lib.length_coeff / ec
            if ctx.needs_input_grad[0]:
                out[0] = -0.5 * (gp["pos"] - gm["pos"]) * lc
            if ctx.needs_input_grad[1]:
                out[1] = -0.5 * (gp["box"] - gm["box"]) * lc
            if ctx.needs_input_grad[5]:
                out[5] = -0.5 * (gp["ds"] - gm["ds"]) * lc
            if ctx.needs_input_grad[4]:
                out[4] = -0.5 * (gp["eta"] - gm["eta"]) * lc
        return tuple(out)


def qeq_solve(module: QEqForceModule, positions, box, chi, hardness, eta, pairs, ds, buffer_scales,
              constraint_matrix=None, constraint_vals=None, q0=None, shift=None, tol: Optional[float] = None,
              max_iter: Optional[int] = None):
    """Differentiable QEq charges q*(positions, box, chi, hardness, eta, ds, shift).

    Gradients of any loss of q* flow back through the implicit adjoint (a second
    projected CG with the same operator)."""
    n = positions.shape[0]
    if q0 is None:
        q0 = torch.zeros(n, dtype=positions.dtype, device=positions.device)
    if constraint_matrix is not None and constraint_vals is None:
        constraint_vals = torch.zeros(constraint_matrix.shape[0], dtype=positions.dtype, device=positions.device)
    if shift is None:
        shift = torch.zeros(n, dtype=positions.dtype, device=positions.device)
    return QEqSolveFn.apply(positions, box, chi, hardness, eta, ds, shift, module, pairs, buffer_scales,
                            constraint_matrix, constraint_vals, q0, module.eps if tol is None else tol,
                            module.max_iter if max_iter is None else max_iter)


# ---------------------------------------------------------------------------
# several frames in one solve (the differentiation batch)
# ---------------------------------------------------------------------------
def _frames_vec(v, nf: int, n: int, dt):
    """[N] (shared by the frames) or [nf, N] -> contiguous [nf * N] of dtype dt."""
    return prep_float(v.detach().reshape(-1, n).expand(nf, n), dt).reshape(-1)


def _qeq_solve_frames_raw(module, q0, positions, box, chi, hardness, eta, pairs, ds, buffer_scales, C, b, project_q0,
                          tol, max_iter, shift=None):
    """admp_qeq_solve_frames over positions [nf, N, 3], box [nf, 3, 3], pairs
    [nf, P, 2] (frame-local indices, padding rows with scale 0), ds / scales
    [nf, P]; chi, hardness, eta, shift [N] or [nf, N].  Returns (q [nf, N],
    iterations [nf], residuals [nf], status)."""
    lib = L.load()
    L.require_cuda(positions, "positions")
    if box is None:
        raise ValueError("admp_b200 QEq solve needs a periodic box")
    nf, n = int(positions.shape[0]), int(positions.shape[1])
    dt = positions.dtype
    dev = positions.device
    ec = module.const_lib.energy_coeff
    lc = module.const_lib.length_coeff
    pos = prep_float(positions.detach() * lc, dt)
    bx = prep_float(box.detach().reshape(nf, 3, 3) * lc, dt)
    P = int(pairs.shape[1])
    offs = (torch.arange(nf, device=dev, dtype=torch.long) * n).view(nf, 1, 1)
    prg = (pairs.to(torch.long) + offs).reshape(-1, 2).contiguous()
    dsc = prep_float(ds.detach() * lc, dt).reshape(-1)
    bsc = prep_float(buffer_scales.reshape(nf, P), dt).reshape(-1)
    chi_c = _frames_vec(chi * ec, nf, n, dt)
    hard_c = _frames_vec(hardness * ec, nf, n, dt)
    eta_c = _frames_vec(eta * lc, nf, n, dt) if eta is not None else torch.zeros(nf * n, dtype=dt, device=dev)
    sh = _frames_vec(shift, nf, n, dt) if shift is not None else None
    q = _frames_vec(q0, nf, n, dt).clone()
    flags = module._flags()
    if project_q0:
        flags |= L.QEQ_PROJECT_Q0
    c = module.submodels["coulomb"]
    km = [[1, 1, 1]] * nf
    if c.kspace_flag:
        km = c.kmesh_for(bx)
        c._kmesh = torch.tensor(km[-1], dtype=torch.long)
    kp, _keep = L.int3([k for row in km for k in row])
    nc = 0 if C is None else int(C.shape[0])
    Cc = prep_float(C.detach().reshape(nc, n), dt) if nc else None
    bvals = (ctypes.c_double * max(nc, 1))(*([float(v) for v in b.detach().reshape(-1).tolist()] if nc else [0.0]))
    nbytes = lib.admp_qeq_frames_workspace_size(L.dtype_code(dt), nf, n, nf * P, kp if c.kspace_flag else None, nc)
    if nbytes == 0:
        L.check(L.BAD_ARG, f"QEq workspace for {nf} frames")
    ws = L.workspace(nbytes, dev)
    iters = (ctypes.c_int * nf)()
    resid = (ctypes.c_double * nf)()
    st = lib.admp_qeq_solve_frames(L.dtype_code(dt), flags, nf, n, kp, L.ptr(pos), L.ptr(bx), nf * P, L.ptr(prg),
                                   L.ptr(dsc), L.ptr(bsc), L.ptr(chi_c), L.ptr(hard_c), L.ptr(eta_c), L.ptr(sh),
                                   float(c.kappa) or 1.0, module.const_lib.dielectric, nc, L.ptr(Cc), bvals, L.ptr(q),
                                   float(tol), int(max_iter), iters, resid, L.ptr(ws), nbytes, L.stream_of(dev))
    if st == L.NOT_CONVERGED:
        L.warn_not_converged(lib.admp_last_error_message().decode())
    elif st != L.OK:
        L.check(st, "QEq solve (frames)")
    return q.reshape(nf, n), list(iters), list(resid), st


def _quadratic_part_grads_frames(module, pos, bx, pr, dsc, bsc, q, eta_c):
    """Gradients of E_J(q) = Coulomb + damping over nf frames w.r.t. positions
    [nf, N, 3], box [nf, 3, 3], ds [nf, P] and eta [nf, N]."""
    c = module.submodels["coulomb"]
    km = c.kmesh_for(bx) if c.kspace_flag else [[1, 1, 1]] * pos.shape[0]
    qf = q.contiguous()
    _, _, g = coulomb_pbc(pos, bx, pr, dsc, bsc, qf, float(c.kappa), km, module.const_lib.dielectric, c.rspace_flag,
                          c.kspace_flag, c.slab_corr_flag, c.slab_axis, True)
    out = {"pos": g["pos"], "box": g["box"], "ds": g["ds"], "eta": torch.zeros_like(qf)}
    if "damping" in module.submodels:
        _, gds, _, geta = damping_raw(dsc, qf, eta_c, pr, bsc, module.const_lib.dielectric, True)
        out["ds"] = out["ds"] + gds
        out["eta"] = geta
    return out


class QEqFramesFn(torch.autograd.Function):
    """Charges q*[nf, N] of several frames, differentiable through the implicit
    adjoint (one batched second CG over all frames)."""

    @staticmethod
    def forward(ctx, positions, box, chi, hardness, eta, ds, shift, module, pairs, buffer_scales, C, b, q0, tol,
                max_iter):
        q, iters, resid, status = _qeq_solve_frames_raw(module, q0, positions, box, chi, hardness, eta, pairs, ds,
                                                        buffer_scales, C, b, True, tol, max_iter, shift)
        module.converge_iter = max(iters) if status == L.OK else -1
        module.frame_iters = iters
        module.frame_residuals = resid
        module.last_residual = max(resid)
        ctx.module = module
        ctx.tol = tol
        ctx.max_iter = max_iter
        ctx.save_for_backward(positions, box, chi, hardness, eta, ds, pairs, buffer_scales,
                              C if C is not None else torch.empty(0), q)
        ctx.has_C = C is not None
        return q

    @staticmethod
    def backward(ctx, gq):
        positions, box, chi, hardness, eta, ds, pairs, bs, C, q = ctx.saved_tensors
        module = ctx.module
        Cm = C if ctx.has_C else None
        zero_b = torch.zeros(Cm.shape[0], dtype=q.dtype, device=q.device) if Cm is not None else None
        lam, _, _, _ = _qeq_solve_frames_raw(module, torch.zeros_like(q), positions, box, -gq.detach(), hardness, eta,
                                             pairs, ds, bs, Cm, zero_b, True, min(ctx.tol, 1e-8),
                                             max(ctx.max_iter, 200))
        lam = lam.to(q.dtype)
        out = [None] * 15
        ec = module.const_lib.energy_coeff
        if ctx.needs_input_grad[2]:
            out[2] = -lam
        if ctx.needs_input_grad[6]:
            out[6] = -lam / ec
        if ctx.needs_input_grad[3]:
            out[3] = -2.0 * q * lam
        if any(ctx.needs_input_grad[i] for i in (0, 1, 4, 5)):
            nf, n = q.shape
            dt = positions.dtype
            lc0 = module.const_lib.length_coeff
            pos = prep_float(positions.detach() * lc0, dt)
            bx = prep_float(box.detach() * lc0, dt)
            pr = pairs.to(torch.long).contiguous()
            dsc = prep_float(ds.detach() * lc0, dt)
            bsc = prep_float(bs, dt)
            eta_c = _frames_vec(eta * lc0, nf, n, dt).reshape(nf, n)
            gp = _quadratic_part_grads_frames(module, pos, bx, pr, dsc, bsc, q + lam, eta_c)
            gm = _quadratic_part_grads_frames(module, pos, bx, pr, dsc, bsc, q - lam, eta_c)
            lc = lc0 / ec
            if ctx.needs_input_grad[0]:
                out[0] = -0.5 * (gp["pos"] - gm["pos"]) * lc
            if ctx.needs_input_grad[1]:
                out[1] = -0.5 * (gp["box"] - gm["box"]) * lc
            if ctx.needs_input_grad[5]:
                out[5] = -0.5 * (gp["ds"] - gm["ds"]) * lc
            if ctx.needs_input_grad[4]:
                out[4] = -0.5 * (gp["eta"] - gm["eta"]) * lc
        return tuple(out)


def qeq_solve_frames(module: QEqForceModule, positions, box, chi, hardness, eta, pairs, ds, buffer_scales,
                     constraint_matrix=None, constraint_vals=None, q0=None, shift=None, tol: Optional[float] = None,
                     max_iter: Optional[int] = None):
    """Differentiable QEq charges of nf frames of N atoms in one batched solve.

    positions [nf, N, 3], box [nf, 3, 3], pairs [nf, P, 2] with frame-local
    atom indices (rows beyond a frame's own pairs carry scale 0), ds and
    buffer_scales [nf, P]; chi, hardness, eta (and shift) [N] shared by the
    frames or [nf, N]; the constraint C [n_const, N], b [n_const] holds in
    every frame.  Returns q* [nf, N]; its gradients flow to positions, box,
    chi, hardness, eta, ds and shift through the implicit adjoint (a second
    batched CG with the same operator).  The reference solves one frame per
    pgrad_optimize call (qeq.py:1117-1270)."""
    nf, n = positions.shape[0], positions.shape[1]
    dev, dt = positions.device, positions.dtype

    def per_frame(v):
        return v.reshape(-1, n).expand(nf, n) if v is not None else None

    if q0 is None:
        q0 = torch.zeros(nf, n, dtype=dt, device=dev)
    if constraint_matrix is not None and constraint_vals is None:
        constraint_vals = torch.zeros(constraint_matrix.shape[0], dtype=dt, device=dev)
    if shift is None:
        shift = torch.zeros(nf, n, dtype=dt, device=dev)
    return QEqFramesFn.apply(positions, box, per_frame(chi), per_frame(hardness), per_frame(eta), ds,
                             per_frame(shift), module, pairs, buffer_scales, constraint_matrix, constraint_vals,
                             q0, module.eps if tol is None else tol, module.max_iter if max_iter is None else max_iter)
