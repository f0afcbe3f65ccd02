"""Autograd functions over the C ABI with hand-written backward passes.

Each forward launches the sm_100a kernels once and, when any input needs a
gradient, produces the energy's gradients in the same pass (they come almost
for free: the reciprocal gradient needs the same potential mesh as the
energy).  The backward multiplies the saved gradients by the incoming
gradient.  Gradients flow to positions, box, the caller's distances ``ds``,
charges and the QEq parameters -- the contract of the reference modules,
whose forces come from torch.autograd (utils.py:85-112).
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import torch

from . import _lib as L


def _zeros_like_opt(t: Optional[torch.Tensor], need: bool):
    return torch.zeros_like(t) if (need and t is not None) else None


def _c(t: Optional[torch.Tensor]):
    return None if t is None else t.contiguous()


def coulomb_pbc(pos, box, pairs, ds, bs, q, kappa: float, kmesh: Sequence[Sequence[int]], ke: float,
                rspace: bool, kspace: bool, slab: bool, axis: int, need_grad: bool):
    """Energies of CoulombForceModule._forward_pbc (pme.py:261-310) for nf frames.

    Returns (E [nf] float64, comps [nf,5] float64 (real, recip, self, non_neutral, slab),
    grads dict or None)."""
    lib = L.load()
    dev = pos.device
    dt = L.dtype_code(pos.dtype)
    nf, N = pos.shape[0], pos.shape[1]
    P = pairs.shape[1]
    st = L.stream_of(dev)
    E_real = torch.zeros(nf, dtype=torch.float64, device=dev)
    E_recip = torch.zeros(nf, dtype=torch.float64, device=dev)
    terms = torch.zeros(nf, 5, dtype=torch.float64, device=dev)
    g = None
    if need_grad:
        g = {"pos": torch.zeros_like(pos), "box": torch.zeros_like(box), "ds": torch.zeros_like(ds),
             "q": torch.zeros_like(q)}
    if rspace and P > 0:
        L.check(lib.admp_pair_energy(dt, L.PAIR_EWALD, nf, N, P, L.ptr(pairs), L.ptr(ds), L.ptr(bs), L.ptr(q), None,
                                     float(kappa), ke, L.ptr(E_real), L.ptr(g["ds"]) if g else None,
                                     L.ptr(g["q"]) if g else None, None, st), "real-space pair energy")
    if kspace and N > 0:
        km_flat = [int(k) for row in kmesh for k in row]
        kp, _keep = L.int3(km_flat)
        nbytes = lib.admp_pme_recip_workspace_size(dt, nf, kp)
        if nbytes == 0:
            L.check(L.MESH, "reciprocal workspace")
        ws = L.workspace(nbytes, dev)
        L.check(lib.admp_pme_recip(dt, nf, N, kp, L.ptr(pos), L.ptr(box), L.ptr(q), float(kappa), ke, L.ptr(E_recip),
                                   L.ptr(g["pos"]) if g else None, L.ptr(g["q"]) if g else None,
                                   L.ptr(g["box"]) if g else None, L.ptr(ws), nbytes, st), "reciprocal PME")
    flags = 0
    if kspace:
        flags |= L.TERM_SELF | L.TERM_NON_NEUTRAL
    if slab:
        flags |= L.TERM_SLAB | (int(axis) << 8)
    if flags and N > 0:
        L.check(lib.admp_atom_terms(dt, flags, nf, N, L.ptr(pos), L.ptr(box), L.ptr(q), None, None, None,
                                    float(kappa), ke, None, L.ptr(terms), L.ptr(g["q"]) if g else None,
                                    L.ptr(g["pos"]) if g else None, L.ptr(g["box"]) if g else None, None, None,
                                    None, st), "self / non-neutral / slab terms")
    comps = torch.stack([E_real, E_recip, terms[:, 0], terms[:, 1], terms[:, 2]], dim=1)
    return comps.sum(1), comps, g


def coulomb_obc(pairs, ds, bs, q, ke: float, need_grad: bool):
    """pme.py:529-561."""
    lib = L.load()
    dev = q.device
    dt = L.dtype_code(q.dtype)
    nf, N = q.shape
    P = pairs.shape[1]
    E = torch.zeros(nf, dtype=torch.float64, device=dev)
    g = {"ds": torch.zeros_like(ds), "q": torch.zeros_like(q)} if need_grad else None
    if P > 0:
        L.check(lib.admp_pair_energy(dt, L.PAIR_OBC, nf, N, P, L.ptr(pairs), L.ptr(ds), L.ptr(bs), L.ptr(q), None,
                                     0.0, ke, L.ptr(E), L.ptr(g["ds"]) if g else None, L.ptr(g["q"]) if g else None,
                                     None, L.stream_of(dev)), "open-boundary Coulomb")
    return E, g


class CoulombFn(torch.autograd.Function):
    """E(pos, box, ds, q) of CoulombForceModule; returns (E [nf], comps [nf,5])."""

    @staticmethod
    def forward(ctx, pos, box, ds, q, pairs, bs, cfg):
        need = any(ctx.needs_input_grad[:4])
        if box is None:
            E, g = coulomb_obc(pairs, ds, bs, q, cfg["ke"], need)
            comps = torch.zeros(q.shape[0], 5, dtype=torch.float64, device=q.device)
            comps[:, 0] = E
        else:
            E, comps, g = coulomb_pbc(pos, box, pairs, ds, bs, q, cfg["kappa"], cfg["kmesh"], cfg["ke"],
                                      cfg["rspace"], cfg["kspace"], cfg["slab"], cfg["axis"], need)
        ctx.has_box = box is not None
        if need:
            ctx.save_for_backward(g.get("pos"), g.get("box"), g["ds"], g["q"])
        ctx.mark_non_differentiable(comps)
        return E.to(q.dtype), comps

    @staticmethod
    def backward(ctx, gE, gcomps):
        gp, gb, gds, gq = ctx.saved_tensors
        w = gE
        out_pos = gp * w[:, None, None] if (gp is not None and ctx.needs_input_grad[0]) else None
        out_box = gb * w[:, None, None] if (gb is not None and ctx.needs_input_grad[1]) else None
        out_ds = gds * w[:, None] if ctx.needs_input_grad[2] else None
        out_q = gq * w[:, None] if ctx.needs_input_grad[3] else None
        return out_pos, out_box, out_ds, out_q, None, None, None


def damping_raw(ds, q, eta, pairs, bs, ke: float, need: bool):
    """Gaussian damping energy (pair + self) and optional gradients (qeq.py:60-129)."""
    lib = L.load()
    dev = q.device
    dt = L.dtype_code(q.dtype)
    nf, N = q.shape
    P = pairs.shape[1]
    st = L.stream_of(dev)
    E = torch.zeros(nf, dtype=torch.float64, device=dev)
    gds = torch.zeros_like(ds) if need else None
    gq = torch.zeros_like(q) if need else None
    geta = torch.zeros_like(eta) if need else None
    if P > 0:
        L.check(lib.admp_pair_energy(dt, L.PAIR_DAMPING, nf, N, P, L.ptr(pairs), L.ptr(ds), L.ptr(bs), L.ptr(q),
                                     L.ptr(eta), 0.0, ke, L.ptr(E), L.ptr(gds), L.ptr(gq), L.ptr(geta), st),
                "damping pair energy")
    if N > 0:
        L.check(lib.admp_atom_terms(dt, L.TERM_DAMP_SELF, nf, N, None, None, L.ptr(q), L.ptr(eta), None, None, 0.0,
                                    ke, L.ptr(E), None, L.ptr(gq), None, None, L.ptr(geta), None, None, st),
                "damping self energy")
    return E, gds, gq, geta


class DampingFn(torch.autograd.Function):
    """GaussianDampingForceModule energy (qeq.py:60-129): E(ds, q, eta)."""

    @staticmethod
    def forward(ctx, ds, q, eta, pairs, bs, ke):
        need = any(ctx.needs_input_grad[:3])
        E, gds, gq, geta = damping_raw(ds, q, eta, pairs, bs, ke, need)
        if need:
            ctx.save_for_backward(gds, gq, geta)
        return E.to(q.dtype)

    @staticmethod
    def backward(ctx, gE):
        gds, gq, geta = ctx.saved_tensors
        w = gE[:, None]
        return (gds * w if ctx.needs_input_grad[0] else None, gq * w if ctx.needs_input_grad[1] else None,
                geta * w if ctx.needs_input_grad[2] else None, None, None, None)


class SiteFn(torch.autograd.Function):
    """SiteForceModule energy sum(chi q + hardness q^2) (qeq.py:159-209)."""

    @staticmethod
    def forward(ctx, q, chi, hard):
        lib = L.load()
        dev = q.device
        dt = L.dtype_code(q.dtype)
        nf, N = q.shape
        need = any(ctx.needs_input_grad[:3])
        E = torch.zeros(nf, dtype=torch.float64, device=dev)
        gq = torch.zeros_like(q) if need else None
        gc = torch.zeros_like(chi) if need else None
        gh = torch.zeros_like(hard) if need else None
        if N > 0:
            L.check(lib.admp_atom_terms(dt, L.TERM_SITE, nf, N, None, None, L.ptr(q), None, L.ptr(chi), L.ptr(hard),
                                        0.0, 0.0, L.ptr(E), None, L.ptr(gq), None, None, None, L.ptr(gc), L.ptr(gh),
                                        L.stream_of(dev)), "site energy")
        if need:
            ctx.save_for_backward(gq, gc, gh)
        return E.to(q.dtype)

    @staticmethod
    def backward(ctx, gE):
        gq, gc, gh = ctx.saved_tensors
        w = gE[:, None]
        return (gq * w if ctx.needs_input_grad[0] else None, gc * w if ctx.needs_input_grad[1] else None,
                gh * w if ctx.needs_input_grad[2] else None)


class PairDistanceFn(torch.autograd.Function):
    """ds = |pbc_shift(r_i - r_j)| (nblist.py:517-551) with a hand-written backward."""

    @staticmethod
    def forward(ctx, pos, box, pairs):
        lib = L.load()
        dt = L.dtype_code(pos.dtype)
        P = pairs.shape[0]
        ds = torch.empty(P, dtype=pos.dtype, device=pos.device)
        pbc = 1 if box is not None else 0
        L.check(lib.admp_pair_distances(dt, pbc, pos.shape[0], P, L.ptr(pairs), L.ptr(pos), L.ptr(box), L.ptr(ds),
                                        L.stream_of(pos.device)), "pair distances")
        ctx.save_for_backward(pos, box if box is not None else torch.empty(0, device=pos.device), pairs)
        ctx.pbc = pbc
        return ds

    @staticmethod
    def backward(ctx, gds):
        pos, box, pairs = ctx.saved_tensors
        lib = L.load()
        dt = L.dtype_code(pos.dtype)
        gpos = torch.zeros_like(pos) if ctx.needs_input_grad[0] else None
        gbox = torch.zeros_like(box) if (ctx.pbc and ctx.needs_input_grad[1]) else None
        if gpos is not None or gbox is not None:
            L.check(lib.admp_pair_distances_backward(dt, ctx.pbc, pos.shape[0], pairs.shape[0], L.ptr(pairs),
                                                     L.ptr(pos), L.ptr(box) if ctx.pbc else None,
                                                     L.ptr(gds.contiguous()), L.ptr(gpos), L.ptr(gbox),
                                                     L.stream_of(pos.device)), "pair distances backward")
        return gpos, gbox, None


def neighbor_pairs(pos: torch.Tensor, box: Optional[torch.Tensor], cutoff: float):
    """Cell-list pair build (nblist.py:304-445): returns pairs [P,2] int64, buffer_scales [P] int64."""
    lib = L.load()
    dev = pos.device
    dt = L.dtype_code(pos.dtype)
    N = pos.shape[0]
    st = L.stream_of(dev)
    nbytes = lib.admp_nblist_workspace_size(N)
    ws = L.workspace(nbytes, dev)
    import ctypes
    npairs = ctypes.c_longlong(0)
    pbc = 1 if box is not None else 0
    L.check(lib.admp_nblist_count(dt, pbc, N, L.ptr(pos), L.ptr(box), float(cutoff), L.ptr(ws), nbytes,
                                  ctypes.byref(npairs), st), "neighbour list")
    P = int(npairs.value)
    pairs = torch.empty((P, 2), dtype=torch.long, device=dev)
    bs = torch.empty(P, dtype=torch.long, device=dev)
    if P > 0:
        L.check(lib.admp_nblist_fill(dt, pbc, N, L.ptr(pos), L.ptr(box), float(cutoff), L.ptr(ws), nbytes,
                                     L.ptr(pairs), L.ptr(bs), P, st), "neighbour list fill")
    return pairs, bs


class ImagePairDistanceFn(torch.autograd.Function):
    """ds = |r_j - r_i + n.B| for pairs with integer image shifts n (make_ds, nblist.py:212-240)."""

    @staticmethod
    def forward(ctx, pos, box, pairs, shifts):
        lib = L.load()
        dt = L.dtype_code(pos.dtype)
        P = pairs.shape[0]
        ds = torch.empty(P, dtype=pos.dtype, device=pos.device)
        L.check(lib.admp_image_pair_distances(dt, pos.shape[0], P, L.ptr(pairs), L.ptr(shifts), L.ptr(pos),
                                              L.ptr(box), L.ptr(ds), L.stream_of(pos.device)), "pair distances")
        ctx.save_for_backward(pos, box if box is not None else torch.empty(0, device=pos.device), pairs, shifts)
        ctx.has_box = box is not None
        return ds

    @staticmethod
    def backward(ctx, gds):
        pos, box, pairs, shifts = ctx.saved_tensors
        lib = L.load()
        dt = L.dtype_code(pos.dtype)
        gpos = torch.zeros_like(pos) if ctx.needs_input_grad[0] else None
        gbox = torch.zeros_like(box) if (ctx.has_box and ctx.needs_input_grad[1]) else None
        if gpos is not None or gbox is not None:
            L.check(lib.admp_image_pair_distances_backward(dt, pos.shape[0], pairs.shape[0], L.ptr(pairs),
                                                           L.ptr(shifts), L.ptr(pos),
                                                           L.ptr(box) if ctx.has_box else None,
                                                           L.ptr(gds.contiguous()), L.ptr(gpos), L.ptr(gbox),
                                                           L.stream_of(pos.device)), "pair distances backward")
        return gpos, gbox, None, None


def image_neighbor_pairs(pos: torch.Tensor, box: Optional[torch.Tensor], cutoff: float, nnei: int):
    """Pairs over periodic images (dp_nblist's pair set, nblist.py:33-93, 173-209).

    Returns pairs [P,2] int64 (i < j images, then self images (i, i)), image
    shifts [P,3] int32, the number of i < j pairs and the number of atoms
    whose list was cut to their nnei nearest images."""
    import ctypes
    lib = L.load()
    dev = pos.device
    dt = L.dtype_code(pos.dtype)
    N = pos.shape[0]
    st = L.stream_of(dev)
    nbytes = lib.admp_image_nblist_workspace_size(N)
    ws = L.workspace(nbytes, dev)
    n_ij, n_ii, ntr = ctypes.c_longlong(0), ctypes.c_longlong(0), ctypes.c_int(0)
    pbc = 1 if box is not None else 0
    L.check(lib.admp_image_nblist_count(dt, pbc, N, L.ptr(pos), L.ptr(box), float(cutoff), int(nnei), L.ptr(ws),
                                        nbytes, ctypes.byref(n_ij), ctypes.byref(n_ii), ctypes.byref(ntr), st),
            "image neighbour list")
    P = int(n_ij.value) + int(n_ii.value)
    pairs = torch.empty((P, 2), dtype=torch.long, device=dev)
    shifts = torch.empty((P, 3), dtype=torch.int32, device=dev)
    if P > 0:
        L.check(lib.admp_image_nblist_fill(dt, pbc, N, L.ptr(pos), L.ptr(box), float(cutoff), L.ptr(ws), nbytes,
                                           L.ptr(pairs), L.ptr(shifts), P, st), "image neighbour list fill")
    return pairs, shifts, int(n_ij.value), int(ntr.value)
