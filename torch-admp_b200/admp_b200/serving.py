"""Continuous-batching server for PME energy+forces and QEq solves on one GPU.

Requests (positions, box and charges -- or QEq parameters) arrive over time.
The engine keeps every admitted system's state resident on the device --
positions, CSR neighbour rows, the CG vectors and scalars, the previous
charges of a QEq system -- in pools carved by offset.  Each scheduler tick:

  1. admits queued requests while slots, atom / pair pool space and the
     mesh scratch budget allow (admission by HBM footprint), copies their
     inputs host->device and builds their neighbour rows in one batched call;
  2. PME requests get energy + forces in one batched call and complete;
     QEq requests get their CG state initialised (warm start from the
     previous charges of the same system id, if any);
  3. runs ``iters_per_tick`` CG iterations over ALL active QEq systems in
     lock-step launches (systems admitted this tick join immediately;
     converged ones are skipped on the device);
  4. reads the per-slot done flags once (the tick's only host sync) and
     retires converged systems: final energy + forces at the solved charges,
     results device->host, resources freed.

All arithmetic runs in libadmp_b200.so (admp_serve_* entry points).
"""
from __future__ import annotations

import bisect
import concurrent.futures
import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from . import _lib as L
from .utils import DIELECTRIC

SYS_PME, SYS_QEQ = 0, 1
MAX_PER_LAUNCH = 256


class AdmpSys(ctypes.Structure):
    _fields_ = [("natoms", ctypes.c_int), ("atom_off", ctypes.c_int), ("slot", ctypes.c_int),
                ("kind", ctypes.c_int), ("kmesh", ctypes.c_int * 3), ("pad", ctypes.c_int),
                ("pair_off", ctypes.c_longlong), ("pair_cap", ctypes.c_longlong), ("green_off", ctypes.c_longlong),
                ("kappa", ctypes.c_double), ("rcut", ctypes.c_double)]


_P = ctypes.c_void_p


class AdmpPools(ctypes.Structure):
    _fields_ = [(n, _P) for n in ("pos", "q", "chi", "hardness", "eta", "force", "frac", "pstart", "pcnt", "cell_of",
                                  "sorted", "col", "coef", "box", "energy", "cg_state", "slot_info", "cg_x", "cg_r",
                                  "cg_diag", "cg_z", "cg_chi", "cg_hx", "cg_p", "cg_hp", "mesh")] + \
               [("mesh_cap", ctypes.c_longlong), ("spec", _P), ("spec_cap", ctypes.c_longlong), ("acc", _P),
                ("acc_cap", ctypes.c_int), ("cells", _P), ("cells_cap", ctypes.c_longlong), ("sys_scratch", _P),
                ("sys_scratch_bytes", ctypes.c_longlong), ("green", _P), ("green_cap", ctypes.c_longlong),
                ("pos64", _P), ("box64", _P), ("frac64", _P), ("flags", ctypes.c_int), ("slot_resid", _P)]

_COPY_THREADS = 4  # host threads copying request arrays into the pinned staging buffers


def _bind_serve(lib):
    if getattr(lib, "_serve_bound", False):
        return
    PP = ctypes.POINTER(AdmpPools)
    SP = ctypes.POINTER(AdmpSys)
    lib.admp_serve_slot_state_bytes.restype = ctypes.c_size_t
    lib.admp_serve_sys_scratch_bytes.restype = ctypes.c_size_t
    lib.admp_serve_sys_scratch_bytes.argtypes = [ctypes.c_int]
    lib.admp_serve_neighbors.argtypes = [ctypes.c_int, PP, SP, ctypes.c_int, _P]
    lib.admp_serve_energy_forces.argtypes = [ctypes.c_int, PP, SP, ctypes.c_int, ctypes.c_double, _P]
    lib.admp_serve_qeq_init.argtypes = [ctypes.c_int, PP, SP, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_double, _P]
    lib.admp_serve_qeq_iterate.argtypes = [ctypes.c_int, PP, SP, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_double, _P]
    lib.admp_serve_qeq_finish.argtypes = [ctypes.c_int, PP, SP, ctypes.c_int, _P]
    for n in ("admp_serve_neighbors", "admp_serve_energy_forces", "admp_serve_qeq_init", "admp_serve_qeq_iterate",
              "admp_serve_qeq_finish"):
        getattr(lib, n).restype = ctypes.c_int
    lib._serve_bound = True


class _Intervals:
    """First-fit allocator of integer ranges inside [0, cap)."""

    def __init__(self, cap: int, align: int = 1):
        self.cap = cap
        self.align = align
        self.free = [(0, cap)]

    def alloc(self, n: int) -> Optional[int]:
        n = (n + self.align - 1) // self.align * self.align
        for k, (a, b) in enumerate(self.free):
            if b - a >= n:
                if b - a == n:
                    self.free.pop(k)
                else:
                    self.free[k] = (a + n, b)
                return a
        return None

    def release(self, off: int, n: int) -> None:
        """Return [off, off + n) to the sorted free list, merged with its neighbours."""
        n = (n + self.align - 1) // self.align * self.align
        fr = self.free
        a, b = off, off + n
        k = bisect.bisect_left(fr, (a, b))
        if k > 0 and fr[k - 1][1] == a:
            k -= 1
            a = fr[k][0]
            del fr[k]
        if k < len(fr) and fr[k][0] == b:
            b = fr[k][1]
            del fr[k]
        fr.insert(k, (a, b))

    def used(self) -> int:
        return self.cap - sum(b - a for a, b in self.free)


@dataclass
class Result:
    rid: int
    kind: str
    energy: float
    forces: np.ndarray
    charges: Optional[np.ndarray]
    iterations: int
    status: int
    t_arrival: float
    t_done: float
    residual: float = 0.0   # QEq: final ||P grad||_2 / N of the charge solve (the reference's criterion)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


@dataclass
class _Active:
    req: object
    slot: int
    atom_off: int
    pair_off: int
    pair_cap: int
    kmesh: List[int]
    kind: int
    t_arrival: float
    green_off: int = -1
    green_n: int = 0
    retries: int = 0
    packed: Optional[bytes] = None


def auto_kmesh(box_diag, kappa: float, ethresh: float) -> List[int]:
    """ceil(2 kappa L / (3 ethresh^0.2)) per axis (pme.py:390-392)."""
    return [int(math.ceil(2 * kappa * float(L) / (3.0 * ethresh ** (1.0 / 5.0)))) for L in box_diag]


class ServingEngine:
    def __init__(self, device="cuda:0", dtype=torch.float32, max_atoms: int = 4_000_000, max_slots: int = 512,
                 pairs_per_atom: float = 150.0, mesh_budget: int = 64_000_000, rcut: float = 6.0,
                 ethresh: float = 5e-4, tol: float = 1e-6, max_iter: int = 300, iters_per_tick: int = 8,
                 ke: float = DIELECTRIC, green_budget: Optional[int] = None, admit_per_tick: int = 512):
        self.lib = L.load()
        _bind_serve(self.lib)
        self.dev = torch.device(device)
        self.dtype = dtype
        self.dt = L.dtype_code(dtype)
        self.rcut, self.ethresh = rcut, ethresh
        self.kappa = math.sqrt(-math.log(2 * ethresh)) / rcut
        self.tol, self.max_iter, self.iters_per_tick, self.ke = tol, max_iter, iters_per_tick, ke
        self.max_slots = max_slots
        # admissions per scheduler step: later ones are uploaded while the device works on earlier ones
        self.admit_per_tick = admit_per_tick
        A = max_atoms
        Pn = int(max_atoms * pairs_per_atom)
        f = dict(dtype=dtype, device=self.dev)
        i32 = dict(dtype=torch.int32, device=self.dev)
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.t = {
            "pos": torch.zeros(A, 3, **f), "q": torch.zeros(A, **f), "chi": torch.zeros(A, **f),
            "hardness": torch.zeros(A, **f), "eta": torch.zeros(A, **f), "force": torch.zeros(A, 3, **f),
            "frac": torch.zeros(A, 4, **f), "pstart": torch.zeros(A, dtype=torch.int64, device=self.dev),
            "pcnt": torch.zeros(A, **i32), "cell_of": torch.zeros(A, **i32), "sorted": torch.zeros(A, **i32),
            "col": torch.zeros(Pn, **i32), "coef": torch.zeros(Pn, **f),
            "box": torch.zeros(max_slots, 3, 3, **f), "energy": torch.zeros(max_slots, **f64),
            "cg_state": torch.zeros(max_slots * self.lib.admp_serve_slot_state_bytes(), dtype=torch.uint8,
                                    device=self.dev),
            "slot_info": torch.zeros(max_slots, 4, **i32),
            "cg_x": torch.zeros(A, **f64), "cg_r": torch.zeros(A, **f64), "cg_diag": torch.zeros(A, **f64),
            "cg_z": torch.zeros(A, **f64), "cg_chi": torch.zeros(A, **f64), "cg_hx": torch.zeros(A, **f64),
            "cg_p": torch.zeros(A, **f), "cg_hp": torch.zeros(A, **f),
            "mesh": torch.zeros(mesh_budget, **f), "spec": torch.zeros(mesh_budget + 1024, 2, **f),
            "acc": torch.zeros(MAX_PER_LAUNCH * 32, **f64),
            "cells": torch.zeros(3 * (2 * A + 129 * MAX_PER_LAUNCH), **i32),
            "sys_scratch": torch.zeros(self.lib.admp_serve_sys_scratch_bytes(MAX_PER_LAUNCH), dtype=torch.uint8,
                                       device=self.dev),
            "green": torch.zeros(green_budget if green_budget is not None else mesh_budget, **f),
            "slot_resid": torch.zeros(max_slots, **f64),
        }
        if dtype == torch.float32:
            # double copies for the neighbour decisions: the FP32 pair set equals the FP64 one
            self.t["pos64"] = torch.zeros(A, 3, **f64)
            self.t["box64"] = torch.zeros(max_slots, 3, 3, **f64)
            self.t["frac64"] = torch.zeros(A, 4, **f64)
        t = self.t
        self.pools = AdmpPools()
        for name in ("pos", "q", "chi", "hardness", "eta", "force", "frac", "pstart", "pcnt", "cell_of", "sorted",
                     "col", "coef", "box", "energy", "cg_state", "slot_info", "cg_x", "cg_r", "cg_diag", "cg_z",
                     "cg_chi", "cg_hx", "cg_p", "cg_hp", "mesh", "spec", "acc", "cells", "sys_scratch", "green"):
            setattr(self.pools, name, t[name].data_ptr())
        for name in ("pos64", "box64", "frac64"):
            setattr(self.pools, name, t[name].data_ptr() if name in t else None)
        self.pools.mesh_cap = mesh_budget
        self.pools.spec_cap = mesh_budget + 1024
        self.pools.acc_cap = MAX_PER_LAUNCH
        self.pools.cells_cap = t["cells"].numel()
        self.pools.sys_scratch_bytes = t["sys_scratch"].numel()
        self.pools.green_cap = t["green"].numel()
        self.pools.flags = 0
        self.pools.slot_resid = t["slot_resid"].data_ptr()
        self.greens = _Intervals(t["green"].numel(), 32)
        self.mesh_budget = mesh_budget
        self.atoms = _Intervals(A, 32)
        self.pairs = _Intervals(Pn, 64)
        self.free_slots = list(range(max_slots - 1, -1, -1))
        self.queue: List = []
        self.active_qeq: Dict[int, _Active] = {}
        self.results: List[Result] = []
        self.warm: Dict[object, np.ndarray] = {}
        self.stream = torch.cuda.current_stream(self.dev)
        # worker threads for the host-side copies of request arrays into the pinned staging buffers
        self._copy_pool = concurrent.futures.ThreadPoolExecutor(max_workers=_COPY_THREADS)
        self.pin = {}
        self.stats = {"ticks": 0, "launch_calls": 0, "admitted": 0, "h2d_bytes": 0, "d2h_bytes": 0, "retries": 0}
        self._fact_cache: Dict[int, tuple] = {}
        self._pair_grow: Dict[int, tuple] = {}   # pair capacity of requests served again after a row overflow
        self._retry: Dict[int, tuple] = {}
        self._inflight: List[tuple] = []  # launched work whose results are not read yet, in launch order
        self._zeros = {dt: torch.zeros(3 * 64, dtype=dt, device=self.dev) for dt in (torch.float32, torch.float64)}
        self._zero_views = {}  # (dtype, rows, width) -> view of _zeros, the padding parts of _fill
        # upload scratch: box rows of one admission on the device, pinned host staging (ring of three)
        self._box_stage = {dt: torch.zeros(max_slots, 9, dtype=dt, device=self.dev)
                           for dt in (torch.float32, torch.float64)}
        self._stage_ring = [[None, None, []] for _ in range(3)]
        self._stage_k = 0
        self._stage_off = 0
        # host seconds per scheduler phase (admission + upload, launches, waiting on the device, reading results)
        self.host_time = {"admit": 0.0, "launch": 0.0, "wait": 0.0, "results": 0.0}
        # when a list: (library call, start event, end event) of every call, for call_timeline()
        self.call_trace = None
        # results as host numpy arrays (True) or device tensors (False)
        self.results_to_host = True

    # -- resources -----------------------------------------------------------
    @staticmethod
    def _box_host(req):
        return np.asarray(getattr(req, "box_host", None) if getattr(req, "box_host", None) is not None else req.box)

    def _pair_estimate(self, req) -> int:
        n = req.natoms
        V = abs(float(np.linalg.det(self._box_host(req))))
        rho = n / V
        mean = rho * 4.0 / 3.0 * math.pi * self.rcut ** 3
        return int(n * (mean * 1.35 + 24)) + 256

    def _mesh_of(self, kmesh) -> int:
        return (kmesh[0] * kmesh[1] * kmesh[2] + 63) // 64 * 64

    def footprint(self, req) -> dict:
        """Device bytes a request holds while resident (atoms, pairs) and its mesh scratch."""
        fb = 4 if self.dtype == torch.float32 else 8
        per_atom = fb * 17 + 8 * 7 + 4 * 3
        per_pair = 4 + fb
        km = auto_kmesh(np.diagonal(self._box_host(req)), self.kappa, self.ethresh)
        return {"atom_bytes": req.natoms * per_atom, "pair_bytes": self._pair_estimate(req) * per_pair,
                "mesh_elems": self._mesh_of(km)}

    # -- API ------------------------------------------------------------------
    def submit(self, req, t_arrival: Optional[float] = None) -> None:
        self.queue.append((req, time.perf_counter() if t_arrival is None else t_arrival))

    def _facts(self, req):
        """(kmesh, mesh elements, pair capacity) of a request, computed once."""
        f = self._fact_cache.get(id(req))
        if f is None or f[0] is not req:
            km = auto_kmesh(np.diagonal(self._box_host(req)), self.kappa, self.ethresh)
            f = (req, km, self._mesh_of(km), self._pair_estimate(req))
            self._fact_cache[id(req)] = f
        grow = self._pair_grow.get(id(req))
        return f[1], f[2], (max(f[3], grow[1]) if grow is not None and grow[0] is req else f[3])

    def _sys_array(self, items: List[_Active]):
        """ctypes array of the launch descriptors; each request's descriptor is
        packed once and reused by every later launch that includes it."""
        for a in items:
            if a.packed is None:
                s = AdmpSys()
                s.natoms = a.req.natoms
                s.atom_off = a.atom_off
                s.slot = a.slot
                s.kind = a.kind
                for d in range(3):
                    s.kmesh[d] = a.kmesh[d]
                s.pair_off = a.pair_off
                s.pair_cap = a.pair_cap
                s.green_off = a.green_off
                s.kappa = self.kappa
                s.rcut = self.rcut
                a.packed = bytes(s)
        return (AdmpSys * len(items)).from_buffer_copy(b"".join(a.packed for a in items))

    def _chunks(self, items: List[_Active]):
        """Split into launches of <= MAX_PER_LAUNCH systems whose meshes fit the scratch budget."""
        out, cur, mesh = [], [], 0
        for a in items:
            m = self._mesh_of(a.kmesh)
            if cur and (len(cur) >= MAX_PER_LAUNCH or mesh + m > self.mesh_budget):
                out.append(cur)
                cur, mesh = [], 0
            cur.append(a)
            mesh += m
        if cur:
            out.append(cur)
        return out

    def _call(self, fn, items, *extra):
        tr = self.call_trace
        if tr is not None:
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
        for ch in self._chunks(items):
            arr = self._sys_array(ch)
            st = fn(self.dt, ctypes.byref(self.pools), arr, len(ch), *extra, self.stream.cuda_stream)
            self.stats["launch_calls"] += 1
            L.check(st, fn.__name__)
        if tr is not None:
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(self.stream)
            tr.append((fn.__name__, e0, e1))

    def call_timeline(self, start, end, top: int = 3) -> dict:
        """Device-side accounting of the calls traced between the events
        `start` and `end` (recorded on the engine's stream around a pass, with
        `call_trace` set to a list meanwhile): the stream time each library
        call's work spans, and the gaps between calls, in which the device ran
        only the engine's own copies or waited for the host."""
        tr = self.call_trace or []
        span, n = {}, {}
        gaps = []
        prev, prev_name = start, "start"
        for name, e0, e1 in tr:
            span[name] = span.get(name, 0.0) + e0.elapsed_time(e1)
            n[name] = n.get(name, 0) + 1
            gaps.append((prev.elapsed_time(e0), prev_name, name))
            prev, prev_name = e1, name
        gaps.append((prev.elapsed_time(end), prev_name, "end"))
        gaps.sort(key=lambda g: -g[0])
        return {"pass_ms": round(start.elapsed_time(end), 3),
                "calls": {k: {"n": n[k], "ms": round(v, 3)} for k, v in span.items()},
                "gap_ms": round(sum(g[0] for g in gaps), 3),
                "largest_gaps": [{"ms": round(g[0], 3), "after": g[1], "before": g[2]} for g in gaps[:top]]}

    def _admit(self, now: float) -> List[_Active]:
        """Admit arrived requests while slots and pool space allow.  Within a
        tick PME requests are placed before QEq requests, so that each kind
        occupies one contiguous run of the atom pool and uploads in one copy
        per field."""
        ready, keep = [], []
        for req, tarr in self.queue:
            (ready if tarr <= now else keep).append((req, tarr))
        ready.sort(key=lambda rt: 0 if rt[0].kind == "pme" else 1)
        admitted = []
        blocked = False
        for req, tarr in ready:
            if blocked or len(admitted) >= self.admit_per_tick:
                keep.append((req, tarr))
                continue
            n = req.natoms
            km, m, pcap = self._facts(req)
            if not self.free_slots or m > self.mesh_budget:
                keep.append((req, tarr))
                continue
            aoff = self.atoms.alloc(n)
            if aoff is None:
                keep.append((req, tarr))
                continue
            poff = self.pairs.alloc(pcap)
            if poff is None:
                self.atoms.release(aoff, n)
                keep.append((req, tarr))
                continue
            kind = SYS_QEQ if req.kind == "qeq" else SYS_PME
            goff, gn = -1, 0
            if kind == SYS_QEQ:
                gn = km[0] * km[1] * (km[2] // 2 + 1)
                goff = self.greens.alloc(gn)
                if goff is None:
                    self.atoms.release(aoff, n)
                    self.pairs.release(poff, pcap)
                    keep.append((req, tarr))
                    continue
            slot = self.free_slots.pop()
            rt = self._retry.pop(id(req), None)
            admitted.append(_Active(req, slot, aoff, poff, pcap, km, kind, tarr, goff, gn,
                                    retries=rt[1] if rt is not None and rt[0] is req else 0))
        keep.sort(key=lambda rt: rt[1])
        self.queue = keep
        if len(self._fact_cache) > 200_000:
            self._fact_cache.clear()
        if admitted:
            self._upload(admitted)
            self.stats["admitted"] += len(admitted)
        return admitted

    def _runs(self, items: List[_Active]):
        """Maximal runs of items whose atom regions follow each other up to the
        allocator's alignment padding."""
        al = self.atoms.align
        runs, cur = [], []
        for a in items:
            if cur:
                end = cur[-1].atom_off + cur[-1].req.natoms
                if a.atom_off != (end + al - 1) // al * al:
                    runs.append(cur)
                    cur = []
            cur.append(a)
        if cur:
            runs.append(cur)
        return runs

    def _stage_begin(self) -> None:
        """Start an upload on the next of three pinned host staging buffers; a
        buffer is reused only after the copies of its previous upload ran."""
        self._stage_k = (self._stage_k + 1) % 3
        buf, ev, _ = self._stage_ring[self._stage_k]
        if ev is not None:
            ev.synchronize()
        self._stage_ring[self._stage_k] = [buf, None, []]
        self._stage_off = 0

    def _stage_end(self) -> None:
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self._stage_ring[self._stage_k][1] = ev

    def _stage_take(self, n: int, npdt) -> np.ndarray:
        """n values of numpy dtype npdt from the current staging buffer (grown,
        keeping the old one alive until this upload's copies ran, if too small)."""
        slot = self._stage_ring[self._stage_k]
        item = np.dtype(npdt).itemsize
        off = (self._stage_off + 63) // 64 * 64
        need = off + n * item
        if slot[0] is None or slot[0].numel() < need:
            if slot[0] is not None:
                slot[2].append(slot[0])
            cap = max(need, 2 * (slot[0].numel() if slot[0] is not None else 0), 1 << 24)
            slot[0] = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
            off, need = 0, n * item
        self._stage_off = need
        return slot[0][off:need].numpy().view(npdt), slot[0][off:need].view(
            {np.float32: torch.float32, np.float64: torch.float64}[npdt])

    def _fill(self, dest, arrays, pads=None, width=1) -> int:
        """Write the request arrays, with pads[k] zero rows (of `width` values)
        after array k, into the contiguous pool slice `dest` without allocating:
        device tensors with one torch.cat into `dest`, host arrays through the
        pinned staging buffer and one copy.  Returns the host bytes copied."""
        pads = pads or [0] * len(arrays)
        dtype = dest.dtype
        if isinstance(arrays[0], torch.Tensor):
            # per part only the checks that decide whether a view is needed: a step admits hundreds of
            # requests and a torch view costs more host time than the check
            parts = []
            zv = self._zero_views
            for a, p in zip(arrays, pads):
                if a.dtype != dtype:
                    a = a.to(dtype)
                if width > 1:
                    if a.dim() != 2 or a.shape[1] != width:
                        a = a.reshape(-1, width)
                elif a.dim() != 1:
                    a = a.reshape(-1)
                parts.append(a)
                if p:
                    z = zv.get((dtype, p, width))
                    if z is None:
                        z = self._zeros[dtype][:p * width]
                        z = zv[(dtype, p, width)] = z.view(p, width) if width > 1 else z
                    parts.append(z)
            torch.cat(parts, out=dest.view(-1, width) if width > 1 else dest.view(-1))
            return 0
        npdt = {torch.float32: np.float32, torch.float64: np.float64}[dtype]
        n = dest.numel()
        host, th = self._stage_take(n, npdt)
        jobs = []
        o = 0
        for a, p in zip(arrays, pads):
            v = np.asarray(a).reshape(-1)
            jobs.append((o, v))
            o += v.size
            if p:
                host[o:o + p * width] = 0
                o += p * width

        def copy_part(k):
            # numpy releases the GIL for these copies, so the parts run in parallel
            for jo, jv in jobs[k::_COPY_THREADS]:
                host[jo:jo + jv.size] = jv

        if len(jobs) > 1 and n * host.itemsize >= (1 << 20):
            list(self._copy_pool.map(copy_part, range(_COPY_THREADS)))
        else:
            for jo, jv in jobs:
                host[jo:jo + jv.size] = jv
        dest.view(-1).copy_(th, non_blocking=True)
        return n * th.element_size()

    @staticmethod
    def _pads(run):
        """Zero rows between consecutive items of a run (alignment padding)."""
        return [run[k + 1].atom_off - (run[k].atom_off + run[k].req.natoms) for k in range(len(run) - 1)] + [0]

    def _upload(self, items: List[_Active]) -> None:
        t = self.t
        nb = 0
        has64 = "pos64" in t
        self._stage_begin()
        n = len(items)
        slots = torch.tensor([a.slot for a in items], dtype=torch.long).to(self.dev, non_blocking=True)
        bdt = torch.float64 if has64 else self.dtype
        boxes = self._box_stage[bdt][:n]
        nb += self._fill(boxes, [a.req.box for a in items], width=9)
        if has64:
            t["box64"].index_copy_(0, slots, boxes.view(-1, 3, 3))
            t["box"].index_copy_(0, slots, boxes.view(-1, 3, 3).to(self.dtype))
        else:
            t["box"].index_copy_(0, slots, boxes.view(-1, 3, 3))
        for run in self._runs(items):
            lo = run[0].atom_off
            hi = run[-1].atom_off + run[-1].req.natoms
            sl = slice(lo, hi)
            pads = self._pads(run)
            if has64:
                # positions arrive in double; the FP32 copy is made on the device
                nb += self._fill(t["pos64"][sl], [a.req.pos for a in run], pads, 3)
                t["pos"][sl].copy_(t["pos64"][sl], non_blocking=True)
            else:
                nb += self._fill(t["pos"][sl], [a.req.pos for a in run], pads, 3)
            # runs of one kind (PME first, then QEq, within a tick)
            k = 0
            while k < len(run):
                j = k
                while j < len(run) and run[j].kind == run[k].kind:
                    j += 1
                sub = run[k:j]
                ssl = slice(sub[0].atom_off, sub[-1].atom_off + sub[-1].req.natoms)
                spads = pads[k:j - 1] + [0]
                if sub[0].kind == SYS_PME:
                    nb += self._fill(t["q"][ssl], [a.req.charges for a in sub], spads)
                else:
                    for name in ("chi", "hardness", "eta"):
                        nb += self._fill(t[name][ssl], [getattr(a.req, name) for a in sub], spads)
                    t["q"][ssl].zero_()
                    for a in sub:
                        key = a.req.meta.get("system_id") if a.req.meta else None
                        w = self.warm.get(key) if key is not None else None
                        if w is not None and len(w) == a.req.natoms:
                            src = w.to(self.dtype) if isinstance(w, torch.Tensor) else torch.from_numpy(
                                np.asarray(w, dtype=np.float32 if self.dtype == torch.float32 else np.float64))
                            t["q"][a.atom_off:a.atom_off + a.req.natoms].copy_(src, non_blocking=True)
                k = j
        self._stage_end()
        self.stats["h2d_bytes"] += nb

    def _launch_finish(self, items: List[_Active]):
        """Launch energy + forces of finished systems and the copies of their
        results (forces and QEq charges of all of them leave the device in one
        gather + one copy); returns the in-flight record that
        _complete_finish reads once the record's event has passed."""
        self._call(self.lib.admp_serve_energy_forces, items, self.ke)
        t = self.t
        host = self.results_to_host
        runs = self._runs(sorted(items, key=lambda a: a.atom_off))
        F_all = torch.cat([t["force"][r[0].atom_off:r[-1].atom_off + r[-1].req.natoms] for r in runs])
        qitems = [a for a in items if a.kind == SYS_QEQ]
        qruns = self._runs(sorted(qitems, key=lambda a: a.atom_off))
        q_all = torch.cat([t["q"][r[0].atom_off:r[-1].atom_off + r[-1].req.natoms] for r in qruns]) if qruns else None
        if host:
            Fh = torch.empty(F_all.shape, dtype=self.dtype, pin_memory=True)
            Fh.copy_(F_all, non_blocking=True)
            qh = None
            if q_all is not None:
                qh = torch.empty(q_all.shape, dtype=self.dtype, pin_memory=True)
                qh.copy_(q_all, non_blocking=True)
            F_all, q_all = Fh, qh
        E = torch.empty(self.max_slots, dtype=torch.float64, pin_memory=True)
        E.copy_(t["energy"], non_blocking=True)
        info = torch.empty(self.max_slots, 4, dtype=torch.int32, pin_memory=True)
        info.copy_(t["slot_info"], non_blocking=True)
        resid = None
        if qitems:
            resid = torch.empty(self.max_slots, dtype=torch.float64, pin_memory=True)
            resid.copy_(t["slot_resid"], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        return ("finish", ev, items, runs, qruns, F_all, q_all, E, info, resid)

    def _complete_finish(self, rec, now_fn) -> None:
        """Results of a finish record out, resources freed (its event has passed)."""
        _, _, items, runs, qruns, F_all, q_all, E, info, resid = rec
        host = self.results_to_host
        tdone = now_fn()
        Fsrc = F_all.numpy() if host else F_all
        qsrc = (q_all.numpy() if host else q_all) if q_all is not None else None
        Eh = E.numpy()
        ih = info.numpy()
        rh = resid.numpy() if resid is not None else None
        # row of each system inside the gathered arrays (runs keep their alignment padding)
        off, qoff = {}, {}
        o = 0
        for r in runs:
            for a in r:
                off[a.slot] = o + a.atom_off - r[0].atom_off
            o += r[-1].atom_off + r[-1].req.natoms - r[0].atom_off
        o = 0
        for r in qruns:
            for a in r:
                qoff[a.slot] = o + a.atom_off - r[0].atom_off
            o += r[-1].atom_off + r[-1].req.natoms - r[0].atom_off
        if not host:  # device views of every system in one call each (per-system slicing costs ~10 us apiece)
            Fv, qv = self._views(Fsrc, off, items), (self._views(qsrc, qoff, items) if qsrc is not None else {})
        for a in items:
            n = a.req.natoms
            if host:
                Fo = Fsrc[off[a.slot]:off[a.slot] + n]
                qo = qsrc[qoff[a.slot]:qoff[a.slot] + n] if a.kind == SYS_QEQ else None
            else:
                Fo = Fv[a.slot]
                qo = qv.get(a.slot) if a.kind == SYS_QEQ else None
            st = int(ih[a.slot, 2])
            if st == L.CAPACITY and a.retries < 2:
                # a neighbour row outgrew its slot: serve the request again with the rows it needs
                need = int(ih[a.slot, 3])
                self._pair_grow[id(a.req)] = (a.req, max(2 * a.pair_cap, need + need // 8 + 1024))
                self._retry[id(a.req)] = (a.req, a.retries + 1)
                self.queue.append((a.req, a.t_arrival))
                self.stats["retries"] += 1
                self._release(a)
                continue
            it = int(ih[a.slot, 1]) if a.kind == SYS_QEQ else 0
            if host:
                self.stats["d2h_bytes"] += n * 3 * Fsrc.itemsize + 8 + (n * qsrc.itemsize if qo is not None else 0)
            if qo is not None and a.req.meta and a.req.meta.get("system_id") is not None:
                self.warm[a.req.meta["system_id"]] = qo.copy() if host else qo.clone()
            res = float(rh[a.slot]) if (rh is not None and a.kind == SYS_QEQ) else 0.0
            self.results.append(Result(a.req.rid, a.req.kind, float(Eh[a.slot]), Fo, qo, it, st, a.t_arrival, tdone,
                                       res))
            self._release(a)

    @staticmethod
    def _views(src, off, items):
        """{slot: src[off[slot]:off[slot] + natoms]} for the items whose slot is in `off`, from one
        torch.split over the gathered rows (gaps between systems become unused pieces)."""
        segs = sorted((off[a.slot], a.req.natoms, a.slot) for a in items if a.slot in off)
        sizes, keys, pos = [], [], 0
        for o, n, slot in segs:
            if o > pos:
                sizes.append(o - pos)
                keys.append(None)
            sizes.append(n)
            keys.append(slot)
            pos = o + n
        if pos < src.shape[0]:
            sizes.append(src.shape[0] - pos)
            keys.append(None)
        return {k: v for k, v in zip(keys, torch.split(src, sizes)) if k is not None}

    def _complete_iterate(self, rec) -> None:
        """Systems whose done flag (or error) showed in an iterate record's
        snapshot leave the CG set; their finish work is launched."""
        _, _, act, info = rec
        ih = info.numpy()
        done = [a for a in act if self.active_qeq.get(a.slot) is a and (ih[a.slot, 0] != 0 or ih[a.slot, 2] != 0)]
        for a in done:
            del self.active_qeq[a.slot]
        if done:
            self._call(self.lib.admp_serve_qeq_finish, done)
            self._inflight.append(self._launch_finish(done))

    def _drain(self, now_fn, max_iter_records: int, keep_new: int = 0) -> None:
        """Complete in-flight records in launch order: every record whose
        event has passed, and the oldest ones (waiting on them) while more than
        `max_iter_records` iterate records are outstanding.  Keeping one
        iterate record in flight lets the host read results while the device
        works on the next batch of CG iterations.  With `max_iter_records` 0
        (no CG batch running) all but the `keep_new` newest records are waited
        for."""
        while self._inflight:
            rec = self._inflight[0]
            if max_iter_records > 0:
                n_iter = sum(1 for r in self._inflight if r[0] == "iter")
                if n_iter <= max_iter_records and not rec[1].query():
                    break
            elif len(self._inflight) <= keep_new and not rec[1].query():
                break
            self._inflight.pop(0)
            h0 = time.perf_counter()
            rec[1].synchronize()
            h1 = time.perf_counter()
            self.host_time["wait"] += h1 - h0
            if rec[0] == "finish":
                self._complete_finish(rec, now_fn)
            else:
                self._complete_iterate(rec)
            self.host_time["results"] += time.perf_counter() - h1

    def _release(self, a: _Active) -> None:
        self.atoms.release(a.atom_off, a.req.natoms)
        self.pairs.release(a.pair_off, a.pair_cap)
        if a.green_off >= 0:
            self.greens.release(a.green_off, a.green_n)
        self.free_slots.append(a.slot)

    def tick(self, now_fn=time.perf_counter) -> int:
        """One scheduler step; returns the number of results completed.

        Work is launched first (neighbour lists, CG set-up and PME
        energy + forces of newly admitted systems, then a batch of CG
        iterations over every active QEq system with a snapshot of the
        per-slot done flags); results of earlier steps are read afterwards,
        so the device stays busy while the host schedules.  While arrived
        requests wait, this step's launches are left in flight even with no
        CG batch running, so the next step's admission overlaps them.

        Every copy and launch goes to the engine's stream (the stream that
        was current when the engine was built), whatever stream is current
        at the call, so the staging-buffer events cover the uploads."""
        with torch.cuda.stream(self.stream):
            return self._tick(now_fn)

    def _tick(self, now_fn) -> int:
        n0 = len(self.results)
        r0 = len(self._inflight)
        now = now_fn()
        h0 = time.perf_counter()
        new = self._admit(now)
        h1 = time.perf_counter()
        self.host_time["admit"] += h1 - h0
        if new:
            self._call(self.lib.admp_serve_neighbors, new)
            pme = [a for a in new if a.kind == SYS_PME]
            qeq = [a for a in new if a.kind == SYS_QEQ]
            if qeq:
                self._call(self.lib.admp_serve_qeq_init, qeq, self.tol, self.max_iter, self.ke)
                for a in qeq:
                    self.active_qeq[a.slot] = a
            if pme:
                self._inflight.append(self._launch_finish(pme))
        if self.active_qeq:
            act = list(self.active_qeq.values())
            self._call(self.lib.admp_serve_qeq_iterate, act, self.iters_per_tick, self.tol, self.max_iter, self.ke)
            info = torch.empty(self.max_slots, 4, dtype=torch.int32, pin_memory=True)
            info.copy_(self.t["slot_info"], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self._inflight.append(("iter", ev, act, info))
        self.host_time["launch"] += time.perf_counter() - h1
        # with arrived requests still waiting (a backlog), this step's records stay in flight so the
        # next step's admission overlaps their device work; otherwise they are waited for at once
        backlog = bool(self.queue) and self.queue[0][1] <= now
        self._drain(now_fn, 1 if self.active_qeq else 0, len(self._inflight) - r0 if backlog else 0)
        self.stats["ticks"] += 1
        return len(self.results) - n0

    def pending(self) -> int:
        return len(self.queue) + len(self.active_qeq) + len(self._inflight)

    def run(self, requests, arrivals: bool = True, time_scale: float = 1.0, max_seconds: float = 1e9):
        """Serve a list of requests.  With ``arrivals`` the request ``arrival``
        times (seconds) are honoured relative to the start; otherwise all are
        available at once.  Returns the results in completion order."""
        t0 = time.perf_counter()
        for r in requests:
            self.submit(r, t0 + (r.arrival * time_scale if arrivals else 0.0))
        with torch.cuda.stream(self.stream):
            return self._run_loop(t0, max_seconds)

    def _run_loop(self, t0: float, max_seconds: float):
        while self.pending():
            if self._tick(time.perf_counter) == 0 and not self.active_qeq and not self._inflight:
                # nothing on the device: wait for the next arrival
                nxt = min(t for _, t in self.queue) if self.queue else None
                if nxt is not None:
                    dt = nxt - time.perf_counter()
                    if dt > 0:
                        time.sleep(min(dt, 0.01))
            if time.perf_counter() - t0 > max_seconds:
                raise TimeoutError("serving run exceeded its time limit")
        return self.results
