"""Benchmark: PME+QEq serving stream (systems/s, p50/p99 latency) on B200.

Workload (one "step" = one pass over the stream): N_REQ requests with atom
counts log-uniform in [200, 20000], cubic boxes at 0.1 atoms/A^3, 60% PME
energy+forces (+-1 charges) and 40% QEq solves on water-like systems, rc 6 A,
ethresh 5e-4 (mesh from the reference's automatic rule), CG to
||P grad|| / N < 1e-7.  Synthetic, seeded (the reference has no dataset).

  value        systems/s of the batched FP32 serving engine with every input
               already resident in HBM (closed loop: all requests available)
  e2e          the same through the public engine API from host numpy
               arrays (H2D inputs and D2H results inside the timed region);
               p50/p99 latency from an open-loop Poisson pass at a stated rate
  plain_gpu    one system at a time through the drop-in modules (FP32)
  roofline     dominant kernel's algorithmic GB/s from CUDA events vs the
               measured HBM copy bandwidth
  cpu_baseline the CPU oracle (restatement of the reference) on a sample

`--impl reference` times the CPU oracle alone (rank 0).  Under torchrun each
rank serves its own stream (replicas; no collective on the data path).
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "torch-admp_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "PME+QEq systems/sec and p50/p99 latency vs plain GPU path at 1e-4 force err"
UNIT = "systems/s"
N_REQ = 2000
SEED = 1024
RATE = 2000.0          # Poisson arrival rate (requests/s) of the synthetic stream
RCUT, ETHRESH = 6.0, 5e-4
# CG stopping rule ||P grad||_2 / N < TOL; 1e-7 keeps the FP32 charges within 1e-5 e and the
# forces within 1e-4 of the FP64 solution (at 1e-6 the charge error reaches ~5e-6 e and the
# force error ~2e-4)
TOL = 1e-7
LAT_RATE = 1000.0      # open-loop Poisson rate (requests/s) for the p50/p99 latency pass
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic byte, from one ncu capture of
# every launch of these kernels in five passes of the 400-request stream (x pass 85.5 MB per launch,
# spread 62.5, gather 58.1); roofline.traffic = ratio x algorithmic bytes per launch of this run
TRAFFIC_PER_ALG_BYTE = {"fft_x_green": 0.600, "spread": 0.959, "gather": 0.857}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nreq", type=int, default=N_REQ)
    ap.add_argument("--latency-rate", type=float, default=LAT_RATE,
                    help="open-loop Poisson arrival rate (requests/s) for p50/p99")
    ap.add_argument("--cpu-reps", type=int, default=None,
                    help="repetitions of the CPU sample (default 3 for --impl reference, 1 beside the GPU arm)")
    ap.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE,
                    help="requests in the size-stratified CPU sample")
    ap.add_argument("--plain-sample", type=int, default=100)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the FP64 serving, electrode and differentiation-batch legs")
    ap.add_argument("--timeline", action="store_true",
                    help="after the timed passes, trace one device-resident pass call by call (CUDA events "
                         "around each library call) and print the accounting as JSON on stderr")
    return ap.parse_args()


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x: float, device=None) -> float:
    """The largest value of x over all ranks (x itself without a process
    group): replicas are timed on their own devices and the job takes as long
    as its slowest rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_stream(nreq: int, rank: int):
    """Each replica serves its own seeded stream of the same distribution."""
    from admp_b200 import synthetic
    return synthetic.serving_stream(nreq, SEED + rank, RATE)


# ---------------------------------------------------------------- CPU oracle
def _cpu_one(req_tuple):
    """One request on the CPU oracle (restatement of the reference path:
    cell-list neighbours, PME energy + forces, or the reference's projected
    nonlinear CG for QEq followed by energy + forces).  Returns (seconds,
    energy, forces, charges or None)."""
    from oracle import admp_oracle as O
    t0 = time.perf_counter()
    kind, pos, box, q, chi, hard, eta = req_tuple
    kappa = O.ewald_kappa(RCUT, ETHRESH)
    km = O.auto_kmesh(box, kappa, ETHRESH)
    pairs = O.nblist_pbc_cells(pos, box, RCUT)
    bs = O.pair_buffer_scales(pairs)
    if kind == "pme":
        o = O.coulomb_forces(pos, box, pairs, bs, q, rcut=RCUT, ethresh=ETHRESH, kmesh=km)
        return time.perf_counter() - t0, o["E"], o["forces"], None
    ds = O.pairs_ds(pos, pairs, box)
    s = O.QEqSystem(pos, box, chi, hard, eta, pairs, ds, bs, rcut=RCUT, ethresh=ETHRESH, kmesh=km)
    n = pos.shape[0]
    qs, _ = O.solve_quadratic(s, np.zeros(n), np.ones((1, n)), np.zeros(1), max_iter=200, eps=TOL)
    E, _ = s.energy_grad(qs)
    o = O.coulomb_forces(pos, box, pairs, bs, qs, rcut=RCUT, ethresh=ETHRESH, kmesh=km)
    _, dds, _, _ = O.damping(qs, eta, pairs, ds, bs)
    dpd, _ = O.ds_backward(pos, box, pairs, dds)
    return time.perf_counter() - t0, E, o["forces"] - dpd, qs


CPU_SAMPLE = 48   # requests of the size-stratified CPU sample


def cpu_sample(stream, k: int = CPU_SAMPLE):
    """k requests of the stream, one from each of k equal-count strata of the
    stream sorted by atom count (the request at each stratum's middle), so
    the sample follows the stream's size distribution and mix of kinds."""
    srt = sorted(stream, key=lambda r: (r.natoms, r.rid))
    n = len(srt)
    return [srt[min(n - 1, int((j + 0.5) * n / k))] for j in range(min(k, n))]


def cpu_baseline(stream, reps: int = 1, k: int = CPU_SAMPLE):
    """CPU oracle throughput, measured: the size-stratified sample of the
    stream runs on every host core at once (spawn pool, one request per
    task, largest first), each request timed on its core while the others
    run.  value = cores x requests / core-seconds of the sample (the rate of
    a stream that keeps every core busy with requests of the sample's size
    mix), the median over `reps` repetitions.  The sample's own wall clock is
    bounded below by its largest request (one core busy at the end), so
    requests / wall seconds is reported beside it as `wall_value`, a lower
    bound.  A secondary figure extrapolates the per-request times per kind
    (power law in N) to the whole stream.  Returns (systems/s, cores,
    description, details dict)."""
    import multiprocessing as mp
    picks = cpu_sample(stream, k)
    cores = min(os.cpu_count() or 1, len(picks))  # pool workers
    order = sorted(range(len(picks)), key=lambda j: -(picks[j].natoms * (8 if picks[j].kind == "qeq" else 1)))
    tasks = [(picks[j].kind, picks[j].pos, picks[j].box, picks[j].charges, picks[j].chi, picks[j].hardness,
              picks[j].eta) for j in order]
    ctx = mp.get_context("spawn")
    walls, rates, times, outs = [], [], None, None
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_warm, range(cores), chunksize=1)
        for _ in range(max(1, reps)):
            t0 = time.perf_counter()
            outs = pool.map(_cpu_one, tasks, chunksize=1)
            walls.append(time.perf_counter() - t0)
            t = [o[0] for o in outs]
            rates.append(cores * len(tasks) / sum(t))
            times = t if times is None else [min(a, b) for a, b in zip(times, t)]
    wall = statistics.median(walls)
    value = statistics.median(rates)
    # secondary: power law t = a N^b per kind over the measured requests, summed over the whole stream
    byreq = [(picks[j], tt) for j, tt in zip(order, times)]
    pred = 0.0
    for kind in ("pme", "qeq"):
        pts = [(r.natoms, tt) for r, tt in byreq if r.kind == kind]
        if not pts:
            continue
        x = np.log([p_[0] for p_ in pts])
        y = np.log([p_[1] for p_ in pts])
        b, a = np.polyfit(x, y, 1) if len(pts) > 1 else (1.0, y[0] - x[0])
        pred += sum(math.exp(a + b * math.log(r.natoms)) for r in stream if r.kind == kind)
    nq = sum(1 for r in picks if r.kind == "qeq")
    desc = (f"{len(tasks)} requests ({len(tasks) - nq} PME, {nq} QEq; {min(r.natoms for r in picks)}-"
            f"{max(r.natoms for r in picks)} atoms, one per atom-count stratum of the stream) on {cores} cores at "
            f"once; value = cores x requests / core-seconds (median of {len(rates)}: "
            f"{', '.join(f'{r_:.2f}' for r_ in rates)} systems/s); wall {wall:.1f} s, bounded by the largest request")
    details = {"wall_s": walls, "wall_value": len(tasks) / wall, "rates": rates, "core_seconds": sum(times),
               "requests": len(tasks),
               "extrapolated_stream_value": cores * len(stream) / pred if pred > 0 else None,
               "rids": [r.rid for r in picks],
               "results": {picks[j].rid: o[1:] for j, o in zip(order, outs)}}
    return value, cores, desc, details


def _cpu_warm(_):
    """Import the oracle in a pool worker before the timed repetitions."""
    from oracle import admp_oracle  # noqa: F401
    return 0


# ---------------------------------------------------------------- GPU helpers
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.time(), ln.strip()))

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0: float = None, t1: float = None):
        """Samples taken in [t0, t1] (all of them when none falls there)."""
        lines = [ln for t, ln in self.lines if t0 is None or t0 <= t <= t1]
        if not lines:
            lines = [ln for _, ln in self.lines]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[3 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def to_device_requests(stream, dev, dtype):
    """Copies of the requests whose arrays live on the GPU."""
    import copy

    import torch
    out = []
    for r in stream:
        c = copy.copy(r)
        c.pos = torch.as_tensor(r.pos, dtype=torch.float64, device=dev)
        c.box_host = r.box
        c.box = torch.as_tensor(r.box, dtype=torch.float64, device=dev)
        if r.kind == "pme":
            c.charges = torch.as_tensor(r.charges, dtype=dtype, device=dev)
        else:
            c.chi = torch.as_tensor(r.chi, dtype=dtype, device=dev)
            c.hardness = torch.as_tensor(r.hardness, dtype=dtype, device=dev)
            c.eta = torch.as_tensor(r.eta, dtype=dtype, device=dev)
        out.append(c)
    return out


def plain_path(stream, dev, dtype, n, eps=TOL):
    """One system at a time through the drop-in modules (what a user of the
    reference API would run on the GPU)."""
    import torch

    from admp_b200.nblist import TorchNeighborList
    from admp_b200.pme import CoulombForceModule
    from admp_b200.qeq import QEqForceModule, pgrad_optimize
    cm = CoulombForceModule(rcut=RCUT, ethresh=ETHRESH)
    qm = QEqForceModule(RCUT, ETHRESH, eps=eps, max_iter=2000)
    nb = TorchNeighborList(RCUT)
    out = {}

    def one(r):
        pos = torch.as_tensor(r.pos, dtype=dtype, device=dev).requires_grad_(True)
        box = torch.as_tensor(r.box, dtype=dtype, device=dev)
        pairs = nb(pos, box)
        if r.kind == "pme":
            E = cm(pos, box, pairs, nb.get_ds(), nb.get_buffer_scales(),
                   {"charge": torch.as_tensor(r.charges, dtype=dtype, device=dev)})
            F = -torch.autograd.grad(E.sum(), pos)[0]
            return float(E.sum()), F.detach().double().cpu().numpy(), None
        n_ = pos.shape[0]
        C = torch.ones(1, n_, dtype=dtype, device=dev)
        E, q = pgrad_optimize(qm, torch.zeros(n_, dtype=dtype, device=dev), pos, box,
                              torch.as_tensor(r.chi, dtype=dtype, device=dev),
                              torch.as_tensor(r.hardness, dtype=dtype, device=dev),
                              torch.as_tensor(r.eta, dtype=dtype, device=dev), pairs, nb.get_ds(),
                              nb.get_buffer_scales(), C, torch.zeros(1, dtype=dtype, device=dev), method="quadratic")
        F = -torch.autograd.grad(E.sum(), pos)[0]
        return float(E.sum()), F.detach().double().cpu().numpy(), q.detach().double().cpu().numpy()

    sample = stream[:n]
    one(sample[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in sample:
        out[r.rid] = one(r)
    torch.cuda.synchronize()
    return len(sample) / (time.perf_counter() - t0), out


def accuracy_vs(results, ref):
    """Largest relative force error (per request, by its largest force) and
    charge error (e) of serving results against reference (E, F, q) tuples."""
    ferr = {"pme": 0.0, "qeq": 0.0}
    qerr = 0.0
    eerr = 0.0
    for rid, (E, F, q) in ref.items():
        o = results[rid]
        k = "qeq" if q is not None else "pme"
        ferr[k] = max(ferr[k], float(np.abs(np.asarray(o.forces, np.float64) - F).max() / np.abs(F).max()))
        eerr = max(eerr, abs(o.energy - E) / abs(E))
        if q is not None:
            qerr = max(qerr, float(np.abs(np.asarray(o.charges, np.float64) - q).max()))
    return {"max_rel_force_err": max(ferr.values()), "max_rel_force_err_pme": ferr["pme"],
            "max_rel_force_err_qeq": ferr["qeq"], "max_charge_err_e": qerr, "max_rel_energy_err": eerr,
            "requests": len(ref)}


def tc_matvec_flops(km) -> float:
    """Tensor-core FLOPs of one FP32 CG matvec's mesh passes on a K0 x K1 x K2 mesh, as the kernels
    issue them: 128-line tiles, 8-column K-steps, three TF32 products per step (head / tail split),
    padding included (csrc/dft_tc.cuh)."""
    K0, K1, K2 = (int(k) for k in km)
    K2h = K2 // 2 + 1

    def cd(a, b):
        return -(-a // b)

    def ks(K):  # K-steps of a contraction over K in two 40-column halves
        return min(5, cd(K, 8)) + (cd(K - 40, 8) if K > 40 else 0)

    def step(n):  # one 3-term K-step: 128 x n x 8 products
        return 3 * 2 * 128 * n * 8

    tz, ty, tx = cd(K0 * K1, 128), cd(K0 * K2h, 128), cd(K1 * K2h, 128)
    n0, n2 = cd(K0, 16) * 16, cd(K2, 16) * 16
    ns0, ns2 = (K0 - 1) // 2, (K2 - 1) // 2
    zf = tz * ks(K2) * step(80)
    y = ty * 2 * ks(K1) * step(80)
    x = tx * 2 * (ks(K0) * step(80) + (cd(K0 // 2 + 1, 8) + (cd(ns0 + 1, 8) if ns0 >= 1 else 0)) * step(n0))
    zi = tz * (cd(K2h, 8) + (cd(ns2 + 1, 8) if ns2 >= 1 else 0)) * step(n2)
    return float(zf + 2 * y + x + zi)


def tensor_roofline(stream, results, prof, peaks, kap):
    """Achieved tensor throughput of the CG matvec's mesh passes in the profiled pass: the FLOPs the
    tensor-core kernels issue ((iterations + 1) matvecs per QEq request) over their CUDA-event time,
    against dense TF32 = half the measured BF16 rate (the tensor cores run TF32 at half the BF16 rate)."""
    from admp_b200.serving import auto_kmesh
    names = ("tc_z_fwd", "tc_y_fwd", "tc_x", "tc_y_inv", "tc_z_inv")
    ms = sum(prof[k]["ms"] for k in names if k in prof)
    if ms <= 0:
        return None
    byrid = {r.rid: r for r in stream}
    flops = 0.0
    for res in results:
        if res.kind != "qeq":
            continue
        km = auto_kmesh(np.diagonal(byrid[res.rid].box), kap, ETHRESH)
        flops += (res.iterations + 1) * tc_matvec_flops(km)
    achieved = flops / (ms / 1e3) / 1e12
    bf16 = float(peaks.get("bf16_tflops", 0.0)) if peaks else 0.0
    peak = bf16 / 2 if bf16 > 0 else 1590.0 / 2
    return {"kernels": list(names), "ms": ms, "tflops": achieved, "peak_tflops": peak,
            "peak_source": "half the measured bf16 burst" if bf16 > 0 else "half the fallback bf16",
            "frac": achieved / peak,
            "flops_note": "TF32 products as issued: three per term (head / tail split), padding included"}


def same_sample_gpu(eng, reqs, passes: int = 3):
    """The FP32 serving engine on the CPU baseline's sample (host numpy in and
    out, as e2e): systems/s over `passes` passes after one untimed pass, and
    the results of the last pass."""
    import torch
    eng.results_to_host = True
    eng.results = []
    eng.run(reqs, arrivals=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(passes):
        eng.results = []
        res = eng.run(reqs, arrivals=False)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / passes
    return {"value": len(reqs) / dt, "unit": UNIT, "requests": len(reqs), "ms_per_pass": dt * 1e3,
            "results": {r.rid: r for r in res}}


def fp64_serving(stream, dev, args, world):
    """The serving engine in FP64 arithmetic (the reference's precision) on
    the same stream: device-resident and host-input (e2e) systems/s."""
    import torch

    from admp_b200.serving import ServingEngine, auto_kmesh
    dstream = to_device_requests(stream, dev, torch.float64)
    kap = math.sqrt(-math.log(2 * ETHRESH)) / RCUT
    mesh_sum = sum(int(np.prod(auto_kmesh(np.diagonal(r.box), kap, ETHRESH))) for r in stream)
    total_atoms = sum(r.natoms for r in stream)
    eng = ServingEngine(device=dev, dtype=torch.float64, max_atoms=min(6_000_000, int(total_atoms * 1.1) + 65536),
                        max_slots=min(1024, len(stream) + 8), mesh_budget=min(64_000_000, mesh_sum + 4_000_000),
                        rcut=RCUT, ethresh=ETHRESH, tol=TOL, max_iter=300, iters_per_tick=8)
    out = {}
    for name, reqs, host in (("value", dstream, False), ("e2e", stream, True)):
        eng.results_to_host = host
        for _ in range(2):
            eng.results = []
            eng.run(reqs, arrivals=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        passes = max(1, min(args.steps, 3))
        for _ in range(passes):
            eng.results = []
            res = eng.run(reqs, arrivals=False)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / passes
        out[name] = len(reqs) * world / max_over_ranks(dt, dev)
        out[f"{name}_failed"] = sum(1 for r in res if r.status != 0)
    del eng
    torch.cuda.empty_cache()
    return {"value": out["value"], "e2e": out["e2e"], "unit": UNIT, "dtype": "f64",
            "failed_requests": out["value_failed"] + out["e2e_failed"],
            "note": "device-resident and host-input passes of the same stream, FP64 bulk arithmetic"}


def electrode_leg(dev):
    """Constant-potential electrodes at their stated size (2 x 1,152 fcc(111)
    electrode atoms at 1 V / 0 V, 3,000 ions, 64 x 64 x 160 mesh, slab
    correction): GPU time of infer() (neighbour list, electrode solve, energy
    and forces) in FP32 and FP64, and the errors against the reference's
    result for the same system (tests/golden/electrode_cfg3.npz)."""
    import torch

    from admp_b200 import synthetic
    from admp_b200.electrode import LAMMPSElectrodeConstraint, PolarizableElectrode, infer, setup_from_lammps
    from admp_b200.nblist import TorchNeighborList
    pos_np, box_np, q_np, top, bot = synthetic.electrode_system(SEED)
    gpath = os.path.join(ROOT, "tests", "golden", "electrode_cfg3.npz")
    g = np.load(gpath) if os.path.exists(gpath) else None
    out = {"electrode_atoms": int(len(top) + len(bot)), "atoms": int(len(q_np)), "kmesh": [64, 64, 160]}
    for dt, eps, tag in ((torch.float32, 1e-7, "fp32"), (torch.float64, 1e-10, "fp64")):
        calc = PolarizableElectrode(rcut=RCUT, ethresh=ETHRESH, kmesh=[64, 64, 160], slab_corr=True, eps=eps,
                                    max_iter=2000)
        cons = [LAMMPSElectrodeConstraint(indices=top, value=1.0, mode="conp", eta=math.sqrt(2.0)),
                LAMMPSElectrodeConstraint(indices=bot, value=0.0, mode="conp", eta=math.sqrt(2.0))]

        def run():
            pos = torch.tensor(pos_np, dtype=dt, device=dev, requires_grad=True)
            box = torch.tensor(box_np, dtype=dt, device=dev)
            ch = torch.tensor(q_np, dtype=dt, device=dev)
            nb = TorchNeighborList(RCUT)
            pairs = nb(pos, box)
            data = setup_from_lammps(len(q_np), cons, True, device=dev, dtype=dt)
            E, F, q = infer(calc, pos, box, ch, pairs, nb.get_ds(), nb.get_buffer_scales(), *data, method="lbfgs")
            return float(E), F.detach().double().cpu().numpy(), q.detach().double().cpu().numpy()

        run()
        torch.cuda.synchronize()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            E, F, q = run()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        r = {"ms": statistics.median(ts) * 1e3, "cg_iterations": calc.converge_iter}
        if g is not None:
            r["max_rel_force_err_vs_reference"] = float(np.abs(F - g["forces"]).max() / np.abs(g["forces"]).max())
            r["max_charge_err_vs_reference_e"] = float(np.abs(q - g["q_ref"]).max())
            r["rel_energy_err_vs_reference"] = abs(E - float(g["E"])) / abs(float(g["E"]))
        out[tag] = r
    # the dense path (method="matinv": Hessian from batched Hessian-vector products + KKT solve), FP64
    calc = PolarizableElectrode(rcut=RCUT, ethresh=ETHRESH, kmesh=[64, 64, 160], slab_corr=True, eps=1e-10,
                                max_iter=2000)
    pos = torch.tensor(pos_np, dtype=torch.float64, device=dev, requires_grad=True)
    box = torch.tensor(box_np, dtype=torch.float64, device=dev)
    ch = torch.tensor(q_np, dtype=torch.float64, device=dev)
    nb = TorchNeighborList(RCUT)
    pairs = nb(pos, box)
    cons = [LAMMPSElectrodeConstraint(indices=top, value=1.0, mode="conp", eta=math.sqrt(2.0)),
            LAMMPSElectrodeConstraint(indices=bot, value=0.0, mode="conp", eta=math.sqrt(2.0))]
    data = setup_from_lammps(len(q_np), cons, True, device=dev, dtype=torch.float64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    E, F, q = infer(calc, pos, box, ch, pairs, nb.get_ds(), nb.get_buffer_scales(), *data, method="matinv")
    torch.cuda.synchronize()
    r = {"ms": (time.perf_counter() - t0) * 1e3}
    if g is not None:
        r["max_charge_err_vs_reference_e"] = float(np.abs(q.detach().cpu().numpy() - g["q_ref"]).max())
    out["fp64_matinv"] = r
    del pos, box, ch, pairs, nb, data, E, F, q
    torch.cuda.empty_cache()
    if g is not None:
        out["reference_cpu_s"] = float(g["time_ref_s"])
        out["reference_cpu_note"] = (f"the reference's infer(method='lbfgs', eps 1e-8) on {int(g['threads'])} CPU "
                                     "threads, timed when the golden file was made (not on this host)")
    return out


def diff_batch_leg(dev, nframes: int = 64):
    """The differentiation batch: 64 jittered frames of the 3,000-atom water
    system (48^3 mesh), neighbour lists + batched charge solve + energy +
    gradients w.r.t. positions, box, chi, hardness and eta through the
    implicit adjoint, in FP32 and FP64 (median of 3 after one warm-up)."""
    import torch

    from admp_b200 import synthetic
    from admp_b200.nblist import frame_pair_lists
    from admp_b200.qeq import QEqForceModule, qeq_solve_frames
    pos_np, box_np, chi_np, hard_np, eta_np, _ = synthetic.water_frames(nframes, SEED)
    out = {"frames": nframes, "atoms_per_frame": int(pos_np.shape[1])}
    for dt, tol, tag in ((torch.float32, 1e-7, "fp32"), (torch.float64, 1e-10, "fp64")):
        m = QEqForceModule(RCUT, ETHRESH, kmesh=48, eps=tol, max_iter=1000)

        def run():
            pos = torch.tensor(pos_np, dtype=dt, device=dev, requires_grad=True)
            box = torch.tensor(box_np, dtype=dt, device=dev, requires_grad=True)
            chi = torch.tensor(chi_np, dtype=dt, device=dev, requires_grad=True)
            hard = torch.tensor(hard_np, dtype=dt, device=dev, requires_grad=True)
            eta = torch.tensor(eta_np, dtype=dt, device=dev, requires_grad=True)
            pairs, ds, bs = frame_pair_lists(pos, box, RCUT)
            n = pos.shape[1]
            C = torch.ones(1, n, dtype=dt, device=dev)
            q = qeq_solve_frames(m, pos, box, chi, hard, eta, pairs, ds, bs, C, tol=tol)
            params = {"charge": q, "chi": chi.expand(nframes, n), "hardness": hard.expand(nframes, n),
                      "eta": eta.expand(nframes, n)}
            E = m(pos, box, pairs, ds, bs, params)
            return torch.autograd.grad(E.sum(), [pos, box, chi, hard, eta])

        run()
        torch.cuda.synchronize()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            run()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        ms = statistics.median(ts) * 1e3
        out[tag] = {"ms": ms, "frames_per_s": nframes / (ms / 1e3), "max_cg_iterations": m.converge_iter}
    return out


def main():
    args = parse()
    rank, world, local = rank_info()
    from admp_b200 import synthetic
    if args.impl == "reference":
        if rank != 0:
            return
        stream = synthetic.serving_stream(args.nreq, SEED, RATE)
        v, cores, sample, det = cpu_baseline(stream, args.cpu_reps or 3, args.cpu_sample)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"serving stream, {args.nreq} requests (200-20000 atoms, 60% PME / 40% QEq)",
                           "rcut": RCUT, "ethresh": ETHRESH, "cg_tol": TOL},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                                 "wall_value": det["wall_value"],
                                 "extrapolated_stream_value": det["extrapolated_stream_value"]},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    from admp_b200 import _lib as L
    from admp_b200.serving import ServingEngine

    stream = rank_stream(args.nreq, rank)
    total_atoms = sum(r.natoms for r in stream)
    dstream = to_device_requests(stream, dev, torch.float32)
    # pools sized to the stream (capped): all requests fit, so admission never stalls the closed loop
    from admp_b200.serving import auto_kmesh
    kap = math.sqrt(-math.log(2 * ETHRESH)) / RCUT
    mesh_sum = sum(int(np.prod(auto_kmesh(np.diagonal(r.box), kap, ETHRESH))) for r in stream)
    eng = ServingEngine(device=dev, dtype=torch.float32, max_atoms=min(6_000_000, int(total_atoms * 1.1) + 65536),
                        max_slots=min(1024, args.nreq + 8), mesh_budget=min(96_000_000, mesh_sum + 4_000_000),
                        rcut=RCUT, ethresh=ETHRESH, tol=TOL, max_iter=300, iters_per_tick=8)

    def one_pass(reqs, to_host=True, arrivals=False, rate_scale=1.0):
        eng.results = []
        eng.results_to_host = to_host
        return eng.run(reqs, arrivals=arrivals, time_scale=rate_scale)

    def barrier():
        if world > 1:
            dist.barrier()

    # the clock sampler (an nvidia-smi process) starts before the warm-up: its start-up attaches to the
    # driver and would otherwise stall launches of the first timed pass; only its samples taken inside
    # the timed region are summarised
    clk = ClockSampler(dev.index).__enter__()
    # warm-up
    for _ in range(args.warmup):
        one_pass(dstream, to_host=False)
    torch.cuda.synchronize()
    # as a long-running server would: the objects that live through warm-up (modules, requests, pools)
    # leave the cyclic collector's scan set, whose full collections otherwise stall a pass by ~30 ms
    gc.collect()
    gc.freeze()

    # timed: device-resident inputs
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = L.launch_count()
    for k in eng.host_time:
        eng.host_time[k] = 0.0
    barrier()
    torch.cuda.synchronize()
    t_clk0 = time.time()
    e0.record(st)
    for _ in range(args.steps):
        res = one_pass(dstream, to_host=False)
    e1.record(st)
    torch.cuda.synchronize()
    t_clk1 = time.time()
    clk.__exit__()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = L.launch_count() - launches0
    ms = max_over_ranks(ms, dev)
    ms_per_step = ms / args.steps
    host_ms = {k: round(v * 1000.0 / args.steps, 3) for k, v in eng.host_time.items()}
    value = args.nreq * world / (ms_per_step / 1000.0)
    n_bad = sum(1 for r in res if r.status != 0)

    # profile pass: per-kernel device time from CUDA events on the launch stream
    L.profile_enable(200000)
    pres = one_pass(dstream, to_host=False)
    torch.cuda.synchronize()
    prof = L.profile_read()
    L.profile_enable(0)

    if args.timeline:
        ts0, ts1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eng.call_trace = []
        torch.cuda.synchronize()
        ts0.record(st)
        one_pass(dstream, to_host=False)
        ts1.record(st)
        torch.cuda.synchronize()
        print(json.dumps({"timeline": eng.call_timeline(ts0, ts1)}), file=sys.stderr, flush=True)
        eng.call_trace = None

    # e2e: host numpy inputs and results, closed loop
    h0 = eng.stats["h2d_bytes"]
    d0 = eng.stats["d2h_bytes"]
    # the same number of untimed passes as the device-resident leg: the first host-input passes grow the
    # pinned staging and result buffers
    for _ in range(args.warmup):
        one_pass(stream, to_host=True)
    torch.cuda.synchronize()
    gc.collect()
    gc.freeze()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one_pass(stream, to_host=True)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps
    e2e_val = args.nreq / e2e_s
    h2d = (eng.stats["h2d_bytes"] - h0) / (args.steps + args.warmup)
    d2h = (eng.stats["d2h_bytes"] - d0) / (args.steps + args.warmup)
    if world > 1:
        e2e_val = args.nreq * world / max_over_ranks(e2e_s, dev)

    # open-loop latency at a stated Poisson rate
    lat_rate = args.latency_rate
    # one untimed open-loop pass first, as a long-running server would have had: its small steps take
    # launch shapes, first kernel loads and pinned result buffers that the closed-loop passes never needed
    one_pass(stream, to_host=True, arrivals=True, rate_scale=RATE / lat_rate)
    lat_res = one_pass(stream, to_host=True, arrivals=True, rate_scale=RATE / lat_rate)
    lats = sorted(r.latency for r in lat_res)
    p50 = lats[len(lats) // 2] * 1000.0
    p99 = lats[min(len(lats) - 1, int(0.99 * len(lats)))] * 1000.0

    # plain one-at-a-time GPU path and accuracy of the FP32 serving results vs FP64
    plain_val, plain_out = plain_path(stream, dev, torch.float32, args.plain_sample)
    # accuracy reference: FP64 drop-in path with the charge solve converged tightly (pinned to the oracle)
    _, ref64 = plain_path(stream, dev, torch.float64, args.plain_sample, eps=1e-10)
    byrid = {r.rid: r for r in one_pass(stream, to_host=True)}
    ferr, qerr, ferr_pme, ferr_qeq = 0.0, 0.0, 0.0, 0.0
    for rid, (E, F, q) in ref64.items():
        o = byrid[rid]
        fe = float(np.abs(o.forces - F).max() / np.abs(F).max())
        ferr = max(ferr, fe)
        if q is not None:
            ferr_qeq = max(ferr_qeq, fe)
            qerr = max(qerr, float(np.abs(o.charges - q).max()))
        else:
            ferr_pme = max(ferr_pme, fe)

    # roofline of the dominant kernel
    import json as _json
    peaks = {}
    try:
        peaks = _json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    dom = max((k for k in prof if prof[k]["bytes"] > 0), key=lambda k: prof[k]["ms"])
    tot_ms = sum(v["ms"] for v in prof.values())
    rf = {}
    for k in ("spread", "gather", dom):
        v = prof[k]
        if v["launches"] and v["ms"] > 0:
            rf[k] = {"gbs": v["bytes"] / (v["ms"] / 1000.0) / 1e9, "ms_per_launch": v["ms"] / v["launches"],
                     "launches": v["launches"], "share": v["ms"] / tot_ms if tot_ms else None}
    achieved = rf[dom]["gbs"]
    alg_per_launch = achieved * 1e9 * rf[dom]["ms_per_launch"] / 1e3
    traffic = TRAFFIC_PER_ALG_BYTE[dom] * alg_per_launch if dom in TRAFFIC_PER_ALG_BYTE else None
    tensor = tensor_roofline(stream, pres, prof, peaks, kap)
    extra = {}
    if not args.no_extra:
        extra["fp64"] = fp64_serving(stream, dev, args, world)
        extra["electrode_cfg3"] = electrode_leg(dev)
        extra["diff_batch_cfg4"] = diff_batch_leg(dev)
    cpu = None
    same = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sample_reqs = cpu_sample(stream, args.cpu_sample)
        same = same_sample_gpu(eng, sample_reqs)
        v, cores, sample, det = cpu_baseline(stream, args.cpu_reps or 1, args.cpu_sample)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
               "wall_value": det["wall_value"], "extrapolated_stream_value": det["extrapolated_stream_value"]}
        same["cpu_value"] = v
        same["accuracy_vs_oracle"] = accuracy_vs(same.pop("results"), det["results"])
    clocks = clk.summary(t_clk0, t_clk1)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"serving stream: {args.nreq} requests, atoms log-uniform 200-20000, "
                                   f"0.1 atoms/A^3, 60% PME / 40% QEq water, rc {RCUT}, ethresh {ETHRESH}, "
                                   f"CG tol {TOL}", "atoms_per_step": total_atoms,
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "meshes and atom pools far exceed L2 across a pass (each step streams all systems)"},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "p50_ms": p50, "p99_ms": p99, "latency_rate_rps": lat_rate},
            "plain_gpu": {"value": plain_val, "unit": UNIT, "sample": f"first {args.plain_sample} requests, FP32, "
                                                                     "one system per call"},
            "speedup_vs_plain": value / plain_val if plain_val else None,
            "accuracy": {"max_rel_force_err_vs_fp64": ferr, "max_charge_err_vs_fp64_e": qerr,
                         "max_rel_force_err_pme": ferr_pme, "max_rel_force_err_qeq": ferr_qeq,
                         "sample": f"first {args.plain_sample} requests vs the FP64 drop-in path "
                                   "(QEq solved to ||P grad||/N < 1e-10)"},
            "tensor_passes": tensor,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": ("ncu DRAM bytes per algorithmic byte of the 400-request stream "
                                            "x this run's algorithmic bytes per launch") if traffic else None,
                         "peak_source": peak_src,
                         "kernels": rf},
            "kernel_ms": {k: round(v["ms"], 3) for k, v in prof.items()},
            "host_ms_per_step": host_ms,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "failed_requests": n_bad,
        }
        if cpu:
            line["cpu_baseline"] = cpu
            line["same_sample"] = same
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
