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
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--plain-sample", type=int, default=100)
    ap.add_argument("--no-cpu", action="store_true")
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
    nonlinear CG for QEq followed by energy + forces).  Returns seconds."""
    from oracle import admp_oracle as O
    t0 = time.perf_counter()
    kind, pos, box, q, chi, hard, eta = req_tuple
    kappa = O.ewald_kappa(RCUT, ETHRESH)
    km = O.auto_kmesh(box, kappa, ETHRESH)
    pairs = O.nblist_pbc_cells(pos, box, RCUT)
    bs = O.pair_buffer_scales(pairs)
    if kind == "pme":
        O.coulomb_forces(pos, box, pairs, bs, q, rcut=RCUT, ethresh=ETHRESH, kmesh=km)
        return time.perf_counter() - t0
    ds = O.pairs_ds(pos, pairs, box)
    s = O.QEqSystem(pos, box, chi, hard, eta, pairs, ds, bs, rcut=RCUT, ethresh=ETHRESH, kmesh=km)
    n = pos.shape[0]
    qs, _ = O.solve_quadratic(s, np.zeros(n), np.ones((1, n)), np.zeros(1), max_iter=200, eps=TOL)
    O.coulomb_forces(pos, box, pairs, bs, qs, rcut=RCUT, ethresh=ETHRESH, kmesh=km)
    return time.perf_counter() - t0


CPU_SAMPLE_SIZES = {"pme": (300, 1000, 3000, 6000), "qeq": (300, 900, 2400)}


def cpu_baseline(stream, seconds: float):
    """CPU oracle throughput on the stream, from a timed sample.

    Requests of each kind closest to the sizes in CPU_SAMPLE_SIZES are run
    one per process on the host cores (spawn pool); a power law t = a N^b
    fitted per kind to their single-core times predicts every request of the
    stream, and the stream throughput is cores / mean(predicted time) (the
    requests are independent, so they spread over the cores).  Returns
    (systems/s, cores, sample text)."""
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    picks = []
    for kind, sizes in CPU_SAMPLE_SIZES.items():
        cand = [r for r in stream if r.kind == kind]
        for n in sizes:
            if cand:
                picks.append(min(cand, key=lambda r: abs(r.natoms - n)))
    tasks = [(r.kind, r.pos, r.box, r.charges, r.chi, r.hardness, r.eta) for r in picks]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(min(cores, len(tasks))) as pool:
        times = pool.map(_cpu_one, tasks, chunksize=1)
    wall = time.perf_counter() - t0
    pred = 0.0
    for kind in CPU_SAMPLE_SIZES:
        pts = [(r.natoms, t) for r, t in zip(picks, times) if r.kind == kind]
        x = np.log([p[0] for p in pts])
        y = np.log([p[1] for p in pts])
        b, a = np.polyfit(x, y, 1) if len(pts) > 1 else (1.0, y[0] - x[0])
        pred += sum(math.exp(a + b * math.log(r.natoms)) for r in stream if r.kind == kind)
    value = cores * len(stream) / pred
    desc = (f"{len(picks)} requests timed single-core ({', '.join(f'{r.kind} {r.natoms}: {t:.2f}s' for r, t in zip(picks, times))}; "
            f"wall {wall:.1f}s), power-law fit per kind extrapolated to all {len(stream)} requests "
            f"(predicted {pred:.0f} core-seconds)")
    return value, cores, desc


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


def main():
    args = parse()
    rank, world, local = rank_info()
    from admp_b200 import synthetic
    if args.impl == "reference":
        if rank != 0:
            return
        stream = synthetic.serving_stream(args.nreq, SEED, RATE)
        vals = []
        for _ in range(max(args.steps, 1)):
            v, cores, sample = cpu_baseline(stream, max(args.cpu_seconds, 5.0))
            vals.append(v)
        v = statistics.median(vals)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"serving stream, {args.nreq} requests (200-20000 atoms, 60% PME / 40% QEq)",
                           "rcut": RCUT, "ethresh": ETHRESH, "cg_tol": TOL},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                                 "sample": sample + " per step"},
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
    one_pass(dstream, to_host=False)
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
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, sample = cpu_baseline(stream, args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
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
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
