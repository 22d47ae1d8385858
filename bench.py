"""Throughput of the SPH geomechanics step: particle-updates/s (soil particles x steps / s).

Default workload: the 1.92M-particle translating retaining wall (soil block 200x80x120
at dx = 2.5 mm, 262,500 Adami/contact boundary particles, FP32), synthetic seeded
inputs from retainwall_code_b200.cases.retaining_wall.  A step is one whole
StepCalculation + PredictorSection + CorrectorSection (src/loquat.cu:548-561), replayed
from a captured CUDA graph; the state (~3.6 GB) is larger than L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload wall2|wall2_half|col1|batch64|batch64_forms|closure] [--precision-report]

Workloads besides the default: batch64 (the 64-case sweep in one graph launch per step),
batch64_forms (the same with the precision form and the learned closure, against plain
FP32), closure (the learned closure on the 1.92M wall), --precision-report (the
precision form against FP64).

--gpus N under torchrun: N independent replicas of the case, one per GPU (the single
case does not shard); value = N x npm x K / max-over-ranks device time.
--impl reference: the reference step on the host cores (the CPU restatement of the
reference's kernels, all threads), rank 0 only, a bounded sample of steps.

Beside the headline the default line carries: `amortized` (the same case over 2000 steps
from step 0, sorts and candidate-list rebuilds included), `reference_cuda` (the
reference's own CUDA build on the same case files and GPU, timed by its driver) and the
CPU baselines.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-updates/s/GPU at 1.92M particles"
METRICS = {"wall2_half": "particle-updates/s/GPU at 0.96M particles (half-length wall)",
           "col1": "particle-updates/s/GPU at 27,648 particles (column collapse)"}


def metric_of(workload: str) -> str:
    """The headline metric for the 1.92M wall; the same quantity named for the other cases."""
    return METRICS.get(workload, METRIC)
# From the ncu capture of the interaction's walk kernel on the 0.96M-particle case
# (profiles/k_interaction_wall2_half.md): DRAM read+write 461.4 + 63.4 MB and 337.2M warp
# instructions per launch.  Both grow with the particle count, so they are scaled per
# soil particle to the benchmarked case.
IX_DRAM_BYTES_PER_SOIL = (461.41e6 + 63.44e6) / 960000
IX_WARP_INSTR_PER_SOIL = 337.22e6 / 960000
# L1 data-stage wavefronts the walk kernel cannot avoid: each listed neighbour's 64-byte
# record is two 32-byte sectors read by one lane (records of a warp's lanes are distinct),
# each list entry an eighth of a sector (a warp's 32 entries are one coalesced 128-byte
# load), each particle's own state and outputs about 240 B.  The L1 data stage retires one
# wavefront per cycle per SM, and scattered sectors cost one wavefront each (ncu: 122.5M
# sectors requested per launch on the 0.96M case, 84% of the stage's peak).
IX_L1_SECTORS_PER_ENTRY = 2 + 1 / 8
IX_L1_SECTORS_PER_SOIL = 240 / 32
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# Host bytes rw_create_from_case copies per particle (int32 x4 codes, double x4 position,
# velocity and id/mass, double x6 stress and strain) and per boundary normal (double x4).
H2D_PER_PARTICLE = 16 + 3 * 32 + 2 * 48
H2D_PER_BOUNDARY = 32


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return dict(PEAKS_FALLBACK), "fallback"


def make_case(workload: str):
    from retainwall_code_b200 import cases as C

    if workload == "wall2":
        return C.retaining_wall(), {"workload": "retaining wall, active translation 1 mm/s",
                                    "soil": "200x80x120", "dx_m": 0.0025, "npm": 1920000,
                                    "wall_friction": "tan(2/3 phi_c)", "trajectory_steps": 20000}
    if workload == "wall2_half":  # half-length block, for profiler captures
        return C.retaining_wall(nx=100), {"workload": "retaining wall (half length)", "soil": "100x80x120",
                                          "dx_m": 0.0025, "npm": 960000, "trajectory_steps": 20000}
    if workload == "col1":
        return C.column_collapse(), {"workload": "column collapse", "soil": "24x24x48", "dx_m": 0.005, "npm": 27648,
                                     "trajectory_steps": 2000}
    raise SystemExit(f"unknown workload {workload}")


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(backend: str = "nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); NCCL on GPUs,
    gloo for host-only runs of the same logic."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def allreduce_max(x: float, ws: int) -> float:
    """Largest value over the ranks (the slowest rank's time)."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def pinned_case(case):
    """A copy of the case whose particle arrays live in page-locked host memory (the
    form a host keeps its inputs in when it streams them to the GPU); the copy is made
    before any clock starts."""
    import copy

    import numpy as np
    import torch

    def pin(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        t = torch.empty(a.shape, dtype={np.int32: torch.int32, np.float64: torch.float64}[dt], pin_memory=True)
        out = t.numpy()
        out[...] = a
        pin.keep.append(t)
        return out

    pin.keep = []
    c = copy.copy(case)
    c.codes = pin(case.codes, np.int32)
    for k in ("pospres", "velrhop", "idmassidx", "stress", "strain", "normal"):
        setattr(c, k, pin(getattr(case, k), np.float64))
    c._pinned = pin.keep
    return c


def timed_steps(sim, steps: int, device: int):
    """Times `steps` graph replays with CUDA events, sampling clocks meanwhile; returns
    (ms, kernels launched, clock sampler).  The launch count is the graph's kernels minus
    the gated bodies the device skipped (searches with no cell change, scan launches
    with every particle on a list, list builds while the kept lists stand), read from
    the context's counters."""
    i0 = sim.info()
    with ClockSampler(device) as clk:
        ms = sim.step_timed(steps)
    sim.synchronize()
    i1 = sim.info()
    launched = (steps * i1.graph_kernels
                - (i1.n_search_skipped - i0.n_search_skipped) * i1.search_body_kernels
                - (i1.n_scan_skipped - i0.n_scan_skipped)
                - (i1.n_build_skipped - i0.n_build_skipped) * i1.build_body_kernels)
    return ms, launched, clk


def interaction_bytes(inf, ncell: int, scalar: int, list_entries: int = 0) -> int:
    """Algorithmic HBM bytes of one interaction launch: every live soil particle's own
    state read once (cell 16, position 4s, velocity 4s, stress 6s, mass 4s, contact
    state 4x4s) and its outputs written once (contact 2x4s, acceleration 4s, strain rate
    6s, spin 4s), plus each particle's neighbour record (16s, position included) read
    once, plus the kept candidate lists (4 B per entry) and the cell ranges (8 B per
    cell)."""
    s = scalar
    per_soil = 16 + (4 + 4 + 6 + 4 + 16) * s + (8 + 4 + 6 + 4) * s
    return inf.npm * per_soil + inf.np * 16 * s + 4 * list_entries + ncell * 8


def cpu_sample(case, threads: int, steps: int, precision: int = 4):
    """The reference step on host cores: the CPU restatement, full case, `steps` steps
    (precision 4: float, as the reference's default build; 8: double)."""
    from oracle.oracle import Oracle

    t0 = time.perf_counter()
    o = Oracle(case, precision, threads)
    t_init = time.perf_counter() - t0
    o.step(1)  # warm-up step
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    npm = o.info().npm
    o.close()
    return npm * steps / dt, dt, t_init


def reference_cuda_sample(case, steps: int, warmup: int, device: int, precision: int = 4):
    """The reference's own CUDA build (oracle/_ref/ref_driver_f32, or ref_driver_f64 for
    FP64, built from the reference's sources) on the same case files and the same GPU:
    its step loop timed with CUDA events by the driver, clocks sampled meanwhile.  The
    reference hard-codes the wall friction (0.58108); the step's work does not depend on
    its value."""
    import tempfile

    from retainwall_code_b200 import cases as C

    name = "ref_driver_f64" if precision == 8 else "ref_driver_f32"
    drv = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(drv):
        return {"unavailable": f"oracle/_ref/{name} not built (needs the reference sources)"}
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    gpu = vis.split(",")[device] if vis else str(device)  # the driver runs on its device 0
    with tempfile.TemporaryDirectory() as d:
        proj = os.path.join(d, "wall")
        C.write_case(case, proj)
        with ClockSampler(device) as clk:
            r = subprocess.run([drv, proj, "--steps", str(steps), "--warmup", str(warmup), "--time"],
                               capture_output=True, text=True, timeout=1200,
                               env=dict(os.environ, CUDA_VISIBLE_DEVICES=gpu))
    if r.returncode != 0:
        return {"unavailable": f"reference driver exited {r.returncode}: {r.stderr[-300:]}"}
    rec = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    return {"value": rec["particle_updates_per_s"], "unit": "particle-updates/s", "ms_per_step": rec["ms_per_step"],
            "steps": steps, "warmup": warmup, "npm": rec["npm"], "dtype": "f64" if precision == 8 else "f32",
            "how": "unmodified reference build (sm_100a), RunSimulation's step loop, CUDA events", "clocks":
            clk.summary()}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    case, cfg = make_case(args.workload)
    threads = os.cpu_count() or 1
    prec = args.precision or (8 if args.workload == "col1" else 4)  # configuration 1 is FP64
    # a bounded sample of about 4M particle-updates of host work (3 steps at 1.92M)
    steps = max(1, min(args.steps, max(3, int(4e6 // max(case.npm, 1)))))
    ups, dt, _ = cpu_sample(case, threads, steps, precision=prec)
    sample = (f"{steps} whole {'FP64' if prec == 8 else 'FP32'} steps of the full {case.npm}-particle case "
              f"after 1 warm-up step")
    line = {
        "impl": "reference", "metric": metric_of(args.workload), "value": ups, "unit": "particle-updates/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": 1, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 8 else "f32", "data": "synthetic (seeded generator)",
        "config": dict(cfg, host_threads=threads),
        "cpu_baseline": {"value": ups, "unit": "particle-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": ups, "unit": "particle-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def shard_cases(specs, ws):
    """Largest-first greedy bin packing of cases over ranks by soil-particle count."""
    sizes = [(s["nx"] * s["ny"] * s["nz"], k) for k, s in enumerate(specs)]
    loads = [0] * ws
    owner = [0] * len(specs)
    for n, k in sorted(sizes, reverse=True):
        r = min(range(ws), key=lambda q: loads[q])
        owner[k] = r
        loads[r] += n
    return owner, loads


def run_batch(args, ws, rank, local):
    """Batched sweep: 64 retaining-wall cases of uneven sizes (50k-400k soil particles),
    sharded across ranks; on each GPU one graph launch per step advances all its cases."""
    from retainwall_code_b200 import Batch, LoquatSph, cases as C

    specs = C.batch_sweep(n_cases=args.batch_cases)
    owner, loads = shard_cases(specs, ws)
    mine = [s for k, s in enumerate(specs) if owner[k] == rank]
    sims, kinds = [], []
    for s in mine:
        c = C.retaining_wall(nx=s["nx"], ny=s["ny"], nz=s["nz"], dx=s["dx"], phi_c=s["phi_c"], e0=s["e0"],
                             mode=s["mode"], seed=s["seed"], name=s["name"])
        sim = LoquatSph(case=c, device=local, precision=4)
        sim.autotune(2)
        inf = sim.info()
        kinds.append((inf.ix_kernel, inf.walk_threads, inf.integrator_threads))
        sims.append(sim)
    npm_local = sum(sim.info().npm for sim in sims)
    b = Batch(sims)
    b.step(args.warmup)
    b.synchronize()
    barrier(ws)
    with ClockSampler(local) as clk:
        ms = b.step_timed(args.steps)
    ms = allreduce_max(ms, ws)
    total_npm = sum(s["nx"] * s["ny"] * s["nz"] for s in specs)
    value = total_npm * args.steps / (ms * 1e-3)
    infos = [sim.info() for sim in sims]
    npb_local = sum(i.npb for i in infos)
    # per particle the step advances (soil and boundary): smaller cases carry more wall
    # and floor per soil particle, which the soil-only metric does not see
    per_particle = {"soil_rank0": npm_local, "boundary_rank0": npb_local,
                    "ns_per_soil_particle": ms / args.steps * 1e6 / max(npm_local, 1) if ws == 1 else None,
                    "ns_per_particle": ms / args.steps * 1e6 / max(npm_local + npb_local, 1) if ws == 1 else None}
    lists = {"sections_that_sorted": sum(i.n_sorts for i in infos),
             "interactions_on_kept_lists": sum(i.n_list_reuse for i in infos),
             "interactions": sum(2 * i.step for i in infos),
             "searches_skipped_by_graph_gates": sum(i.n_search_skipped for i in infos)}
    for sim in sims:
        if sim.info().device_err:
            raise SystemExit("device error word set")
    # e2e: host case arrays -> contexts (upload) -> batched steps, one wall-force read per
    # case per step; the cases are generated on the host before the clock starts
    host_cases = [pinned_case(C.retaining_wall(nx=s["nx"], ny=s["ny"], nz=s["nz"], dx=s["dx"], phi_c=s["phi_c"],
                                               e0=s["e0"], mode=s["mode"], seed=s["seed"], name=s["name"]))
                  for s in mine]
    for sim in sims:
        sim.close()
    b.close()
    barrier(ws)
    t0 = time.perf_counter()
    # contexts are independent: a host creates them from several threads (each call
    # holds no Python lock while the library uploads and converts its case)
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=8) as ex:
        sims2 = list(ex.map(lambda c: LoquatSph(case=c, device=local, precision=4), host_cases))
    b2 = Batch(sims2)
    for _ in range(args.steps):
        b2.step(1)
        b2.wall_force(0)  # every case's resultant, one D2H of 24 B per case
    e2e_s = allreduce_max(time.perf_counter() - t0, ws)
    line = {
        "metric": "aggregate particle-updates/s, batched sweep of 64 retaining-wall cases", "value": value,
        "unit": "particle-updates/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generator, config-5 sweep)",
        "config": {"workload": "batched sweep", "cases": len(specs), "soil_particles_total": total_npm,
                   "cases_on_rank0": len(mine), "soil_on_rank0": npm_local,
                   "autotuned_shapes_rank0": {f"kernel{k}/walk{w}/integ{i}": kinds.count((k, w, i))
                                              for (k, w, i) in sorted(set(kinds))},
                   "parallelism": f"cases sharded over {ws} GPU(s), largest first"},
        "e2e": {"value": total_npm * args.steps / e2e_s, "unit": "particle-updates/s",
                "h2d_bytes_per_step": int(sum(c.np_ * H2D_PER_PARTICLE + c.npb * H2D_PER_BOUNDARY
                                              for c in host_cases) / args.steps),
                "d2h_bytes_per_step": 24 * len(mine),
                "note": "upload of every case from pinned host arrays + batched steps + one wall-force read per step (rank 0)"},
        "candidate_lists_rank0": lists,
        "per_particle": per_particle,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batch_forms(args, ws, rank, local):
    """The three forms together on the batched sweep: the 64 cases advanced in one graph
    launch per step with the precision form (compensated integration, FP64 norms) and the
    learned closure (trained as in the closure workload), against the same batch in plain
    FP32.  value = aggregate particle-updates/s of the combined form.  Each case's wall
    resultant after the timed steps (averaged over 50 further steps) is compared with its
    plain FP32 run and, together with the plain run's, with an FP64 run of the same batch
    (the FP64 step is pinned to the oracle's double-precision restatement)."""
    import numpy as np

    from retainwall_code_b200 import Batch, LoquatSph, _abi, cases as C

    specs = C.batch_sweep(n_cases=args.batch_cases)
    owner, loads = shard_cases(specs, ws)
    mine = [s for k, s in enumerate(specs) if owner[k] == rank]
    cases = [C.retaining_wall(nx=s["nx"], ny=s["ny"], nz=s["nz"], dx=s["dx"], phi_c=s["phi_c"], e0=s["e0"],
                              mode=s["mode"], seed=s["seed"], name=s["name"]) for s in mine]
    net, training = train_closure(args, local) if args.batch_forms != "precision" else (None, None)
    res = {}
    for form in ("plain", "forms", "f64"):
        sims = []
        for c in cases:
            sim = LoquatSph(case=c, device=local, precision=8 if form == "f64" else 4)
            if form == "forms":
                if args.batch_forms in ("both", "precision"):
                    sim.set_option(_abi.OPT_MIXED_PRECISION, 1)
                if args.batch_forms in ("both", "closure"):
                    sim.set_closure(net, margin=0.05)
                    sim.set_option(_abi.OPT_CLOSURE_MAX_ERR, args.closure_max_err)
            sims.append(sim)
        b = Batch(sims)
        b.step(args.warmup)
        b.synchronize()
        barrier(ws)
        with ClockSampler(local) as clk:
            ms = b.step_timed(args.steps)
        ms = allreduce_max(ms, ws)
        # the lateral resultant averaged over 50 further steps: one step's contact force
        # flickers with single contacts opening and closing
        navg = 50
        forces = np.zeros(len(sims))
        for _ in range(navg):
            b.step(1)
            forces += b.wall_force(0)[:, 0] / navg
        stats = [sim.closure_stats() for sim in sims] if form == "forms" and net is not None else []
        errs = [sim.info().device_err for sim in sims]
        res[form] = {"ms": ms, "forces": forces, "stats": stats, "clocks": clk.summary(), "err": max(errs)}
        b.close()
        for sim in sims:
            sim.close()
    total_npm = sum(s["nx"] * s["ny"] * s["nz"] for s in specs)
    value = total_npm * args.steps / (res["forms"]["ms"] * 1e-3)
    plain = total_npm * args.steps / (res["plain"]["ms"] * 1e-3)
    fp, ff, fd = res["plain"]["forces"], res["forms"]["forces"], res["f64"]["forces"]
    scale = np.maximum(np.abs(fp), 1e-9)
    rel = np.abs(ff - fp) / scale
    scale64 = np.maximum(np.abs(fd), 1e-9)
    rel64 = {"forms": np.abs(ff - fd) / scale64, "plain": np.abs(fp - fd) / scale64}
    offered = sum(st["offered"] for st in res["forms"]["stats"])
    used = sum(st["used"] for st in res["forms"]["stats"])
    judged = [st["mean_rel_err"] for st in res["forms"]["stats"] if st["used"] > 0]
    line = {
        "metric": "aggregate particle-updates/s, batched sweep of 64 retaining-wall cases, precision form + learned closure",
        "value": value, "unit": "particle-updates/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["forms"]["ms"] / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32+bf16", "data": "synthetic (seeded generator, config-5 sweep)",
        "config": {"workload": "batched sweep, combined forms", "forms": args.batch_forms, "cases": len(specs),
                   "soil_particles_total": total_npm,
                   "cases_on_rank0": len(mine), "parallelism": f"cases sharded over {ws} GPU(s), largest first"},
        "plain_batch": {"value": plain, "ms_per_step": res["plain"]["ms"] / args.steps},
        "forms_over_plain_batch": value / plain,
        "wall_force_vs_plain_fp32": {"averaged_over_steps": 50,
                                     "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
                                     "cases_within_1pct": int((rel <= 0.01).sum()), "cases": int(len(rel)),
                                     "per_case": [[s["mode"], s["nx"] * s["ny"] * s["nz"], float(a), float(b)]
                                                  for s, a, b in zip(mine, fp, ff)]},
        "wall_force_vs_fp64": {"averaged_over_steps": 50, "f64_ms_per_step": res["f64"]["ms"] / args.steps,
                               **{k: {"max_rel": float(v.max()), "median_rel": float(np.median(v)),
                                      "cases_within_1pct": int((v <= 0.01).sum()),
                                      "cases_within_half_pct": int((v <= 0.005).sum())}
                                  for k, v in rel64.items()},
                               "per_case_f64": [float(x) for x in fd]},
        "closure": {"offered": offered, "used": used, "used_share": used / max(offered, 1),
                    "mean_judged_rel_err_over_cases": float(np.mean(judged)) if judged else None},
        "training": training,
        "clocks": res["forms"]["clocks"],
        "device_err": max(res["forms"]["err"], res["plain"]["err"], res["f64"]["err"]),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import numpy as np

    from retainwall_code_b200 import LoquatSph
    from retainwall_code_b200 import _abi

    case, cfg = make_case(args.workload)
    # ---- device-resident throughput ----------------------------------------------------
    prec = args.precision or (8 if args.workload == "col1" else 4)  # configuration 1 is FP64
    sim = LoquatSph(case=case, device=local, precision=prec)
    if args.ix_kernel is not None:
        sim.set_option(_abi.OPT_INTERACTION_KERNEL, args.ix_kernel)
    if args.strict:
        sim.set_option(_abi.OPT_STRICT_FP, 1)
    if args.skin is not None:
        sim.set_option(_abi.OPT_LIST_SKIN, args.skin)
    if args.no_gates:
        sim.set_option(_abi.OPT_GRAPH_GATES, 0)
    inf = sim.info()
    sim.step(args.warmup)
    sim.synchronize()
    barrier(ws)
    ms, launched, clk = timed_steps(sim, args.steps, local)
    ms = allreduce_max(ms, ws)
    barrier(ws)
    npm = sim.info().npm
    value = ws * npm * args.steps / (ms * 1e-3)
    inf = sim.info()
    le, lp = sim.list_stats()
    lists = {"skin_h": 0.02 if args.skin is None else args.skin, "sections_that_sorted": inf.n_sorts,
             "interactions_on_kept_lists": inf.n_list_reuse, "interactions": 2 * inf.step,
             "mean_list_length": le / max(lp, 1)}
    if inf.device_err:
        raise SystemExit(f"device error word {inf.device_err}")
    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": metric_of(args.workload), "value": ws * npm * args.steps / (ms * 1e-3),
                              "ms_per_step": ms / args.steps, "steps": args.steps, "partial": True}), flush=True)
        return
    # ---- stage profile (CUDA events on the library's stream, per-stage launches) -------
    stages, kps = sim.profile(5)
    ix_ms = 0.5 * (stages["interaction_p"] + stages["interaction_c"])
    sim.close()
    # ---- end to end through the public API: upload from host, step, read the result ---
    host_case = pinned_case(case)
    barrier(ws)
    t0 = time.perf_counter()
    sim2 = LoquatSph(case=host_case, device=local, precision=prec)
    e2e_steps = args.steps
    for _ in range(e2e_steps):
        sim2.step(1)
        sim2.wall_force(0)  # D2H of the step's result (3 doubles)
    sim2.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, ws)
    sim2_lists = sim2.list_stats()
    sim2.close()
    e2e = ws * npm * e2e_steps / e2e_s
    # bytes uploaded by rw_create_from_case: the caller's arrays as they are (codes 16 B,
    # position, velocity, id/mass 32 B each, stress and strain 48 B each; normals 32 B
    # per boundary particle), converted on the device
    h2d = inf.np * H2D_PER_PARTICLE + inf.npb * H2D_PER_BOUNDARY
    # ---- roofline of the dominant kernel ------------------------------------------------
    pk, kind = peaks()
    list_entries, list_parts = sim2_lists
    ib = interaction_bytes(inf, inf.ncell, prec, list_entries)
    achieved = ib / (ix_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": "k_interaction", "achieved": achieved, "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "peak_source": kind,
            "traffic": IX_DRAM_BYTES_PER_SOIL * npm, "algorithmic_bytes_per_launch": ib, "launch_ms": ix_ms,
            "note": "not HBM-bound: bound by the L1 data stage (record gathers), see roofline_l1"}
    # whole step against the compulsory traffic of the algorithm: FP32 compact state of
    # 104 B per soil particle moved through two sections (bin, sort, permute, contact
    # preparation, interaction + integration) = 1276 B per soil particle, 644 B per
    # boundary particle and 32 B per cell per step
    b_alg = 1276 * npm + 644 * inf.npb + 32 * inf.ncell
    step_ach = b_alg / (ms / args.steps * 1e-3) / 1e9
    roof_step = {"bound": "hbm", "achieved": step_ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
                 "frac": step_ach / pk["hbm_gbs"], "peak_source": kind, "algorithmic_bytes_per_step": b_alg,
                 "note": "1276 B/soil + 644 B/boundary + 32 B/cell per step; FP32 issue is the tighter bound"}
    clocks = clk.summary()
    mhz = clocks.get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
    issue_peak = 148 * 4 * mhz * 1e6  # warp instructions per second
    issue_ach = IX_WARP_INSTR_PER_SOIL * npm / (ix_ms * 1e-3)
    issue = {"bound": "instruction issue", "kernel": "k_interaction", "achieved": issue_ach, "peak": issue_peak,
             "unit": "warp-instructions/s", "frac": issue_ach / issue_peak,
             "note": "instructions per launch from the ncu capture, scaled per soil particle"}
    l1_sectors = IX_L1_SECTORS_PER_ENTRY * list_entries + IX_L1_SECTORS_PER_SOIL * npm
    l1_peak = 148 * mhz * 1e6  # one L1 data-stage wavefront per cycle per SM
    roof_l1 = {"bound": "L1 data stage", "kernel": "k_interaction", "achieved": l1_sectors / (ix_ms * 1e-3),
               "peak": l1_peak, "unit": "sectors/s", "frac": l1_sectors / (ix_ms * 1e-3) / l1_peak,
               "sectors_per_launch": l1_sectors,
               "note": "2 sectors per listed neighbour (64-B record) + 1/8 per list entry + 7.5 per particle"}
    line = {
        "metric": metric_of(args.workload), "value": value, "unit": "particle-updates/s", "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 8 else "f32", "data": "synthetic (seeded generator)",
        "config": dict(cfg, parallelism=f"replicas x{ws}", np=inf.np, npb=inf.npb, ncell=inf.ncell,
                       l2=("device state 3.6 GB (double-buffered candidate lists included) > L2 (126 MB): "
                           "no flush needed") if inf.np > 1_000_000 else
                          ("the state fits in L2 (126 MB): steps run L2-warm, as a run of this case does; "
                           "not flushed")),
        "e2e": {"value": e2e, "unit": "particle-updates/s", "h2d_bytes_per_step": int(h2d / e2e_steps),
                "d2h_bytes_per_step": 24, "note": "case upload from pinned host arrays + per-step rw_step + wall-force read"},
        "roofline": roof,
        "roofline_l1": roof_l1,
        "roofline_issue": issue,
        "roofline_step": roof_step,
        "stage_ms": stages,
        "candidate_lists": lists,
        "gpu_launches": launched,
        "clocks": clocks,
    }
    # ---- the same case over a long window from step 0: sorts and list rebuilds included --
    # (a property of one case on one GPU: single-GPU runs only, so that a multi-GPU run
    # does not hold every GPU while rank 0 runs it)
    n_am = min(args.amortized_steps, cfg.get("trajectory_steps", args.amortized_steps))
    if rank == 0 and ws == 1 and n_am > 0:
        sim3 = LoquatSph(case=case, device=local, precision=prec)
        with ClockSampler(local) as clk3:
            ms3 = sim3.step_timed(n_am)
        i3 = sim3.info()
        line["amortized"] = {
            "value": i3.npm * n_am / (ms3 * 1e-3), "unit": "particle-updates/s",
            "steps": n_am, "ms_per_step": ms3 / n_am, "from_step": 0,
            "sections_that_sorted": i3.n_sorts, "searches_skipped": i3.n_search_skipped,
            "interactions": 2 * i3.step, "interactions_on_kept_lists": i3.n_list_reuse,
            "list_updates": i3.n_list_updates,
            "lists_rebuilt_per_update": i3.n_lists_rebuilt / max(i3.n_list_updates, 1),
            "full_list_builds": 2 * i3.step - i3.n_build_skipped - i3.n_list_updates,
            "vs_headline_window": (ms3 / n_am) / (ms / args.steps),
            "clocks": clk3.summary()}
        sim3.close()
    if rank == 0 and ws == 1 and not args.no_reference_cuda:
        line["reference_cuda"] = reference_cuda_sample(case, args.reference_cuda_steps, 3, local, prec)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        n_cpu = max(2, min(100, int(4e6 // max(npm, 1))))  # about 4M particle-updates of host work
        ups, dt, _ = cpu_sample(case, threads, n_cpu, precision=prec)
        line["cpu_baseline"] = {"value": ups, "unit": "particle-updates/s", "cores": threads, "kind": "port",
                                "sample": f"{n_cpu} whole {'FP64' if prec == 8 else 'FP32'} steps of the full "
                                          f"{npm}-particle case (+1 warm-up)"}
        if prec == 4:
            ups64, _, _ = cpu_sample(case, threads, 1, precision=8)
            line["cpu_baseline_f64"] = {"value": ups64, "unit": "particle-updates/s", "cores": threads,
                                        "kind": "port",
                                        "sample": f"1 whole FP64 step of the full {npm}-particle case (+1 warm-up)"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def invariants(sig):
    """p = -tr(sigma)/3 and q = sqrt(3/2 s:s) per particle (sigma: n x 6, xx yy zz xy xz yz)."""
    import numpy as np

    sig = np.asarray(sig, np.float64)
    p = -(sig[:, 0] + sig[:, 1] + sig[:, 2]) / 3.0
    s = sig.copy()
    s[:, :3] += p[:, None]
    ss = (s[:, 0] ** 2 + s[:, 1] ** 2 + s[:, 2] ** 2 + 2 * (s[:, 3] ** 2 + s[:, 4] ** 2 + s[:, 5] ** 2))
    return p, np.sqrt(1.5 * ss)


def precision_report(args):
    """Precision form against FP64 runs of the same seed: the column collapse (config 1)
    for positions and stress invariants, a retaining wall for the wall resultant."""
    import numpy as np

    from retainwall_code_b200 import LoquatSph, _abi, cases as C

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))

    out = {"metric": "precision form error vs FP64", "steps": {}}
    col = C.column_collapse()
    wall = C.retaining_wall(nx=48, ny=24, nz=36, dx=0.0025)
    runs = {}
    for name, case, steps in (("column_collapse_27648", col, args.precision_steps),
                              ("retaining_wall_41472", wall, args.precision_steps)):
        res = {}
        for mode in ("f64", "f32", "f32_mixed"):
            sim = LoquatSph(case=case, precision=8 if mode == "f64" else 4)
            if mode == "f32_mixed":
                sim.set_option(_abi.OPT_MIXED_PRECISION, 1)
            x0 = sim.get("pos_abs")[:, :3].astype(np.float64)
            wf = []
            chunk = max(1, steps // 20)
            done = 0
            while done < steps:
                n = min(chunk, steps - done)
                sim.step(n)
                done += n
                wf.append(sim.wall_force(0)[0])
            sim.synchronize()
            inf = sim.info()
            mat = slice(inf.npb, inf.npb + inf.npm)
            res[mode] = dict(x=sim.get("pos_abs")[:, :3].astype(np.float64)[mat], x0=x0[mat],
                             sig=sim.get("str")[mat], wf=np.array(wf))
            sim.close()
        ref = res["f64"]
        p64, q64 = invariants(ref["sig"])
        disp = ref["x"] - ref["x0"]
        entry = {"steps": steps}
        for mode in ("f32", "f32_mixed"):
            r = res[mode]
            p, q = invariants(r["sig"])
            entry[mode] = {"displacement_rel_l2": rel(r["x"] - r["x0"], disp),
                           "position_max_abs_m": float(np.abs(r["x"] - ref["x"]).max()),
                           "p_rel_l2": rel(p, p64), "q_rel_l2": rel(q, q64),
                           "wall_force_max_rel": float(np.max(np.abs(r["wf"] - ref["wf"])) /
                                                       max(np.abs(ref["wf"]).max(), 1e-30))}
        entry["wall_force_f64_N"] = float(ref["wf"][-1])
        out["steps"][name] = entry
    print(json.dumps(out), flush=True)


def wallforce_report(args, device):
    """The wall's lateral resultant over the 1.92M retaining wall's full trajectory
    (20,000 steps at dt = 5e-6 s), in plain FP32 and in the precision form, against an
    FP64 run of the same case.  The resultant (nearest-wall sum, FP64 accumulation) is
    sampled every `--wallforce-every` steps.  A second FP64 run, whose positions start
    one float ulp away (a random sign per coordinate), measures how far the trajectory's
    own sensitivity moves the resultant: wall-contact decisions switch on velocity
    signs, so differences of one rounding grow into discrete jumps.  Reported per run:
    the largest deviation from FP64 over the trajectory relative to the largest FP64
    magnitude, for the sampled resultant and for its moving averages over windows of
    1, 10, 50 and 100 samples, the RMS deviation, and the deviation of the trajectory
    mean."""
    import copy

    import numpy as np

    from retainwall_code_b200 import LoquatSph, _abi, cases as C

    case = C.retaining_wall()
    pert = copy.deepcopy(case)
    rng = np.random.default_rng(7)
    p32 = pert.pospres[:, :3].astype(np.float32)
    away = np.where(rng.random(p32.shape) < 0.5, np.float32(-np.inf), np.float32(np.inf))
    soil = np.arange(pert.np_) >= pert.npb
    p32[soil] = np.nextafter(p32[soil], away[soil])
    pert.pospres[:, :3] = p32.astype(np.float64)
    steps, every = args.wallforce_steps, args.wallforce_every
    hist, times = {}, {}
    for mode, c in (("f64", case), ("f64_one_ulp", pert), ("f32", case), ("f32_precision", case)):
        sim = LoquatSph(case=c, device=device, precision=8 if mode.startswith("f64") else 4)
        if mode == "f32_precision":
            sim.set_option(_abi.OPT_MIXED_PRECISION, 1)
        wf, done, ms = [], 0, 0.0
        while done < steps:
            n = min(every, steps - done)
            ms += sim.step_timed(n)
            done += n
            wf.append(sim.wall_force(0)[0])
        if sim.info().device_err:
            raise SystemExit(f"{mode}: device error word {sim.info().device_err}")
        hist[mode], times[mode] = np.array(wf), ms / steps
        sim.close()
    ref = hist["f64"]
    top = np.abs(ref).max()
    out = {"metric": "wall lateral resultant vs FP64 over the full trajectory", "case": "retaining wall 200x80x120",
           "steps": steps, "sample_every": every, "dt_s": 5e-6,
           "f64_resultant_N": {"first": float(ref[0]), "last": float(ref[-1]), "max_abs": float(top),
                               "mean": float(ref.mean())},
           "ms_per_step": times, "windows_samples": [1, 10, 50, 100]}

    def smooth(x, w):
        return np.convolve(x, np.ones(w) / w, mode="valid") if w > 1 else x

    for mode in ("f64_one_ulp", "f32", "f32_precision"):
        d = hist[mode] - ref
        out[mode] = {"max_dev_over_max_f64": {str(w): float(np.abs(smooth(hist[mode], w) - smooth(ref, w)).max() / top)
                                              for w in out["windows_samples"]},
                     "rms_dev_over_max_f64": float(np.sqrt(np.mean(d * d)) / top),
                     "mean_dev_over_mean_f64": float(abs(hist[mode].mean() - ref.mean()) / abs(ref.mean())),
                     "final_rel": float(abs(d[-1]) / abs(ref[-1]))}
    out["history_N"] = {k: [float(x) for x in v[:: max(1, len(v) // 40)]] for k, v in hist.items()}
    print(json.dumps(out), flush=True)


def closure_accuracy(net, steps, device, max_err=0.02):
    """FP64 runs against plain FP32 and FP32 with the learned closure, same seeds: the
    column collapse (config 1's case) for positions and stress invariants, a 41k
    retaining wall for the wall resultant (largest deviation over the run)."""
    import numpy as np

    from retainwall_code_b200 import LoquatSph, _abi, cases as C

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))

    out = {"steps": steps}
    for name, case in (("column_collapse_27648", C.column_collapse()),
                       ("retaining_wall_41472", C.retaining_wall(nx=48, ny=24, nz=36, dx=0.0025))):
        res = {}
        for mode in ("f64", "f32", "closure"):
            sim = LoquatSph(case=case, precision=8 if mode == "f64" else 4, device=device)
            if mode == "closure":
                sim.set_closure(net, margin=0.05)
                sim.set_option(_abi.OPT_CLOSURE_MAX_ERR, max_err)
            x0 = sim.get("pos_abs")[:, :3].astype(np.float64)
            wf, done, chunk = [], 0, max(1, steps // 20)
            while done < steps:
                n = min(chunk, steps - done)
                sim.step(n)
                done += n
                wf.append(sim.wall_force(0)[0])
            inf = sim.info()
            mat = slice(inf.npb, inf.npb + inf.npm)
            res[mode] = dict(x=sim.get("pos_abs")[:, :3].astype(np.float64)[mat], x0=x0[mat], sig=sim.get("str")[mat],
                             wf=np.array(wf), stats=sim.closure_stats() if mode == "closure" else None)
            sim.close()
        ref = res["f64"]
        p64, q64 = invariants(ref["sig"])
        entry = {}
        for mode in ("f32", "closure"):
            r = res[mode]
            p, q = invariants(r["sig"])
            entry[mode] = {"displacement_rel_l2": rel(r["x"] - r["x0"], ref["x"] - ref["x0"]),
                           "p_rel_l2": rel(p, p64), "q_rel_l2": rel(q, q64)}
            if np.abs(ref["wf"]).max() > 0:
                entry[mode]["wall_force_max_rel"] = float(np.max(np.abs(r["wf"] - ref["wf"])) /
                                                          np.abs(ref["wf"]).max())
        entry["closure"]["judged"] = res["closure"]["stats"]
        out[name] = entry
    return out


def train_closure(args, device):
    """The closure network trained on plain runs of the column collapse and of retaining
    walls of the batched sweep's kind (phi_c 28-40 deg, e0 0.55-0.80, three wall modes,
    per-sample material augmentation); returns (network, training record)."""
    from retainwall_code_b200 import cases as C
    from retainwall_code_b200.closure import Mlp, training_run

    net = Mlp(device=device, seed=1, sample_capacity=args.closure_samples)
    t0 = time.perf_counter()
    runs = 0
    while net.sample_count() < args.closure_samples:
        # low-discrepancy sweep of the friction angle and the initial void ratio, so that
        # a few runs already span both ranges (end points first)
        u = (0.0, 1.0)[runs] if runs < 2 else (runs * 0.6180339887) % 1.0
        v = (1.0, 0.0)[runs] if runs < 2 else (runs * 0.7548776662) % 1.0
        phi, e0 = 28.0 + 12.0 * u, 0.55 + 0.25 * v
        if runs % 2 == 0:  # the column collapse (24 x 24 x 48, 5 mm), every 2nd particle
            case, stride = C.column_collapse(phi_c=phi, e0=e0, seed=100 + runs), 2
        else:  # a retaining wall of the batched sweep's kind (102k soil particles), every 16th
            mode = ("active", "passive", "rotation")[runs % 3]
            case = C.retaining_wall(nx=80, ny=32, nz=40, dx=0.004, phi_c=phi, e0=e0, mode=mode, seed=100 + runs)
            stride = 16
        training_run(net, case, steps=args.closure_run_steps, every=max(4, args.closure_run_steps // 100),
                     stride=stride, device=device, seed=runs)
        runs += 1
    collect_s = time.perf_counter() - t0
    n_samples = net.sample_count()
    t0 = time.perf_counter()
    loss = net.train(epochs=args.closure_epochs, batch=8192, lr=2e-3, seed=1)
    train_s = time.perf_counter() - t0
    return net, {"samples": n_samples, "runs": runs, "collect_s": collect_s, "epochs": args.closure_epochs,
                 "train_s": train_s, "samples_per_s": n_samples * args.closure_epochs / train_s,
                 "final_mse": loss}


def run_closure(args, ws, rank, local):
    """The learned-closure form: a network trained on plain runs of the column collapse
    and retaining-wall configurations (phi_c 28-40 deg, e0 0.55-0.80), then the 1.92M
    retaining wall stepped with and without it.  value = particle-updates/s with the
    closure; the plain throughput, the closure's judged error, its fallback share and the
    wall force against the plain run are reported beside it."""
    import numpy as np

    from retainwall_code_b200 import LoquatSph, _abi, cases as C

    net, training = train_closure(args, local)
    acc = closure_accuracy(net, args.closure_acc_steps, local, args.closure_max_err)
    case, cfg = make_case("wall2")
    res = {}
    for mode in ("plain", "closure"):
        sim = LoquatSph(case=case, device=local)
        if mode == "closure":
            sim.set_closure(net, margin=0.05)
            sim.set_option(_abi.OPT_CLOSURE_MAX_ERR, args.closure_max_err)
        sim.step(args.warmup)
        sim.synchronize()
        barrier(ws)
        ms, launched, clk = timed_steps(sim, args.steps, local)
        ms = allreduce_max(ms, ws)
        stages, kps = sim.profile(3)
        res[mode] = {"ms": ms, "npm": sim.info().npm, "stages": stages, "launched": launched,
                     "clocks": clk.summary(),
                     "wall_force_N": float(sim.wall_force(0)[0]), "stats": sim.closure_stats(),
                     "err": sim.info().device_err}
        sim.close()
    npm = res["closure"]["npm"]
    value = ws * npm * args.steps / (res["closure"]["ms"] * 1e-3)
    plain = ws * res["plain"]["npm"] * args.steps / (res["plain"]["ms"] * 1e-3)
    st = res["closure"]["stats"]
    # tensor work of one closure launch: 128-row tiles of five layers (K, N padded)
    macs = 16 * 64 + 3 * 64 * 64 + 64 * 16
    extra_ms = 0.5 * ((res["closure"]["stages"]["predictor"] - res["plain"]["stages"]["predictor"]) +
                      (res["closure"]["stages"]["corrector"] - res["plain"]["stages"]["corrector"]))
    pk, kind = peaks()
    tflops = 2.0 * macs * npm / (max(extra_ms, 1e-6) * 1e-3) / 1e12
    wf_p, wf_c = res["plain"]["wall_force_N"], res["closure"]["wall_force_N"]
    if rank == 0:
        print(json.dumps({
            "metric": METRIC + " (learned closure)", "value": value, "unit": "particle-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["closure"]["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
            "data": "synthetic (seeded generator)", "config": dict(cfg, parallelism=f"replicas x{ws}"),
            "plain": {"value": plain, "ms_per_step": res["plain"]["ms"] / args.steps},
            "closure": {"offered": st["offered"], "used": st["used"],
                        "used_share": st["used"] / max(st["offered"], 1.0), "mean_rel_err": st["mean_rel_err"],
                        "max_rel_err": st["max_rel_err"],
                        "wall_force_rel_diff_vs_plain": abs(wf_c - wf_p) / max(abs(wf_p), 1e-30),
                        "extra_ms_per_launch": extra_ms,
                        "tensor_roofline": {"bound": "tensor", "achieved": tflops, "peak": pk["bf16_tflops"] * 1.0,
                                            "unit": "TFLOP/s", "frac": tflops / pk["bf16_tflops"],
                                            "note": "two launches per step; MACs of the padded 16-64-64-64-64-16 net"}},
            "accuracy_vs_fp64": acc,
            "training": training,
            "stage_ms": res["closure"]["stages"], "gpu_launches": res["closure"]["launched"],
            "clocks": res["closure"]["clocks"], "device_err": res["closure"]["err"],
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="wall2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end and stage-profile passes")
    ap.add_argument("--no-reference-cuda", action="store_true", help="skip timing the reference's CUDA build")
    ap.add_argument("--reference-cuda-steps", type=int, default=50)
    ap.add_argument("--amortized-steps", type=int, default=20000,
                    help="steps of the long window from step 0 (sorts, list updates and rebuilds included; "
                         "default: the 1.92M wall's whole 20,000-step trajectory); 0: skip")
    ap.add_argument("--ix-kernel", type=int, default=None, help="interaction kernel: 0 global (default), 1 chunked")
    ap.add_argument("--precision", type=int, choices=[4, 8], default=None,
                    help="bytes per scalar of the single-case workloads (default: 8 for col1, which the "
                         "configuration runs in FP64, else 4)")
    ap.add_argument("--skin", type=float, default=None, help="kept candidate-list skin in units of h (0: scan cells)")
    ap.add_argument("--strict", action="store_true", help="separately rounded interaction arithmetic")
    ap.add_argument("--no-gates", action="store_true",
                    help="plain step graph without conditional nodes (for ncu, which replays single graph kernels)")
    ap.add_argument("--precision-report", action="store_true", help="precision form vs FP64 (configs 1 and 3)")
    ap.add_argument("--precision-steps", type=int, default=2000)
    ap.add_argument("--wallforce-report", action="store_true",
                    help="wall resultant of FP32 and the precision form vs FP64 over the 1.92M wall's trajectory")
    ap.add_argument("--wallforce-steps", type=int, default=20000)
    ap.add_argument("--wallforce-every", type=int, default=20)
    ap.add_argument("--batch-cases", type=int, default=64)
    ap.add_argument("--batch-forms", choices=["both", "closure", "precision"], default="both",
                    help="forms applied in the batch64_forms workload")
    ap.add_argument("--closure-samples", type=int, default=10_000_000)
    ap.add_argument("--closure-epochs", type=int, default=30)
    ap.add_argument("--closure-run-steps", type=int, default=2000)
    ap.add_argument("--closure-acc-steps", type=int, default=2000)
    ap.add_argument("--closure-max-err", type=float, default=0.02,
                    help="judged-error bound of the closure (RW_OPT_CLOSURE_MAX_ERR)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.precision_report:
        precision_report(args)
        return
    if args.wallforce_report:
        wallforce_report(args, 0)
        return
    if args.impl == "reference":  # host cores only: rank 0 runs, the other ranks exit
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, ws, int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = dist_setup()
    try:
        if args.workload == "batch64":
            run_batch(args, ws, rank, local)
        elif args.workload == "batch64_forms":
            run_batch_forms(args, ws, rank, local)
        elif args.workload == "closure":
            run_closure(args, ws, rank, local)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
