"""Benchmark of the LIJ (line-implicit Jacobi) solver on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2|c3a|c3b] [--algo fp64|ref|mixed]

A step is one LIJ solve of the configured system from U = 0 to the relative
residual tolerance (default: 1200 lines x 1280 cells = 1,536,000 cells, 9x9
FP64 blocks, seeded synthetic values with shift 4, tolerance 1e-10; the
mixed-precision solve of the same system is timed beside it).  The
metric is LIJ sweeps per second: total sweeps of all steps on all GPUs
divided by the device time (CUDA events, max over ranks).  The blocks stay
resident in HBM for `value`; `e2e` repeats the step through the C ABI from
pinned host buffers (Jacobian upload, factorization, solve, solution
read-back every step).

With N > 1 (torchrun) the mesh is split into N contiguous line ranges, one
per rank (strong scaling): each sweep exchanges the halo lines' updates
with the neighbouring ranks (NCCL send/recv) and all-reduces one double
for the global norm.  --replicas gives every rank its own independent
system instead (weak scaling, no data-path collective).  --impl reference times the CPU restatement of the reference path
(oracle/, OpenMP over lines on all host cores) on the same system: one
sweep per step, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (lines L, cells per line K, diagonal shift, tolerance)
    "c1": (60, 64, 9.0, 1e-12),
    "c2": (360, 384, 9.0, 1e-12),
    "c3a": (600, 640, 4.0, 1e-10),
    "c3b": (1200, 1280, 4.0, 1e-10),
}
SEED = 1
# batched uneven systems: 64 meshes, lines log-uniform in [60, 1200], cells per line
# log-uniform in [32, 1280], shift 9, tolerance 1e-10
BATCH_CONFIGS = {"c4": {"nsys": 64, "L": (60, 1200), "K": (32, 1280), "shift": 9.0,
                        "tol": 1e-10, "seed": 4}}
# paper Table 5 (V100, FP64): 5 LIJ iterations on ex06 (138,240 cells) in 8.470 ms
PUBLISHED_SWEEPS_PER_S = {"c2": 5 / 0.008470, "c3a": 5 / 0.018741, "c3b": 5 / 0.076733}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def aggregate(values, op):
    """max / sum of per-rank values (plain Python; the NCCL path mirrors it)."""
    return max(values) if op == "max" else sum(values)


class Dist:
    def __init__(self, ws, rank, local, backend):
        self.ws, self.rank, self.local = ws, rank, local
        self.pg = None
        if ws > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def reduce(self, value, op):
        if not self.pg:
            return value
        import torch
        dev = "cuda" if torch.cuda.is_available() and self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX if op == "max" else self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons while the measurement runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        import tempfile
        self.path = os.path.join(tempfile.gettempdir(), f"tbs_clocks_{os.getpid()}_{gpu_index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        loaded = [r for r in rows if r[2] > 200.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in loaded for i, v in enumerate(r[3]) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": loaded[0][1],
                "reasons": reasons, "samples": len(rows), "samples_under_load": len(loaded)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_problem(L, K, shift, pinned, nvar=9):
    from triblocksolve_b200 import Mesh
    from triblocksolve_b200 import _native as N
    mesh = Mesh.structured(L, K, nvar=nvar)
    nb = nvar * nvar
    sizes = {"jacD": nb * mesh.nelem, "jacO1": nb * mesh.nintface, "jacO2": nb * mesh.nintface,
             "rhs": nvar * mesh.nelem}
    if pinned:
        import torch
        host = {k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
                for k, n in sizes.items()}
    else:
        host = {k: np.empty(n) for k, n in sizes.items()}
    N.check(N.lib.tbs_gen_jacobian(nvar, mesh.nelem, mesh.nintface, float(shift), SEED,
                                   N.dptr(host["jacD"]), N.dptr(host["jacO1"]),
                                   N.dptr(host["jacO2"]), N.dptr(host["rhs"]), None))
    return mesh, host


def reference_model_bytes(mesh) -> float:
    """Bytes per sweep by the reference's own count (src/main.cxx:146-175):
    duMem (jacDLU, DinvC, A once, dU twice loaded and twice stored, res, the
    line index arrays), cpMem (five dU-sized vectors) and lrMem (jacD, jacO1,
    jacO2, U five times, res loaded and stored, all mesh index arrays).
    Times sweeps/s it gives the GB/s in which the paper quotes its figures
    (about 6.45 KB per cell for 9x9 blocks)."""
    nv = int(mesh.nvar)
    nb = nv * nv
    N, F, L, eft = int(mesh.nelem), int(mesh.nintface), int(mesh.nline), int(mesh.eftot)
    du = 8.0 * (3 * nb * N + 4 * nv * N + nv * N) + 4.0 * (L + (L + 1) + N + N)
    cp = 8.0 * 5 * nv * N
    lr = (8.0 * (nb * N + 2 * nb * F + 5 * nv * N + 2 * nv * N)
          + 4.0 * ((N + 1) + eft + 2 * F + L + (L + 1) + N + N))
    return du + cp + lr


def cpu_system(L, K, shift, nvar=9):
    """The same seeded system for the CPU legs, built by the oracle's numpy
    generator (bit-identical to the library's) so that the CPU legs never
    load the product library."""
    from oracle import synthetic
    mesh = synthetic.structured_mesh(L, K, nvar=nvar)
    D, O1, O2, rhs = synthetic.jacobian(nvar, mesh.nelem, mesh.nintface, shift, SEED)
    return mesh, {"jacD": D, "jacO1": O1, "jacO2": O2, "rhs": rhs}


def cpu_impl():
    """The CPU implementation of the reference path: the reference's own
    kernels (OKL translated to C, oracle/_ref, kind "reference") where they
    were built, else the oracle's restatement (kind "port")."""
    import oracle
    if oracle.ref_available():
        return oracle.RefBaseline, "reference", ("the reference's own OKL kernels (lineLU_v2, "
                                                 "linesmoothLU_TriBlock_v3, linesmoothLU_v5) "
                                                 "translated to C with OCCA's OpenMP semantics, "
                                                 "oracle/_ref")
    return oracle.Baseline, "port", "oracle/lij_oracle.c, OpenMP over lines"


def cpu_model() -> str:
    """The host CPU's model name, as /proc/cpuinfo gives it."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(mesh, host, budget_s=12.0, sweeps=None):
    """The CPU reference path on all host cores (and a one-thread sample); sweeps/s."""
    import oracle
    cls, kind, what = cpu_impl()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    b = cls(mesh, host["jacD"], host["jacO1"], host["jacO2"], host["rhs"], threads)
    t_factor = time.perf_counter() - t0
    if sweeps is None:
        t0 = time.perf_counter()
        b.sweeps(1)
        t1 = time.perf_counter() - t0
        sweeps = int(max(1, min(200, budget_s / max(t1, 1e-6))))
        b.reset()
    t0 = time.perf_counter()
    b.sweeps(sweeps)
    dt = time.perf_counter() - t0
    del b
    # (i) one thread, what the reference's serial mode runs: a bounded sample
    t0 = time.perf_counter()
    b1 = cls(mesh, host["jacD"], host["jacO1"], host["jacO2"], host["rhs"], 1)
    t_factor1 = time.perf_counter() - t0
    n1, t1_total = 0, 0.0
    while t1_total < budget_s / 4 and n1 < sweeps:
        t0 = time.perf_counter()
        b1.sweeps(1)
        t1_total += time.perf_counter() - t0
        n1 += 1
    del b1
    oracle.set_threads(threads)
    return {"value": sweeps / dt, "unit": "sweeps/s", "cores": threads, "kind": kind,
            "cpu_model": cpu_model(), "nproc": os.cpu_count(),
            "sample": f"{sweeps} FP64 sweeps of the same {mesh.nline}x{mesh.max_line_nelem} system "
                      f"after one factorization ({t_factor:.2f} s), {what}, {threads} threads",
            "factor_s": t_factor, "seconds": dt,
            "single_thread": {"value": n1 / t1_total, "unit": "sweeps/s", "cores": 1,
                              "factor_s": t_factor1, "sweeps": n1, "seconds": t1_total}}


def batch_shapes(cfg):
    """Seeded (lines, cells per line) of every system of a batched workload."""
    rng = np.random.default_rng(cfg["seed"])
    lo, hi = cfg["L"]
    Ls = np.exp(rng.uniform(np.log(lo), np.log(hi), cfg["nsys"])).round().astype(int)
    lo, hi = cfg["K"]
    Ks = np.exp(rng.uniform(np.log(lo), np.log(hi), cfg["nsys"])).round().astype(int)
    return [(int(a), int(b)) for a, b in zip(Ls, Ks)]


def run_batch(args):
    """A step is one batched solve of all systems from U = 0 to the tolerance."""
    import torch

    import triblocksolve_b200 as tbs
    from triblocksolve_b200 import _native as N
    cfg = BATCH_CONFIGS[args.config]
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = Dist(ws, rank, local, "nccl")
    algo = {"fp64": tbs.ALGO_FP64, "mixed": tbs.ALGO_MIXED}[args.algo]
    tol, shift = cfg["tol"], cfg["shift"]
    shapes = batch_shapes(cfg)
    solvers, meshes, rhs_h = [], [], []
    t_setup = time.perf_counter()
    for k, (L, K) in enumerate(shapes):
        mesh = tbs.Mesh.structured(L, K)
        nb = 81
        jacD = np.empty(nb * mesh.nelem)
        O1 = np.empty(nb * mesh.nintface)
        O2 = np.empty(nb * mesh.nintface)
        rhs = torch.empty(9 * mesh.nelem, dtype=torch.float64, pin_memory=True).numpy()
        N.check(N.lib.tbs_gen_jacobian(9, mesh.nelem, mesh.nintface, shift, 1000 * SEED + k,
                                       N.dptr(jacD), N.dptr(O1), N.dptr(O2), N.dptr(rhs), None))
        s = tbs.Solver(local)
        s.set_mesh(mesh)
        s.set_jacobian_arrays(jacD, O1, O2, rhs)
        s.factor(algo)
        del jacD, O1, O2
        solvers.append(s)
        meshes.append(mesh)
        rhs_h.append(rhs)
    setup_s = time.perf_counter() - t_setup
    batch = tbs.Batch(solvers)
    # a dedicated stream for the batch's graph launches, visible to the CUDA events
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    batch.set_stream(stream.cuda_stream)
    footprint = sum(s.memory_allocated() for s in solvers)
    cells = np.array([m.nelem for m in meshes], dtype=np.int64)
    max_sweeps = 400
    inner = None
    ctas, stages, order, tune_ms = batch.tune()
    if args.algo == "mixed":
        # the FP32 inner sweep schedule (first outer step, the others) timed on the batch
        f_in, r_in, _ = batch.tune_inner(tol, max_sweeps)
        inner = [f_in, r_in]
    with ClockSampler(local) as clocks:
        for _ in range(max(args.warmup, 0)):
            batch.solve(tol, max_sweeps)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        cell_sweeps = 0
        sw = None
        for _ in range(args.steps):
            sw, hist = batch.solve(tol, max_sweeps)
            cell_sweeps += int((cells * sw).sum())
        ev1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        elapsed_ms = ev0.elapsed_time(ev1)
        batch.profile(True)
        batch.profile_reset()
        nprof = max(1, min(args.steps, 3))
        for _ in range(nprof):
            swp, _h = batch.solve(tol, max_sweeps)
        prof = batch.profile_read()
        batch.profile(False)
        # e2e: new right-hand sides from pinned host memory, batched solve, solutions back
        ne2e = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 5))
        sol_h = [torch.empty(9 * m.nelem, dtype=torch.float64, pin_memory=True).numpy()
                 for m in meshes]
        for s in solvers:
            s.set_stream(stream.cuda_stream)
        torch.cuda.synchronize()
        ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev2.record(stream)
        e2e_cs = 0
        for _ in range(ne2e):
            for s, r in zip(solvers, rhs_h):
                s.set_rhs(r)
            swe, _h = batch.solve(tol, max_sweeps)
            for s, u in zip(solvers, sol_h):
                N.check(N.lib.tbs_get_solution(s.ctx, N.dptr(u)), s.ctx)
            e2e_cs += int((cells * swe).sum())
        ev3.record(stream)
        torch.cuda.synchronize()
        e2e_ms = ev2.elapsed_time(ev3)
    clk = clocks.summary()
    max_ms = dist.reduce(elapsed_ms, "max")
    all_cs = dist.reduce(cell_sweeps, "sum")
    max_e2e = dist.reduce(e2e_ms, "max")
    all_e2e = dist.reduce(e2e_cs, "sum")
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        kern = {}
        # the batch engine's line solves write dU (d) only, its residuals add it to U (c)
        names = {"fast_thomas": "fast_thomas_dU", "fast_resid": "fast_resid_U",
                 "fast_thomas32": "fast_thomas32", "fast_resid32": "fast_resid32_U",
                 "full_resid": "full_resid", "fast_resid32_rhs": "fast_resid32_rhs"}
        for name, (launches, ms) in prof.items():
            b = None
            if name in names:
                # every system contributes its bytes once per launch it takes part in
                def runs(n_sw):
                    n_sw = int(n_sw)
                    if not inner or n_sw == 0:
                        return n_sw
                    th = inner[0] + (n_sw - 1) * inner[1]
                    return {"fast_thomas32": th, "fast_resid32": th - n_sw}.get(name, n_sw)
                b = nprof * sum(s.kernel_bytes(names[name]) * runs(n_sw) for s, n_sw in zip(solvers, swp))
            kern[name] = {"launches": launches, "total_ms": round(ms, 3),
                          "avg_us": round(1e3 * ms / launches, 2) if launches else None,
                          "bytes_total": b,
                          "gbs": round(b / (ms * 1e-3) / 1e9, 1) if b and ms > 0 else None}
        hot = [k for k in kern if kern[k]["bytes_total"]]
        dom = max(hot, key=lambda k: kern[k]["total_ms"]) if hot else None
        roof = None
        if dom:
            ach = kern[dom]["gbs"]
            roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "traffic": None,
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes": "sum over systems of the kernel's bytes x sweeps run",
                    "avg_launch_us": kern[dom]["avg_us"]}
        launches_per_solve = sum(v["launches"] for v in kern.values()) / nprof
        value = all_cs / (max_ms * 1e-3)
        line = {
            "metric": "batched LIJ cell-sweeps/s", "value": round(value, 1), "unit": "cell-sweeps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.algo == "fp64" else "f32+f64",
            "data": "synthetic: seeded structured meshes and values (shift %g)" % shift,
            "config": {
                "workload": f"{len(shapes)} independent LIJ systems solved together to {tol:g} "
                            f"relative residual each, lines log-U[{cfg['L'][0]},{cfg['L'][1]}], "
                            f"cells per line log-U[{cfg['K'][0]},{cfg['K'][1]}], 9x9 blocks, "
                            f"algo {args.algo}",
                "systems": len(shapes), "cells_total": int(cells.sum()),
                "cells_min": int(cells.min()), "cells_max": int(cells.max()),
                "lines_total": int(sum(m.nline for m in meshes)),
                "device_footprint_gb": round(footprint / 1e9, 2),
                "sweeps_min": int(sw.min()), "sweeps_max": int(sw.max()),
                "inner_sweeps": inner,
                "schedule": {"ctas_per_sm": ctas, "stages": stages,
                             "warps_per_line": batch.warps_per_line(),
                             "order": "longest lines first" if order == 0 else "mesh order",
                             "tuned_thomas_ms": round(tune_ms, 4)},
                "setup_s": round(setup_s, 1),
                "time_per_batch_ms": round(max_ms / args.steps, 3),
                "l2": "no flush: every sweep streams %.1f GB of blocks, > 126 MB L2" %
                      (8 * 81 * 5 * cells.sum() / 1e9),
                "timing": "CUDA events on the batch's stream around the synchronous batched "
                          "solves (one graph launch each)",
                "parallelism": f"{ws} ranks, each its own batch" if ws > 1 else "1 GPU",
            },
            "roofline": roof,
            "kernels": kern,
            "e2e": {"value": round(all_e2e / (max_e2e * 1e-3), 1), "unit": "cell-sweeps/s",
                    "h2d_bytes_per_step": int(sum(r.nbytes for r in rhs_h)),
                    "d2h_bytes_per_step": int(sum(u.nbytes for u in sol_h)), "steps": ne2e,
                    "what": "per step: tbs_set_rhs of every system from pinned host memory, "
                            "tbs_batch_solve, tbs_get_solution of every system"},
            "gpu_launches": int(round(launches_per_solve * args.steps)),
            "clocks": clk,
        }
        if ws == 1 and not args.no_cpu_baseline:
            # bounded sample: the oracle on the median-size system of the batch
            k = int(np.argsort(cells)[len(cells) // 2])
            L, K = shapes[k]
            m2, host = cpu_system(L, K, shift)
            cb = cpu_baseline(m2, host, budget_s=10.0)
            cb["value"] = cb["value"] * m2.nelem
            cb["unit"] = "cell-sweeps/s"
            cb["sample"] = f"median system of the batch ({L}x{K}): " + cb["sample"]
            line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    batch.close()
    for s in solvers:
        s.close()
    dist.close()
    return 0


# serving: Poisson arrivals over the 60x64, 360x384, 600x640 and 1200x1280 systems, 1-8
# right-hand sides per request, 20% of requests bring new Jacobian values (re-factor),
# tolerance 1e-10 for every right-hand side
SERVE_CONFIGS = {"c5": {"systems": [(60, 64, 9.0), (360, 384, 9.0), (600, 640, 4.0),
                                    (1200, 1280, 4.0)],
                        "rhs": (1, 8), "refactor": 0.2, "tol": 1e-10, "seed": 5,
                        "load": 0.6}}


def run_serving(args):
    """Steps are requests.  Phase 1 submits all requests at once (saturation:
    the server's capacity in right-hand-side solves/s); phase 2 replays them
    as a Poisson process at `load` x that capacity and reports p50/p99
    latency.  Latency is host wall clock from submit to the solution in host
    memory, as a client sees it."""
    import threading

    import torch

    import triblocksolve_b200 as tbs
    from triblocksolve_b200 import _native as N
    cfg = SERVE_CONFIGS[args.config]
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = Dist(ws, rank, local, "nccl")
    algo = {"fp64": tbs.ALGO_FP64, "mixed": tbs.ALGO_MIXED}[args.algo]
    tol = cfg["tol"]
    rng = np.random.default_rng(cfg["seed"] + 7 * rank)

    def pinned(n):
        return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()

    srv = tbs.Server(local, algo, budget_bytes=64 << 30, max_rhs=64, chunk=4)
    sys_ids, meshes, rhs_pool, alt = [], [], [], []
    t_setup = time.perf_counter()
    for k, (L, K, shift) in enumerate(cfg["systems"]):
        mesh = tbs.Mesh.structured(L, K)
        jac = types.SimpleNamespace(jacD=np.empty(81 * mesh.nelem), jacO1=np.empty(81 * mesh.nintface),
                                    jacO2=np.empty(81 * mesh.nintface), rhs=np.empty(9 * mesh.nelem))
        N.check(N.lib.tbs_gen_jacobian(9, mesh.nelem, mesh.nintface, shift, 2000 + k,
                                       N.dptr(jac.jacD), N.dptr(jac.jacO1), N.dptr(jac.jacO2),
                                       N.dptr(jac.rhs), None))
        sys_ids.append(srv.add_system(mesh, jac))
        # the values a re-factoring request brings (pinned, as a serving client would stage them)
        a = types.SimpleNamespace(jacD=pinned(81 * mesh.nelem), jacO1=pinned(81 * mesh.nintface),
                                  jacO2=pinned(81 * mesh.nintface))
        junk = np.empty(9 * mesh.nelem)
        N.check(N.lib.tbs_gen_jacobian(9, mesh.nelem, mesh.nintface, shift, 3000 + k,
                                       N.dptr(a.jacD), N.dptr(a.jacO1), N.dptr(a.jacO2),
                                       N.dptr(junk), None))
        alt.append(a)
        pool = pinned(8 * 9 * mesh.nelem).reshape(8, 9 * mesh.nelem)
        pool[:] = rng.uniform(-1.0, 1.0, pool.shape)
        rhs_pool.append(pool)
        meshes.append(mesh)
        del jac
    setup_s = time.perf_counter() - t_setup
    nreq = max(1, args.steps)
    lo, hi = cfg["rhs"]
    plan = [(int(rng.integers(len(sys_ids))), int(rng.integers(lo, hi + 1)),
             bool(rng.random() < cfg["refactor"])) for _ in range(nreq)]
    outs = [pinned(8 * 9 * m.nelem).reshape(8, 9 * m.nelem) for m in meshes]

    def submit(s, nrhs, refac):
        return srv.submit(sys_ids[s], rhs_pool[s][:nrhs], tol, 400,
                          new_jacobian=alt[s] if refac else None, out=outs[s][:nrhs])

    # warm-up: every system once, and a re-factor of the smallest
    for _ in range(max(args.warmup, 1)):
        for s in range(len(sys_ids)):
            submit(s, 2, False).wait()
    submit(0, 1, True).wait()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        # phase 1: saturation
        st0 = srv.stats()
        t0 = time.perf_counter()
        reqs = [submit(*p) for p in plan]
        res = [r.wait() for r in reqs]
        sat_s = time.perf_counter() - t0
        st1 = srv.stats()
        rhs_done = sum(p[1] for p in plan)
        capacity = rhs_done / sat_s
        sat_lat = np.array([r[3] for r in res])
        worst_rel = max(float(r[2].max()) for r in res)
        # phase 2: Poisson arrivals at load x capacity (requests per second)
        rate = cfg["load"] * capacity / ((lo + hi) / 2.0)
        gaps = rng.exponential(1.0 / rate, nreq)
        lat, qms = [None] * nreq, [None] * nreq
        handles = [None] * nreq
        ready = threading.Semaphore(0)

        def waiter():
            for i in range(nreq):
                ready.acquire()
                _U, _sw, _rel, lat[i], qms[i] = handles[i].wait()

        th = threading.Thread(target=waiter)
        th.start()
        t1 = time.perf_counter()
        due = t1
        for i, p in enumerate(plan):
            due += gaps[i]
            d = due - time.perf_counter()
            if d > 0:
                time.sleep(d)
            handles[i] = submit(*p)
            ready.release()
        th.join()
        open_s = time.perf_counter() - t1
        st2 = srv.stats()
    clk = clocks.summary()
    lat = np.array(lat)
    qms = np.array(qms)
    if rank == 0:
        per_shape = {}
        for (s, nrhs, refac), l in zip(plan, lat):
            key = f"{cfg['systems'][s][0]}x{cfg['systems'][s][1]}"
            per_shape.setdefault(key, []).append(l)
        line = {
            "metric": "serving right-hand-side solves/s", "value": round(capacity, 2),
            "unit": "rhs-solves/s", "n_gpus": ws, "steps": nreq, "warmup": args.warmup,
            "ms_per_step": round(1e3 * sat_s / nreq, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.algo == "fp64" else "f32+f64",
            "data": "synthetic: seeded structured meshes, values and right-hand sides",
            "config": {
                "workload": f"{nreq} requests over {len(sys_ids)} resident systems "
                            f"({', '.join(f'{a}x{b}' for a, b, _ in cfg['systems'])}), "
                            f"{lo}-{hi} right-hand sides each, {int(100 * cfg['refactor'])}% "
                            f"re-factor with new Jacobian values, {tol:g} relative residual "
                            f"per right-hand side, algo {args.algo}",
                "requests": nreq, "rhs_total": rhs_done,
                "refactor_requests": int(sum(p[2] for p in plan)),
                "saturation": {"seconds": round(sat_s, 3),
                               "requests_per_s": round(nreq / sat_s, 2),
                               "rhs_solves_per_s": round(capacity, 2),
                               "p50_ms": round(float(np.percentile(sat_lat, 50)), 3),
                               "p99_ms": round(float(np.percentile(sat_lat, 99)), 3),
                               "graph_launches": st1["graph_launches"] - st0["graph_launches"]},
                "poisson": {"offered_requests_per_s": round(rate, 2),
                            "load": cfg["load"], "seconds": round(open_s, 3),
                            "rhs_solves_per_s": round(rhs_done / open_s, 2),
                            "p50_ms": round(float(np.percentile(lat, 50)), 3),
                            "p90_ms": round(float(np.percentile(lat, 90)), 3),
                            "p99_ms": round(float(np.percentile(lat, 99)), 3),
                            "queue_p50_ms": round(float(np.percentile(qms, 50)), 3),
                            "queue_p99_ms": round(float(np.percentile(qms, 99)), 3),
                            "p50_ms_by_shape": {k: round(float(np.percentile(v, 50)), 3)
                                                for k, v in per_shape.items()},
                            "p99_ms_by_shape": {k: round(float(np.percentile(v, 99)), 3)
                                                for k, v in per_shape.items()}},
                "loop_ms": {k: round((st1[k] - st0[k]) / 1e3, 1)
                            for k in ("us_start", "us_members", "us_run", "us_retire")},
                "peak_rhs_in_flight": st2["peak_rhs_in_flight"],
                "peak_rhs_gb": round(st2["peak_rhs_bytes"] / 1e9, 2),
                "resident_systems_gb": round(st2["resident_system_bytes"] / 1e9, 2),
                "worst_rel_residual": worst_rel,
                "setup_s": round(setup_s, 1),
                "timing": "host wall clock: saturation = first submit to last solution in host "
                          "memory; latency per request = submit to its solution in host memory",
                "parallelism": f"{ws} ranks, each its own server" if ws > 1 else "1 GPU",
            },
            "e2e": {"value": round(capacity, 2), "unit": "rhs-solves/s",
                    "h2d_bytes_per_step": int(sum(8 * 9 * meshes[p[0]].nelem * p[1] for p in plan)
                                              / nreq),
                    "d2h_bytes_per_step": int(sum(8 * 9 * meshes[p[0]].nelem * p[1] for p in plan)
                                              / nreq),
                    "what": "the value itself: right-hand sides from pinned host memory, "
                            "solutions back to pinned host memory, re-factor uploads included"},
            "gpu_launches": int(st1["graph_launches"] - st0["graph_launches"]),
            "clocks": clk,
        }
        if ws == 1 and not args.no_cpu_baseline:
            L, K, shift = cfg["systems"][1]
            m2, host = cpu_system(L, K, shift)
            cb = cpu_baseline(m2, host, budget_s=8.0)
            # sweeps per solve of that shape from the saturation run
            sw = [int(r[1].mean()) for p, r in zip(plan, res) if p[0] == 1] or [10]
            cb["value"] = cb["value"] / max(1.0, float(np.mean(sw)))
            cb["unit"] = "rhs-solves/s"
            cb["sample"] = (f"{L}x{K} system only, solves/s = oracle sweeps/s / "
                            f"{np.mean(sw):.1f} sweeps per solve: " + cb["sample"])
            line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    srv.close()
    dist.close()
    return 0


def run_serving_reference(args):
    """The oracle on the host cores for the serving workload: per step one FP64
    sweep of the 360x384 system (a bounded sample), reported as right-hand-side
    solves/s with the sweeps per solve of that shape at the tolerance."""
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    cfg = SERVE_CONFIGS[args.config]
    L, K, shift = cfg["systems"][1]
    mesh, host = cpu_system(L, K, shift)
    cls, kind, what = cpu_impl()
    threads = os.cpu_count() or 1
    b = cls(mesh, host["jacD"], host["jacO1"], host["jacO2"], host["rhs"], threads)
    for _ in range(args.warmup):
        b.sweeps(1)
    b.reset()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        b.sweeps(1)
    dt = time.perf_counter() - t0
    sweeps_per_solve = 7.0  # 360x384, shift 9, 1e-10 (the GPU solve's count)
    v = args.steps / dt / sweeps_per_solve
    line = {"impl": "reference", "metric": "serving right-hand-side solves/s", "value": round(v, 3),
            "unit": "rhs-solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * dt / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded structured mesh and values",
            "config": {"workload": f"one FP64 sweep per step of the {L}x{K} system; solves/s = "
                                   f"sweeps/s / {sweeps_per_solve:g} sweeps per solve",
                       "cells": mesh.nelem},
            "cpu_baseline": {"value": round(v, 3), "unit": "rhs-solves/s", "cores": threads,
                             "kind": kind,
                             "sample": f"{args.steps} sweeps of the {L}x{K} system; {what}"},
            "e2e": {"value": round(v, 3), "unit": "rhs-solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_batch_reference(args):
    """The oracle on the host cores for a batched workload: one FP64 sweep of
    the batch's median-size system per step (a bounded sample), in cell-sweeps/s."""
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    cfg = BATCH_CONFIGS[args.config]
    shapes = batch_shapes(cfg)
    cells = np.array([L * K for L, K in shapes])
    L, K = shapes[int(np.argsort(cells)[len(cells) // 2])]
    mesh, host = cpu_system(L, K, cfg["shift"])
    cls, kind, what = cpu_impl()
    threads = os.cpu_count() or 1
    b = cls(mesh, host["jacD"], host["jacO1"], host["jacO2"], host["rhs"], threads)
    for _ in range(args.warmup):
        b.sweeps(1)
    b.reset()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        b.sweeps(1)
    dt = time.perf_counter() - t0
    v = mesh.nelem * args.steps / dt
    line = {"impl": "reference", "metric": "batched LIJ cell-sweeps/s", "value": round(v, 1),
            "unit": "cell-sweeps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * dt / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded structured meshes and values",
            "config": {"workload": f"one FP64 sweep per step of the median system ({L}x{K}) of "
                                   f"the {len(shapes)}-system batch", "cells": mesh.nelem},
            "cpu_baseline": {"value": round(v, 1), "unit": "cell-sweeps/s", "cores": threads,
                             "kind": kind,
                             "sample": f"{args.steps} sweeps of the {L}x{K} system; {what}"},
            "e2e": {"value": round(v, 1), "unit": "cell-sweeps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_multi(args, L, K, shift, tol):
    """--nrhs N (N > 1): N right-hand sides of one system solved together per
    step through tbs_solve_multi_device (FP64; groups of up to 8 read the
    line blocks once per sweep).  value = right-hand-side sweeps per second;
    e2e = tbs_solve_multi from pinned host arrays (right-hand sides in,
    solutions out)."""
    import torch

    import triblocksolve_b200 as tbs
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = Dist(ws, rank, local, "nccl")
    nrhs = args.nrhs
    mesh, host = build_problem(L, K, shift, pinned=True)
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    solver = tbs.Solver(local)
    solver.set_stream(stream.cuda_stream)
    solver.set_mesh(mesh)
    solver.set_jacobian_arrays(host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
    solver.factor(tbs.ALGO_FP64)
    n = 9 * mesh.nelem
    rows = torch.empty((nrhs, n), dtype=torch.float64, pin_memory=True).numpy()
    rows[0] = host["rhs"]
    rng = np.random.default_rng(SEED)
    for r in range(1, nrhs):
        rows[r] = rng.uniform(-1, 1, n)
    d_rhs = torch.from_numpy(rows).to(f"cuda:{local}", non_blocking=False)
    d_U = torch.zeros_like(d_rhs)
    Uh = torch.empty((nrhs, n), dtype=torch.float64, pin_memory=True).numpy()
    max_sweeps = 400
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for _ in range(max(args.warmup, 0)):
            solver.solve_multi_device(d_rhs.data_ptr(), d_U.data_ptr(), nrhs, tol, max_sweeps)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        sweeps_total = 0
        for _ in range(args.steps):
            sw, _h = solver.solve_multi_device(d_rhs.data_ptr(), d_U.data_ptr(), nrhs, tol,
                                               max_sweeps)
            sweeps_total += int(sw.sum())
        t1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        elapsed_ms = t0.elapsed_time(t1)
        solver.profile(True)
        solver.profile_reset()
        nprof = max(1, min(args.steps, 10))
        for _ in range(nprof):
            solver.solve_multi_device(d_rhs.data_ptr(), d_U.data_ptr(), nrhs, tol, max_sweeps)
        prof = solver.profile_read()
        solver.profile(False)
        ne2e = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 10))
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_sweeps = 0
        for _ in range(ne2e):
            _U, sw, _h = solver.solve_multi(rows, tol, max_sweeps, out=Uh)
            e2e_sweeps += int(sw.sum())
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
    clk = clocks.summary()
    max_ms = dist.reduce(elapsed_ms, "max")
    all_sweeps = dist.reduce(sweeps_total, "sum")
    max_e2e_ms = dist.reduce(e2e_ms, "max")
    all_e2e = dist.reduce(e2e_sweeps, "sum")
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        g = min(nrhs, 8)
        kern = {}
        for name, (launches, ms) in prof.items():
            b = None
            if name in ("multi_thomas", "multi_resid"):
                b = solver.kernel_bytes(f"{name}/{g}")
            avg_us = 1e3 * ms / launches if launches else 0.0
            kern[name] = {"launches": launches, "total_ms": round(ms, 4), "avg_us": round(avg_us, 3),
                          "bytes_per_launch": b,
                          "gbs": round(b / (avg_us * 1e-6) / 1e9, 1) if b and avg_us > 0 else None}
        hot = [k for k in kern if kern[k]["bytes_per_launch"]]
        dom = max(hot, key=lambda k: kern[k]["total_ms"]) if hot else None
        roof = None
        if dom:
            ach = kern[dom]["gbs"]
            roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "traffic": None,
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes_per_launch": kern[dom]["bytes_per_launch"],
                    "avg_launch_us": kern[dom]["avg_us"],
                    "note": "algorithmic bytes with every right-hand side of the group active"}
        line = {
            "metric": "LIJ sweeps/s", "value": round(all_sweeps / (max_ms * 1e-3), 2),
            "unit": "sweeps/s (one right-hand side each)", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded structured mesh and values (shift %g, seed %d); right-hand "
                    "side 0 is the generated rhs, the others seeded U(-1,1)" % (shift, SEED),
            "config": {
                "workload": f"{nrhs} right-hand sides of one LIJ system solved together to {tol:g} "
                            f"from U=0, {L} lines x {K} cells ({mesh.nelem} cells), FP64, "
                            f"groups of up to 8",
                "cells": mesh.nelem, "nrhs": nrhs, "tol": tol,
                "rhs_sweeps_per_step": all_sweeps / ws / args.steps,
                "ms_per_rhs_solve": round(max_ms / args.steps / nrhs, 4),
                "l2": "no flush: every sweep streams the line blocks (> 126 MB L2)",
                "parallelism": f"{ws} independent systems, one per GPU" if ws > 1 else "1 GPU",
            },
            "roofline": roof, "kernels": kern,
            "e2e": {"value": round(all_e2e / (max_e2e_ms * 1e-3), 2),
                    "unit": "sweeps/s (one right-hand side each)",
                    "h2d_bytes_per_step": int(rows.nbytes), "d2h_bytes_per_step": int(Uh.nbytes),
                    "steps": ne2e,
                    "what": "per step: tbs_solve_multi from pinned host arrays (right-hand "
                            "sides in, solutions out), factors resident"},
            "gpu_launches": int(round(sum(v["launches"] for v in kern.values()) / nprof * args.steps)),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    dist.close()
    return 0


def run_partition(args, L, K, shift, tol):
    """--partition: ONE mesh of the config split into N contiguous line
    ranges, one per rank (strong scaling).  Each sweep: line solves, the
    halo lines' dU exchanged with the neighbouring ranks (NCCL send/recv of
    one line of 9 doubles per cell per boundary), residual, all-reduce of
    the owned norms.  value = sweeps of the whole mesh per second; e2e adds
    the partition's Jacobian upload, factorization and the owned solution's
    read-back to every step.  At N = 1 the mesh is one partition without
    halo lines: the host-driven sweep loop beside the graph-launched solve."""
    import torch

    import triblocksolve_b200 as tbs
    from triblocksolve_b200 import _native as N
    from triblocksolve_b200.partition import (DistExchange, PartitionedSolve, PartitionSolver,
                                              owned_norm_sq, partition_lines)
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = Dist(ws, rank, local, "nccl")
    mesh, whole = build_problem(L, K, shift, pinned=False)
    parts = partition_lines(mesh, ws)
    part = parts[rank]
    host = {}
    for k, a in zip(("jacD", "jacO1", "jacO2", "rhs"),
                    part.sub_arrays(whole["jacD"], whole["jacO1"], whole["jacO2"], whole["rhs"])):
        host[k] = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy()
        host[k][:] = a
    del whole
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    solver = PartitionSolver(part, local)
    solver.set_stream(stream.cuda_stream)  # the stream the CUDA events below are recorded on
    solver.set_jacobian_arrays(host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
    solver.factor(tbs.ALGO_FP64)
    ex = DistExchange(part, solver, device=f"cuda:{local}", group=None) if ws > 1 else None

    class _Single:  # one partition, nothing to exchange
        def exchange(self, which):
            pass

        def allreduce_sum(self, x):
            return x

        def norm_sq_async(self, sweepers):
            return owned_norm_sq(sweepers, torch.device(f"cuda:{local}"))

    run = PartitionedSolve([solver], ex if ex else _Single())
    max_sweeps = 400
    Uh = torch.empty(9 * part.mesh.nelem, dtype=torch.float64, pin_memory=True).numpy()
    with ClockSampler(local) as clocks:
        for _ in range(max(args.warmup, 0)):
            run.solve(tol, max_sweeps)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        sweeps_total = 0
        hist = None
        for _ in range(args.steps):
            n, hist = run.solve(tol, max_sweeps)
            sweeps_total += n
        t1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        elapsed_ms = t0.elapsed_time(t1)
        solver.profile(True)
        solver.profile_reset()
        nprof = max(1, min(args.steps, 10))
        for _ in range(nprof):
            run.solve(tol, max_sweeps)
        prof = solver.profile_read()
        solver.profile(False)
        ne2e = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 10))
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_sweeps = 0
        for _ in range(ne2e):
            solver.set_jacobian_arrays(host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
            solver.factor(tbs.ALGO_FP64)
            n, _h = run.solve(tol, max_sweeps)
            solver.solution(out=Uh)
            e2e_sweeps += n
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
    clk = clocks.summary()
    tn = solver.true_residual_norm()
    true_rel = float(np.sqrt(dist.reduce(tn * tn, "sum"))) / float(hist[0])
    max_ms = dist.reduce(elapsed_ms, "max")
    max_e2e_ms = dist.reduce(e2e_ms, "max")
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        kern = {}
        for name, (launches, ms) in prof.items():
            try:
                # the owned lines' solves add dU to U; the residual adds it for the
                # halo lines only (a few lines: counted as the single-system form)
                b = solver.kernel_bytes(name)
            except Exception:
                b = None
            avg_us = 1e3 * ms / launches if launches else 0.0
            kern[name] = {"launches": launches, "total_ms": round(ms, 4), "avg_us": round(avg_us, 3),
                          "bytes_per_launch": b,
                          "gbs": round(b / (avg_us * 1e-6) / 1e9, 1) if b and avg_us > 0 else None}
        hot = [k for k in kern if kern[k]["bytes_per_launch"] and k != "fast_resid_rhs"]
        dom = max(hot, key=lambda k: kern[k]["total_ms"]) if hot else None
        roof = None
        if dom:
            ach = kern[dom]["gbs"]
            roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "traffic": None,
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes_per_launch": kern[dom]["bytes_per_launch"],
                    "avg_launch_us": kern[dom]["avg_us"], "rank": 0}
        halo_bytes = sum(8 * 9 * int(part.mesh.linesize[k]) for ks in part.recvs.values() for k in ks)
        line = {
            "metric": "LIJ sweeps/s", "value": round(sweeps_total / (max_ms * 1e-3), 2),
            "unit": "sweeps/s (of the whole mesh)", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 5),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded structured mesh and values (shift %g, seed %d)" % (shift, SEED),
            "config": {
                "workload": f"one LIJ system of {L} lines x {K} cells ({mesh.nelem} cells) split "
                            f"into {ws} line partitions, solved to {tol:g} from U=0, FP64",
                "cells": mesh.nelem, "tol": tol, "partitions": ws,
                "owned_lines_rank0": part.nowned, "halo_lines_rank0": part.nhalo,
                "halo_bytes_per_sweep_rank0": halo_bytes,
                "sweeps_per_solve": sweeps_total / args.steps, "true_rel_residual": true_rel,
                "true_residual_check": {"checks": run.checks, "restarts": run.restarts},
                "l2": "no flush: every sweep streams the line blocks (> 126 MB L2)",
                "parallelism": f"line partitions of one mesh over {ws} GPUs, NCCL halo exchange"
                               if ws > 1 else "1 GPU, one partition (host-driven sweep loop)",
            },
            "roofline": roof, "kernels": kern,
            "e2e": {"value": round(e2e_sweeps / (max_e2e_ms * 1e-3), 2),
                    "unit": "sweeps/s (of the whole mesh)",
                    "h2d_bytes_per_step": int(sum(a.nbytes for a in host.values())),
                    "d2h_bytes_per_step": int(Uh.nbytes), "steps": ne2e,
                    "what": "per step on every rank: tbs_set_jacobian of the partition from "
                            "pinned host memory, tbs_factor, the partitioned solve, "
                            "tbs_get_solution (rank 0's bytes)"},
            "gpu_launches": int(round(sum(v["launches"] for v in kern.values()) / nprof * args.steps)),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    del ex
    solver.close()
    dist.close()
    return 0


def run_gmres(args, L, K, shift, tol):
    """--gmres M: restarted GMRES(M) on the system, right preconditioned by
    one LIJ sweep (tbs_gmres, FP64 line factors), to the config's tolerance
    from U = 0; value = solves per second, with the plain LIJ solve of the
    same system timed beside it.  e2e: tbs_set_rhs from pinned host memory,
    tbs_gmres, tbs_get_solution per step."""
    import torch

    import triblocksolve_b200 as tbs
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = Dist(ws, rank, local, "nccl")
    mesh, host = build_problem(L, K, shift, pinned=True)
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    solver = tbs.Solver(local)
    solver.set_stream(stream.cuda_stream)
    solver.set_mesh(mesh)
    solver.set_jacobian_arrays(host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
    solver.factor(tbs.ALGO_FP64)
    m, max_iters = args.gmres, 400
    with ClockSampler(local) as clocks:
        for _ in range(max(args.warmup, 0)):
            solver.gmres(tol, m, 1, max_iters)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        iters = 0
        for _ in range(args.steps):
            it, h = solver.gmres(tol, m, 1, max_iters)
            iters += it
        t1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        elapsed_ms = t0.elapsed_time(t1)
        true_rel = solver.true_residual_norm() / float(h[0])
        # the plain line sweep on the same system, for comparison
        solver.solve(tol, max_iters)
        torch.cuda.synchronize()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(stream)
        nl = max(1, min(args.steps, 20))
        for _ in range(nl):
            lij_sweeps, lh = solver.solve(tol, max_iters)
        l1.record(stream)
        torch.cuda.synchronize()
        lij_ms = l0.elapsed_time(l1) / nl
        solver.profile(True)
        solver.profile_reset()
        nprof = max(1, min(args.steps, 10))
        for _ in range(nprof):
            solver.gmres(tol, m, 1, max_iters)
        prof = solver.profile_read()
        solver.profile(False)
        ne2e = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 10))
        Uh = torch.empty(9 * mesh.nelem, dtype=torch.float64, pin_memory=True).numpy()
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ne2e):
            solver.set_rhs(host["rhs"])
            solver.gmres(tol, m, 1, max_iters)
            solver.solution(out=Uh)
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
    clk = clocks.summary()
    max_ms = dist.reduce(elapsed_ms, "max")
    max_e2e = dist.reduce(e2e_ms, "max")
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        kern = {}
        for name, (launches, ms) in prof.items():
            try:
                b = solver.kernel_bytes(name)
            except Exception:
                b = None
            avg_us = 1e3 * ms / launches if launches else 0.0
            kern[name] = {"launches": launches, "total_ms": round(ms, 4), "avg_us": round(avg_us, 3),
                          "bytes_per_launch": b,
                          "gbs": round(b / (avg_us * 1e-6) / 1e9, 1) if b and avg_us > 0 else None}
        hot = [k for k in kern if kern[k]["bytes_per_launch"] and k != "fast_resid_rhs"]
        dom = max(hot, key=lambda k: kern[k]["total_ms"]) if hot else None
        roof = None
        if dom:
            ach = kern[dom]["gbs"]
            roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "traffic": None,
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes_per_launch": kern[dom]["bytes_per_launch"],
                    "avg_launch_us": kern[dom]["avg_us"]}
        line = {
            "metric": "GMRES solves/s", "value": round(ws * args.steps / (max_ms * 1e-3), 3),
            "unit": "solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded structured mesh and values (shift %g, seed %d)" % (shift, SEED),
            "config": {
                "workload": f"GMRES({m}) right-preconditioned by one LIJ sweep, to {tol:g} from "
                            f"U=0, {L} lines x {K} cells ({mesh.nelem} cells), FP64",
                "cells": mesh.nelem, "restart": m, "tol": tol,
                "arnoldi_steps_per_solve": iters / args.steps,
                "time_to_tol_ms": round(max_ms / args.steps, 4),
                "true_rel_residual": true_rel,
                "lij_sweeps_to_tol": int(lij_sweeps), "lij_time_to_tol_ms": round(lij_ms, 4),
                "l2": "no flush: every step streams the line blocks and the basis (> 126 MB L2)",
                "parallelism": f"{ws} independent systems, one per GPU" if ws > 1 else "1 GPU",
            },
            "roofline": roof, "kernels": kern,
            "e2e": {"value": round(ws * ne2e / (max_e2e * 1e-3), 3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(host["rhs"].nbytes), "d2h_bytes_per_step": int(Uh.nbytes),
                    "steps": ne2e,
                    "what": "per step: tbs_set_rhs from pinned host memory, tbs_gmres, tbs_get_solution"},
            "gpu_launches": int(round(sum(v["launches"] for v in kern.values()) / nprof * args.steps)),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    dist.close()
    return 0


def run_reference(args, L, K, shift, tol):
    """The reference's CPU path on the host cores, one FP64 sweep per step
    (a bounded sample of a solve), rank 0 only; the factorization is timed
    apart and reported."""
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    mesh, host = cpu_system(L, K, shift)
    cls, kind, what = cpu_impl()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    b = cls(mesh, host["jacD"], host["jacO1"], host["jacO2"], host["rhs"], threads)
    t_factor = time.perf_counter() - t0
    for _ in range(args.warmup):
        b.sweeps(1)
    b.reset()
    t0 = time.perf_counter()
    done = 0
    for _ in range(args.steps):
        b.sweeps(1)
        done += 1
    dt = time.perf_counter() - t0
    v = done / dt
    line = {"impl": "reference", "metric": "LIJ sweeps/s", "value": v, "unit": "sweeps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded structured mesh and values (shift %g, seed %d)" % (shift, SEED),
            "config": {"workload": f"LIJ solve to {tol:g} relative residual from U=0, {L} lines x {K} "
                                   f"cells ({mesh.nelem} cells, {mesh.nintface} faces), 9x9 blocks, "
                                   f"algo fp64",
                       "cells": mesh.nelem, "lines": L, "cells_per_line": K, "tol": tol,
                       "algo": "fp64", "factor_s": round(t_factor, 3),
                       "step": "one FP64 sweep of the solve (a bounded sample; sweeps/s does not "
                               "depend on how many are timed)"},
            "cpu_baseline": {"value": v, "unit": "sweeps/s", "cores": threads, "kind": kind,
                             "cpu_model": cpu_model(), "nproc": os.cpu_count(),
                             "sample": f"{done} sweeps (one per step) after one factorization "
                                       f"({t_factor:.2f} s); {what} (OCCA, MPI and gfortran, "
                                       "which the reference builds with, are absent)"},
            "e2e": {"value": v, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3b",
                    choices=sorted(CONFIGS) + sorted(BATCH_CONFIGS) + sorted(SERVE_CONFIGS))
    ap.add_argument("--algo", default="fp64", choices=["fp64", "ref", "mixed", "pij"])
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nvar", type=int, default=9,
                    help="block size of the generated system (the reference's block-size study)")
    ap.add_argument("--gmres", type=int, default=0,
                    help="restart length: time line-preconditioned GMRES instead of the sweep loop")
    ap.add_argument("--nrhs", type=int, default=1,
                    help="right-hand sides per solve (> 1: tbs_solve_multi, FP64)")
    ap.add_argument("--partition", action="store_true",
                    help="one mesh split into line partitions over the ranks (strong scaling)")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1: N independent systems, one per rank (weak scaling), "
                         "instead of one mesh split into line partitions")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision solve timed beside the FP64 one")
    args = ap.parse_args()
    if args.config in SERVE_CONFIGS:
        if args.impl == "reference":
            return run_serving_reference(args)
        return run_serving(args)
    if args.config in BATCH_CONFIGS:
        if args.impl == "reference":
            return run_batch_reference(args)
        return run_batch(args)
    L, K, shift, tol = CONFIGS[args.config]
    if args.impl == "reference":
        return run_reference(args, L, K, shift, tol)
    ws_env = dist_env()[0]
    if args.partition or (ws_env > 1 and not args.replicas and args.algo == "fp64"
                          and args.nvar == 9 and args.nrhs == 1 and not args.gmres):
        if args.algo != "fp64" or args.nvar != 9 or args.nrhs > 1 or args.gmres:
            ap.error("--partition runs the FP64 sweep at nvar 9")
        return run_partition(args, L, K, shift, tol)
    if args.gmres > 0:
        return run_gmres(args, L, K, shift, tol)
    if args.nrhs > 1:
        if args.algo != "fp64":
            ap.error("--nrhs > 1 needs --algo fp64")
        return run_multi(args, L, K, shift, tol)

    import torch

    import triblocksolve_b200 as tbs
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = Dist(ws, rank, local, "nccl")
    algo = {"fp64": tbs.ALGO_FP64, "ref": tbs.ALGO_REFERENCE, "mixed": tbs.ALGO_MIXED,
            "pij": tbs.ALGO_PIJ}[args.algo]

    nvar = args.nvar
    if nvar != 9:
        if args.algo not in ("fp64", "ref"):
            ap.error("--nvar other than 9 needs --algo fp64 or ref")
        shift = max(shift, float(nvar))  # keeps the generated blocks diagonally dominant
    mesh, host = build_problem(L, K, shift, pinned=True, nvar=nvar)
    # a dedicated stream: CUDA graphs cannot be captured on the legacy default stream
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    solver = tbs.Solver(local)
    solver.set_stream(stream.cuda_stream)
    solver.set_mesh(mesh)
    solver.set_jacobian_arrays(host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    solver.factor(algo)
    f1.record()
    torch.cuda.synchronize()
    factor_ms = f0.elapsed_time(f1)
    max_sweeps = 400
    inner = None
    if args.algo == "mixed":
        solver.tune_inner(tol, max_sweeps)
        inner = list(solver.inner_schedule())  # [first outer step, the others]

    with ClockSampler(local) as clocks:
        for _ in range(max(args.warmup, 0)):
            solver.solve(tol, max_sweeps)
        # ---------------- timed region: K solves, blocks resident in HBM
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if nvar == 9:
            solver.resid_timer(reset=True)
        t0.record(stream)
        sweeps_total = 0
        last_hist = None
        for _ in range(args.steps):
            s, last_hist = solver.solve(tol, max_sweeps)
            sweeps_total += s
        t1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        elapsed_ms = t0.elapsed_time(t1)
        # the sweeps' residual launches inside those graph solves, on the device clock
        in_graph = solver.resid_timer() if nvar == 9 else (0.0, 0)
        # ---------------- per-kernel CUDA-event timing (same solves, eager launch)
        solver.profile(True)
        solver.profile_reset()
        nprof = max(1, min(args.steps, 20))
        prof_sweeps = 0
        for _ in range(nprof):
            s, _h = solver.solve(tol, max_sweeps)
            prof_sweeps += s
        prof = solver.profile_read()
        solver.profile(False)
        # ---------------- e2e: upload + factor + solve + read back, from pinned host memory
        ne2e = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 20))
        Uh = torch.empty(nvar * mesh.nelem, dtype=torch.float64, pin_memory=True).numpy()
        for _ in range(1):
            solver.set_jacobian_arrays(host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
            torch.cuda.synchronize()
            f2, f3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f2.record(stream)
            solver.factor(algo)
            f3.record(stream)
            torch.cuda.synchronize()
            factor_warm_ms = f2.elapsed_time(f3)
            solver.solve(tol, max_sweeps)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        # (a) one system after another: upload, factor, solve, read back
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        seq_sweeps = 0
        for _ in range(ne2e):
            solver.set_jacobian_arrays(host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
            solver.factor(algo)
            s, hh = solver.solve(tol, max_sweeps)
            solver.solution(out=Uh)  # straight into pinned host memory
            seq_sweeps += s
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        seq_ms = e0.elapsed_time(e1)
        # (b) a stream of systems: the next two Jacobians are staged (uploaded
        # back to back on the context's copy stream) while the current one is
        # factored and solved; the same uploads, factorizations, solves and
        # read-backs, step for step
        jac_h = (host["jacD"], host["jacO1"], host["jacO2"], host["rhs"])
        e0.record(stream)
        e2e_sweeps = 0
        solver.stage_jacobian_arrays(*jac_h)
        if ne2e > 1:
            solver.stage_jacobian_arrays(*jac_h)
        solver.factor(algo)
        for k in range(ne2e):
            s, hh = solver.solve(tol, max_sweeps)
            solver.solution(out=Uh)
            e2e_sweeps += s
            if k + 2 < ne2e:
                solver.stage_jacobian_arrays(*jac_h)
            if k + 1 < ne2e:
                solver.factor(algo)
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        check = solver.solve_check() if args.algo == "fp64" else None
        true_rel = solver.true_residual_norm() / float(last_hist[0])
        # ---------------- the mixed form beside it: FP32 line factors and inner sweeps,
        # FP64 outer residual, same system and tolerance, same number of timed solves
        mixed = None
        if (args.algo == "fp64" and nvar == 9 and not args.no_mixed
                and args.config in ("c3a", "c3b")):
            U64 = solver.solution()
            solver.factor(tbs.ALGO_MIXED)
            solver.tune_inner(tol, max_sweeps)
            for _ in range(max(args.warmup, 0)):
                solver.solve(tol, max_sweeps)
            torch.cuda.synchronize()
            dist.barrier()
            torch.cuda.synchronize()
            m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            msteps = 0
            for _ in range(args.steps):
                ms_, mh = solver.solve(tol, max_sweeps)
                msteps += ms_
            m1.record(stream)
            torch.cuda.synchronize()
            dist.barrier()
            torch.cuda.synchronize()
            mixed_ms = dist.reduce(m0.elapsed_time(m1), "max") / args.steps
            Um = solver.solution()
            mixed = {
                "ms_per_solve": round(mixed_ms, 4),
                "outer_steps_per_solve": msteps / args.steps,
                "inner_sweeps": list(solver.inner_schedule()),
                "true_rel_residual": solver.true_residual_norm() / float(mh[0]),
                "rel_error_vs_fp64_solution": float(np.linalg.norm(Um - U64) / np.linalg.norm(U64)),
                "what": "TBS_ALGO_MIXED: FP32 line factors and inner sweeps, FP64 outer "
                        "residual from the original blocks, autotuned inner sweep schedule; "
                        "CUDA events around the same number of graph-launched solves",
            }
    clk = clocks.summary()

    max_ms = dist.reduce(elapsed_ms, "max")
    all_sweeps = dist.reduce(sweeps_total, "sum")
    max_e2e_ms = dist.reduce(e2e_ms, "max")
    all_e2e_sweeps = dist.reduce(e2e_sweeps, "sum")
    max_seq_ms = dist.reduce(seq_ms, "max")
    all_seq_sweeps = dist.reduce(seq_sweeps, "sum")

    if rank == 0:
        value = all_sweeps / (max_ms * 1e-3)
        peak, peak_kind = measured_peak_hbm()
        kern = {}
        for name, (launches, ms) in prof.items():
            try:
                b = solver.kernel_bytes(name)
            except Exception:
                b = None
            avg_us = 1e3 * ms / launches if launches else 0.0
            kern[name] = {"launches": launches, "total_ms": round(ms, 4),
                          "avg_us": round(avg_us, 3),
                          "bytes_per_launch": b,
                          "gbs": round(b / (avg_us * 1e-6) / 1e9, 1) if b and avg_us > 0 else None}
        hot = [k for k in kern if kern[k]["bytes_per_launch"] and k not in ("fast_resid_rhs",
                                                                             "fast_resid32_rhs")]
        dom = max(hot, key=lambda k: kern[k]["total_ms"]) if hot else None
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if dom and os.path.exists(tpath) and nvar == 9:
            t = json.load(open(tpath)).get(args.config, {}).get(dom)
            if t:
                traffic = t
        roof = None
        if dom:
            ach = kern[dom]["gbs"]
            roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "traffic": traffic,
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes_per_launch": kern[dom]["bytes_per_launch"],
                    "avg_launch_us": kern[dom]["avg_us"]}
            if dom == "fast_resid" and in_graph[1] > 0:
                g_us = in_graph[0] / in_graph[1]
                g_ach = kern[dom]["bytes_per_launch"] / (g_us * 1e-6) / 1e9
                roof["in_timed_region"] = {
                    "launches": in_graph[1], "avg_launch_us": round(g_us, 3),
                    "achieved": round(g_ach, 1), "frac": round(g_ach / peak, 4),
                    "how": "the same kernel's launches inside the timed graph solves, each from "
                           "its earliest CTA start to its last CTA's finish on the GPU's "
                           "%globaltimer (CUDA events cannot sit inside the solve graph's loop); "
                           "achieved/frac above are from CUDA events around eager launches of "
                           "the same solves"}
        # the profiled kernels of a solve, plus the two each graph-launched
        # solve adds around its graph (control block in, state read back)
        launches_per_solve = sum(v["launches"] for v in kern.values()) / nprof + 2
        sweeps_per_solve = sweeps_total / args.steps
        h2d = sum(host[k].nbytes for k in ("jacD", "jacO1", "jacO2", "rhs"))
        d2h = Uh.nbytes + 8 * (max_sweeps + 1)
        nb_ = nvar * nvar
        ref_bytes = reference_model_bytes(mesh)
        line = {
            "metric": "LIJ sweeps/s", "value": round(value, 2), "unit": "sweeps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": (round(value / ws / PUBLISHED_SWEEPS_PER_S[args.config], 3)
                            if args.config in PUBLISHED_SWEEPS_PER_S and args.algo in ("fp64", "ref")
                            and nvar == 9
                            else None),
            "dtype": "f64" if args.algo != "mixed" else "f32+f64",
            "data": "synthetic: seeded structured mesh and values (shift %g, seed %d); the "
                    "reference's real Jacobians are not available" % (shift, SEED),
            "config": {
                "workload": f"LIJ solve to {tol:g} relative residual from U=0, {L} lines x {K} "
                            f"cells ({mesh.nelem} cells, {mesh.nintface} faces), {nvar}x{nvar} blocks, "
                            f"algo {args.algo}",
                "cells": mesh.nelem, "lines": L, "cells_per_line": K, "tol": tol,
                "algo": args.algo, "sweeps_per_solve": sweeps_per_solve,
                "inner_sweeps": inner,
                "time_to_tol_ms": round(max_ms / args.steps, 4),
                "kernel_ms_per_solve_eager": round(sum(v["total_ms"] for v in kern.values()) / nprof, 4),
                "kernel_times": "per-kernel times from a separate pass of the same solves launched eagerly with CUDA events around every launch (the timed solves are graph launches)",
                "factor_ms": round(factor_ms, 3),
                "factor_ms_warm": round(factor_warm_ms, 3),
                "true_rel_residual": true_rel,
                "true_residual_check": (None if check is None else
                                        {"true_norm": check[0], "checks": check[1],
                                         "restarts": check[2]}),
                "l2": "no flush: every sweep streams %.0f MB of blocks, > 126 MB L2" %
                      (8 * nvar * nvar * 5 * mesh.nelem / 1e6),
                "reference_model_gbs": round(ref_bytes * value / ws / 1e9, 1),
                "reference_model_bytes_per_sweep": int(ref_bytes),
                "published_baseline": "V100 FP64 LIJ, paper Table 5 (5 sweeps); vs_baseline "
                                      "is per GPU",
                "parallelism": f"{ws} independent systems, one per GPU" if ws > 1 else "1 GPU",
            },
            "roofline": roof,
            "kernels": kern,
            "e2e": {"value": round(all_e2e_sweeps / (max_e2e_ms * 1e-3), 2), "unit": "sweeps/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "steps": ne2e,
                    "what": "per step, through the C ABI from pinned host memory: tbs_solve, "
                            "tbs_get_solution, the system two ahead staged (tbs_stage_jacobian: "
                            "uploads back to back on the context's copy stream while the "
                            "systems before it are factored and solved), tbs_factor of the next "
                            "staged system; every step's upload, factorization, solve and "
                            "read-back inside the timed region",
                    "sequential": {"value": round(all_seq_sweeps / (max_seq_ms * 1e-3), 2),
                                   "what": "per step: tbs_set_jacobian, tbs_factor, tbs_solve, "
                                           "tbs_get_solution, one after another"}},
            "gpu_launches": int(round(launches_per_solve * args.steps)),
            "clocks": clk,
        }
        if mixed is not None:
            fp64_ms = max_ms / args.steps
            mixed["fp64_ms_per_solve"] = round(fp64_ms, 4)
            mixed["speedup_vs_fp64"] = round(fp64_ms / mixed["ms_per_solve"], 3)
            line["mixed"] = mixed
        if ws == 1 and not args.no_cpu_baseline:
            if args.algo == "pij":
                import oracle
                line["cpu_baseline"] = cpu_baseline(oracle.point_lines(mesh), host)
                line["cpu_baseline"]["sample"] += " (one-cell lines: the point-implicit sweep)"
            else:
                line["cpu_baseline"] = cpu_baseline(mesh, host)
        print(json.dumps(line), flush=True)
    solver.close()
    dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
