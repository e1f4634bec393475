#!/usr/bin/env python
"""Shell solves/sec (p50/p99 latency), mixed precision vs FP64 on the GPU.

Workload: 64 independent clamped plates, element grids log-uniform 16^2 ..
256^2 with aspect 1..4 (seed 4321), t ~ U(2, 8) mm, p ~ U(0.5, 2) kPa,
E = 70 GPa, nu = 0.3. A step assembles the 6x6-block BSR Jacobian (fused
BCs), factors the block ILU(k) preconditioner (k per problem from the
autotuner's table) and solves every problem to ||b - A x|| / ||b|| <= 1e-8
with FP32 ILU factors inside FP64 GMRES, all 64 problems as one batch.
`value` is whole-job solves/s with inputs resident in HBM; `e2e` repeats the
step through the public API with the load vectors copied from pinned host
memory and the displacements copied back inside the timed region. Beside
it: the same batch with FP64 factors, the plain FP64 GPU path (each problem
alone through gf_gmres_solve), the per-solve mixed-vs-FP64 displacement
difference, the sweep kernel's roofline and a CPU baseline.

--impl reference times the CPU path (the oracle's compiled restatement of
the reference's CPU assembly plus FP64 block ILU(k) and GMRES, with the same
fill and ordering) on a pool of single-threaded worker processes.

Multi-GPU (torchrun): every rank solves its own full batch (replicas, weak
scaling); the step time is the max over ranks.
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

METRIC = "shell solves/sec + p50/p99 latency, mixed vs FP64 GPU at 1e-8 rel residual"
WORKLOAD = ("64 clamped plates, grids 16^2-256^2 log-uniform, aspect 1-4, seed 4321; "
            "assemble + block ILU(k) + GMRES/IR to 1e-8")


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--problems", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain (one problem at a time) FP64 GPU path")
    ap.add_argument("--tune", action="store_true",
                    help="re-run the fill autotuner instead of the committed table")
    ap.add_argument("--tune-log", default=None,
                    help="with --tune: write the autotuner's trial log (JSON) to this file")
    ap.add_argument("--serve-seconds", type=float, default=8.0,
                    help="length of the Poisson request stream of the serving run (0 skips it)")
    ap.add_argument("--assembly-case", action="store_true",
                    help="small profiling case: Jacobian assembly (fused BCs) of the 400x200 "
                         "jittered cantilever plate, 5 times (no JSON line)")
    ap.add_argument("--sweep-case", choices=["dataflow", "level"], default=None,
                    help="small profiling case: the triangular sweeps of one 256x128 plate, "
                         "natural ordering, ILU(6), FP32 factors, applied 5 times with the "
                         "given sweep kernel (no JSON line)")
    return ap.parse_args()


SERVE_RATE, SERVE_MAX_CLASS = 20.0, 4


def serving_run(seconds):
    """Continuous-batching server on a Poisson stream of plate and stiffened-box
    requests (rate 20/s, size classes 0..4 = 5e3..2.5e4 DOF, per-request
    thickness field and load from the request seed), once with FP32 ILU
    factors (mixed) and once with FP64 factors, each to a 1e-8 relative
    residual. Size classes are built, their fill tuned and their slot groups
    reserved before the stream starts."""
    from gpu_fem_b200 import serve
    out, fills, n = {}, None, 0
    for prec, name in (("fp32", "mixed"), ("fp64", "fp64")):
        reqs = serve.poisson_requests(rate=SERVE_RATE, duration=seconds, seed=99,
                                      max_class=SERVE_MAX_CLASS)
        n = len(reqs)
        try:
            srv = serve.Server(budget_gb=40.0, streams=4, max_batch=8, precision=prec,
                               fills=fills)
            srv.warm({(r.family, r.cls) for r in reqs})
            fills = dict(srv.fills)
            res = srv.run(reqs)
            out[name] = {k: res[k] for k in ("requests", "solved", "solves_per_s", "p50_ms",
                                              "p99_ms", "wall_s", "reserved_gb")}
            out[name]["fills"] = {f"{f}{k}": int(v) for (f, k), v in sorted(srv.fills.items())}
            del srv
        except Exception as e:  # report the failure in the line, keep the rest
            out[name] = {"error": repr(e)[:300]}
    out["stream"] = (f"Poisson {SERVE_RATE:g} req/s for {seconds:g} s, {n} requests, plates and "
                     f"stiffened boxes, size classes 0..{SERVE_MAX_CLASS} (5e3..2.5e4 DOF); "
                     f"latency = completion - arrival; slot groups of 8/4/2/1 per class reserved "
                     f"before the stream")
    return out


def assembly_case():
    """Jacobian assembly with fused BCs of the 400x200 plate (80,601 nodes,
    ~209 MB of block values, above L2), 5 times with the coloured scatter:
    the small case on which the assembly kernel is profiled. Then prints the
    event-timed Jacobian with the coloured and the atomic scatter, alone and
    for the 64-plate batch (one launch per colour over all problems, or one
    launch with atomics)."""
    import torch
    from gpu_fem_b200 import mesh as M
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner, createBsrMat
    from gpu_fem_b200.batch import Batch
    m = M.plate_config2()
    A = ElementAssembler.from_mesh(m, ordering="rcm")
    K = createBsrMat(A)
    res = A.createVarsVec()
    for _ in range(5):
        A.add_jacobian(res, K, fuse_bcs=True)
    torch.cuda.synchronize()
    print("assembly case", A.get_nnzb())

    def timed(fn, reps=10):
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"400x200 coloured ms": timed(lambda: A.add_jacobian(None, K, fuse_bcs=True)),
           "400x200 atomic ms": timed(lambda: A.add_jacobian(None, K, fuse_bcs=True, atomic=True))}
    meshes = M.batch_config4(64)
    asms = [ElementAssembler.from_mesh(mm, ordering="natural") for mm in meshes]
    mats = [createBsrMat(a) for a in asms]
    pcs = [ILUk_Preconditioner(a, fill_level=0) for a in asms]
    bt = Batch(asms, mats, pcs)
    out["batch64 coloured ms"] = timed(bt.assemble)
    bt.set_scatter(True)
    out["batch64 atomic ms"] = timed(bt.assemble)
    print("assembly scatter", json.dumps({k: round(v, 3) for k, v in out.items()}))


def sweep_case(kind):
    """One preconditioner (256x128 clamped plate, t = 2 mm, natural ordering,
    ILU(6), FP32 factors, ~150 MB of factor) applied 5 times with the given
    sweep kernel: the small case on which the sweep and factorization kernels
    are profiled (its levels are large enough that the factorization and the
    level-synchronous sweeps run on a two-CTA cluster). Prints the mean
    event-timed apply (both sweeps)."""
    import torch
    from gpu_fem_b200 import mesh as M
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner, createBsrMat
    m = M.plate(256, 128, 1.0, 0.5, lambda x, y: 0.002 + 0 * x, "all_edges",
                lambda q: 1e3 + 0 * q[:, 0])
    A = ElementAssembler.from_mesh(m, ordering="natural")
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    P = ILUk_Preconditioner(A, fill_level=6, precision="fp32", sweep=kind)
    P.factor(K)
    r = torch.randn(m.num_dof, dtype=torch.float64, device="cuda")
    z = torch.zeros_like(r)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    P.apply(r, z)
    e0.record()
    for _ in range(5):
        P.apply(r, z)
    e1.record()
    torch.cuda.synchronize()
    print("sweep case", kind, P.info(), P.sweeps(), f"{e0.elapsed_time(e1) / 5:.3f} ms per apply",
          float(z.abs().max()))


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = []
        reasons = set()
        smax = None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def job_ms(ms, ws, device):
    """Per-step time of the whole job: the maximum over ranks of each rank's
    device-timed step (every rank runs its own replica of the batch)."""
    if ws == 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(problems_per_rank, ws, ms):
    """Solves per second of the whole job: every rank's problems over the
    slowest rank's step time."""
    return ws * problems_per_rank / (ms / 1e3)


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# DRAM bytes (read + write) of a sweep launch over its algorithmic bytes,
# from an ncu capture of the 256x128 ILU(6) FP32 sweep case (the batch's
# launches are too large to capture): 85.1 MB / 80.2 MB for L, 89.7 MB /
# 85.1 MB for U (profiles/bsweep_tma_256x128_ilu6_traffic.md). Traffic per
# launch grows with the blocks streamed, so the bench scales the ratio by its
# own algorithmic bytes per launch.
SWEEP_TRAFFIC_RATIO = 1.055

# Fill level k and node ordering of each of the 64 problems, as chosen by the
# batch autotuner (gpu_fem_b200/batch.py: ordering by ILU(8) levels x blocks
# per row, then the converging k of smallest modelled factor + solve time) on
# a B200. Both arms run every problem with these, so their configs match;
# `--tune` re-runs the autotuner and prints the table it finds. This table
# measured 268 solves/s; re-tuning with the current cost models picks higher
# fills for the large plates (17 instead of 23 GMRES steps) and measured
# 249 solves/s, because the batched factorization's time is not yet modelled
# well enough (the problems share the SMs).
FILLS = [12, 16, 12, 7, 6, 6, 10, 8, 8, 5, 8, 6, 10, 6, 12, 12, 8, 8, 8, 12, 12, 6, 10, 10, 6,
         16, 12, 6, 7, 8, 10, 12, 5, 12, 5, 10, 7, 6, 5, 12, 16, 16, 5, 12, 6, 10, 10, 12, 10,
         12, 8, 7, 16, 8, 6, 5, 8, 10, 12, 16, 4, 4, 10, 12]
ORDERS = "n" * 64  # one character per problem: "n" natural, "r" RCM


def bench_config(meshes, fills, orders, ws):
    """The workload description both arms print (identical for the same table)."""
    return {"workload": WORKLOAD, "problems": len(meshes),
            "dofs": int(sum(m.num_dof for m in meshes)),
            "fill_levels": [int(k) for k in fills], "orderings": "".join(o[0] for o in orders),
            "rtol": 1e-8, "gmres": "right-preconditioned GMRES(100), FP64 Krylov vectors",
            "l2": "inputs larger than L2 (all 64 systems resident, ~GB)",
            "parallelism": f"replicas x{ws}"}


def table_or_none(n):
    if FILLS is None or ORDERS is None or len(FILLS) != n or len(ORDERS) != n:
        return None, None
    return list(FILLS), ["natural" if c == "n" else "rcm" for c in ORDERS]


# ---------------------------------------------------------------- CPU arm
# The CPU path (the oracle's compiled restatement of the reference's CPU
# assembly, add_jacobian_cpu, plus block ILU(k) and right-preconditioned
# GMRES in FP64) runs one problem per process on a pool of single-threaded
# workers (spawned, so no worker inherits a CUDA context): independent
# problems are the CPU's natural parallelism, as they are the GPU batch's.
_CPU = {}


def _cpu_init(root, nprob):
    sys.path.insert(0, root)
    from gpu_fem_b200 import mesh as M
    _CPU["meshes"] = M.batch_config4(nprob)


def _cpu_solve(task):
    """One problem: pattern, assembly + BCs, ILU(k), GMRES to 1e-8 (1 thread)."""
    import numpy as np

    from oracle import pyoracle as po
    i, fill, order = task
    m = _CPU["meshes"][i]
    if order == "rcm":
        rowp0, cols0 = po.bsr_pattern(m.conn, m.num_nodes)
        perm = po.rcm(rowp0, cols0, 0, 1)
    else:
        perm = np.arange(m.num_nodes, dtype=np.int32)
    t0 = time.perf_counter()
    st, x, it, rel, ph = po.solve_problem(m, perm, fill, restart=100, rtol=1e-8, maxit=20000,
                                          nthreads=1)
    # the timed CPU solve is assembly + factorization + GMRES; pattern, RCM
    # and symbolic ILU are set-up kept between steps on both paths
    return i, time.perf_counter() - t0 - ph[0], st, it, rel


def cpu_groups(meshes, ngroups):
    """Problems by size rank, dealt into ngroups groups (every ngroups-th),
    so each group spans the whole size distribution."""
    order = sorted(range(len(meshes)), key=lambda i: meshes[i].num_elements)
    return [order[g::ngroups] for g in range(ngroups)]


class CpuPool:
    def __init__(self, nprob, cores=None):
        import multiprocessing as mp
        self.cores = cores or os.cpu_count() or 1
        self.pool = mp.get_context("spawn").Pool(self.cores, initializer=_cpu_init,
                                                 initargs=(ROOT, nprob))

    def run(self, idx, fills, orders, meshes):
        """Solve the problems idx, largest first; (wall s, sum of per-problem s)."""
        tasks = sorted(((i, fills[i], orders[i]) for i in idx),
                       key=lambda t: -meshes[t[0]].num_elements)
        t0 = time.perf_counter()
        out = list(self.pool.imap_unordered(_cpu_solve, tasks))
        wall = time.perf_counter() - t0
        bad = [o for o in out if o[2] != 0]
        if bad:
            raise RuntimeError(f"CPU solves did not converge: {bad[:3]}")
        return wall, sum(o[1] for o in out)

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_measure(meshes, fills, orders, groups, pool):
    n = sum(len(g) for g in groups)
    wall = ssum = 0.0
    for g in groups:
        w, t = pool.run(g, fills, orders, meshes)
        wall += w
        ssum += t
    # all_core: measured solves / wall time of the pool; single_thread: solves
    # / summed per-problem times (each worker runs one problem on one core);
    # ideal_packing: cores x single_thread, the pool's rate if no worker ever
    # waited for the largest problem of a step
    return {"all_core": n / wall, "single_thread": n / ssum, "ideal_packing": pool.cores * n / ssum,
            "n": n, "wall_s": wall, "cores": pool.cores}


def run_reference(args):
    from gpu_fem_b200 import mesh as M
    ws, rank, _ = _dist()
    if rank != 0:
        return
    meshes = M.batch_config4(args.problems)
    fills, orders = table_or_none(len(meshes))
    if fills is None:
        print(json.dumps({"impl": "reference", "unavailable": "no fill/ordering table for "
                          "this problem count (run bench.py --tune on a GPU)"}), flush=True)
        return
    quarters = cpu_groups(meshes, 4)
    everything = list(range(len(meshes)))
    pool = CpuPool(len(meshes))
    try:
        # warm-up steps: a quarter of the batch each (every 4th by size)
        for s in range(args.warmup):
            pool.run(quarters[s % 4], fills, orders, meshes)
        per = [cpu_measure(meshes, fills, orders, [everything], pool) for _ in range(args.steps)]
    finally:
        pool.close()
    n = sum(p["n"] for p in per)
    wall = sum(p["wall_s"] for p in per)
    value = n / wall
    single = n / sum(p["n"] / p["single_thread"] for p in per)
    sample = (f"every step the whole 64-problem batch, largest first on {pool.cores} "
              f"single-threaded worker processes; each problem: assembly + BCs, ILU(k), "
              f"right-preconditioned GMRES to 1e-8 with the GPU path's fill and ordering; "
              f"value = solves / wall time")
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded meshes)", "impl": "reference",
            "config": bench_config(meshes, fills, orders, ws),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": pool.cores,
                             "kind": "port", "sample": sample,
                             "single_thread": {"value": single, "unit": "solves/s", "cores": 1},
                             "ideal_packing": {"value": single * pool.cores, "unit": "solves/s",
                                               "note": "cores x single-thread rate"}},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def plain_fp64_run(bs):
    """The plain FP64 GPU path: each problem alone through the single-problem
    entry points (gf_add_jacobian with fused BCs, gf_precond_factor with FP64
    factors, gf_gmres_solve), one after another on one stream. Returns ms for
    all problems (one warm-up pass first)."""
    import torch

    from gpu_fem_b200.assembler import gmres_solve
    from gpu_fem_b200.batch import solve_opts
    opts = solve_opts(bs.rtol, False, bs.restart)

    def one_pass():
        for a, k, p, b, x in zip(bs.asms, bs.mats, bs.P64, bs.bs, bs.xs):
            a.add_jacobian(None, k, fuse_bcs=True)
            p.factor(k)
            x.zero_()
            st, stats = gmres_solve(a, k, p, b, x, opts)
            if stats["rel_residual"] > bs.rtol:
                raise RuntimeError(f"plain FP64 solve did not converge: {stats}")

    one_pass()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    one_pass()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def main():
    args = _args()
    if args.sweep_case:
        return sweep_case(args.sweep_case)
    if args.assembly_case:
        return assembly_case()
    if args.impl == "reference":
        return run_reference(args)
    import numpy as np
    import torch

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from gpu_fem_b200 import _lib as L
    from gpu_fem_b200 import mesh as M
    from gpu_fem_b200.batch import BatchSolver

    meshes = M.batch_config4(args.problems)
    fills, orders = table_or_none(len(meshes))
    t0 = time.perf_counter()
    if fills is None or args.tune:
        bs = BatchSolver(meshes, tune=True)
    else:
        bs = BatchSolver(meshes, ordering=orders, fill=fills, tune=False)
    setup_s = time.perf_counter() - t0

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    timed_phases = []

    def timed(mixed, host_io=None, sweep_timing=False):
        import ctypes as C
        for _ in range(args.warmup):
            bs.step(mixed, host_io)
        barrier()
        if sweep_timing:
            L.check(L.lib().gf_timing_enable(1), "timing")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        c0 = L.lib().gf_launch_count()
        torch.cuda.nvtx.range_push("timed")
        ev[0].record()
        its = []
        phase_ms = [0.0, 0.0, 0.0]
        for k in range(args.steps):
            pe = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            stats = bs.step(mixed, host_io, phases=pe)
            ev[k + 1].record()
            its.append(max(s["iterations"] for s in stats))
            timed_phases.append(pe)
        torch.cuda.synchronize()
        for pe in timed_phases:
            for q in range(3):
                phase_ms[q] += pe[q].elapsed_time(pe[q + 1]) / args.steps
        timed_phases.clear()
        timed.phases = phase_ms
        barrier()
        torch.cuda.nvtx.range_pop()
        timed.launches = L.lib().gf_launch_count() - c0
        if sweep_timing:
            sm, sl, sb = C.c_double(), C.c_longlong(), C.c_double()
            L.check(L.lib().gf_timing_read(C.byref(sm), C.byref(sl), C.byref(sb)), "timing")
            L.check(L.lib().gf_timing_enable(0), "timing")
            timed.sweep = (sm.value, sl.value, sb.value)
        lat = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
        ms = job_ms(ev[0].elapsed_time(ev[-1]) / args.steps, ws, "cuda")
        timed.iters = its
        return ms, lat

    clocks = ClockSampler(local)
    clocks.start()
    ms_mixed, lat_mixed = timed(True, sweep_timing=True)
    launches = timed.launches
    sweep_ms, sweep_launches, sweep_bytes = timed.sweep
    phases_mixed = timed.phases
    its_mixed = timed.iters
    clk = clocks.stop()
    ms_fp64, lat_fp64 = timed(False)
    its_fp64 = timed.iters
    # end to end through the public API with host buffers
    host_b = [torch.tensor(m.loads).pin_memory() for m in meshes]
    host_x = [torch.empty(m.num_dof, dtype=torch.float64).pin_memory() for m in meshes]
    ms_e2e, _ = timed(True, (host_b, host_x))
    h2d = sum(8 * m.num_dof for m in meshes)
    nprob = len(meshes)
    value = job_throughput(nprob, ws, ms_mixed)
    # per-solve displacement difference of the mixed path (FP32 factors)
    # against the FP64 path, on the same problems
    bs.step(True)
    x_mixed = [x.cpu().numpy().copy() for x in bs.xs]
    bs.step(False)
    errs = [float(np.linalg.norm(a - x.cpu().numpy()) / np.linalg.norm(x.cpu().numpy()))
            for a, x in zip(x_mixed, bs.xs)]
    # the plain FP64 GPU path: one problem at a time (not batched)
    ms_plain = None if args.no_plain else job_ms(plain_fp64_run(bs), ws, "cuda")

    # roofline of the dominant kernel, the block triangular sweeps
    # (bsweep_tma), from CUDA events around every sweep pair inside the timed
    # mixed-precision region and the algorithmic bytes the sweeps report
    peak, peak_kind = _peaks()
    sweep_s = sweep_ms / 1e3
    achieved = sweep_bytes / sweep_s / 1e9 if sweep_s > 0 else 0.0
    orders_used = bs.orderings
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 assembly, SpMV and GMRES; f32 ILU factor values",
        "data": "synthetic (seeded meshes)",
        "config": bench_config(meshes, bs.fills, orders_used, ws),
        "setup_s": round(setup_s, 2),
        "gmres_steps_max": {"mixed": its_mixed, "fp64": its_fp64},
        "latency_ms": {"p50": float(np.percentile(lat_mixed, 50)),
                       "p99": float(np.percentile(lat_mixed, 99)),
                       "note": "all 64 requests of a step complete together"},
        "fp64_gpu": {"value": job_throughput(nprob, ws, ms_fp64), "unit": "solves/s",
                     "ms_per_step": ms_fp64, "note": "the same batch with FP64 factors",
                     "latency_ms": {"p50": float(np.percentile(lat_fp64, 50)),
                                    "p99": float(np.percentile(lat_fp64, 99))}},
        "mixed_over_fp64": ms_fp64 / ms_mixed,
        "mixed_vs_fp64_error": {"max": max(errs), "median": float(np.median(errs)),
                                "per_solve": [float(f"{e:.3g}") for e in errs],
                                "note": "||x_mixed - x_fp64|| / ||x_fp64|| per problem"},
        "phase_ms": {"assemble": phases_mixed[0], "factor": phases_mixed[1],
                     "solve": phases_mixed[2]},
        "e2e": {"value": job_throughput(nprob, ws, ms_e2e), "unit": "solves/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
        "roofline": {"kernel": "bsweep_tma (block L and U sweeps, FP32 factor values)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": SWEEP_TRAFFIC_RATIO * sweep_bytes / max(sweep_launches, 1),
                     "traffic_note": "DRAM read+write per launch: ncu ratio traffic/algorithmic "
                                     "bytes of the 256x128 ILU(6) sweep case x this run's "
                                     "algorithmic bytes per launch",
                     "launches": sweep_launches,
                     "ms_per_launch": sweep_ms / max(sweep_launches, 1),
                     "algorithmic_bytes_per_launch": sweep_bytes / max(sweep_launches, 1),
                     "share_of_step": sweep_ms / (ms_mixed * args.steps)},
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    if ms_plain is not None:
        line["plain_fp64_gpu"] = {
            "value": job_throughput(nprob, ws, ms_plain), "unit": "solves/s",
            "ms_per_step": ms_plain,
            "note": "each problem alone: gf_add_jacobian + gf_precond_factor (FP64 factors) + "
                    "gf_gmres_solve, one after another"}
        line["mixed_batched_over_plain_fp64"] = ms_plain / ms_mixed
    if fills is None or args.tune:
        line["tuned_table"] = {"fills": [int(k) for k in bs.fills],
                               "orders": "".join(o[0] for o in bs.orderings)}
        if args.tune_log:
            with open(args.tune_log, "w") as f:
                json.dump([[str(x) for x in e] for e in (bs.tune_log or [])], f)
    if args.serve_seconds > 0:
        line["serving"] = serving_run(args.serve_seconds)
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        pool = CpuPool(len(meshes))
        try:
            cb = cpu_measure(meshes, bs.fills, bs.orderings, [list(range(len(meshes)))], pool)
        finally:
            pool.close()
        line["cpu_baseline"] = {
            "value": cb["all_core"], "unit": "solves/s", "cores": cb["cores"], "kind": "port",
            "sample": f"the whole 64-problem batch once, largest first on {cb['cores']} "
                      f"single-threaded worker processes with the GPU's fill and ordering "
                      f"({cb['wall_s']:.1f} s)",
            "single_thread": {"value": cb["single_thread"], "unit": "solves/s", "cores": 1},
            "ideal_packing": {"value": cb["ideal_packing"], "unit": "solves/s",
                              "note": "cores x single-thread rate"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
