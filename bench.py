#!/usr/bin/env python
"""Shell solves/sec (p50/p99 latency), mixed precision vs FP64 on the GPU.

Workload: 64 independent clamped plates, element grids log-uniform 16^2 ..
256^2 with aspect 1..4 (seed 4321), t ~ U(2, 8) mm, p ~ U(0.5, 2) kPa,
E = 70 GPa, nu = 0.3. A step assembles the 6x6-block BSR Jacobian (fused
BCs), factors the block ILU(k) preconditioner (k autotuned per problem) and
solves every problem to ||b - A x|| / ||b|| <= 1e-8 with FP32 ILU + FP32
SpMV inside FP64 GMRES / iterative refinement. `value` is whole-job solves/s
with inputs resident in HBM; `e2e` repeats the step through the public API
with the load vectors copied from pinned host memory and the displacements
copied back inside the timed region. The FP64 GPU path is timed beside it.

--impl reference times the CPU oracle (a restatement of the reference's CPU
assembly plus FP64 ILU-GMRES) on a bounded sample of the same problems.

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
    ap.add_argument("--serve-seconds", type=float, default=0.0,
                    help="length of the Poisson request stream of the serving run (0 skips it)")
    ap.add_argument("--assembly-case", action="store_true",
                    help="small profiling case: Jacobian assembly (fused BCs) of the 400x200 "
                         "jittered cantilever plate, 5 times (no JSON line)")
    ap.add_argument("--sweep-case", action="store_true",
                    help="small profiling case: the triangular sweeps of one 256x128 plate, "
                         "natural ordering, ILU(6), FP32 factors, applied 5 times (no JSON line)")
    return ap.parse_args()


SERVE_RATE, SERVE_MAX_CLASS = 20.0, 6


def serving_run(seconds):
    """Continuous-batching server on a Poisson stream of plate and box
    requests (rate 20/s, size classes 5e3..5.5e4 DOF, per-request thickness
    field and load from the request seed), once with FP32 ILU factors
    (mixed) and once with FP64 factors, each to a 1e-8 relative residual.
    Size classes are built and their fill tuned before the stream starts."""
    from gpu_fem_b200 import serve
    out, fills, n = {}, None, 0
    for prec, name in (("fp32", "mixed"), ("fp64", "fp64")):
        reqs = serve.poisson_requests(rate=SERVE_RATE, duration=seconds, seed=99,
                                      max_class=SERVE_MAX_CLASS)
        n = len(reqs)
        srv = serve.Server(budget_gb=40.0, streams=4, max_batch=16, precision=prec, fills=fills)
        srv.warm({(r.family, r.cls) for r in reqs})
        fills = dict(srv.fills)
        res = srv.run(reqs)
        out[name] = {k: res[k] for k in ("requests", "solved", "solves_per_s", "p50_ms", "p99_ms",
                                          "wall_s")}
    out["stream"] = (f"Poisson {SERVE_RATE:g} req/s for {seconds:g} s, {n} requests, plates and "
                     f"stiffened boxes, size classes 0..{SERVE_MAX_CLASS} (5e3..5.5e4 DOF); "
                     f"latency = completion - arrival")
    return out


def assembly_case():
    """Jacobian assembly with fused BCs of the 400x200 plate (80,601 nodes,
    ~209 MB of block values, above L2), 5 times: the small case on which the
    assembly kernel is profiled."""
    import torch
    from gpu_fem_b200 import mesh as M
    from gpu_fem_b200.assembler import ElementAssembler, createBsrMat
    m = M.plate_config2()
    A = ElementAssembler.from_mesh(m, ordering="rcm")
    K = createBsrMat(A)
    res = A.createVarsVec()
    for _ in range(5):
        A.add_jacobian(res, K, fuse_bcs=True)
    torch.cuda.synchronize()
    print("assembly case", A.get_nnzb())


def sweep_case():
    """One preconditioner (256x128 clamped plate, t = 2 mm, natural ordering,
    ILU(6), FP32 factors, ~150 MB of factor) applied 5 times: the small case
    on which the sweep and factorization kernels are profiled (its levels
    are large enough that both run on a two-CTA cluster)."""
    import torch
    from gpu_fem_b200 import mesh as M
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner, createBsrMat
    m = M.plate(256, 128, 1.0, 0.5, lambda x, y: 0.002 + 0 * x, "all_edges",
                lambda q: 1e3 + 0 * q[:, 0])
    A = ElementAssembler.from_mesh(m, ordering="natural")
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    P = ILUk_Preconditioner(A, fill_level=6, precision="fp32")
    P.factor(K)
    r = torch.randn(m.num_dof, dtype=torch.float64, device="cuda")
    z = torch.zeros_like(r)
    for _ in range(5):
        P.apply(r, z)
    torch.cuda.synchronize()
    print("sweep case", P.info(), float(z.abs().max()))


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


def systematic_sample(meshes, offset, k=4):
    """Indices of k problems spread evenly over the size ranking (ranks
    offset, offset + n/k, ...): solves/s over such a sample estimates the
    whole batch's solves/s without running every large problem on the CPU."""
    order = sorted(range(len(meshes)), key=lambda i: meshes[i].num_elements)
    stride = max(len(order) // k, 1)
    return [order[(offset % stride) + j * stride] for j in range(k) if (offset % stride) + j * stride < len(order)]


def cpu_ordering(mesh, fill=8):
    """The GPU path's ordering rule on the oracle: natural or RCM, whichever
    gives fewer ILU(fill) levels x blocks per row."""
    import numpy as np

    from oracle import pyoracle as po
    rowp0, cols0 = po.bsr_pattern(mesh.conn, mesh.num_nodes)
    best = None
    for name, perm in (("natural", np.arange(mesh.num_nodes, dtype=np.int32)),
                       ("rcm", po.rcm(rowp0, cols0, 0, 1))):
        rowp, cols = po.permute_pattern(rowp0, cols0, perm)
        rk, ck = po.iluk_pattern(rowp, cols, fill)
        nl, _ = po.levels(rk, ck, True)
        nu, _ = po.levels(rk, ck, False)
        score = (nl + nu) * len(ck) / mesh.num_nodes
        if best is None or score < best[0]:
            best = (score, name)
    return best[1]


def cpu_baseline_run(problems, fills, budget_s=25.0, threads=None, orders=None):
    """Oracle (restated reference CPU path): assembly (OpenMP over elements),
    FP64 block ILU(k), right-preconditioned GMRES, in the same ordering and
    fill as the GPU path; on as many of the given problems as fit in about
    budget_s. Returns (solves/s, n, seconds, cores)."""
    import numpy as np

    from oracle import pyoracle as po
    threads = threads or os.cpu_count() or 1
    orders = orders or ["rcm"] * len(problems)
    t_total, n = 0.0, 0
    for m, k, o in zip(problems, fills, orders):
        t0 = time.perf_counter()
        rowp0, cols0 = po.bsr_pattern(m.conn, m.num_nodes)
        perm = (po.rcm(rowp0, cols0, 0, 1) if o == "rcm"
                else np.arange(m.num_nodes, dtype=np.int32))
        rowp, cols, A, _, perm = po.assemble_jacobian(m, perm=perm, nthreads=threads)
        po.apply_bcs_mat(rowp, cols, A, perm, m.bcs)
        b = np.zeros(6 * m.num_nodes)
        b.reshape(-1, 6)[perm] = m.loads.reshape(-1, 6)
        if k:
            rk, ck = po.iluk_pattern(rowp, cols, k)
            Ak = po.scatter_to_pattern(rowp, cols, A, rk, ck)
        else:
            rk, ck, Ak = rowp, cols, A
        st, LU = po.ilu0(rk, ck, Ak)
        # right preconditioning with the ILU(k) factors over A's pattern
        st2, x, its, rel = _oracle_gmres_right(po, rowp, cols, A, rk, ck, LU, b)
        dt = time.perf_counter() - t0
        t_total += dt
        n += 1
        if t_total >= budget_s:
            break
    return n / t_total, n, t_total, threads


def _oracle_gmres_right(po, rowp, cols, A, rk, ck, LU, b, m=200, rtol=1e-8, maxit=5000):
    """FP64 right-preconditioned GMRES(m) on the oracle kernels (numpy
    Arnoldi, C SpMV and ILU apply)."""
    import numpy as np
    x = np.zeros_like(b)
    bn = np.linalg.norm(b)
    r = b - po.spmv(rowp, cols, A, x)
    rel = np.linalg.norm(r) / bn
    it = 0
    while rel > rtol and it < maxit:
        beta = np.linalg.norm(r)
        V = [r / beta]
        H = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        g[0] = beta
        cs, ss = np.zeros(m), np.zeros(m)
        j = 0
        for j in range(m):
            w = po.spmv(rowp, cols, A, po.ilu0_apply(rk, ck, LU, V[j]))
            for i in range(j + 1):
                H[i, j] = w @ V[i]
                w = w - H[i, j] * V[i]
            H[j + 1, j] = np.linalg.norm(w)
            V.append(w / H[j + 1, j])
            for i in range(j):
                a, c = H[i, j], H[i + 1, j]
                H[i, j], H[i + 1, j] = cs[i] * a + ss[i] * c, -ss[i] * a + cs[i] * c
            a, c = H[j, j], H[j + 1, j]
            h = np.hypot(a, c)
            cs[j], ss[j] = a / h, c / h
            H[j, j], H[j + 1, j] = cs[j] * a + ss[j] * c, 0.0
            g[j + 1], g[j] = -ss[j] * g[j], cs[j] * g[j]
            it += 1
            if abs(g[j + 1]) <= rtol * bn:
                break
        jj = j + 1
        y = np.linalg.solve(np.triu(H[:jj, :jj]), g[:jj])
        x += po.ilu0_apply(rk, ck, LU, sum(y[i] * V[i] for i in range(jj)))
        r = b - po.spmv(rowp, cols, A, x)
        rel = np.linalg.norm(r) / bn
    return (0 if rel <= rtol else 1), x, it, rel


def run_reference(args):
    from gpu_fem_b200 import mesh as M
    ws, rank, _ = _dist()
    if rank != 0:
        return
    probs = M.batch_config4(args.problems)
    vals = []
    for s in range(args.warmup + args.steps):
        idx = systematic_sample(probs, 2 + 5 * s)
        sample = [probs[i] for i in idx]
        v, n, sec, cores = cpu_baseline_run(sample, [_default_fill(p) for p in sample],
                                            budget_s=1e9,
                                            orders=[cpu_ordering(p) for p in sample])
        if s >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * n / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded meshes)", "impl": "reference",
            "config": {"workload": WORKLOAD,
                       "sample": "4 problems per step spread over the size ranking"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": "per step 4 of the 64 problems at size ranks o, o+16, "
                                       "o+32, o+48 (o varies by step); ILU(8), same "
                                       "ordering rule as the GPU path"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _default_fill(mesh):
    # offline sweep: thin, coarse plates need more fill (see DESIGN notes)
    return 8


def main():
    args = _args()
    if args.sweep_case:
        return sweep_case()
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
    t0 = time.perf_counter()
    bs = BatchSolver(meshes, tune=True)
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

    # roofline of the dominant kernel, the block triangular sweeps
    # (bsweep_tma), from CUDA events around every sweep pair inside the timed
    # mixed-precision region and the algorithmic bytes the sweeps report
    peak, peak_kind = _peaks()
    sweep_s = sweep_ms / 1e3
    achieved = sweep_bytes / sweep_s / 1e9 if sweep_s > 0 else 0.0

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 assembly, SpMV and GMRES; f32 ILU factor values", "data": "synthetic (seeded meshes)",
        "config": {"workload": WORKLOAD, "problems": nprob,
                   "dofs": int(sum(m.num_dof for m in meshes)),
                   "fill_levels": bs.fills,
                   "gmres_steps_max": {"mixed": its_mixed, "fp64": its_fp64},
                   "l2": "inputs larger than L2 (all 64 systems resident, ~GB)",
                   "setup_s": round(setup_s, 2), "parallelism": f"replicas x{ws}"},
        "latency_ms": {"p50": float(np.percentile(lat_mixed, 50)),
                       "p99": float(np.percentile(lat_mixed, 99)),
                       "note": "all 64 requests of a step complete together"},
        "fp64_gpu": {"value": job_throughput(nprob, ws, ms_fp64), "unit": "solves/s",
                     "ms_per_step": ms_fp64,
                     "latency_ms": {"p50": float(np.percentile(lat_fp64, 50)),
                                    "p99": float(np.percentile(lat_fp64, 99))}},
        "mixed_over_fp64": ms_fp64 / ms_mixed,
        "phase_ms": {"assemble": phases_mixed[0], "factor": phases_mixed[1],
                     "solve": phases_mixed[2]},
        "e2e": {"value": job_throughput(nprob, ws, ms_e2e), "unit": "solves/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
        "roofline": {"kernel": "bsweep_tma (block L and U sweeps, FP32 factor values)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "launches": sweep_launches,
                     "ms_per_launch": sweep_ms / max(sweep_launches, 1),
                     "algorithmic_bytes_per_launch": sweep_bytes / max(sweep_launches, 1),
                     "share_of_step": sweep_ms / (ms_mixed * args.steps)},
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    if args.serve_seconds > 0:
        line["serving"] = serving_run(args.serve_seconds)
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        idx = systematic_sample(meshes, 2)
        v, n_cpu, sec, cores = cpu_baseline_run([meshes[i] for i in idx],
                                                [bs.fills[i] for i in idx], budget_s=1e9,
                                                orders=[bs.orderings[i] for i in idx])
        line["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                                "sample": f"{n_cpu} of the 64 problems at size ranks 2, 18, 34, "
                                          f"50, same fill and ordering as the GPU ({sec:.1f} s)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
