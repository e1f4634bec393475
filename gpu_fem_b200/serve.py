"""Continuous-batching shell-solve server.

Requests (a plate or a stiffened box, a size class, a per-request thickness
field and load, all generated from the request seed) arrive as a Poisson
stream. The server keeps, per size class, one device-resident assembler
(mesh, node ordering, BSR pattern, coloured scatter schedule) and slot
groups reserved before the stream starts: groups of 8, 4, 2 and 1 slots
(BSR matrix, ILU(k) symbolic + factor streams, load / displacement /
thickness vectors) with a persistent batch handle and solver workspace
each, as many as the class's share of the HBM budget holds (measured).
Nothing is allocated while requests stream in. A request is admitted when a
reserved group of its class is free; the dispatcher fills the best-fitting
free group with the class's queued requests and a worker thread runs it on
its own CUDA stream with the batched engine (gf_batch_*), so requests that
arrive while others are on the device start as soon as a group frees up,
and batches overlap on the device. Latency = completion - arrival.

Each request is solved with its own per-problem GMRES state and reductions,
so its result does not depend on what else is in the batch (tested).
Precision: FP32 ILU(k) factors inside FP64 GMRES; the fill level is tuned
per size class at the thinnest thickness a request can carry.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from . import mesh as M
from .assembler import BsrMat, ILUk_Preconditioner, _stream
from .batch import Batch, BatchSolver, choose_ordering, solve_opts

import ctypes as C


def size_classes(n=16, lo=5e3, hi=2e6):
    return [lo * (hi / lo) ** (k / (n - 1)) for k in range(n)]


def class_mesh(family, dof):
    """Base mesh of a size class (thickness and load are per request)."""
    if family == "plate":
        ne = max(4, int(round(math.sqrt(dof / 6.0))) - 1)
        return M.plate(ne, ne, 1.0, 1.0, lambda x, y: 0.005 + 0 * x, "all_edges",
                       lambda q: 1e3 + 0 * q[:, 0], name=f"plate_{ne}x{ne}")
    s = max(2, int(round(math.sqrt(dof / 444.0))))
    return M.box(nx=9 * s, ny=2 * s, nz=max(1, s), nribs=10)


# thinnest element a request can carry: t0 >= 2 mm scaled by (1 - 0.25)
T_MIN = 0.0015


def tune_class_fill(mesh, ordering, rtol=1e-8, margin=2):
    """ILU fill level of a size class: the autotuner's choice for the class
    mesh alone at the thinnest thickness any request of the class can carry
    (the hardest case for block ILU on shells), plus a margin where the
    factor's rows still fit the triangular sweep, so every request
    converges."""
    import dataclasses
    m = dataclasses.replace(mesh, thick=np.full(mesh.num_elements, T_MIN))
    bs = BatchSolver([m], ordering=ordering, tune=True, rtol=rtol, build=False,
                     objective="problem")
    k = bs.fills[0]
    if k >= L.GF_FILL_FULL:
        return k
    return fit_fill(bs.asms[0], k + margin, "fp32")


@dataclass
class Request:
    rid: int
    arrival: float
    family: str
    cls: int
    seed: int
    t0: float = 0.0
    done: float = 0.0
    rel: float = float("nan")
    iters: int = 0
    status: int = -1


def poisson_requests(rate, duration, seed=99, nclasses=16, families=("plate", "box"),
                     max_class=None):
    g = M.MT19937_64(seed)
    reqs, t, rid = [], 0.0, 0
    classes = size_classes(nclasses)
    # sizes log-uniform over 5e3..2e6 DOF, or up to the largest allowed class
    lo = math.log(5e3)
    hi = math.log(2e6 if max_class is None else classes[max_class])
    while True:
        u = g.uniform(4)
        t += -math.log(max(u[0], 1e-300)) / rate
        if t > duration:
            break
        fam = families[int(u[1] * len(families)) % len(families)]
        dof = math.exp(lo + u[2] * (hi - lo))
        cls = int(np.argmin([abs(math.log(dof / c)) for c in classes]))
        reqs.append(Request(rid, t, fam, cls, int(u[3] * 2 ** 31)))
        rid += 1
    return reqs


class Group:
    """A fixed set of slots of one size class with a persistent batch handle:
    a dispatch fills up to len(slots) requests into it; slots it leaves empty
    get a zero load and drop out of the solve at its first residual check."""

    def __init__(self, cls, size, scatter="tune"):
        self.cls = cls
        self.slots = [cls.make_slot() for _ in range(size)]
        self.batch = Batch([cls.asm] * size, [s["K"] for s in self.slots],
                           [s["P"] for s in self.slots])
        n = size
        self.thick_ptrs = (C.c_void_p * n)(*[s["thick"].data_ptr() for s in self.slots])
        # assembly scatter: timed per group ("tune"), or fixed
        if scatter == "tune":
            self.atomic = self.tune_scatter()
        else:
            self.atomic = scatter == "atomic"
            self.batch.set_scatter(self.atomic)

    def tune_scatter(self, reps=3):
        """Times this group's assembly with the coloured scatter (one launch
        per colour) and the atomic one (one launch, FP64 atomics) and keeps
        the faster: atomics pay where the colours' launches dominate."""
        def timed():
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            L.check(L.lib().gf_batch_assemble_ex(self.batch.h, self.thick_ptrs, _stream()),
                    "assemble")
            e0.record()
            for _ in range(reps):
                L.check(L.lib().gf_batch_assemble_ex(self.batch.h, self.thick_ptrs, _stream()),
                        "assemble")
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1)
        self.batch.set_scatter(False)
        t_col = timed()
        self.batch.set_scatter(True)
        t_atom = timed()
        atomic = t_atom < t_col
        self.batch.set_scatter(atomic)
        return atomic

    def run(self, reqs, server):
        """Assemble, factor and solve the group with `reqs` in its first slots."""
        cls = self.cls
        for k, slot in enumerate(self.slots):
            if k < len(reqs):
                thick, loads = cls.request_data(reqs[k].seed)
                slot["thick"].copy_(torch.from_numpy(thick), non_blocking=False)
                slot["b"].copy_(torch.from_numpy(loads), non_blocking=False)
            else:
                slot["b"].zero_()
            slot["x"].zero_()
        L.check(L.lib().gf_batch_assemble_ex(self.batch.h, self.thick_ptrs, _stream()),
                "assemble")
        self.batch.factor()
        st, stats = self.batch.solve([s["b"] for s in self.slots], [s["x"] for s in self.slots],
                                     solve_opts(server.rtol, False, server.restart,
                                                server.max_iters))
        torch.cuda.current_stream().synchronize()
        return stats[:len(reqs)]


def fit_fill(asm, fill, precision):
    """The highest fill level <= `fill` whose factor rows fit the triangular
    sweep's shared-memory stage for factors of `precision` (FP64 factor rows
    take twice the bytes of FP32 ones, so a fill tuned with FP32 factors may
    not fit with FP64 factors)."""
    if fill >= L.GF_FILL_FULL:
        return fill
    k = fill
    while k > 0:
        try:
            ILUk_Preconditioner(asm, k, precision)
            return k
        except L.GpuFemError as e:
            if e.status != L.GF_INVALID_ARG:
                raise
            k -= 1
    return 0


class SizeClass:
    """Device-resident mesh, ordering, pattern and scatter schedule of one size
    class, with slot groups reserved at warm-up (nothing is allocated while
    requests stream in)."""

    def __init__(self, family, k, dof, fill=None, rtol=1e-8, precision="fp32"):
        self.family, self.k = family, k
        self.mesh = class_mesh(family, dof)
        self.ordering, self.asm = choose_ordering(self.mesh)
        fill = fill if fill is not None else tune_class_fill(self.mesh, self.ordering, rtol)
        self.fill = fit_fill(self.asm, fill, precision)
        self.precision = precision
        self.groups = []       # reserved
        self.free = []         # groups not running
        self.lock = threading.Lock()
        self.reserved_bytes = 0

    def make_slot(self):
        K = BsrMat(self.asm)
        P = ILUk_Preconditioner(self.asm, self.fill, self.precision)
        n = self.mesh.num_dof
        return {"K": K, "P": P, "b": torch.zeros(n, dtype=torch.float64, device="cuda"),
                "x": torch.zeros(n, dtype=torch.float64, device="cuda"),
                "thick": torch.tensor(self.mesh.thick, dtype=torch.float64, device="cuda")}

    def reserve(self, sizes, budget_bytes, server):
        """Builds slot groups of the given sizes (largest first) while the
        device memory they take (measured) stays within budget_bytes; each
        group is run once with zero loads so its solver workspace exists
        before the stream starts. Returns the bytes reserved."""
        for size in sorted(sizes, reverse=True):
            torch.cuda.synchronize()
            before = torch.cuda.mem_get_info()[0]
            g = Group(self, size, server.scatter)
            g.run([], server)
            used = before - torch.cuda.mem_get_info()[0]
            if self.groups and self.reserved_bytes + used > budget_bytes:
                del g  # over this class's share: released again
                continue
            self.reserved_bytes += used
            self.groups.append(g)
            self.free.append(g)
        return self.reserved_bytes

    def take_group(self, pending):
        """The free group that best fits `pending` requests: the smallest one
        that holds them all, else the largest free one; None if none is free."""
        with self.lock:
            if not self.free:
                return None
            fits = [g for g in self.free if len(g.slots) >= pending]
            g = (min(fits, key=lambda x: len(x.slots)) if fits
                 else max(self.free, key=lambda x: len(x.slots)))
            self.free.remove(g)
            return g

    def give_back(self, g):
        with self.lock:
            self.free.append(g)

    def request_data(self, seed):
        """Thickness field and load vector of a request (from its seed)."""
        r = M.MT19937_64(seed).uniform(5)
        m = self.mesh
        cen = m.xpts[m.conn].mean(axis=1)
        t0 = 0.002 + 0.006 * r[0]
        amp = 0.25 * r[1]
        thick = t0 * (1 + amp * np.sin(2 * np.pi * (1 + r[2]) * cen[:, 0]) *
                      np.cos(np.pi * cen[:, 1]))
        loads = m.loads * (0.5 + 1.5 * r[3])
        return thick, loads


class Server:
    """Continuous batching over reserved slot groups. Admission: a request
    waits in its class's queue until a reserved group of the class is free;
    the dispatcher then moves up to the group's size of queued requests into
    it and hands it to a worker thread, which runs it on its own CUDA stream,
    so batches of different classes (and several of one class) overlap on
    the device while new requests keep arriving."""

    GROUP_SIZES = (8, 4, 2, 1)

    def __init__(self, budget_gb=120.0, streams=4, max_batch=8, classes=None, restart=100,
                 rtol=1e-8, fills=None, max_iters=3000, precision="fp32", scatter="tune"):
        self.budget = budget_gb * 1e9
        # assembly scatter of the slot groups: "tune" (each group times the
        # coloured and the atomic scatter and keeps the faster), "coloured"
        # (bitwise reproducible) or "atomic"
        self.scatter = scatter
        self.max_batch = max_batch
        self.restart, self.rtol, self.max_iters = restart, rtol, max_iters
        self.precision = precision  # ILU factor values: "fp32" (mixed) or "fp64"
        self.classes = {}
        self.streams = [torch.cuda.Stream() for _ in range(streams)]
        self.work = queue.Queue()
        self.completed = []
        self.done_lock = threading.Lock()
        self.errors = []
        self.fills = fills or {}
        self.keep_results = False
        self.results = {}
        self.reserved_bytes = 0

    def get_class(self, family, k):
        key = (family, k)
        if key not in self.classes:
            dof = size_classes()[k]
            self.classes[key] = SizeClass(family, k, dof, self.fills.get(key), self.rtol,
                                          self.precision)
            self.fills[key] = self.classes[key].fill
        return self.classes[key]

    def warm(self, keys):
        """Builds the size classes and reserves their slot groups (sizes up to
        max_batch), the HBM budget shared equally by the classes."""
        keys = sorted(keys)
        share = self.budget / max(len(keys), 1)
        sizes = [s for s in self.GROUP_SIZES if s <= self.max_batch]
        for fam, k in keys:
            c = self.get_class(fam, k)
            if not c.groups:
                self.reserved_bytes += c.reserve(sizes, share, self)
        torch.cuda.synchronize()

    def _worker(self, stream):
        while True:
            item = self.work.get()
            if item is None:
                break
            group, reqs = item
            try:
                with torch.cuda.stream(stream):
                    stats = group.run(reqs, self)
                now = time.perf_counter()
                for req, s in zip(reqs, stats):
                    req.done = now
                    req.rel = s["rel_residual"]
                    req.iters = s["iterations"]
                    req.status = s["status"]
                if self.keep_results:
                    for req, slot in zip(reqs, group.slots):
                        self.results[req.rid] = slot["x"].cpu().numpy().copy()
            except Exception as e:  # keep serving; record the failure
                self.errors.append(repr(e))
                for req in reqs:
                    req.status = -2
                    req.done = time.perf_counter()
            finally:
                group.cls.give_back(group)
                with self.done_lock:
                    self.completed += reqs

    def solve_alone(self, req):
        """Solve one request by itself (a group of one built for it) and return x."""
        cls = self.get_class(req.family, req.cls)
        g = Group(cls, 1, self.scatter)
        g.run([req], self)
        torch.cuda.synchronize()
        return g.slots[0]["x"].cpu().numpy().copy()

    def run(self, requests, time_scale=1.0):
        """Serve a request stream in real time; returns per-request records."""
        missing = {(r.family, r.cls) for r in requests} - set(self.classes)
        if missing:
            raise ValueError(f"size classes not warmed: {sorted(missing)}")
        threads = [threading.Thread(target=self._worker, args=(s,), daemon=True)
                   for s in self.streams]
        for t in threads:
            t.start()
        queues = {key: [] for key in self.classes}
        i = 0
        t_start = time.perf_counter()
        nreq = len(requests)
        while True:
            now = time.perf_counter() - t_start
            while i < nreq and requests[i].arrival * time_scale <= now:
                requests[i].t0 = t_start + requests[i].arrival * time_scale
                queues[(requests[i].family, requests[i].cls)].append(requests[i])
                i += 1
            dispatched = False
            for key, q in queues.items():
                while q:
                    g = self.classes[key].take_group(len(q))
                    if g is None:
                        break
                    take, q[:] = q[:len(g.slots)], q[len(g.slots):]
                    self.work.put((g, take))
                    dispatched = True
            with self.done_lock:
                ndone = len(self.completed)
            if i >= nreq and ndone >= nreq:
                break
            if not dispatched:
                time.sleep(0.001)
        for _ in threads:
            self.work.put(None)
        for t in threads:
            t.join()
        t_end = time.perf_counter()
        lat = [(r.done - r.t0) * 1e3 for r in requests]
        ok = [r for r in requests if r.status == L.GF_OK]
        return {"requests": nreq, "solved": len(ok), "wall_s": t_end - t_start,
                "solves_per_s": len(ok) / (t_end - t_start),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "reserved_gb": self.reserved_bytes / 1e9, "errors": self.errors[:3]}
