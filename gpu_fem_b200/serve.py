"""Continuous-batching shell-solve server.

Requests (a plate or a stiffened box, a size class, a per-request thickness
field and load, all generated from the request seed) arrive as a Poisson
stream. The server keeps, per size class, one device-resident assembler
(mesh, node ordering, BSR pattern, coloured scatter schedule) and a pool of
slots (BSR matrix, ILU(k) symbolic + factors, load / displacement vectors).
A request is admitted when its slot memory fits the HBM budget; admitted
requests are batched and solved with the batched engine (gf_batch_*) on a
pool of CUDA streams served by worker threads, so requests that arrive
while others are on the device start as soon as a slot and a stream free
up, and their work overlaps on the device. Latency = completion - arrival.

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
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import mesh as M
from .assembler import BsrMat, ElementAssembler, ILUk_Preconditioner, _stream
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
    """ILU fill level of a size class: the batch autotuner's choice at the
    thinnest thickness any request of the class can carry (the hardest case
    for block ILU on shells), plus a margin, so every request converges."""
    import dataclasses
    m = dataclasses.replace(mesh, thick=np.full(mesh.num_elements, T_MIN))
    return BatchSolver([m], ordering=ordering, tune=True, rtol=rtol,
                       build=False).fills[0] + margin


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


class SizeClass:
    def __init__(self, family, k, dof, fill=None, rtol=1e-8, precision="fp32"):
        self.family, self.k = family, k
        self.mesh = class_mesh(family, dof)
        self.ordering, self.asm = choose_ordering(self.mesh)
        self.fill = fill if fill is not None else tune_class_fill(self.mesh, self.ordering, rtol)
        self.precision = precision
        self.free = []
        self.lock = threading.Lock()
        nn, ne = self.mesh.num_nodes, self.mesh.num_elements
        # per-slot footprint estimate: FP64+FP32 matrix, FP64+FP32 factors, vectors
        nnzb = self.asm.get_nnzb()
        self.slot_bytes = int(nnzb * 36 * 12 * (1 + 1.5 * (self.fill > 0)) * 2 + 6 * nn * 8 * 8 +
                              ne * 8)

    def make_slot(self):
        K = BsrMat(self.asm)
        P = ILUk_Preconditioner(self.asm, self.fill, self.precision)
        n = self.mesh.num_dof
        return {"K": K, "P": P, "b": torch.zeros(n, dtype=torch.float64, device="cuda"),
                "x": torch.zeros(n, dtype=torch.float64, device="cuda"),
                "thick": torch.zeros(self.mesh.num_elements, dtype=torch.float64, device="cuda")}

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
    def __init__(self, budget_gb=120.0, streams=4, max_batch=64, classes=None, restart=100,
                 rtol=1e-8, fills=None, max_iters=3000, precision="fp32"):
        self.budget = budget_gb * 1e9
        self.used = 0.0
        self.mem_lock = threading.Lock()
        self.max_batch = max_batch
        self.restart, self.rtol, self.max_iters = restart, rtol, max_iters
        self.precision = precision  # ILU factor values: "fp32" (mixed) or "fp64"
        self.classes = {}
        self.streams = [torch.cuda.Stream() for _ in range(streams)]
        self.work = queue.Queue()
        self.completed = []
        self.done_lock = threading.Lock()
        self.errors = []
        self.class_spec = classes or []
        self.fills = fills or {}
        self.keep_results = False
        self.results = {}

    def get_class(self, family, k):
        key = (family, k)
        if key not in self.classes:
            dof = size_classes()[k]
            self.classes[key] = SizeClass(family, k, dof, self.fills.get(key), self.rtol,
                                          self.precision)
            self.fills[key] = self.classes[key].fill
        return self.classes[key]

    def warm(self, keys, slots=1):
        for fam, k in keys:
            c = self.get_class(fam, k)
            for _ in range(slots):
                c.free.append(c.make_slot())
        torch.cuda.synchronize()

    def _worker(self, stream):
        while True:
            item = self.work.get()
            if item is None:
                break
            batch = item
            try:
                with torch.cuda.stream(stream):
                    self._run_batch(batch)
            except Exception as e:  # keep serving; record the failure
                self.errors.append(repr(e))
                for req, cls, slot in batch:
                    req.status = -2
                    req.done = time.perf_counter()
            finally:
                for req, cls, slot in batch:
                    with cls.lock:
                        cls.free.append(slot)
                    with self.mem_lock:
                        self.used -= cls.slot_bytes
                with self.done_lock:
                    self.completed += [r for r, _, _ in batch]

    def _run_batch(self, batch):
        asms = [cls.asm for _, cls, _ in batch]
        mats = [slot["K"] for _, _, slot in batch]
        pcs = [slot["P"] for _, _, slot in batch]
        for req, cls, slot in batch:
            thick, loads = cls.request_data(req.seed)
            slot["thick"].copy_(torch.from_numpy(thick), non_blocking=False)
            slot["b"].copy_(torch.from_numpy(loads), non_blocking=False)
            slot["x"].zero_()
        bt = Batch(asms, mats, pcs)
        n = len(batch)
        T = (C.c_void_p * n)(*[slot["thick"].data_ptr() for _, _, slot in batch])
        L.check(L.lib().gf_batch_assemble_ex(bt.h, T, _stream()), "assemble")
        bt.factor()
        st, stats = bt.solve([s["b"] for _, _, s in batch], [s["x"] for _, _, s in batch],
                             solve_opts(self.rtol, False, self.restart, self.max_iters))
        torch.cuda.current_stream().synchronize()
        now = time.perf_counter()
        for (req, _, slot), s in zip(batch, stats):
            req.done = now
            req.rel = s["rel_residual"]
            req.iters = s["iterations"]
            req.status = s["status"]
            if self.keep_results:
                self.results[req.rid] = slot["x"].cpu().numpy().copy()

    def solve_alone(self, req):
        """Solve one request by itself (batch of one) and return x."""
        cls = self.get_class(req.family, req.cls)
        slot = cls.make_slot()
        self._run_batch([(req, cls, slot)])
        torch.cuda.synchronize()
        return slot["x"].cpu().numpy().copy()

    def run(self, requests, time_scale=1.0):
        """Serve a request stream in real time; returns per-request records."""
        threads = [threading.Thread(target=self._worker, args=(s,), daemon=True)
                   for s in self.streams]
        for t in threads:
            t.start()
        pending = []
        i = 0
        t_start = time.perf_counter()
        nreq = len(requests)
        while True:
            now = time.perf_counter() - t_start
            while i < nreq and requests[i].arrival * time_scale <= now:
                requests[i].t0 = t_start + requests[i].arrival * time_scale
                pending.append(requests[i])
                i += 1
            # admit FIFO while slots and memory allow; one batch per size class
            # (requests of a class cost alike, so none waits on a slower kind)
            groups = {}
            keep = []
            for req in pending:
                cls = self.get_class(req.family, req.cls)
                batch = groups.setdefault((req.family, req.cls), [])
                ok = len(batch) < self.max_batch
                if ok:
                    with self.mem_lock:
                        ok = self.used + cls.slot_bytes <= self.budget
                        if ok:
                            self.used += cls.slot_bytes
                if not ok:
                    keep.append(req)
                    continue
                with cls.lock:
                    slot = cls.free.pop() if cls.free else None
                if slot is None:
                    slot = cls.make_slot()
                batch.append((req, cls, slot))
            pending = keep
            dispatched = False
            for batch in groups.values():
                if batch:
                    self.work.put(batch)
                    dispatched = True
            with self.done_lock:
                ndone = len(self.completed)
            if i >= nreq and not pending and ndone >= nreq:
                break
            if not dispatched:
                time.sleep(0.002)
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
                "errors": self.errors[:3]}
