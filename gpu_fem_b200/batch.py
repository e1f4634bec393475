"""Batched uneven shell solves and the fill-level autotuner.

A batch holds many independent plate / panel problems. Per problem the mesh,
BSR pattern, coloured scatter schedule and ILU(k) symbolic data stay
device-resident; a step re-assembles K (fused BCs) for every problem,
refactors all preconditioners in one level-ordered launch and solves all
problems together (gf_batch_*): one SpMV launch and one launch per
triangular sweep for the whole batch, per-problem GMRES states. Precision:
FP64, or FP32 ILU factors inside FP64 GMRES (mixed); FP32 ILU + FP32 SpMV
inside FP64 iterative refinement is available as well.

Autotuner: block ILU(0) is unstable on thin shells (Schur complements of the
membrane-dominated rows lose definiteness), so the fill level k of the
symbolic ILU(k) (computeILUk, include/linalg/bsr_utils.h:678-807) is chosen
per problem: every candidate k is tried on the whole batch in one batched
solve (FP32 factors, the less forgiving precision, inside FP64 GMRES) with
an iteration cap, and the converging candidates are combined so that the
modelled time of the batched factor + solve is smallest (batch_cost_us):
the batch runs as many GMRES steps as its slowest-converging problem needs
and each launch lasts as long as its longest level chain, so a problem that
converges early can take a lower fill (fewer levels, a cheaper
factorization) at no cost in steps.
The node ordering (natural or RCM) is chosen first, by levels x blocks per
row of ILU(8).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .assembler import BsrMat, ElementAssembler, ILUk_Preconditioner, SolveOptions, _stream

FILL_CANDIDATES = (0, 1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 16, 24)  # then GF_FILL_FULL (see _autotune)


class Batch:
    """gf_batch handle over lists of assemblers, matrices, preconditioners."""

    def __init__(self, asms, mats, pcs):
        n = len(asms)
        self.keep = (asms, mats, pcs)
        A = (C.c_void_p * n)(*[a.h.value for a in asms])
        K = (C.c_void_p * n)(*[m.h.value for m in mats])
        P = (C.c_void_p * n)(*[p.h.value for p in pcs])
        h = C.c_void_p()
        L.check(L.lib().gf_batch_create(n, A, K, P, C.byref(h)), "gf_batch_create")
        self.h = h
        self.n = n

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and L._LIB is not None:
            L.lib().gf_batch_destroy(h)
            self.h = None

    def assemble(self):
        L.check(L.lib().gf_batch_assemble(self.h, _stream()), "gf_batch_assemble")

    def set_scatter(self, atomic):
        """Batched assembly scatter: coloured (bitwise reproducible, one launch
        per colour over all problems) or FP64 atomics (one launch)."""
        L.check(L.lib().gf_batch_set_scatter(self.h, L.GF_ASSEMBLE_ATOMIC if atomic else 0),
                "gf_batch_set_scatter")

    def factor(self):
        L.check(L.lib().gf_batch_factor(self.h, _stream()), "gf_batch_factor")

    def solve(self, bs, xs, opts):
        n = self.n
        B = (C.c_void_p * n)(*[b.data_ptr() for b in bs])
        X = (C.c_void_p * n)(*[x.data_ptr() for x in xs])
        stats = (L.gf_solve_stats * n)()
        st = L.lib().gf_batch_solve(self.h, B, X, C.byref(opts), stats, _stream())
        if st not in (L.GF_OK, L.GF_NOT_CONVERGED):
            L.check(st, "gf_batch_solve")
        return st, [{"iterations": s.iterations, "restarts": s.restarts,
                     "refinements": s.refinements, "status": s.status,
                     "rel_residual": s.rel_residual} for s in stats]


def solve_opts(rtol=1e-8, mixed=False, restart=100, max_iters=20000, inner_rtol=1e-4):
    return SolveOptions(restart=restart, max_iters=max_iters, rtol=rtol, side=1,
                        mixed=1 if mixed else 0, inner_rtol=inner_rtol, max_refine=30,
                        check_every=25)


ORDERINGS = ("natural", "rcm")


def factor_work(nrow, inf):
    """Block updates of one factorization: ~nrow x lower x (lower + 1), with
    lower the blocks left of the diagonal per row."""
    lower = max(inf["nnzb"] - nrow, 0) / (2.0 * nrow)
    return nrow * lower * (lower + 1.0)


def factor_cost_us(nrow, inf, warps=None):
    """One numeric factorization of a problem (microseconds), fitted to B200
    runs of single plates (16^2 to 256^2 elements, fills 1 to 16) on the
    dataflow factorization with dependency-ordered steps: ~7-9 us a lower
    level (a row waits for its last-finishing dependency, then has only the
    steps that depend on it left), a little more per level as rows get
    longer, and a small throughput term for the block updates
    (~nrow x lower x (lower + 1), lower = blocks left of the diagonal per
    row) spread over the warps."""
    lvl, nnzb = inf["levels_L"], inf["nnzb"]
    lower = max(nnzb - nrow, 0) / (2.0 * nrow)
    if warps is None:  # alone: up to 128 CTAs of 8 warps
        warps = 8 * max(1, min(128, nrow // 32))
    work = factor_work(nrow, inf)
    if inf.get("ordering", "natural") == "rcm":
        t = 7.19 * lvl - 0.0132 * lvl * lower + 0.0031 * lvl * lower * lower + 0.028 * work / warps - 2.9
    else:
        t = 8.56 * lvl - 0.101 * lvl * lower + 0.0040 * lvl * lower * lower + 0.143 * work / warps - 40.9
    return max(t, 20.0)


def sweep_cost_us(inf):
    """Both triangular sweeps of one preconditioner apply (microseconds),
    fitted to B200 applies of the batch's plates: ~1.1 us a level plus
    ~2.3 ns per block of the level on one CTA, or ~1.6 us plus ~1.6 ns when
    the level's rows outnumber one CTA's warps or its blocks fill the stage
    and two CTAs share it (meeting once per chunk)."""
    lvl, lvu, nnzb = inf["levels_L"], inf["levels_U"], inf["nnzb"]
    nrow = inf.get("nrow") or 0
    blocks = max(nnzb - nrow, 0) / 2.0 / max(lvl, 1)
    rows = nrow / max(lvl, 1)
    split = rows > 13 or blocks > 380
    per_level = 1.6 + 0.0016 * blocks if split else 1.1 + 0.0023 * blocks
    return (lvl + lvu) * per_level


STEP_OVERHEAD_US = 150.0  # SpMV, orthogonalisation and launches of one GMRES step


def step_cost_us(nrow, inf, iterations):
    """Factor + solve time of a problem alone (microseconds): the
    factorization plus, per GMRES step, both sweeps and ~150 us of SpMV,
    reductions and launches."""
    inf = dict(inf, nrow=nrow)
    return factor_cost_us(nrow, inf) + iterations * (sweep_cost_us(inf) + STEP_OVERHEAD_US)


def batch_cost_us(choice):
    """Modelled time of one batched factor + solve (microseconds). choice:
    per problem (iterations, factor us, sweep us per GMRES step). The
    factorization of a batch is one launch, so it costs its slowest
    problem's; GMRES step s costs the slowest sweep among the problems still
    iterating at s (a sweep launch lasts as long as its longest level chain)."""
    fac = max(c[1] for c in choice)
    total, run_max, prev = 0.0, 0.0, 0
    # walk the steps from the last backwards: problems join the running set
    # in order of decreasing iteration count
    for its, _, sw in sorted(choice, key=lambda c: -c[0]):
        if its < prev or prev == 0:
            total += (prev - its) * (run_max + STEP_OVERHEAD_US) if prev else 0.0
            prev = its
        run_max = max(run_max, sw)
    total += prev * (run_max + STEP_OVERHEAD_US)
    return fac + total


def shared_factor_costs(cands, fills, sms=148):
    """Candidates with the factor cost of a batched factorization: when the
    problems' picks are `fills`, a candidate of problem p gets the SMs'
    share (one 8-warp CTA each) that its block updates take of the batch's,
    at most 128 CTAs (weights: block updates ** 0.7, as in the library's
    plan). fills=None keeps the alone costs. Candidates without
    their (nrow, info) keep their cost."""
    if fills is None:
        return [[c[:4] for c in cs] for cs in cands]
    # the library's CTA plan weights problems by block updates ** 0.7
    chosen = []
    for cs, k in zip(cands, fills):
        c = next(c for c in cs if c[0] == k)
        chosen.append(factor_work(*c[4]) ** 0.7 if len(c) > 4 else 0.0)
    total = sum(chosen)
    out = []
    for p, cs in enumerate(cands):
        row = []
        for c in cs:
            if len(c) <= 4 or total <= 0.0:
                row.append(c[:4])
                continue
            nrow, inf = c[4]
            w = factor_work(nrow, inf) ** 0.7
            share = w / max(total - chosen[p] + w, 1e-30)
            ctas = max(1, min(128, nrow // 32, int(sms * share)))
            row.append((c[0], c[1], factor_cost_us(nrow, inf, warps=8 * ctas), c[3]))
        out.append(row)
    return out


def choose_batch_fills(cands, rounds=8):
    """Per-problem fill levels that minimise batch_cost_us. cands[p]: list of
    (k, iterations, factor us, sweep us) of the converging candidates of
    problem p. Starts from every problem's own cheapest candidate and
    changes one problem at a time while the batch's modelled time drops."""
    pick = [min(c, key=lambda t: t[2] + t[1] * (t[3] + STEP_OVERHEAD_US)) for c in cands]
    best = batch_cost_us([p[1:] for p in pick])
    for _ in range(rounds):
        improved = False
        for p in range(len(cands)):
            for cand in cands[p]:
                if cand is pick[p]:
                    continue
                trial = pick[:p] + [cand] + pick[p + 1:]
                t = batch_cost_us([q[1:] for q in trial])
                if t < best - 1e-9:
                    best, pick, improved = t, trial, True
        if not improved:
            break
    return [p[0] for p in pick], best


def choose_ordering(mesh, fill=8):
    """Assembler of the mesh in the node ordering whose ILU(fill) triangles
    have the fewest levels (the sweeps' critical path). Line-by-line
    (natural) numbering of a structured plate gives levels ~ n_long +
    (fill + 2) n_short, several times fewer than RCM's diagonal wavefronts,
    whose nodes chain up through the element diagonals; RCM stays the choice
    for meshes whose generator numbering is poor."""
    best = None
    for o in ORDERINGS:
        a = ElementAssembler.from_mesh(mesh, ordering=o)
        try:
            inf = ILUk_Preconditioner(a, fill, "fp64").info()
        except L.GpuFemError:  # fill rows too long for the sweep kernel
            continue
        # levels x blocks per row: both the sweep and the factorization
        # critical paths grow with it (a poor numbering fills in heavily)
        score = (inf["levels_L"] + inf["levels_U"]) * inf["nnzb"] / a.get_num_nodes()
        if best is None or score < best[0]:
            best = (score, o, a)
    if best is None:
        raise RuntimeError(f"no ordering of {mesh.name} gives a usable ILU({fill})")
    return best[1], best[2]


class BatchSolver:
    """Problems resident on the current device, solved as one batch."""

    def __init__(self, meshes, ordering="auto", tune=True, fill=None, rtol=1e-8, restart=100,
                 build=True, objective="batch"):
        self.rtol, self.restart = rtol, restart
        # autotuner objective: "batch" minimises the modelled time of the
        # batched factor + solve (batch_cost_us), "problem" each problem's
        # own factor + solve time
        self.objective = objective
        self.meshes = meshes
        # assemblers (host symbolic work in the library, GIL released) are
        # built on host threads
        from concurrent.futures import ThreadPoolExecutor
        workers = max(1, min(8, len(meshes)))
        if ordering == "auto":
            with ThreadPoolExecutor(max_workers=workers) as ex:
                picked = list(ex.map(choose_ordering, meshes))
            self.orderings = [o for o, _ in picked]
            self.asms = [a for _, a in picked]
        else:  # one ordering for all, or one per problem
            self.orderings = ([ordering] * len(meshes) if isinstance(ordering, str)
                              else list(ordering))
            with ThreadPoolExecutor(max_workers=workers) as ex:
                self.asms = list(ex.map(lambda mo: ElementAssembler.from_mesh(mo[0], ordering=mo[1]),
                                        zip(meshes, self.orderings)))
        self.mats = [BsrMat(a) for a in self.asms]
        self.bs = [torch.tensor(m.loads, device="cuda") for m in meshes]
        self.xs = [torch.zeros_like(b) for b in self.bs]
        for a, k in zip(self.asms, self.mats):
            a.add_jacobian(None, k, fuse_bcs=True)
        n = len(meshes)
        if fill is not None:
            self.fills = [fill] * n if np.isscalar(fill) else list(fill)
            self.tune_log = None
        elif tune:
            self.fills, self.tune_log = self._autotune()
        else:
            self.fills, self.tune_log = [0] * n, None
        if not build:  # fill levels only (the server tunes its size classes this way)
            return
        # the preconditioners' host setup (orderings of the steps, chunk
        # streams) runs in the library with the GIL released: build them on
        # host threads
        from concurrent.futures import ThreadPoolExecutor
        jobs = [(a, k, pr) for pr in ("fp64", "fp32") for a, k in zip(self.asms, self.fills)]
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            built = list(ex.map(lambda j: ILUk_Preconditioner(*j), jobs))
        n = len(self.asms)
        self.P64, self.P32 = built[:n], built[n:]
        self.b64 = Batch(self.asms, self.mats, self.P64)
        self.b32 = Batch(self.asms, self.mats, self.P32)
        torch.cuda.synchronize()

    def _trial(self, k, todo, cap, best, cands, log):
        """Factor and solve problems `todo` with fill k (FP32 factors inside
        FP64 GMRES, at most `cap` steps); records the converging ones."""
        try:
            P = [ILUk_Preconditioner(self.asms[i], k, "fp32") for i in todo]
        except L.GpuFemError:  # a factor row longer than the sweep's stage
            log.append((k, "precond create failed"))
            return False
        bt = Batch([self.asms[i] for i in todo], [self.mats[i] for i in todo], P)
        try:
            bt.factor()
        except L.GpuFemError:
            log.append((k, "factor failed"))
            return True
        for i in todo:
            self.xs[i].zero_()
        st, stats = bt.solve([self.bs[i] for i in todo], [self.xs[i] for i in todo],
                             solve_opts(self.rtol, False, restart=self.restart, max_iters=cap))
        for j, i in enumerate(todo):
            s = stats[j]
            nrow = self.asms[i].get_num_nodes()
            inf = dict(P[j].info(), nrow=nrow, ordering=self.orderings[i])
            nlev = inf["levels_L"] + inf["levels_U"]
            ok = s["status"] == L.GF_OK
            log.append((i, k, s["iterations"], s["rel_residual"], nlev, ok))
            if ok:
                cands[i].append((k, s["iterations"], factor_cost_us(nrow, inf),
                                 sweep_cost_us(inf), (nrow, inf)))
                cost = step_cost_us(nrow, inf, s["iterations"])
                if best[i] is None or cost < best[i][0]:
                    best[i] = (cost, k, k)
        return True

    def _autotune(self, cap=400):
        n = len(self.meshes)
        best = [None] * n
        cands = [[] for _ in range(n)]
        log = []
        for k in FILL_CANDIDATES:
            todo = [i for i in range(n) if best[i] is None or k <= best[i][2] + 4]
            if not todo:
                break
            if not self._trial(k, todo, cap, best, cands, log):
                break
            if all(b is not None for b in best) and k >= max(b[1] for b in best) + 4:
                break
        missing = [self.meshes[i].name for i in range(n) if best[i] is None]
        if missing:
            raise RuntimeError(f"no ILU fill level converged for {missing}")
        if self.objective == "problem":
            return [b[1] for b in best], log
        # A batch runs as many GMRES steps as its slowest-converging problem
        # needs: the problems that need many steps even at their best fill
        # also get every higher fill and the complete factor (GF_FILL_FULL,
        # a direct solve where its rows fit the sweep kernel) tried.
        steps = [min(c[1] for c in cands[i]) for i in range(n)]
        slow = [i for i in range(n) if steps[i] >= 0.6 * max(steps)]
        for k in FILL_CANDIDATES + (L.GF_FILL_FULL,):
            todo = [i for i in slow if all(c[0] != k for c in cands[i])
                    and k > max(c[0] for c in cands[i])]
            if todo:
                self._trial(k, todo, cap, best, cands, log)
        fills, _ = choose_batch_fills(shared_factor_costs(cands, fills=None))
        # the batch's factorizations share the SMs in proportion to their
        # block updates: re-cost every candidate with its share of the SMs
        # given the other problems' picks, and choose again
        for _ in range(3):
            new, _ = choose_batch_fills(shared_factor_costs(cands, fills))
            if new == fills:
                break
            fills = new
        return fills, log

    def step(self, mixed: bool, host_io=None, spmv32=False, phases=None):
        """Assemble, factor and solve every problem once. mixed: FP32 ILU
        factors (half the bytes of the sweeps' factor streams) inside FP64
        GMRES; with spmv32 also FP32 SpMV in an inner GMRES under FP64
        iterative refinement, whose reachable residual is limited by
        cond(A) x 6e-8 and so fails on the thinnest shells. phases: optional
        list of 4 CUDA events recorded before assembly, factorization, solve
        and after the solve."""
        ev = phases if phases is not None else [None] * 4
        if host_io is not None:
            for b, hb in zip(self.bs, host_io[0]):
                b.copy_(hb, non_blocking=True)
        bt = self.b32 if mixed else self.b64
        if ev[0] is not None:
            ev[0].record()
        bt.assemble()
        if ev[1] is not None:
            ev[1].record()
        bt.factor()
        if ev[2] is not None:
            ev[2].record()
        for x in self.xs:
            x.zero_()
        st, stats = bt.solve(self.bs, self.xs,
                             solve_opts(self.rtol, mixed and spmv32, self.restart))
        if ev[3] is not None:
            ev[3].record()
        if st != L.GF_OK:
            raise RuntimeError(f"batch solve failed: {[s for s in stats if s['status']]}")
        if host_io is not None:
            for x, hx in zip(self.xs, host_io[1]):
                hx.copy_(x, non_blocking=True)
        return stats
