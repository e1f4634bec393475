"""Seeded synthetic shell meshes for the plate / box workloads.

The reference's only mesh generator is the plate of
examples/plate_demo/_plate_utils.h:9-144 (createPlateAssembler). It emits
element nodes counter-clockwise ({n, n+1, n+nnx+1, n+nnx}, :103-104), while
the basis expects tensor-product order (getNodePoint, include/shell/basis.h:138-142),
which makes every element a bow-tie. The generators here emit tensor order
{n, n+1, n+nnx, n+nnx+1}.

All randomness comes from a bit-exact std::mt19937_64 (seeded with one
64-bit integer) with uniforms (x >> 11) * 2**-53, so C++ callers can
regenerate the same inputs.

Every mesh is returned as a :class:`ShellMesh` holding natural-order arrays:
``conn`` (Ne, 4) int32, ``xpts`` (Nn, 3) float64, ``thick`` (Ne,) float64,
``bcs`` (nbc,) int32 natural DOF indices (6*node + dof), ``loads`` (6*Nn,)
float64, plus ``E``/``nu``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

__all__ = ["MT19937_64", "ShellMesh", "plate", "plate_config1", "plate_config2",
           "box_config3", "batch_config4", "box"]

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


class MT19937_64:
    """std::mt19937_64 with the C++ standard's seeding (seed(value))."""

    NN, MM = 312, 156
    MATRIX_A = np.uint64(0xB5026F5AA96619E9)
    UM = np.uint64(0xFFFFFFFF80000000)
    LM = np.uint64(0x7FFFFFFF)

    def __init__(self, seed: int = 5489):
        mt = [0] * self.NN
        mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, self.NN):
            prev = mt[i - 1]
            mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
        self.mt = np.array(mt, dtype=np.uint64)
        self.idx = self.NN

    def _twist(self):
        mt, NN, MM = self.mt, self.NN, self.MM
        one, zero = np.uint64(1), np.uint64(0)
        x = (mt[0:NN - MM] & self.UM) | (mt[1:NN - MM + 1] & self.LM)
        mag = np.where((x & one) != zero, self.MATRIX_A, zero)
        mt[0:NN - MM] = mt[MM:NN] ^ (x >> one) ^ mag
        x = (mt[NN - MM:NN - 1] & self.UM) | (mt[NN - MM + 1:NN] & self.LM)
        mag = np.where((x & one) != zero, self.MATRIX_A, zero)
        mt[NN - MM:NN - 1] = mt[0:MM - 1] ^ (x >> one) ^ mag
        x = (mt[NN - 1] & self.UM) | (mt[0] & self.LM)
        mag = self.MATRIX_A if (int(x) & 1) else zero
        mt[NN - 1] = mt[MM - 1] ^ (x >> one) ^ mag
        self.idx = 0

    def raw(self, n: int) -> np.ndarray:
        """Next n raw 64-bit outputs (tempered), as uint64."""
        out = np.empty(n, dtype=np.uint64)
        k = 0
        while k < n:
            if self.idx >= self.NN:
                self._twist()
            take = min(n - k, self.NN - self.idx)
            out[k:k + take] = self.mt[self.idx:self.idx + take]
            self.idx += take
            k += take
        y = out
        y = y ^ ((y >> np.uint64(29)) & np.uint64(0x5555555555555555))
        y = y ^ ((y << np.uint64(17)) & np.uint64(0x71D67FFFEDA60000))
        y = y ^ ((y << np.uint64(37)) & np.uint64(0xFFF7EEE000000000))
        y = y ^ (y >> np.uint64(43))
        return y

    def uniform(self, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
        u = (self.raw(n) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
        return lo + (hi - lo) * u


@dataclass
class ShellMesh:
    conn: np.ndarray
    xpts: np.ndarray
    thick: np.ndarray
    bcs: np.ndarray
    loads: np.ndarray
    E: float = 70e9
    nu: float = 0.3
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def num_nodes(self) -> int:
        return int(self.xpts.shape[0])

    @property
    def num_elements(self) -> int:
        return int(self.conn.shape[0])

    @property
    def num_dof(self) -> int:
        return 6 * self.num_nodes


def _pressure_loads(conn, xpts, pfun):
    """Consistent nodal loads f_i = int p N_i dA on the w DOF, 2x2 Gauss with
    the reference's point/weight convention (include/shell/quadrature.h)."""
    rt3 = 0.577350269189626
    nn = xpts.shape[0]
    f = np.zeros(6 * nn)
    X = xpts[conn]  # (Ne, 4, 3)
    for iq in range(4):
        xi = (-rt3, rt3)[iq % 2]
        eta = (-rt3, rt3)[iq // 2]
        na = np.array([0.5 * (1 - xi), 0.5 * (1 + xi)])
        nb = np.array([0.5 * (1 - eta), 0.5 * (1 + eta)])
        N = np.array([na[0] * nb[0], na[1] * nb[0], na[0] * nb[1], na[1] * nb[1]])
        Nxi = np.array([-0.5 * nb[0], 0.5 * nb[0], -0.5 * nb[1], 0.5 * nb[1]])
        Neta = np.array([-0.5 * na[0], -0.5 * na[1], 0.5 * na[0], 0.5 * na[1]])
        xq = np.einsum("n,enk->ek", N, X)
        dxi = np.einsum("n,enk->ek", Nxi, X)
        deta = np.einsum("n,enk->ek", Neta, X)
        dA = np.linalg.norm(np.cross(dxi, deta), axis=1)
        p = pfun(xq)
        contrib = (p * dA)[:, None] * N[None, :]
        np.add.at(f, 6 * conn + 2, contrib)
    return f


def plate(nxe, nye, Lx, Ly, thick_fn, clamp, pressure, jitter=0.0, seed=1234,
          E=70e9, nu=0.3, name="plate"):
    """Rectangular flat plate in the z=0 plane with tensor-ordered quads.

    thick_fn(xc, yc) -> thickness at element centroids; clamp in
    {"all_edges", "x0"}; pressure(xq) -> transverse pressure at points.
    jitter: in-plane node jitter as a fraction of the element size; per node
    (natural order) two uniforms U(-1, 1) are drawn (x then y); interior nodes
    move in x and y, edge nodes only along their edge, corners stay fixed.
    """
    nnx, nny = nxe + 1, nye + 1
    dx, dy = Lx / nxe, Ly / nye
    ix, iy = np.meshgrid(np.arange(nnx), np.arange(nny))
    ix, iy = ix.ravel(), iy.ravel()
    x = ix * dx
    y = iy * dy
    if jitter > 0.0:
        r = MT19937_64(seed).uniform(2 * nnx * nny, -1.0, 1.0).reshape(-1, 2)
        onx = (ix == 0) | (ix == nxe)
        ony = (iy == 0) | (iy == nye)
        movex = ~onx
        movey = ~ony
        x = x + np.where(movex, r[:, 0] * jitter * dx, 0.0)
        y = y + np.where(movey, r[:, 1] * jitter * dy, 0.0)
    xpts = np.stack([x, y, np.zeros_like(x)], axis=1)
    ex, ey = np.meshgrid(np.arange(nxe), np.arange(nye))
    n0 = (nnx * ey + ex).ravel()
    conn = np.stack([n0, n0 + 1, n0 + nnx, n0 + nnx + 1], axis=1).astype(np.int32)
    cen = xpts[conn].mean(axis=1)
    thick = np.asarray(thick_fn(cen[:, 0], cen[:, 1]), dtype=np.float64)
    thick = np.broadcast_to(thick, (conn.shape[0],)).copy()
    if clamp == "all_edges":
        bnodes = np.nonzero((ix == 0) | (ix == nxe) | (iy == 0) | (iy == nye))[0]
    elif clamp == "x0":
        bnodes = np.nonzero(ix == 0)[0]
    else:
        raise ValueError(clamp)
    bcs = (6 * bnodes[:, None] + np.arange(6)[None, :]).ravel().astype(np.int32)
    loads = _pressure_loads(conn, xpts, pressure)
    loads[bcs] = 0.0
    return ShellMesh(conn, xpts, thick, bcs, loads, E, nu, name,
                     {"nxe": nxe, "nye": nye, "Lx": Lx, "Ly": Ly})


def plate_config1():
    """1.0 x 1.0 m, 10x10 elements, t = 5 mm, all edges clamped, 1 kPa."""
    return plate(10, 10, 1.0, 1.0, lambda x, y: 0.005 + 0 * x, "all_edges",
                 lambda q: 1.0e3 + 0 * q[:, 0], name="plate_10x10")


def plate_config2(nxe=400, nye=200):
    """2 x 1 m, 400x200 elements, t = 4 mm (1 + 0.25 sin 2 pi x cos pi y) at
    element centroids, +/-10 % in-plane jitter (seed 1234), edge x = 0
    clamped, p = 1 kPa sin(pi x / 2)."""
    return plate(nxe, nye, 2.0, 1.0,
                 lambda x, y: 0.004 * (1.0 + 0.25 * np.sin(2 * np.pi * x) * np.cos(np.pi * y)),
                 "x0", lambda q: 1.0e3 * np.sin(np.pi * q[:, 0] / 2.0), jitter=0.1, seed=1234,
                 name=f"plate_{nxe}x{nye}_jitter")


def box(nx=603, ny=150, nz=45, Lx=4.0, Ly=1.0, Lz=0.3, nribs=10, t_skin=0.003,
        t_web=0.006, tip_load=1.0e4, E=70e9, nu=0.3):
    """Closed rectangular box (skins z=0, z=Lz; spars y=0, y=Ly; ribs at
    x = k Lx/(nribs-1)); the root face x = 0 is clamped and a tip load in z is
    spread equally over the tip-rib nodes. Node indices: structured nodes are
    created on demand and deduplicated by integer grid coordinates."""
    if nx % (nribs - 1) != 0:
        raise ValueError("nx must be divisible by nribs-1")
    ids = {}
    coords = []

    def node(i, j, k):
        key = (i, j, k)
        v = ids.get(key)
        if v is None:
            v = len(coords)
            ids[key] = v
            coords.append((i * Lx / nx, j * Ly / ny, k * Lz / nz))
        return v

    conn, thick = [], []
    # skins (bottom k=0, top k=nz), element grid over (i, j)
    for k in (0, nz):
        for j in range(ny):
            for i in range(nx):
                conn.append((node(i, j, k), node(i + 1, j, k), node(i, j + 1, k),
                             node(i + 1, j + 1, k)))
                thick.append(t_skin)
    # spars (y=0, y=ny), element grid over (i, k)
    for j in (0, ny):
        for k in range(nz):
            for i in range(nx):
                conn.append((node(i, j, k), node(i + 1, j, k), node(i, j, k + 1),
                             node(i + 1, j, k + 1)))
                thick.append(t_web)
    # ribs, element grid over (j, k)
    step = nx // (nribs - 1)
    for r in range(nribs):
        i = r * step
        for k in range(nz):
            for j in range(ny):
                conn.append((node(i, j, k), node(i, j + 1, k), node(i, j, k + 1),
                             node(i, j + 1, k + 1)))
                thick.append(t_web)
    conn = np.asarray(conn, dtype=np.int32)
    xpts = np.asarray(coords, dtype=np.float64)
    thick = np.asarray(thick, dtype=np.float64)
    root = np.nonzero(np.abs(xpts[:, 0]) < 1e-12)[0]
    bcs = (6 * root[:, None] + np.arange(6)[None, :]).ravel().astype(np.int32)
    tip = np.nonzero(np.abs(xpts[:, 0] - Lx) < 1e-12)[0]
    loads = np.zeros(6 * xpts.shape[0])
    loads[6 * tip + 2] = tip_load / len(tip)
    return ShellMesh(conn, xpts, thick, bcs, loads, E, nu, f"box_{nx}x{ny}x{nz}",
                     {"nx": nx, "ny": ny, "nz": nz})


def box_config3():
    return box()


def batch_config4(n=64, seed=4321, E=70e9, nu=0.3):
    """64 plates: nx = round(exp U(ln 16, ln 256)), aspect a ~ U(1, 4),
    ny = max(16, round(nx / a)), element size 1/nx m, t ~ U(2, 8) mm uniform,
    p ~ U(0.5, 2) kPa, all edges clamped. Four uniforms per problem in that
    order."""
    r = MT19937_64(seed).uniform(4 * n).reshape(n, 4)
    out = []
    for k in range(n):
        nx = int(round(math.exp(math.log(16) + r[k, 0] * (math.log(256) - math.log(16)))))
        a = 1.0 + 3.0 * r[k, 1]
        ny = max(16, int(round(nx / a)))
        t = 0.002 + 0.006 * r[k, 2]
        p = 500.0 + 1500.0 * r[k, 3]
        h = 1.0 / nx
        out.append(plate(nx, ny, nx * h, ny * h, lambda x, y, t=t: t + 0 * x, "all_edges",
                         lambda q, p=p: p + 0 * q[:, 0], E=E, nu=nu,
                         name=f"plate_{nx}x{ny}"))
    return out


def write_bdf(mesh, path, fmt="small", node_ids=None, elem_ids=None, pid=1):
    """Writes the mesh as a NASTRAN bulk-data file: GRID, CQUAD4 (nodes around
    the element: tensor order n0 n1 n3 n2 becomes G1 G2 G3 G4 = n0 n1 n3 n2)
    and one SPC entry per constrained node. fmt: "small" (8-column fields),
    "large" (16-column fields, GRID* / CQUAD4* with '*' continuation lines) or
    "free" (comma separated). node_ids / elem_ids: file ids (default 1..n)."""
    nn, ne = mesh.num_nodes, mesh.num_elements
    nid = np.arange(1, nn + 1) if node_ids is None else np.asarray(node_ids)
    eid = np.arange(1, ne + 1) if elem_ids is None else np.asarray(elem_ids)
    bc_nodes = {}
    for d in np.asarray(mesh.bcs):
        bc_nodes.setdefault(int(d) // 6, []).append(int(d) % 6 + 1)

    def small(key, fields):
        return key.ljust(8) + "".join(str(f)[:8].rjust(8) for f in fields)

    def real8(x):
        s = f"{x:.6g}"
        if len(s) > 8:
            s = f"{x:.2e}"
        return s if ("." in s or "e" in s) else s + "."

    lines = ["$ shell mesh", "BEGIN BULK"]
    for k in range(nn):
        x, y, z = mesh.xpts[k]
        if fmt == "small":
            lines.append(small("GRID", [nid[k], 0, real8(x), real8(y), real8(z)]))
        elif fmt == "large":
            f16 = [f"{float(v):.8e}" for v in (x, y, z)]  # at most 16 characters
            lines.append("GRID*".ljust(8) + str(nid[k]).rjust(16) + "0".rjust(16) +
                         f16[0].rjust(16) + f16[1].rjust(16))
            lines.append("*".ljust(8) + f16[2].rjust(16))
        else:
            lines.append(f"GRID,{nid[k]},0,{float(x)!r},{float(y)!r},{float(z)!r}")
    for e in range(ne):
        c = mesh.conn[e]
        g = [nid[c[0]], nid[c[1]], nid[c[3]], nid[c[2]]]
        if fmt == "small":
            lines.append(small("CQUAD4", [eid[e], pid] + g))
        elif fmt == "large":
            lines.append("CQUAD4*".ljust(8) + "".join(str(v).rjust(16) for v in [eid[e], pid] + g[:2]))
            lines.append("*".ljust(8) + "".join(str(v).rjust(16) for v in g[2:]))
        else:
            lines.append("CQUAD4," + ",".join(str(v) for v in [eid[e], pid] + g))
    for node, dofs in bc_nodes.items():
        c = "".join(str(d) for d in sorted(dofs))
        if fmt == "free":
            lines.append(f"SPC,1,{nid[node]},{c},0.0")
        else:
            lines.append(small("SPC", [1, nid[node], c, "0."]))
    lines.append("ENDDATA")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
