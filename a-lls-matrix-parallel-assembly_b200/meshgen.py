"""Seeded synthetic FEM meshes for the assembly path (host side, numpy).

The reference generates structured, unperturbed meshes inside each benchmark
program:

* Q4 grid            ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:575-603
* T3 grid (n0-n2 split) ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:373-400
* mixed Q4/T3 grid   ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:447-485
* Hex20 lattice      ALLS_Hex20_3D_Assembly_Performance.cu:324-362

The generators here keep the reference's node numbering (``j*(nx+1)+i`` in
2-D), per-element node order and interleaved DOF numbering
(``dof = node*dpn + d``), and add what the benchmark configurations ask for:
seeded jitter of interior nodes, random T3 diagonals, shuffled element order,
per-element E and nu, and a *compact* Hex20 node numbering (corner and
mid-edge nodes only; the reference lattice also keeps face- and body-centre
points that no element uses, ``ALLS_Hex20_3D_Assembly_Performance.cu:326-338``).

Every generator is deterministic for a given seed (numpy PCG64) and checks that
every element has a positive Jacobian determinant at all of its Gauss points.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

Q4, T3, HEX20, MIXED_2D = 0, 1, 2, 3
KIND_NAMES = {Q4: "q4", T3: "t3", HEX20: "hex20", MIXED_2D: "mixed"}
NPE = {Q4: 4, T3: 3, HEX20: 20}
DPN = {Q4: 2, T3: 2, MIXED_2D: 2, HEX20: 3}

# Q4 2x2 Gauss abscissa as written in the reference (Q4A:48).
_G2 = 0.577350269189626
# Hex20 3-point Gauss abscissa (H20:45).
_G3 = 0.774596669241483


@dataclasses.dataclass
class Mesh:
    """A mesh in the layout the C ABI takes (structure-of-arrays coordinates)."""

    kind: int
    x: np.ndarray                 # float64 [num_nodes]
    y: np.ndarray                 # float64 [num_nodes]
    z: Optional[np.ndarray]       # float64 [num_nodes] (Hex20 only)
    conn: np.ndarray              # int32 [num_elems, stride]
    types: Optional[np.ndarray]   # uint8 [num_elems] (mixed meshes only)
    E: Optional[np.ndarray]       # float64 [num_elems] or None (uniform E0)
    nu: Optional[np.ndarray]      # float64 [num_elems] or None (uniform nu0)
    E0: float = 1.0
    nu0: float = 0.3
    thickness: float = 1.0
    name: str = ""
    seed: int = 0

    @property
    def num_nodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def num_elems(self) -> int:
        return int(self.conn.shape[0])

    @property
    def stride(self) -> int:
        return int(self.conn.shape[1])

    @property
    def dpn(self) -> int:
        return DPN[self.kind]

    @property
    def num_dofs(self) -> int:
        return self.num_nodes * self.dpn

    def nodes_per_elem(self) -> np.ndarray:
        if self.kind == MIXED_2D:
            return np.where(self.types == Q4, 4, 3).astype(np.int64)
        return np.full(self.num_elems, NPE[self.kind], dtype=np.int64)

    def contributions(self) -> int:
        """Sum over elements of ndof_e^2 (scalar Ke entries scattered)."""
        npe = self.nodes_per_elem()
        return int(np.sum((npe * self.dpn) ** 2))

    def element_E(self) -> np.ndarray:
        return self.E if self.E is not None else np.full(self.num_elems, self.E0)

    def element_nu(self) -> np.ndarray:
        return self.nu if self.nu is not None else np.full(self.num_elems, self.nu0)


# ----------------------------------------------------------------------------
# 2-D helpers
# ----------------------------------------------------------------------------

def _grid_nodes(nx: int, ny: int, lx: float, ly: float):
    i = np.arange(nx + 1, dtype=np.float64)
    j = np.arange(ny + 1, dtype=np.float64)
    X, Y = np.meshgrid(i * lx / nx, j * ly / ny)      # [ny+1, nx+1], node id j*(nx+1)+i
    return X.ravel().copy(), Y.ravel().copy()


def _interior_mask_2d(nx: int, ny: int) -> np.ndarray:
    m = np.zeros((ny + 1, nx + 1), dtype=bool)
    m[1:-1, 1:-1] = True
    return m.ravel()


def _cell_corners(nx: int, ny: int):
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (j * (nx + 1) + i).ravel()
    n1 = n0 + 1
    n2 = n0 + (nx + 1) + 1
    n3 = n0 + (nx + 1)
    return n0, n1, n2, n3


def _q4_detj_min(x, y, conn):
    """Minimum Jacobian determinant of Q4 elements over the 2x2 Gauss points."""
    xe, ye = x[conn], y[conn]
    out = np.inf
    for xi in (-_G2, _G2):
        for eta in (-_G2, _G2):
            dxi = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
            deta = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
            j00, j01 = xe @ dxi, ye @ dxi
            j10, j11 = xe @ deta, ye @ deta
            out = min(out, float(np.min(j00 * j11 - j01 * j10)))
    return out


def _t3_detj(x, y, conn):
    x0, x1, x2 = (x[conn[:, k]] for k in range(3))
    y0, y1, y2 = (y[conn[:, k]] for k in range(3))
    return (x1 - x0) * (y2 - y0) - (y1 - y0) * (x2 - x0)


def _jitter_until_valid(rng, x0, y0, interior, amp, check, max_halvings=8):
    """Jitter interior nodes by U(-amp, amp) and halve the jitter of nodes that
    belong to inverted elements until every element is valid (deterministic)."""
    dx = rng.uniform(-amp, amp, size=x0.shape) * interior
    dy = rng.uniform(-amp, amp, size=y0.shape) * interior
    for _ in range(max_halvings + 1):
        x, y = x0 + dx, y0 + dy
        bad_nodes = check(x, y)
        if bad_nodes is None or bad_nodes.size == 0:
            return x, y
        dx[bad_nodes] *= 0.5
        dy[bad_nodes] *= 0.5
    raise RuntimeError("could not produce a mesh with positive Jacobians")


# ----------------------------------------------------------------------------
# Generators
# ----------------------------------------------------------------------------

def q4_grid(nx: int = 100, ny: int = 100, *, jitter: float = 0.1, seed: int = 1,
            E: float = 1.0, nu: float = 0.3, thickness: float = 1.0,
            lx: float = 1.0, ly: float = 1.0) -> Mesh:
    """Structured Q4 plane-stress mesh in natural element order (Q4A:575-603),
    interior nodes jittered by U(+-jitter*h)."""
    rng = np.random.default_rng(seed)
    x0, y0 = _grid_nodes(nx, ny, lx, ly)
    n0, n1, n2, n3 = _cell_corners(nx, ny)
    conn = np.stack([n0, n1, n2, n3], axis=1).astype(np.int32)
    h = min(lx / nx, ly / ny)

    def check(x, y):
        xe, ye = x[conn], y[conn]
        bad = np.zeros(conn.shape[0], dtype=bool)
        for xi in (-_G2, _G2):
            for eta in (-_G2, _G2):
                dxi = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
                deta = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
                d = (xe @ dxi) * (ye @ deta) - (ye @ dxi) * (xe @ deta)
                bad |= d <= 0.05 * 0.25 * h * h
        return np.unique(conn[bad].ravel())

    x, y = _jitter_until_valid(rng, x0, y0, _interior_mask_2d(nx, ny), jitter * h, check)
    return Mesh(Q4, x, y, None, conn, None, None, None, E0=E, nu0=nu,
                thickness=thickness, name=f"q4_{nx}x{ny}", seed=seed)


def t3_grid(nx: int = 1000, ny: int = 1000, *, jitter: float = 0.2, seed: int = 2,
            random_diagonal: bool = True, shuffle: bool = True,
            E_sigma: float = 0.5, nu: float = 0.3, thickness: float = 1.0,
            lx: float = 1.0, ly: float = 1.0) -> Mesh:
    """T3 mesh of a structured grid, each cell split into two triangles.

    The reference split is (n0,n1,n2),(n0,n2,n3) (T3:385-392); with
    ``random_diagonal`` each cell instead draws its diagonal from a Bernoulli(0.5)
    (the other split is (n0,n1,n3),(n1,n2,n3)). Element order is shuffled,
    E ~ LogNormal(0, E_sigma) per element (E_sigma=0 gives E=1)."""
    rng = np.random.default_rng(seed)
    x0, y0 = _grid_nodes(nx, ny, lx, ly)
    n0, n1, n2, n3 = _cell_corners(nx, ny)
    if random_diagonal:
        alt = rng.random(n0.shape[0]) < 0.5
    else:
        alt = np.zeros(n0.shape[0], dtype=bool)
    a = np.where(alt[:, None], np.stack([n0, n1, n3], 1), np.stack([n0, n1, n2], 1))
    b = np.where(alt[:, None], np.stack([n1, n2, n3], 1), np.stack([n0, n2, n3], 1))
    conn = np.empty((2 * n0.shape[0], 3), dtype=np.int32)
    conn[0::2] = a
    conn[1::2] = b
    h = min(lx / nx, ly / ny)

    def check(x, y):
        bad = _t3_detj(x, y, conn) <= 0.05 * h * h
        return np.unique(conn[bad].ravel())

    x, y = _jitter_until_valid(rng, x0, y0, _interior_mask_2d(nx, ny), jitter * h, check)
    if shuffle:
        conn = conn[rng.permutation(conn.shape[0])]
    E = rng.lognormal(0.0, E_sigma, size=conn.shape[0]) if E_sigma > 0 else None
    return Mesh(T3, x, y, None, np.ascontiguousarray(conn), None, E, None, E0=1.0,
                nu0=nu, thickness=thickness, name=f"t3_{nx}x{ny}", seed=seed)


def mixed_grid(nx: int = 1500, ny: int = 1500, *, jitter: float = 0.15, seed: int = 3,
               q4_ratio: float = 0.5, shuffle: bool = True, E_sigma: float = 0.5,
               nu_range=(0.2, 0.4), thickness: float = 1.0,
               lx: float = 1.0, ly: float = 1.0) -> Mesh:
    """Mixed Q4/T3 mesh (MIX:447-485): each cell is a Q4 with probability
    ``q4_ratio``, else the reference's two-triangle split (n0,n1,n2),(n0,n2,n3).
    Connectivity rows have stride 4; T3 rows carry -1 in the 4th column as the
    reference Element does (MIX:473-476). Element order shuffled; E lognormal,
    nu uniform in ``nu_range``."""
    rng = np.random.default_rng(seed)
    x0, y0 = _grid_nodes(nx, ny, lx, ly)
    n0, n1, n2, n3 = _cell_corners(nx, ny)
    is_q4 = rng.random(n0.shape[0]) < q4_ratio
    neg = np.full_like(n0, -1)
    q = np.stack([n0, n1, n2, n3], 1)[is_q4]
    t1 = np.stack([n0, n1, n2, neg], 1)[~is_q4]
    t2 = np.stack([n0, n2, n3, neg], 1)[~is_q4]
    # keep the reference's cell-by-cell emission order before shuffling
    order_q = np.nonzero(is_q4)[0]
    order_t = np.nonzero(~is_q4)[0]
    keys = np.concatenate([order_q * 2, order_t * 2, order_t * 2 + 1])
    rows = np.concatenate([q, t1, t2]).astype(np.int32)
    types = np.concatenate([np.full(q.shape[0], Q4), np.full(2 * t1.shape[0], T3)]).astype(np.uint8)
    srt = np.argsort(keys, kind="stable")
    conn, types = rows[srt], types[srt]
    h = min(lx / nx, ly / ny)

    def check(x, y):
        bad_nodes = []
        tmask = types == T3
        tc = conn[tmask][:, :3]
        bad = _t3_detj(x, y, tc) <= 0.05 * h * h
        bad_nodes.append(tc[bad].ravel())
        qc = conn[~tmask]
        xe, ye = x[qc], y[qc]
        qb = np.zeros(qc.shape[0], dtype=bool)
        for xi in (-_G2, _G2):
            for eta in (-_G2, _G2):
                dxi = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
                deta = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
                d = (xe @ dxi) * (ye @ deta) - (ye @ dxi) * (xe @ deta)
                qb |= d <= 0.05 * 0.25 * h * h
        bad_nodes.append(qc[qb].ravel())
        return np.unique(np.concatenate(bad_nodes))

    x, y = _jitter_until_valid(rng, x0, y0, _interior_mask_2d(nx, ny), jitter * h, check)
    if shuffle:
        p = rng.permutation(conn.shape[0])
        conn, types = conn[p], types[p]
    E = rng.lognormal(0.0, E_sigma, size=conn.shape[0]) if E_sigma > 0 else None
    nu = rng.uniform(nu_range[0], nu_range[1], size=conn.shape[0]) if nu_range else None
    return Mesh(MIXED_2D, x, y, None, np.ascontiguousarray(conn), np.ascontiguousarray(types),
                E, nu, E0=1.0, nu0=0.3, thickness=thickness, name=f"mixed_{nx}x{ny}", seed=seed)


# Hex20 local node offsets on the (2n+1)^3 lattice, in the reference order
# (H20:349-353): 8 corners, 4 bottom mid-edges, 4 top mid-edges, 4 vertical mid-edges.
HEX20_OFFSETS = np.array([
    (0, 0, 0), (2, 0, 0), (2, 2, 0), (0, 2, 0),
    (0, 0, 2), (2, 0, 2), (2, 2, 2), (0, 2, 2),
    (1, 0, 0), (2, 1, 0), (1, 2, 0), (0, 1, 0),
    (1, 0, 2), (2, 1, 2), (1, 2, 2), (0, 1, 2),
    (0, 0, 1), (2, 0, 1), (2, 2, 1), (0, 2, 1)], dtype=np.int64)


def hex20_shape_derivs(xi: float, eta: float, zeta: float) -> np.ndarray:
    """dN/d(xi,eta,zeta) [3,20] of the serendipity Hex20 (formulas of H20:95-128)."""
    xn = np.array([-1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1, -1], float)
    yn = np.array([-1, -1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1], float)
    zn = np.array([-1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0], float)
    d = np.zeros((3, 20))
    for i in range(8):
        a, b, c = xn[i], yn[i], zn[i]
        d[0, i] = 0.125 * a * (1 + b * eta) * (1 + c * zeta) * (2 * a * xi + b * eta + c * zeta - 1)
        d[1, i] = 0.125 * b * (1 + a * xi) * (1 + c * zeta) * (a * xi + 2 * b * eta + c * zeta - 1)
        d[2, i] = 0.125 * c * (1 + a * xi) * (1 + b * eta) * (a * xi + b * eta + 2 * c * zeta - 1)
    for i in (8, 10, 12, 14):
        b, c = yn[i], zn[i]
        d[0, i] = -0.5 * xi * (1 + b * eta) * (1 + c * zeta)
        d[1, i] = 0.25 * b * (1 - xi * xi) * (1 + c * zeta)
        d[2, i] = 0.25 * c * (1 - xi * xi) * (1 + b * eta)
    for i in (9, 11, 13, 15):
        a, c = xn[i], zn[i]
        d[0, i] = 0.25 * a * (1 - eta * eta) * (1 + c * zeta)
        d[1, i] = -0.5 * eta * (1 + a * xi) * (1 + c * zeta)
        d[2, i] = 0.25 * c * (1 + a * xi) * (1 - eta * eta)
    for i in (16, 17, 18, 19):
        a, b = xn[i], yn[i]
        d[0, i] = 0.25 * a * (1 + b * eta) * (1 - zeta * zeta)
        d[1, i] = 0.25 * b * (1 + a * xi) * (1 - zeta * zeta)
        d[2, i] = -0.5 * zeta * (1 + a * xi) * (1 + b * eta)
    return d


def hex20_grid(nx: int = 64, ny: Optional[int] = None, nz: Optional[int] = None, *,
               jitter: float = 0.05, seed: int = 4, E: float = 1.0, nu: float = 0.3,
               lx: float = 1.0, ly: float = 1.0, lz: float = 1.0,
               compact: bool = True) -> Mesh:
    """Hex20 serendipity mesh of an nx*ny*nz box (H20:324-362).

    With ``compact`` only lattice points used by some element are nodes (corners
    and mid-edge points), numbered in the reference lattice order; otherwise the
    full (2n+1)^3 lattice of the reference is kept (orphan nodes included).
    All non-boundary nodes are jittered by U(+-jitter*h) per coordinate."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    rng = np.random.default_rng(seed)
    Lx, Ly, Lz = 2 * nx + 1, 2 * ny + 1, 2 * nz + 1
    k, j, i = np.meshgrid(np.arange(Lz), np.arange(Ly), np.arange(Lx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    odd = (i & 1) + (j & 1) + (k & 1)
    used = odd <= 1 if compact else np.ones(i.shape[0], dtype=bool)
    lattice_to_node = np.full(i.shape[0], -1, dtype=np.int64)
    lattice_to_node[used] = np.arange(int(used.sum()))
    x0 = i[used] * 0.5 * lx / nx
    y0 = j[used] * 0.5 * ly / ny
    z0 = k[used] * 0.5 * lz / nz
    ii, jj, kk = i[used], j[used], k[used]
    boundary = (ii == 0) | (ii == Lx - 1) | (jj == 0) | (jj == Ly - 1) | (kk == 0) | (kk == Lz - 1)
    ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    bx, by, bz = 2 * ex.ravel(), 2 * ey.ravel(), 2 * ez.ravel()
    lat = ((bz[:, None] + HEX20_OFFSETS[None, :, 2]) * (Lx * Ly)
           + (by[:, None] + HEX20_OFFSETS[None, :, 1]) * Lx
           + (bx[:, None] + HEX20_OFFSETS[None, :, 0]))
    conn = lattice_to_node[lat].astype(np.int32)
    assert conn.min() >= 0
    h = min(lx / nx, ly / ny, lz / nz)
    amp = jitter * h
    interior = ~boundary
    d = rng.uniform(-amp, amp, size=(3, x0.shape[0])) * interior
    x, y, z = x0 + d[0], y0 + d[1], z0 + d[2]
    mesh = Mesh(HEX20, x, y, z, np.ascontiguousarray(conn), None, None, None, E0=E, nu0=nu,
                thickness=1.0, name=f"hex20_{nx}x{ny}x{nz}", seed=seed)
    if hex20_min_detj(mesh) <= 0:
        raise RuntimeError("Hex20 jitter produced a non-positive Jacobian")
    return mesh


def hex20_min_detj(mesh: Mesh, chunk: int = 1 << 16) -> float:
    """Minimum detJ over all 27 Gauss points of all Hex20 elements."""
    g = (-_G3, 0.0, _G3)
    dn = np.stack([hex20_shape_derivs(a, b, c) for a in g for b in g for c in g])  # [27,3,20]
    out = np.inf
    for s in range(0, mesh.num_elems, chunk):
        cn = mesh.conn[s:s + chunk]
        X = np.stack([mesh.x[cn], mesh.y[cn], mesh.z[cn]], axis=-1)          # [e,20,3]
        J = np.einsum("gan,enb->egab", dn, X)                                   # [e,27,3,3]
        out = min(out, float(np.linalg.det(J).min()))
    return out


def min_detj(mesh: Mesh) -> float:
    if mesh.kind == HEX20:
        return hex20_min_detj(mesh)
    if mesh.kind == Q4:
        return _q4_detj_min(mesh.x, mesh.y, mesh.conn)
    if mesh.kind == T3:
        return float(_t3_detj(mesh.x, mesh.y, mesh.conn).min())
    t = mesh.types == T3
    a = float(_t3_detj(mesh.x, mesh.y, mesh.conn[t][:, :3]).min()) if t.any() else np.inf
    b = _q4_detj_min(mesh.x, mesh.y, mesh.conn[~t]) if (~t).any() else np.inf
    return min(a, b)


def batch_meshes(n: int = 256, *, seed: int = 5, emin: int = 1000, emax: int = 200_000,
                 kinds=("q4", "t3", "mixed", "hex20")) -> list:
    """The batched configuration: n independent meshes, kind drawn uniformly
    from `kinds`, element count log-uniform over [emin, emax] (the grid is the
    nearest box of that many elements), jitter and material distributions of
    each kind's own generator, one seed per mesh."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = kinds[int(rng.integers(len(kinds)))]
        target = float(np.exp(rng.uniform(np.log(emin), np.log(emax))))
        s = int(rng.integers(1 << 30))
        if kind == "q4":
            nx = max(1, int(round(np.sqrt(target))))
            m = q4_grid(nx, nx, seed=s)
        elif kind == "t3":
            nx = max(1, int(round(np.sqrt(target / 2))))
            m = t3_grid(nx, nx, seed=s)
        elif kind == "mixed":
            nx = max(1, int(round(np.sqrt(target / 1.5))))
            m = mixed_grid(nx, nx, seed=s)
        else:
            nx = max(1, int(round(np.cbrt(target))))
            m = hex20_grid(nx, seed=s)
        m.name = f"batch{i}_{m.name}"
        out.append(m)
    return out


def by_name(name: str) -> Mesh:
    """The benchmark meshes by short name ('q4', 't3', 'mixed', 'hex20') and a few
    small variants used in tests ('q4_small', ...)."""
    table = {
        "q4": lambda: q4_grid(100, 100),
        "t3": lambda: t3_grid(1000, 1000),
        "mixed": lambda: mixed_grid(1500, 1500),
        "hex20": lambda: hex20_grid(64),
        "q4_small": lambda: q4_grid(12, 9, seed=11),
        "t3_small": lambda: t3_grid(13, 10, seed=12),
        "mixed_small": lambda: mixed_grid(11, 14, seed=13),
        "hex20_small": lambda: hex20_grid(3, 4, 2, seed=14),
    }
    return table[name]()
