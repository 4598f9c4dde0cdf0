"""Deterministic generators for the FE-assembled systems the PCG path solves.

HiFlow3 assembles these matrices through its FE stack (mesh -> dof -> fem ->
assembly, out of scope here); this module restates the matrices that stack
produces for bilinear/trilinear (Q1) elements on uniform grids, so that the
solver path can be fed identical systems on the CPU oracle and on the GPU:

* element stiffness of -div(kappa grad u) on one cell, by Hamming distance of
  the two local nodes: 2D [2/3, -1/6, -1/3]; 3D h*[1/3, 0, -1/12, -1/12];
  a global entry is the element entry times the sum of kappa over the cells
  that hold both nodes (exact 2x2(x2) Gauss integration of Q1 gradients);
* homogeneous Dirichlet rows as produced by CoupledMatrix::diagonalize_rows
  -> CPU_CSR_lMatrix::ZeroRows (linear_algebra/coupled_matrix.cc:452-477,
  lmp/lmatrix_csr_cpu.cc:908-927): a boundary row keeps its full sparsity
  pattern, 1 on the diagonal and stored zeros elsewhere; columns are not
  zeroed (set_constraint_rows_to_identity, assembly/all_assembly.h:478-498);
* lexicographic DOF numbering, x fastest, so rows are banded and every row's
  column indices ascend.

Random inputs use a counter-based splitmix64 stream (Steele, Lea & Flood,
"Fast splittable pseudorandom number generators", OOPSLA 2014), so a given
(seed, index) maps to the same value in any implementation.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)

# Fixed seeds of the standard workloads.
SEED_POISSON_2D = 20240601
SEED_POISSON_3D = 20240602
SEED_VARCOEF_3D = 20240603
SEED_BATCH = 20240604
SEED_SERVE = 20240605


def splitmix64(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """splitmix64 output for indices 0..count-1 of (seed, stream)."""
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 0x100000001B3 + stream * 0x51_7CC1_B727_220A_95) % (1 << 64))
        z = base + (np.arange(1, count + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """Doubles in [0, 1) from the top 53 bits of splitmix64."""
    return (splitmix64(seed, count, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def standard_normal(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """N(0,1) samples by the Box-Muller transform of two uniform streams."""
    u1 = uniform01(seed, count, 2 * stream + 1)
    u2 = uniform01(seed, count, 2 * stream + 2)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * math.pi * u2)


@dataclass
class CSRSystem:
    """One assembled system A x = b in CSR (int32 indices, float64 values)."""

    dim: int
    cells: int
    rowptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    b: np.ndarray
    boundary: np.ndarray  # bool per row: Dirichlet row
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.rowptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])


def _assemble(dim: int, n: int, kappa: np.ndarray | None) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """Q1 stiffness on an n^dim cell grid with Dirichlet identity rows."""
    m = n + 1  # nodes per axis
    h = 1.0 / n
    if dim == 2:
        elem = {0: 2.0 / 3.0, 1: -1.0 / 6.0, 2: -1.0 / 3.0}
    else:
        elem = {0: h / 3.0, 1: 0.0, 2: -h / 12.0, 3: -h / 12.0}
    shape_nodes = (m,) * dim
    shape_cells = (n,) * dim
    if kappa is None:
        kappa = np.ones(shape_cells, dtype=np.float64)
    kappa = np.asarray(kappa, dtype=np.float64).reshape(shape_cells)
    # kappa padded by one zero cell on each side: cell c sits at index c+1.
    kp = np.zeros((n + 2,) * dim, dtype=np.float64)
    kp[(slice(1, n + 1),) * dim] = kappa

    # offsets in ascending linear order (slowest axis first in the tuple).
    offs = [o for o in np.ndindex(*((3,) * dim))]
    offs = [tuple(int(v) - 1 for v in o) for o in offs]  # (d_slow, ..., d_x)
    N = m**dim
    idx = np.indices(shape_nodes, dtype=np.int32)  # idx[0] slowest axis
    boundary = np.zeros(shape_nodes, dtype=bool)
    for a in range(dim):
        boundary |= (idx[a] == 0) | (idx[a] == m - 1)
    strides = [m ** (dim - 1 - a) for a in range(dim)]

    cols = np.empty((N, len(offs)), dtype=np.int32)
    vals = np.empty((N, len(offs)), dtype=np.float64)
    mask = np.empty((N, len(offs)), dtype=bool)
    lin = np.arange(N, dtype=np.int64).reshape(shape_nodes)
    for k, d in enumerate(offs):
        ok = np.ones(shape_nodes, dtype=bool)
        for a in range(dim):
            if d[a] == -1:
                ok &= idx[a] >= 1
            elif d[a] == 1:
                ok &= idx[a] <= m - 2
        off_lin = sum(d[a] * strides[a] for a in range(dim))
        # sum of kappa over the cells holding node p and node p+d: per axis,
        # cell start c in {p-1, p} if d=0, {p} if d=+1, {p-1} if d=-1.
        choices = [((-1, 0) if d[a] == 0 else ((0,) if d[a] == 1 else (-1,))) for a in range(dim)]
        ksum = np.zeros(shape_nodes, dtype=np.float64)
        for cs in np.ndindex(*[len(c) for c in choices]):
            sl = tuple(slice(1 + choices[a][cs[a]], 1 + choices[a][cs[a]] + m) for a in range(dim))
            ksum += kp[sl]
        ham = sum(1 for v in d if v != 0)
        v = elem[ham] * ksum
        if ham == 0:
            v = np.where(boundary, 1.0, v)
        else:
            v = np.where(boundary, 0.0, v)
        cols[:, k] = (lin + off_lin).reshape(-1).astype(np.int32)
        vals[:, k] = v.reshape(-1)
        mask[:, k] = ok.reshape(-1)
    counts = mask.sum(axis=1)
    rowptr = np.zeros(N + 1, dtype=np.int32)
    np.cumsum(counts, out=rowptr[1:])
    col = cols[mask]
    val = vals[mask]
    # a stored +0.0 for face couplings in 3D stays stored, as in the reference
    return rowptr, col.astype(np.int32), val.astype(np.float64), boundary.reshape(-1)


def q1_system(dim: int, n: int, seed: int, sigma: float = 0.0, name: str = "") -> CSRSystem:
    """Q1 diffusion on the unit square/cube, n cells per axis.

    sigma == 0 gives the Poisson matrix; sigma > 0 a per-cell coefficient
    kappa = exp(sigma * g), g ~ N(0,1) from the seed.  RHS: U[0,1) on interior
    rows, 0 on Dirichlet rows (x0 = 0 is the start vector)."""
    kappa = None
    if sigma > 0.0:
        kappa = np.exp(sigma * standard_normal(seed, n**dim, stream=7))
    rowptr, col, val, boundary = _assemble(dim, n, kappa)
    N = rowptr.shape[0] - 1
    b = uniform01(seed, N, stream=3)
    b[boundary] = 0.0
    return CSRSystem(dim, n, rowptr, col, val, b, boundary, name or f"q1_{dim}d_{n}",
                     {"seed": seed, "sigma": sigma})


def poisson_2d(n: int = 256, seed: int = SEED_POISSON_2D) -> CSRSystem:
    """2D Q1 Poisson, n x n cells: (n+1)^2 DOFs, 9-point rows."""
    return q1_system(2, n, seed, 0.0, f"poisson2d_{n}")


def poisson_3d(n: int = 128, seed: int = SEED_POISSON_3D) -> CSRSystem:
    """3D Q1 Poisson, n^3 cells: (n+1)^3 DOFs, 27-point rows."""
    return q1_system(3, n, seed, 0.0, f"poisson3d_{n}")


def varcoef_3d(n: int = 128, sigma: float = 2.0, seed: int = SEED_VARCOEF_3D) -> CSRSystem:
    """3D Q1 diffusion with lognormal per-cell coefficient exp(sigma*g)."""
    return q1_system(3, n, seed, sigma, f"varcoef3d_{n}_s{sigma:g}")


def batch_sizes(count: int = 1024, lo: int = 16, hi: int = 256, seed: int = SEED_BATCH) -> np.ndarray:
    """Cells per axis n ~ round(exp(U[ln lo, ln hi])) for a batch of 2D systems."""
    u = uniform01(seed, count, stream=11)
    return np.rint(np.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))).astype(np.int64)


def batch_systems(count: int = 1024, sigma: float = 1.0, seed: int = SEED_BATCH,
                  lo: int = 16, hi: int = 256) -> list[CSRSystem]:
    """The batched workload: independent 2D Q1 systems of uneven size with a
    lognormal (sigma) per-cell coefficient; system k uses seed + k."""
    sizes = batch_sizes(count, lo, hi, seed)
    return [q1_system(2, int(n), seed + 1 + k, sigma, f"batch{k}_n{int(n)}") for k, n in enumerate(sizes)]


def stratified_sample(sizes, m: int) -> list[int]:
    """Indices of m items spread evenly over the items ranked by size (the
    middle item of each of m equal-count strata), in ascending index order:
    a fixed sample whose mean cost tracks the whole set's."""
    order = sorted(range(len(sizes)), key=lambda i: (int(sizes[i]), i))
    m = min(int(m), len(order))
    return sorted(order[int((j + 0.5) * len(order) / m)] for j in range(m))


# Solution fingerprints: comparing solutions of multi-million-row systems
# without storing them.
PROBE_SEED = 20240610
PROBE_VECTORS = 64
PROBE_SAMPLES = 2048


def solution_probe(x) -> dict:
    """Fingerprint of a solution vector: its 2-norm, its projections on
    PROBE_VECTORS seeded Rademacher (+-1) vectors and its values at
    PROBE_SAMPLES seeded positions.  For e = x - y and Rademacher v,
    E[(e.v)^2] = ||e||^2, so probe_error() estimates ||x - y|| / ||y|| from
    two fingerprints alone (64 draws: within about +-20%)."""
    x = np.ascontiguousarray(x, np.float64)
    n = x.shape[0]
    proj = []
    for k in range(PROBE_VECTORS):
        v = 1.0 - 2.0 * (splitmix64(PROBE_SEED, n, stream=100 + k) >> np.uint64(63)).astype(np.float64)
        proj.append(float(np.sum(x * v)))  # pairwise summation
    idx = (splitmix64(PROBE_SEED, PROBE_SAMPLES, stream=99) % np.uint64(n)).astype(np.int64)
    return {"n": int(n), "norm": float(np.linalg.norm(x)), "proj": proj, "sample": x[idx].tolist()}


def probe_error(got: dict, ref: dict) -> dict:
    """Relative error of a solution against a reference solution, from their
    fingerprints: `proj` = sqrt(mean (p_got - p_ref)^2) / ||x_ref|| (an
    unbiased estimate of ||x_got - x_ref||^2 under the square root), `sample`
    = the same estimate from the sampled entries, `max_sample` = the largest
    sampled |x_got - x_ref| over the largest sampled |x_ref|."""
    if got["n"] != ref["n"]:
        raise ValueError("fingerprints of different sizes")
    dp = np.asarray(got["proj"]) - np.asarray(ref["proj"])
    ds = np.asarray(got["sample"]) - np.asarray(ref["sample"])
    m = ds.shape[0]
    return {"proj": float(np.sqrt(np.mean(dp * dp)) / ref["norm"]),
            "sample": float(np.sqrt(ref["n"] / m * np.sum(ds * ds)) / ref["norm"]),
            "max_sample": float(np.max(np.abs(ds)) / max(np.max(np.abs(ref["sample"])), 1e-300))}


def serve_stream(count: int = 20000, rate: float = 100.0, lo_dofs: float = 1e3, hi_dofs: float = 2e6,
                 seed: int = SEED_SERVE) -> list[dict]:
    """The served workload: `count` Q1 diffusion solve requests arriving as a
    Poisson process of `rate` requests/s.  Each request is 2D or 3D (equal
    odds), has a DOF count log-uniform in [lo_dofs, hi_dofs] (cells per axis
    rounded from it, at least 1), a lognormal coefficient with sigma uniform
    in [0.5, 2], and its own seed.  Returns dicts with keys
    t (arrival, s), dim, cells, dofs, sigma, seed."""
    u_dim = uniform01(seed, count, stream=21)
    u_dofs = uniform01(seed, count, stream=22)
    u_sig = uniform01(seed, count, stream=23)
    u_gap = uniform01(seed, count, stream=24)
    gaps = -np.log1p(-u_gap) / rate
    t = np.cumsum(gaps) - gaps[0]
    out = []
    for k in range(count):
        dim = 2 if u_dim[k] < 0.5 else 3
        dofs = math.exp(math.log(lo_dofs) + u_dofs[k] * (math.log(hi_dofs) - math.log(lo_dofs)))
        cells = max(1, int(round(dofs ** (1.0 / dim))) - 1)
        out.append(dict(t=float(t[k]), dim=dim, cells=cells, dofs=(cells + 1) ** dim,
                        sigma=0.5 + 1.5 * float(u_sig[k]), seed=seed + 1 + k))
    return out


def known_answer_3x3() -> CSRSystem:
    """tests/cg_test.cc:44-94: [[2,-1,0],[-1,2,-1],[0,-1,2]] x = (1,-2,0),
    all 9 entries stored (explicit zeros), answer (-0.25, -1.5, -0.75)."""
    rowptr = np.array([0, 3, 6, 9], dtype=np.int32)
    col = np.array([0, 1, 2, 0, 1, 2, 0, 1, 2], dtype=np.int32)
    val = np.array([2, -1, 0, -1, 2, -1, 0, -1, 2], dtype=np.float64)
    b = np.array([1.0, -2.0, 0.0])
    return CSRSystem(0, 0, rowptr, col, val, b, np.zeros(3, dtype=bool), "cg_test_3x3")


def lmp_test_3x3() -> CSRSystem:
    """tests/lmp_test.cc:52-61: the same stencil with only its 7 nonzeros."""
    rowptr = np.array([0, 2, 5, 7], dtype=np.int32)
    col = np.array([0, 1, 0, 1, 2, 1, 2], dtype=np.int32)
    val = np.array([2, -1, -1, 2, -1, -1, 2], dtype=np.float64)
    b = np.array([1.0, -2.0, 0.0])
    return CSRSystem(0, 0, rowptr, col, val, b, np.zeros(3, dtype=bool), "lmp_test_3x3")


def convdiff_2d(n: int, peclet: float = 20.0, seed: int = 7, name: str = "") -> CSRSystem:
    """Non-symmetric test system for BiCGSTAB and Jacobi: -lap u + beta.grad u
    on the n x n interior nodes of the unit square (h = 1/(n+1), Dirichlet
    nodes eliminated), 5-point diffusion and first-order upwind convection,
    scaled by h^2, beta = peclet (cos 0.3, sin 0.3).  The matrix is an
    M-matrix (diagonally dominant, strictly in rows next to the boundary);
    columns ascend within each row; b ~ U[0,1) from the seed's stream 0."""
    h = 1.0 / (n + 1)
    bx, by = peclet * np.cos(0.3), peclet * np.sin(0.3)
    ix, iy = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    ix, iy = ix.ravel(), iy.ravel()
    N = n * n
    rows = np.arange(N)
    # (offset, coefficient, neighbour exists) in ascending column order
    nb = [(-n, -1.0 - h * max(by, 0.0), iy > 0), (-1, -1.0 - h * max(bx, 0.0), ix > 0),
          (0, 4.0 + h * (abs(bx) + abs(by)), np.ones(N, bool)),
          (1, -1.0 + h * min(bx, 0.0), ix < n - 1), (n, -1.0 + h * min(by, 0.0), iy < n - 1)]
    cnt = sum(m.astype(np.int32) for _, _, m in nb)
    rowptr = np.zeros(N + 1, dtype=np.int32)
    np.cumsum(cnt, out=rowptr[1:])
    col = np.empty(rowptr[-1], dtype=np.int32)
    val = np.empty(rowptr[-1], dtype=np.float64)
    pos = rowptr[:-1].copy()
    for off, c, m in nb:
        r = rows[m]
        col[pos[m]] = r + off
        val[pos[m]] = c
        pos[m] += 1
    b = uniform01(seed, N, stream=0)
    return CSRSystem(2, n, rowptr, col, val, b, np.zeros(N, dtype=bool), name or f"convdiff2d_{n}_pe{peclet:g}")


def random_spd(n: int, seed: int, density: float = 0.1, empty_rows: int = 0) -> CSRSystem:
    """Small random symmetric diagonally dominant matrix (ragged rows) for
    edge-case parity: the first `empty_rows` rows hold only their diagonal."""
    rng = np.random.default_rng(seed)
    a = np.zeros((n, n))
    m = rng.random((n, n)) < density
    m = m | m.T
    w = rng.standard_normal((n, n))
    w = (w + w.T) * 0.5
    a[m] = w[m]
    np.fill_diagonal(a, 0.0)
    a[:empty_rows, :] = 0.0
    a[:, :empty_rows] = 0.0
    np.fill_diagonal(a, np.abs(a).sum(axis=1) + 1.0 + rng.random(n))
    rows, cols = np.nonzero(a)
    rowptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(rows, minlength=n), out=rowptr[1:])
    b = rng.random(n)
    return CSRSystem(0, 0, rowptr, cols.astype(np.int32), a[rows, cols].astype(np.float64), b,
                     np.zeros(n, dtype=bool), f"random_spd_{n}")
