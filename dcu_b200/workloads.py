"""Seeded synthetic matrices for the SPAI + BiCGSTAB path.

Every generator returns a square matrix in CSC form (int32 column pointers,
int32 row indices ascending inside each column, float64 values), the layout
the reference reads into ``CSC_Matrix`` (include/common/dataType.h:33-41).
The reference measures on the MatrixMarket fixture ``matrices/circuit_2.mtx``
and on nothing else; these generators stand in for its workloads:

* :func:`convdiff2d`   2D 5-point upwind convection-diffusion (64x64, Pe 10)
* :func:`convdiff3d`   3D 7-point upwind convection-diffusion (128^3, Pe 20)
* :func:`circuit_like` seeded power-law "circuit" matrix shaped like
  circuit_2 (n = 4510, ~21.2k nonzeros, hub rows and columns)
* :func:`varcoef2d`    2D variable-coefficient diffusion, kappa = exp(GRF)
* :func:`batch_systems` 512 independent stencil systems of uneven size

Ordering of grid unknowns is natural with x fastest: k = (z*m + y)*m + x.
Upwinding is along +x: row k couples to its west neighbour k-1 with
-(1 + Pe) and to its east neighbour k+1 with -1.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class CSC:
    """Square sparse matrix in compressed sparse column form."""

    n: int
    ptr: np.ndarray  # int32 [n+1]
    idx: np.ndarray  # int32 [nnz] row indices
    val: np.ndarray  # float64 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.ptr[-1])

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x (float64, numpy; test helper)."""
        y = np.zeros(self.n, dtype=np.float64)
        cols = np.repeat(np.arange(self.n), np.diff(self.ptr))
        np.add.at(y, self.idx, self.val * x[cols])
        return y

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csc_matrix((self.val, self.idx, self.ptr), shape=(self.n, self.n))


def _from_stencil(n: int, rows: np.ndarray, vals: np.ndarray) -> CSC:
    """Build CSC from per-column candidate rows [n, w] (-1 = absent), ascending."""
    valid = rows >= 0
    counts = valid.sum(axis=1).astype(np.int64)
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    idx = rows[valid].astype(np.int32)
    val = vals[valid].astype(np.float64)
    return CSC(n, ptr.astype(np.int32), idx, val)


def convdiff2d(m: int = 64, pe: float = 10.0) -> CSC:
    """2D 5-point upwind convection-diffusion on an m x m grid.

    a_kk = 4 + Pe, a_{k,k-1} = -(1 + Pe), a_{k,k+1} = -1, a_{k,k+-m} = -1,
    Dirichlet boundary (couplings leaving the grid are dropped).
    m = 64, Pe = 10 gives n = 4096, nnz = 20224.
    """
    n = m * m
    c = np.arange(n, dtype=np.int64)
    x = c % m
    # column c holds A(row, c); rows ascending: c-m, c-1, c, c+1, c+m
    rows = np.full((n, 5), -1, dtype=np.int64)
    vals = np.zeros((n, 5), dtype=np.float64)
    rows[:, 0] = np.where(c - m >= 0, c - m, -1); vals[:, 0] = -1.0          # a_{c-m, c}: north of row c-m
    rows[:, 1] = np.where(x >= 1, c - 1, -1); vals[:, 1] = -1.0               # a_{c-1, c}: east coupling of row c-1
    rows[:, 2] = c; vals[:, 2] = 4.0 + pe
    rows[:, 3] = np.where(x <= m - 2, c + 1, -1); vals[:, 3] = -(1.0 + pe)    # a_{c+1, c}: upwind coupling of row c+1
    rows[:, 4] = np.where(c + m < n, c + m, -1); vals[:, 4] = -1.0
    return _from_stencil(n, rows, vals)


def convdiff3d(m: int = 128, pe: float = 20.0) -> CSC:
    """3D 7-point upwind convection-diffusion on an m^3 grid.

    a_kk = 6 + Pe, a_{k,k-1} = -(1 + Pe), the other five couplings -1.
    m = 128, Pe = 20 gives n = 2,097,152, nnz = 14,581,760.
    """
    n = m * m * m
    m2 = m * m
    c = np.arange(n, dtype=np.int64)
    x = c % m
    y = (c // m) % m
    z = c // m2
    rows = np.full((n, 7), -1, dtype=np.int64)
    vals = np.full((n, 7), -1.0, dtype=np.float64)
    rows[:, 0] = np.where(z >= 1, c - m2, -1)
    rows[:, 1] = np.where(y >= 1, c - m, -1)
    rows[:, 2] = np.where(x >= 1, c - 1, -1)
    rows[:, 3] = c; vals[:, 3] = 6.0 + pe
    rows[:, 4] = np.where(x <= m - 2, c + 1, -1); vals[:, 4] = -(1.0 + pe)
    rows[:, 5] = np.where(y <= m - 2, c + m, -1)
    rows[:, 6] = np.where(z <= m - 2, c + m2, -1)
    return _from_stencil(n, rows, vals)


def convdiff(dim: int, m: int, pe: float) -> CSC:
    return convdiff2d(m, pe) if dim == 2 else convdiff3d(m, pe)


def circuit_like(n: int = 4510, seed: int = 2024, target_nnz: int = 21200, alpha: float = 2.1,
                 n_hubs: int = 8, hub_lo: int = 200, hub_hi: int = 400, deg_cap: int = 64,
                 min_mag: float = 0.1) -> CSC:
    """Seeded circuit-like unsymmetric matrix shaped like circuit_2.

    Construction (numpy PCG64(seed)):
      1. 8 hub rows and 8 hub columns (distinct random indices), each with
         U{hub_lo..hub_hi} off-diagonal entries at distinct random positions.
      2. Every row gets a power-law off-diagonal degree: Zipf(alpha) capped at
         deg_cap, min 1, then scaled so that the total reaches the nonzero
         budget target_nnz - n - (hub entries) (rounded, min 1).
      3. Off-diagonal values N(0,1) times a random sign, with magnitudes
         below ``min_mag`` redrawn (a row whose only entry is ~1e-5 would make
         the diagonal ~1e-5 too and leave a row scaled 1e-7 below its
         neighbours, which no right SPAI on A's pattern can correct);
         duplicates merged.
      4. Full diagonal a_ii = 1.1 * sum_{j != i} |a_ij|.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    ent_r, ent_c = [], []
    hub_rows = rng.choice(n, n_hubs, replace=False)
    hub_cols = rng.choice(n, n_hubs, replace=False)
    for r in hub_rows:
        d = int(rng.integers(hub_lo, hub_hi + 1))
        cols = rng.choice(n - 1, d, replace=False)
        cols = cols + (cols >= r)
        ent_r.append(np.full(d, r)); ent_c.append(cols)
    for cidx in hub_cols:
        d = int(rng.integers(hub_lo, hub_hi + 1))
        rows = rng.choice(n - 1, d, replace=False)
        rows = rows + (rows >= cidx)
        ent_r.append(rows); ent_c.append(np.full(d, cidx))
    hub_total = sum(len(a) for a in ent_r)
    budget = max(n, target_nnz - n - hub_total)
    deg = np.minimum(rng.zipf(alpha, n), deg_cap).astype(np.float64)
    deg = np.maximum(1, np.round(deg * budget / deg.sum())).astype(np.int64)
    for r in range(n):
        d = int(deg[r])
        cols = rng.choice(n - 1, d, replace=False)
        cols = cols + (cols >= r)
        ent_r.append(np.full(d, r)); ent_c.append(cols)
    R = np.concatenate(ent_r).astype(np.int64)
    C = np.concatenate(ent_c).astype(np.int64)
    key = np.unique(C * n + R)          # merge duplicates, column-major order
    C = key // n
    R = key % n
    V = rng.standard_normal(len(key))
    small = np.abs(V) < min_mag
    while small.any():
        V[small] = rng.standard_normal(int(small.sum()))
        small = np.abs(V) < min_mag
    V = V * rng.choice([-1.0, 1.0], len(key))
    rowabs = np.zeros(n)
    np.add.at(rowabs, R, np.abs(V))
    # insert the diagonal, keep rows ascending inside each column
    C = np.concatenate([C, np.arange(n)])
    R = np.concatenate([R, np.arange(n)])
    V = np.concatenate([V, 1.1 * rowabs])
    order = np.lexsort((R, C))
    C, R, V = C[order], R[order], V[order]
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ptr, C + 1, 1)
    ptr = np.cumsum(ptr)
    return CSC(n, ptr.astype(np.int32), R.astype(np.int32), V.astype(np.float64))


def gaussian_random_field(m: int, corr: float, seed: int) -> np.ndarray:
    """Stationary Gaussian field on an m x m periodic grid, unit variance,
    squared-exponential covariance with correlation length ``corr`` cells,
    made by FFT filtering of white noise."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal((m, m))
    k = np.fft.fftfreq(m) * 2.0 * np.pi
    kx, ky = np.meshgrid(k, k, indexing="ij")
    filt = np.exp(-0.25 * (kx ** 2 + ky ** 2) * corr ** 2)
    g = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    g -= g.mean()
    g /= g.std()
    return g


def varcoef2d(m: int = 512, seed: int = 5, corr: float = 16.0, adv: float = 0.05) -> CSC:
    """2D variable-coefficient diffusion with small upwind advection.

    kappa = exp(g), g a unit-variance Gaussian random field (correlation
    length ``corr`` cells).  Face coefficients are harmonic means of the two
    cells; a Dirichlet face uses the cell's own kappa.  Row k:
      a_kk = sum of its four face coefficients + adv,
      a_{k,nb} = -kappa_face (and -adv more on the west neighbour).
    m = 512 gives n = 262,144, nnz = 1,308,672.
    """
    kap = np.exp(gaussian_random_field(m, corr, seed))  # indexed [y, x]
    n = m * m
    c = np.arange(n, dtype=np.int64)
    x = c % m
    y = c // m
    K = kap.reshape(-1)

    def harm(a, b):
        return 2.0 * a * b / (a + b)

    # face coefficient of row r towards each neighbour
    def face(r, nb, valid):
        out = np.where(valid, harm(K[r], K[np.where(valid, nb, r)]), K[r])
        return out

    kw = face(c, c - 1, x >= 1)
    ke = face(c, c + 1, x <= m - 2)
    ks = face(c, c - m, y >= 1)
    kn = face(c, c + m, y <= m - 2)
    diag = kw + ke + ks + kn + adv
    # column c holds A(row, c) for rows c-m, c-1, c, c+1, c+m
    rows = np.full((n, 5), -1, dtype=np.int64)
    vals = np.zeros((n, 5), dtype=np.float64)
    # row c-m couples to c through its north face
    rows[:, 0] = np.where(y >= 1, c - m, -1)
    vals[:, 0] = np.where(y >= 1, -kn[np.maximum(c - m, 0)], 0.0)
    rows[:, 1] = np.where(x >= 1, c - 1, -1)
    vals[:, 1] = np.where(x >= 1, -ke[np.maximum(c - 1, 0)], 0.0)
    rows[:, 2] = c
    vals[:, 2] = diag
    rows[:, 3] = np.where(x <= m - 2, c + 1, -1)
    vals[:, 3] = np.where(x <= m - 2, -kw[np.minimum(c + 1, n - 1)] - adv, 0.0)
    rows[:, 4] = np.where(y <= m - 2, c + m, -1)
    vals[:, 4] = np.where(y <= m - 2, -ks[np.minimum(c + m, n - 1)], 0.0)
    return _from_stencil(n, rows, vals)


@dataclass
class Batch:
    """Independent systems assembled as one block-diagonal matrix."""

    A: CSC                 # block-diagonal matrix of all systems
    offsets: np.ndarray    # int64 [S+1] first unknown of each system
    dims: np.ndarray       # 2 or 3 per system
    pes: np.ndarray        # Peclet number per system
    B: np.ndarray          # float64 [N, nrhs] right-hand sides (rows follow A)


def batch_systems(count: int = 512, nrhs: int = 8, n_lo: float = 1e3, n_hi: float = 5e4,
                  seed: int = 3, pe_hi: float = 50.0) -> Batch:
    """``count`` stencil systems, n log-uniform in [n_lo, n_hi]; each is 2D
    5-point (m = round(sqrt n)) or 3D 7-point (m = round(cbrt n)) upwind
    convection-diffusion, 50/50 by seed, Pe ~ U[0, pe_hi]; ``nrhs``
    right-hand sides per system ~ U[-1, 1]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), count))
    dims = np.where(rng.uniform(size=count) < 0.5, 2, 3)
    pes = rng.uniform(0.0, pe_hi, count)
    ptrs, idxs, vals, offs = [], [], [], [0]
    base_nnz = 0
    for s in range(count):
        if dims[s] == 2:
            m = max(2, int(round(np.sqrt(ns[s]))))
            A = convdiff2d(m, pes[s])
        else:
            m = max(2, int(round(np.cbrt(ns[s]))))
            A = convdiff3d(m, pes[s])
        ptrs.append((A.ptr[:-1].astype(np.int64) + base_nnz))
        idxs.append(A.idx.astype(np.int64) + offs[-1])
        vals.append(A.val)
        base_nnz += A.nnz
        offs.append(offs[-1] + A.n)
    N = offs[-1]
    ptr = np.concatenate(ptrs + [np.array([base_nnz])]).astype(np.int32)
    big = CSC(N, ptr, np.concatenate(idxs).astype(np.int32), np.concatenate(vals))
    B = rng.uniform(-1.0, 1.0, (N, nrhs))
    return Batch(big, np.array(offs, dtype=np.int64), dims, pes, B)


def rhs_ones_product(A: CSC) -> np.ndarray:
    """b = A * ones (the right-hand side of the convection-diffusion configs)."""
    return A.matvec(np.ones(A.n))


def rhs_from_solution(A: CSC, seed: int = 7):
    """x_true ~ N(0,1) (seeded) and b = A x_true."""
    rng = np.random.Generator(np.random.PCG64(seed))
    xt = rng.standard_normal(A.n)
    return A.matvec(xt), xt
