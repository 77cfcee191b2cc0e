"""Seeded synthetic sparse systems in Seldon's CSR layout (numpy, host side).

Every generator returns ``(ptr, ind, val)`` as int32/int32/float64 arrays with
0-based indices and columns sorted inside each row, the layout of
``Matrix<double, General, RowSparse>`` (``ptr_``, ``ind_``, ``data_``).
``upper()`` turns a symmetric full CSR into the upper-triangle storage of
``Matrix<double, Symmetric, RowSymSparse>``.

Workloads (sizes follow the configurations the path is measured on):
  lap2d(g)          2D 5-point Laplacian, diag 4, off -1, Dirichlet (g^2 rows)
  poisson3d(g)      3D 7-point Poisson, diag 6, off -1 (g^3 rows)
  convdiff3d(g)     3D 7-point first-order upwind convection-diffusion
  zipf_csr(n)       random nonsymmetric CSR with Zipf(1.5) row lengths
  aniso2d(g, theta) 2D weighted graph Laplacian + 1e-3 I (per-edge weights)
"""
import numpy as np


def _stencil_csr(dims, offsets, coefs, diag):
    """CSR of a constant-coefficient stencil on a box grid (x fastest).

    offsets: list of (dx, dy, dz) neighbour offsets; coefs: their values
    (scalars); diag: diagonal value.  Entries are emitted in increasing
    column order, neighbours outside the box are dropped (Dirichlet)."""
    dims = list(dims) + [1] * (3 - len(dims))
    gx, gy, gz = dims
    n = gx * gy * gz
    idx = np.arange(n, dtype=np.int64)
    ix = idx % gx
    iy = (idx // gx) % gy
    iz = idx // (gx * gy)
    entries = [((0, 0, 0), float(diag))] + list(zip(offsets, coefs))
    # column offset of each entry, used to order the row
    stride = lambda o: o[0] + o[1] * gx + o[2] * gx * gy  # noqa: E731
    entries.sort(key=lambda e: stride(e[0]))
    cols = np.empty((n, len(entries)), dtype=np.int64)
    vals = np.empty((n, len(entries)), dtype=np.float64)
    valid = np.empty((n, len(entries)), dtype=bool)
    for k, (o, c) in enumerate(entries):
        ok = ((ix + o[0] >= 0) & (ix + o[0] < gx) & (iy + o[1] >= 0) & (iy + o[1] < gy)
              & (iz + o[2] >= 0) & (iz + o[2] < gz))
        valid[:, k] = ok
        cols[:, k] = idx + stride(o)
        vals[:, k] = c
    counts = valid.sum(axis=1)
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    ind = cols[valid].astype(np.int32)
    val = vals[valid]
    return ptr.astype(np.int32), ind, val


def lap2d(g, shift=0.0):
    """2D 5-point Laplacian on a g x g grid: diag 4 (+shift), off-diagonal -1."""
    offs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0)]
    return _stencil_csr((g, g), offs, [-1.0] * 4, 4.0 + shift)


def poisson3d(g):
    """3D 7-point Poisson on a g^3 grid: diag 6, off-diagonal -1 (SPD)."""
    offs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    return _stencil_csr((g, g, g), offs, [-1.0] * 6, 6.0)


def convdiff3d(g, velocity=(1.0, 0.5, 0.25), peclet=10.0):
    """3D 7-point first-order upwind convection-diffusion on the unit cube.

    -eps*Lap(u) + v.grad(u) on a g^3 interior grid, h = 1/(g+1), Dirichlet.
    The global Peclet number is |v| * L / eps with L = 1, so
    eps = |v| / peclet.  Rows are scaled by h^2: diagonal
    6*eps + h*(|vx|+|vy|+|vz|), downstream neighbours -eps, upstream
    neighbours -eps - h*|v_d| (nonsymmetric M-matrix)."""
    v = np.asarray(velocity, dtype=np.float64)
    eps = float(np.linalg.norm(v)) / peclet
    h = 1.0 / (g + 1)
    offs, coefs = [], []
    for d in range(3):
        e = [0, 0, 0]
        e[d] = -1
        up_lo = v[d] > 0  # flow in +d: the upstream neighbour is at -1
        offs.append(tuple(e))
        coefs.append(-eps - (h * abs(v[d]) if up_lo else 0.0))
        e = [0, 0, 0]
        e[d] = 1
        offs.append(tuple(e))
        coefs.append(-eps - (0.0 if up_lo else h * abs(v[d])))
    diag = 6.0 * eps + h * float(np.abs(v).sum())
    return _stencil_csr((g, g, g), offs, coefs, diag)


def zipf_csr(n, seed=0, a=1.5, lo=1, hi=2000):
    """Random nonsymmetric CSR: row lengths Zipf(a) clipped to [lo, hi],
    uniform column indices (deduplicated, sorted), values N(0,1), diagonal
    set to 1 + sum|row| (inserted where absent)."""
    rng = np.random.default_rng(seed)
    lens = np.clip(rng.zipf(a, n), lo, hi).astype(np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = rng.integers(0, n, rows.size, dtype=np.int64)
    keys = rows * n + cols
    keys = keys[rows != cols]
    # sorted distinct keys: an in-place sort and a neighbour test (the same
    # array np.unique gives, without its cost on tens of millions of keys)
    keys.sort()
    if keys.size:
        first = np.empty(keys.size, dtype=bool)
        first[0] = True
        np.not_equal(keys[1:], keys[:-1], out=first[1:])
        keys = keys[first]
    r = keys // n
    c = keys % n
    v = rng.standard_normal(keys.size)
    absum = np.bincount(r, weights=np.abs(v), minlength=n)
    # the diagonal entries merged in column order (no off-diagonal key equals
    # a diagonal one)
    dkeys = np.arange(n, dtype=np.int64) * (n + 1)
    at = np.searchsorted(keys, dkeys)
    allk = np.insert(keys, at, dkeys)
    allv = np.insert(v, at, 1.0 + absum)
    r = allk // n
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=ptr[1:])
    return ptr.astype(np.int32), (allk % n).astype(np.int32), allv


def grid_edges(g):
    """Edges (i, j), i < j, of the g x g grid graph (x fastest)."""
    idx = np.arange(g * g, dtype=np.int64).reshape(g, g)
    h = np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], axis=1)
    v = np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], axis=1)
    return np.concatenate([h, v], axis=0)


def aniso2d(g, theta, shift=1e-3):
    """Weighted graph Laplacian of the g x g grid plus shift*I.

    theta: per-edge conductivity, ordered as grid_edges(g).  A_ii =
    sum of incident theta + shift, A_ij = -theta_e.  Returns the full CSR and
    a map `edge_pos` (2, E) giving the positions of A_ij and A_ji in val."""
    n = g * g
    e = grid_edges(g)
    th = np.asarray(theta, dtype=np.float64)
    rows = np.concatenate([e[:, 0], e[:, 1], np.arange(n)])
    cols = np.concatenate([e[:, 1], e[:, 0], np.arange(n)])
    deg = np.bincount(e[:, 0], weights=th, minlength=n) + np.bincount(e[:, 1], weights=th, minlength=n)
    vals = np.concatenate([-th, -th, deg + shift])
    keys = rows * n + cols
    order = np.argsort(keys, kind="stable")
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=ptr[1:])
    inv = np.empty_like(order)
    inv[order] = np.arange(order.size)
    E = e.shape[0]
    edge_pos = np.stack([inv[:E], inv[E:2 * E]])
    return ptr.astype(np.int32), cols[order].astype(np.int32), vals[order], edge_pos


def upper(ptr, ind, val):
    """Upper triangle (diagonal included) of a full CSR: RowSymSparse storage."""
    ptr = np.asarray(ptr, dtype=np.int64)
    rows = np.repeat(np.arange(ptr.size - 1, dtype=np.int64), np.diff(ptr))
    keep = ind >= rows
    uptr = np.zeros_like(ptr)
    np.cumsum(np.bincount(rows[keep], minlength=ptr.size - 1), out=uptr[1:])
    return uptr.astype(np.int32), np.ascontiguousarray(ind[keep]), np.ascontiguousarray(val[keep])


def random_csr(m, n, density, seed=0, dtype=np.float64, empty_rows=0.0):
    """Small random CSR for tests: uniform pattern, N(0,1) values; a fraction
    `empty_rows` of the rows is left empty."""
    rng = np.random.default_rng(seed)
    mask = rng.random((m, n)) < density
    if empty_rows > 0:
        mask[rng.random(m) < empty_rows, :] = False
    r, c = np.nonzero(mask)
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=m), out=ptr[1:])
    return ptr.astype(np.int32), c.astype(np.int32), rng.standard_normal(r.size).astype(dtype)


def matvec(ptr, ind, val, x):
    """y = A x for a full CSR (numpy, vectorised; used to build b = A x*)."""
    ptr = np.asarray(ptr, dtype=np.int64)
    rows = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
    return np.bincount(rows, weights=val * x[ind], minlength=ptr.size - 1)
