"""Synthetic particle states for the tests (reference checkpoint layout)."""
import numpy as np

from cube_nu_b200.params import Params


def cell_order(p: Params, cell):
    """Storage index of global coarse cells (N,3) in the reference order."""
    nt, nnt = p.nt, p.nnt
    cell = np.asarray(cell) % p.nc
    t = cell // nt
    l = cell - t * nt
    return ((((t[:, 2] * nnt + t[:, 1]) * nnt + t[:, 0]) * nt + l[:, 2]) * nt + l[:, 1]) * nt + l[:, 0]


def state_from_positions(p: Params, X, V, pid=None):
    """Encode global coarse-unit positions X (N,3) into (xp, vp, pid, rhoc) sorted by cell
    (arrival order = input order)."""
    X = np.mod(np.asarray(X, dtype=np.float64), p.nc)
    cell = np.floor(X).astype(np.int64)
    mod = 1 << (8 * p.izipx)
    code = np.floor((X - cell) * mod).astype(np.int64) % mod
    code = np.where(code >= mod // 2, code - mod, code).astype(p.xdtype)
    order = cell_order(p, cell)
    perm = np.argsort(order, kind="stable")
    n = X.shape[0]
    if pid is None:
        pid = np.arange(1, n + 1, dtype=np.int64)
    rhoc = np.bincount(order, minlength=p.ncells).astype(np.int32)
    return (np.ascontiguousarray(code[perm]), np.ascontiguousarray(np.asarray(V, np.float32)[perm]),
            np.ascontiguousarray(np.asarray(pid, np.int64)[perm]), rhoc)


def uniform_state(p: Params, n, seed=0, vscale=1.0):
    rng = np.random.default_rng(seed)
    X = rng.random((n, 3)) * p.nc
    V = rng.normal(size=(n, 3)) * vscale
    return state_from_positions(p, X, V)


def clustered_state(p: Params, n, seed=0, nblob=6, sigma=0.6, frac=0.7, vscale=1.0):
    """A mix of uniform particles and tight Gaussian blobs (sigma in coarse cells), so PP
    pairs and the heavier PM3 classes occur."""
    rng = np.random.default_rng(seed)
    nb = int(n * frac)
    centers = rng.random((nblob, 3)) * p.nc
    which = rng.integers(0, nblob, nb)
    Xb = centers[which] + rng.normal(size=(nb, 3)) * sigma
    Xu = rng.random((n - nb, 3)) * p.nc
    X = np.concatenate([Xb, Xu])
    V = rng.normal(size=(n, 3)) * vscale
    return state_from_positions(p, X, V)


def lattice_state(p: Params, seed=0, disp=0.2, vscale=1.0):
    """Perturbed lattice with np_nc particles per coarse cell per dimension."""
    rng = np.random.default_rng(seed)
    m = p.nc * p.np_nc
    g = (np.arange(m) + 0.5) / p.np_nc
    Z, Y, Xg = np.meshgrid(g, g, g, indexing="ij")
    X = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=-1)
    X = X + rng.normal(size=X.shape) * disp
    V = rng.normal(size=X.shape) * vscale
    return state_from_positions(p, X, V)
