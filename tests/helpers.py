"""Shared test systems (small, seeded) for the parity tests."""
import numpy as np

from lynx_b200 import cell as C
from lynx_b200 import pseudo as P


def si8_small(grid=(20, 21, 22), displace=0.05, seed=3):
    """Si8 conventional cell on a small ragged grid, atoms displaced (seeded)."""
    cl, pos = C.diamond_si(1, 20, displace=displace, seed=seed)
    cl.shape = tuple(grid)
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=seed)
    return cl, pos, V


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def subspace_distance(A, B, dV=1.0):
    """Largest principal-angle sine between the column spaces of A and B."""
    qa, _ = np.linalg.qr(np.asarray(A))
    qb, _ = np.linalg.qr(np.asarray(B))
    s = np.linalg.svd(qa.conj().T @ qb, compute_uv=False)
    return float(np.sqrt(max(0.0, 1.0 - s.min() ** 2)))
