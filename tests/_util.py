"""Shared helpers for the parity tests."""
import numpy as np


def vec(d, pre):
    return np.stack([d[pre + "x"], d[pre + "y"], d[pre + "z"]], 1)


def rel_vec_err(a, b):
    """Per-particle |a - b| / |b| with a normwise floor (bodies whose |b| is tiny compared
    with the rms are measured against the rms instead)."""
    nb = np.linalg.norm(b, axis=1)
    floor = 1e-3 * np.sqrt(np.mean(nb ** 2))
    return np.linalg.norm(a - b, axis=1) / np.maximum(nb, floor)


def rel_err(a, b):
    floor = 1e-3 * np.sqrt(np.mean(b ** 2))
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def ref_cell_levels(nchild, child):
    """Levels of cells stored in the reference's depth-first order (root = 0)."""
    lev = np.zeros(len(nchild), dtype=np.int64)
    for c in range(len(nchild)):
        if nchild[c] > 0:
            lev[child[c]:child[c] + nchild[c]] = lev[c] + 1
    return lev


def cell_keys(begin, nbody, level):
    return [(int(b), int(n), int(l)) for b, n, l in zip(begin, nbody, level)]


def pair_set(t, s, keys):
    return set((keys[a], keys[b]) for a, b in zip(t.tolist(), s.tolist()))
