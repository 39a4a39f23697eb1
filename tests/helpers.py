"""Shared comparison helpers for the parity tests."""
import numpy as np


def rel_err(a, b, scale=None):
    """max |a - b| / max |b| (or / scale), the norm-wise relative error."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / s)


def gpu_state(sim):
    p = sim.particles()
    return dict(den=p["den"].astype(np.float64), pos=p["pos"].astype(np.float64), vel=p["vel"].astype(np.float64))


def oracle_csr(buckets, n, ncells):
    """Mobile section of the oracle's buckets as CSR (cell_start, members) with
    members ascending inside each cell, plus the boundary section."""
    counts = buckets["counts"].astype(np.int64)
    contents = buckets["contents"]
    start = np.zeros(ncells + 1, np.int64)
    start[1:] = np.cumsum(counts[:, 2])
    members = np.zeros(int(start[-1]), np.uint32)
    bstart = np.zeros(ncells + 1, np.int64)
    bstart[1:] = np.cumsum(counts[:, 0])
    bmembers = np.zeros(int(bstart[-1]), np.uint32)
    for c in np.nonzero(counts.sum(axis=1))[0]:
        bc, rc, cn = counts[c]
        members[start[c]:start[c + 1]] = np.sort(contents[c, bc + rc:bc + rc + cn])
        bmembers[bstart[c]:bstart[c + 1]] = np.sort(contents[c, :bc])
    return start, members, bstart, bmembers
