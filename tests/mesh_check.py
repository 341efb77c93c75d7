"""Comparison helpers for surface-mesher outputs (test infrastructure).

A mesh is the reference's output layout: one record per occupied marching
cube, 15 vertex slots of (position xyz, normal xyz); slots a cube's triangles
do not use stay zero.  The reference appends records in atomic order, so
records are compared as a set: canonically ordered by the centroid of their
used slots, matched by nearest centroid.
"""
from __future__ import annotations

import numpy as np


def used_slots(records: np.ndarray) -> np.ndarray:
    """[k, 15] bool: slots a record's triangles use (any nonzero or NaN)."""
    r = np.asarray(records, np.float32).reshape(-1, 15, 6)
    return np.any((r != 0) | np.isnan(r), axis=2)


def centroids(records: np.ndarray) -> np.ndarray:
    r = np.asarray(records, np.float64).reshape(-1, 15, 6)
    u = used_slots(r)
    cnt = np.maximum(u.sum(1), 1)
    return (np.where(u[..., None], r[..., :3], 0.0).sum(1)) / cnt[:, None]


def canonical_records(records: np.ndarray) -> np.ndarray:
    """Records sorted by centroid (x, then y, then z)."""
    r = np.asarray(records, np.float32).reshape(-1, 15, 6)
    c = centroids(r)
    order = np.lexsort((c[:, 2], c[:, 1], c[:, 0]))
    return r[order]


def record_aggregates(records: np.ndarray) -> dict:
    """Order-independent summaries of a whole mesh."""
    r = np.asarray(records, np.float64).reshape(-1, 15, 6)
    u = used_slots(r)
    pos = np.where(u[..., None], r[..., :3], 0.0)
    nrm = np.where(u[..., None] & ~np.isnan(r[..., 3:]), r[..., 3:], 0.0)
    return {
        "records": int(r.shape[0]),
        "vertices": int(u.sum()),
        "nan_normals": int(np.isnan(r[..., 3:]).any(axis=2).sum()),
        "position_sum": pos.sum(axis=(0, 1)),
        "position_sq_sum": (pos * pos).sum(),
        "normal_sum": nrm.sum(axis=(0, 1)),
    }


def match_records(a: np.ndarray, b: np.ndarray, tol: float):
    """Pairs records of a with records of b by nearest centroid.

    Returns (pairs [m, 2] of indices, unmatched count in a, unmatched in b);
    a pair needs centroids closer than tol and the same used-slot pattern."""
    from scipy.spatial import cKDTree

    a = np.asarray(a, np.float32).reshape(-1, 15, 6)
    b = np.asarray(b, np.float32).reshape(-1, 15, 6)
    if len(a) == 0 or len(b) == 0:
        return np.zeros((0, 2), np.int64), len(a), len(b)
    ca, cb = centroids(a), centroids(b)
    d, j = cKDTree(cb).query(ca, k=1)
    ua, ub = used_slots(a), used_slots(b)
    ok = (d < tol) & np.all(ua == ub[j], axis=1)
    pairs = np.stack([np.nonzero(ok)[0], j[ok]], 1)
    # each b record used once
    _, first = np.unique(pairs[:, 1], return_index=True)
    pairs = pairs[np.sort(first)]
    return pairs, len(a) - len(pairs), len(b) - len(pairs)


def compare_meshes(a: np.ndarray, b: np.ndarray, h_mesh: float) -> dict:
    """Matched fraction and the worst position / normal differences."""
    pairs, ma, mb = match_records(a, b, 0.25 * h_mesh)
    a = np.asarray(a, np.float32).reshape(-1, 15, 6)
    b = np.asarray(b, np.float32).reshape(-1, 15, 6)
    out = {"a": len(a), "b": len(b), "matched": len(pairs), "unmatched_a": ma, "unmatched_b": mb,
           "pos_err": 0.0, "normal_err": 0.0, "nan_mismatch": 0}
    if len(pairs):
        ra, rb = a[pairs[:, 0]], b[pairs[:, 1]]
        u = used_slots(ra)
        dp = np.abs(ra[..., :3] - rb[..., :3])[u]
        out["pos_err"] = float(dp.max()) if dp.size else 0.0
        na, nb = ra[..., 3:][u], rb[..., 3:][u]
        nan_a, nan_b = np.isnan(na).any(1), np.isnan(nb).any(1)
        out["nan_mismatch"] = int((nan_a != nan_b).sum())
        fin = ~nan_a & ~nan_b
        out["normal_err"] = float(np.abs(na[fin] - nb[fin]).max()) if fin.any() else 0.0
    return out
