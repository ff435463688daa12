"""Accuracy measures of a precision form against the FP64 form.

rel_l1          relative L1 per conserved variable, sum|a - b| / sum|b| (the
                measure the precision forms are stated in);
shock_offsets   positions of the discontinuities of a 1D profile (sub-zone,
                the centroid of |jump| around each steep feature of the
                reference profile) in both profiles, and their distance in
                zones: the "shock positions within one zone" measure.
"""
import numpy as np


def rel_l1(a, b):
    """sum|a - b| / sum|b| over every axis but the last (the variables)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, np.shape(a)[-1])
    b = np.asarray(b, dtype=np.float64).reshape(-1, np.shape(b)[-1])
    den = np.abs(b).sum(axis=0)
    return np.abs(a - b).sum(axis=0) / np.where(den == 0, 1.0, den)


def features(q, rel=0.05, half=4):
    """Indices j of the steep features of profile q: local maxima of
    |q[j+1] - q[j]| above rel * (max q - min q), at least `half` zones apart
    (the largest kept first)."""
    q = np.asarray(q, dtype=np.float64)
    d = np.abs(np.diff(q))
    span = float(q.max() - q.min())
    if span <= 0.0 or d.size < 3:
        return []
    cand = [j for j in range(1, d.size - 1) if d[j] >= d[j - 1] and d[j] >= d[j + 1] and d[j] > rel * span]
    cand.sort(key=lambda j: -d[j])
    kept = []
    for j in cand:
        if all(abs(j - k) > half for k in kept):
            kept.append(j)
    return sorted(kept)


def _centroid(q, j, half):
    d = np.abs(np.diff(np.asarray(q, dtype=np.float64)))
    lo, hi = max(0, j - half), min(d.size, j + half + 1)
    w = d[lo:hi]
    s = w.sum()
    return float((np.arange(lo, hi) * w).sum() / s) if s > 0 else float(j)


def shock_offsets(q_ref, q, rel=0.05, half=4):
    """For each steep feature of q_ref: (position in q_ref, position in q,
    |difference|), positions in zones (sub-zone, jump-weighted centroids over
    +-half zones).  Returns (list of triples, max difference or 0.0)."""
    out = []
    for j in features(q_ref, rel, half):
        a, b = _centroid(q_ref, j, half), _centroid(q, j, half)
        out.append((a, b, abs(a - b)))
    return out, max((t[2] for t in out), default=0.0)
