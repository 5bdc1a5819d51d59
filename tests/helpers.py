"""Shared helpers of the test-suite: relative L1 per variable and oracle runs."""
import numpy as np


def interior(U, s):
    m = s.margin
    if s.ndim == 1:
        return U[:, :, m[0]:U.shape[2] - m[0]]
    return U[:, m[1]:U.shape[1] - m[1], m[0]:U.shape[2] - m[0]]


def rel_l1(a, b):
    """Relative L1 error per variable: sum|a-b| / sum|b|.  A variable that is zero in
    both arrays scores 0; one that is zero only in b scores its absolute L1."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = np.abs(a - b).reshape(a.shape[0], -1).sum(axis=1)
    den = np.abs(b).reshape(b.shape[0], -1).sum(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


def max_rel_l1(pairs):
    return max(float(rel_l1(a, b).max()) for a, b in pairs)
