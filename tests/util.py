"""Helpers shared by the tests."""
import numpy as np


def leaf_magnetizations(R, handle):
    """ObjM of every leaf of a container, flattened in traversal order."""
    out = []

    def rec(x):
        if isinstance(x[0], list) and x and isinstance(x[0][0], list):
            for y in x:
                rec(y)
        else:
            out.append(x[1])

    rec(R.ObjM(handle))
    return np.array(out, dtype=float)


def rel_err(a, b):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
