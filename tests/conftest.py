import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        with open(os.path.join(GOLDEN, name)) as f:
            return json.load(f)
    return load


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


def dense_from_coo(n, rows, cols, vals):
    A = np.zeros((n, n))
    for r, c, v in zip(rows, cols, vals):
        A[r, c] = v
    return A


def scalar_to_block(A, b):
    """Embed a scalar SPD system into 3x3-block CSR (padding rows get an identity diagonal)."""
    n = A.shape[0]
    nb = (n + 2) // 3
    Ap = np.eye(3 * nb)
    Ap[:n, :n] = A
    bp = np.zeros(3 * nb)
    bp[:n] = b
    row_ptr = [0]
    cols, vals = [], []
    for i in range(nb):
        for j in range(nb):
            blk = Ap[3 * i:3 * i + 3, 3 * j:3 * j + 3]
            if np.any(blk != 0.0):
                cols.append(j)
                vals.append(blk)
        row_ptr.append(len(cols))
    return (np.asarray(row_ptr, np.int64), np.asarray(cols, np.int32), np.asarray(vals, np.float64), bp)
