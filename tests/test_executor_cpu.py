"""Host logic of the batched executor (no GPU): readback and time-step validation as the reference's
SceneBatchExecutorV2 does it (scene_batch_executor_v2.cpp:614-745)."""
import numpy as np
import pytest

from project_superdex_b200 import executor as X


def test_time_step_validation():
    assert X.validate_time_step("step", 1 / 240) == 1 / 240
    for bad in (0.0, -1e-3, float("nan"), float("inf")):
        with pytest.raises(ValueError):
            X.validate_time_step("step", bad)


def test_readback_validation():
    n, s = 12, 2
    q, v = np.zeros(n), np.zeros(n)
    c, d = np.zeros(s), np.zeros(s, np.uint8)
    X.validate_readback(X.READ_QPOS | X.READ_QVEL | X.READ_CONTACTS | X.READ_DIVERGED, n, s, q, v, None, c, d)
    X.validate_readback(0, n, s, None, None, None, None, None)
    with pytest.raises(ValueError):  # unknown bit
        X.validate_readback(1 << 7, n, s, None, None, None, None, None)
    with pytest.raises(ValueError):  # selected but missing
        X.validate_readback(X.READ_QPOS, n, s, None, None, None, None, None)
    with pytest.raises(ValueError):  # given but not selected
        X.validate_readback(0, n, s, q, None, None, None, None)
    with pytest.raises(ValueError):  # wrong size
        X.validate_readback(X.READ_QPOS, n, s, np.zeros(n + 1), None, None, None, None)
    with pytest.raises(ValueError):  # wrong dtype
        X.validate_readback(X.READ_DIVERGED, n, s, None, None, None, None, np.zeros(s))
    with pytest.raises(ValueError):  # not contiguous
        X.validate_readback(X.READ_QVEL, n, s, None, np.zeros(2 * n)[::2], None, None, None)
    with pytest.raises(ValueError):  # soft envs have no links
        X.validate_readback(X.READ_LINKS, n, s, None, None, np.zeros(4), None, None)
