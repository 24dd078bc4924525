"""The reference's BSR3 storage at the linear-solver boundary (CPU): BlockSparseMatrix<T,3>::Values()
keeps each block row as one row-major 3 x 3nb strip (block_sparse_matrix.h:459-475). The golden fixture
holds Values() of matrices filled through the reference class's own SetValue (tests/golden/bsr3_reference.json,
made by tests/golden/make_golden.py from oracle/_ref); the layout helpers and the header constants follow it."""
import numpy as np

from project_superdex_b200 import capi
from project_superdex_b200.linear_solver import BlockSparseMatrix, ValueLayout, blocks_to_strips, strips_to_blocks


def test_strip_helpers_match_the_reference_storage(golden):
    g = golden("bsr3_reference.json")
    assert len(g["layout"]) == 3
    for case in g["layout"]:
        rp, blocks, vals = np.array(case["row_ptr"]), np.array(case["blocks"]).reshape(-1, 3, 3), np.array(case["values"])
        assert np.array_equal(blocks_to_strips(rp, blocks), vals)
        assert np.array_equal(strips_to_blocks(rp, vals), blocks)
        m = BlockSparseMatrix.from_blocks(rp, case["col"], blocks)
        assert m.layout == ValueLayout.RowStrips and np.array_equal(m.values, vals)


def test_strip_offset_formula():
    """Entry (lr, lc) of block k of block row br sits at 9 ptr[br] + 3 (lr nb + k) + lc."""
    rng = np.random.default_rng(0)
    rp = np.array([0, 3, 4, 8])
    blocks = rng.normal(size=(8, 3, 3))
    v = blocks_to_strips(rp, blocks)
    for br in range(3):
        nb = rp[br + 1] - rp[br]
        for k in range(nb):
            for lr in range(3):
                for lc in range(3):
                    assert v[9 * rp[br] + 3 * (lr * nb + k) + lc] == blocks[rp[br] + k, lr, lc]


def test_layout_constants_and_default():
    assert (capi.SDX_BSR_ROW_STRIPS, capi.SDX_BSR_BLOCKS) == (0, 1)
    assert capi.default_linear_params().value_layout == capi.SDX_BSR_ROW_STRIPS


def test_reference_pcg_fixture_is_consistent(golden):
    """The fixture's reference solutions meet the stop test they were run with (rel 1e-6, residual L2)."""
    for sysd in golden("bsr3_reference.json")["pcg"]:
        rp, col = np.array(sysd["row_ptr"]), np.array(sysd["col"])
        blocks = strips_to_blocks(rp, np.array(sysd["values"]))
        b = np.array(sysd["b"])
        for run in sysd["runs"]:
            x = np.array(run["x"])
            y = np.zeros_like(b)
            for i in range(rp.size - 1):
                for k in range(rp[i], rp[i + 1]):
                    y[3 * i:3 * i + 3] += blocks[k] @ x[3 * col[k]:3 * col[k] + 3]
            assert run["convergence"] == 1
            assert np.linalg.norm(b - y) <= 1.0001e-6 * np.linalg.norm(b)
