"""Host side of the batched engine: the block-diagonal stacking that
pdhg_load_batch takes (no GPU needed)."""
import dataclasses

import numpy as np


def test_stacking_is_block_diagonal(pkg):
    ps = [pkg.lpgen.random_equality_lp(m, n, 3, seed=s)
          for s, (m, n) in enumerate([(10, 30), (4, 9), (25, 60)])]
    ps[1] = dataclasses.replace(ps[1], maximize=True, obj_const=-2.5)
    b = pkg.pdhg.stack_batch(ps)
    assert list(b["row_off"]) == [0, 10, 14, 39] and list(b["col_off"]) == [0, 30, 39, 99]
    assert b["nnz"] == sum(p.nnz for p in ps) == b["row_ptr"][-1]
    assert list(b["maximize"]) == [0, 1, 0] and b["obj_const"][1] == -2.5
    for k, p in enumerate(ps):
        r0, r1 = b["row_off"][k], b["row_off"][k + 1]
        c0, c1 = b["col_off"][k], b["col_off"][k + 1]
        e0, e1 = b["row_ptr"][r0], b["row_ptr"][r1]
        assert np.array_equal(b["row_ptr"][r0:r1 + 1] - e0, p.row_ptr)
        assert np.array_equal(b["col_idx"][e0:e1] - c0, p.col_idx)
        assert np.all((b["col_idx"][e0:e1] >= c0) & (b["col_idx"][e0:e1] < c1))
        assert np.array_equal(b["val"][e0:e1], p.val)
        for f in ("c", "col_lo", "col_hi"):
            assert np.array_equal(b[f][c0:c1], getattr(p, f))
        for f in ("row_lo", "row_hi"):
            assert np.array_equal(b[f][r0:r1], getattr(p, f))


def test_stacking_keeps_empty_instances(pkg):
    p = pkg.lpgen.random_equality_lp(5, 12, 2, seed=1)
    empty = dataclasses.replace(p, m=0, n=0, row_ptr=np.zeros(1, np.int32),
                                col_idx=np.zeros(0, np.int32), val=np.zeros(0), c=np.zeros(0),
                                col_lo=np.zeros(0), col_hi=np.zeros(0), row_lo=np.zeros(0),
                                row_hi=np.zeros(0))
    b = pkg.pdhg.stack_batch([p, empty, p])
    assert list(b["row_off"]) == [0, 5, 5, 10] and list(b["col_off"]) == [0, 12, 12, 24]
    assert np.all(np.diff(b["row_ptr"]) >= 0)
