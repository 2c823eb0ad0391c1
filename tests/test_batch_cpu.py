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


def test_threaded_stacking_matches_concatenation(pkg):
    # enough instances for several filling threads: the result must be the
    # plain concatenation with rows, columns and entries offset per instance
    ps = [pkg.lpgen.random_equality_lp(5 + s % 7, 11 + s % 13, 2, seed=s) for s in range(400)]
    b = pkg.pdhg.stack_batch(ps)
    roff = np.concatenate([[0], np.cumsum([p.m for p in ps])])
    coff = np.concatenate([[0], np.cumsum([p.n for p in ps])])
    zoff = np.concatenate([[0], np.cumsum([p.nnz for p in ps])])
    rp = np.concatenate([p.row_ptr[:-1] + z for p, z in zip(ps, zoff)] + [[zoff[-1]]])
    assert np.array_equal(b["row_ptr"], rp)
    assert np.array_equal(b["col_idx"], np.concatenate([p.col_idx + c for p, c in zip(ps, coff)]))
    assert np.array_equal(b["val"], np.concatenate([p.val for p in ps]))
    for f in ("c", "col_lo", "col_hi", "row_lo", "row_hi"):
        assert np.array_equal(b[f], np.concatenate([getattr(p, f) for p in ps])), f
    assert np.array_equal(b["row_off"], roff) and np.array_equal(b["col_off"], coff)
