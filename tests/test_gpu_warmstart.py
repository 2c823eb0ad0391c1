"""Learned warm start on a small parametric family (config-2-structure base
with 500 rows and 1,200 columns, b and c moved by ~9% along 64 parameters).

The batched engine solves the training instances; the basis and the network
(tensor-core training) are fitted; on held-out parameters the gated starts
must (a) replace the cold start only where their KKT residual is lower,
(b) be taken for most instances (the gate's measure is PDLP's l2 relative
KKT, evaluated on the device), (c) reach every optimum that the cold start
reaches, each reported solve meeting the same relative-KKT tolerance, and
(d) need fewer iterations on average than the cold start.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPT = dict(precision="mixed", termination_rule="relative_kkt", restart_rule="adaptive",
           primal_weight_update=True, tolerance=1e-4, max_iterations=300_000)


def test_learned_warm_start_beats_the_cold_start(pkg):
    fam = pkg.lpgen.parametric_family(500, 1200, 5, seed=4001)
    opt = pkg.PdhgOptions(**OPT)
    train_th = fam.thetas(256, seed=1)
    test_th = fam.thetas(32, seed=2)
    train = [fam.instance(t) for t in train_th]
    test = [fam.instance(t) for t in test_th]
    with pkg.Engine(0) as e:
        res = pkg.warmstart.solve_family(e, train, opt)
        assert sum(r.status == "optimal" for r in res) >= 240
        ws = pkg.warmstart.LearnedWarmStart(fam, rank=32, hidden=256)
        rep = ws.fit(train_th, res, epochs=400, batch=32, lr=1e-3)
        assert rep.losses[-1] < 0.5 * rep.losses[0], rep.losses[[0, -1]]
        assert ws.val_loss < 1.0  # better than predicting the mean coefficients
        x0s, y0s, used, kw, kc = ws.starts(e, test, test_th, opt)
        assert np.all(kw[used] < kc[used])
        assert used.sum() >= 0.75 * len(test), (used.sum(), kw, kc)
        cold = pkg.warmstart.solve_family(e, test, opt)
        warm = pkg.warmstart.solve_family(e, test, opt, x0s, y0s)
    for c, w in zip(cold, warm):
        if c.status == "optimal":
            assert w.status == "optimal"
        if w.status == "optimal":
            assert w.relative_kkt < 1e-4
    it_c = np.mean([r.iterations for r in cold])
    it_w = np.mean([r.iterations for r in warm])
    assert it_w < it_c, (it_w, it_c)
