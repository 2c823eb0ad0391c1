"""The warm start's run-time fallback on the CPU, against a fake engine.

A warm-started batch gets the family's iteration budget; instances not
optimal by then are solved again from the cold start with the full cap, in
one batch, and report the iterations of both attempts."""
import numpy as np


class FakeEngine:
    """solve_batch answers from a table: per instance id, the iterations a
    warm start needs and the iterations the cold start needs."""

    def __init__(self, pkg, need):
        self.pkg = pkg
        self.need = need
        self.calls = []
        self.batch = None

    def load_batch(self, problems):
        self.batch = list(problems)

    def solve_batch(self, opt, x0=None, y0=None):
        warm = x0 is not None
        self.calls.append(([p for p in self.batch], opt.max_iterations, warm))
        out = []
        for k, p in enumerate(self.batch):
            need = self.need[p][0 if warm else 1]
            if warm:
                assert x0[k][0] == p and y0[k][0] == -p
            ok = need <= opt.max_iterations
            out.append(self.pkg.PdhgResult(status="optimal" if ok else "iteration_limit",
                                           iterations=min(need, opt.max_iterations)))
        return out


def test_fallback_resolves_only_the_stragglers_cold(pkg):
    # instance id -> (warm iterations needed, cold iterations needed)
    need = {0: (100, 400), 1: (5_000, 300), 2: (250, 260), 3: (10**9, 900)}
    e = FakeEngine(pkg, need)
    probs = [0, 1, 2, 3]
    x0s = [np.array([p, 0.0]) for p in probs]
    y0s = [np.array([-p, 0.0]) for p in probs]
    opt = pkg.PdhgOptions(max_iterations=300_000)
    rs = pkg.warmstart.solve_family_with_fallback(e, probs, opt, x0s, y0s, budget=1_000, chunk=2)
    assert [r.status for r in rs] == ["optimal"] * 4
    assert [r.iterations for r in rs] == [100, 1_000 + 300, 250, 1_000 + 900]
    # two warm chunks at the budget, then one cold batch of the stragglers at the cap
    assert [(c[0], c[1], c[2]) for c in e.calls] == [([0, 1], 1_000, True), ([2, 3], 1_000, True),
                                                    ([1, 3], 300_000, False)]
    assert opt.max_iterations == 300_000  # the caller's options are not changed


def test_no_budget_or_no_starts_is_the_plain_batched_solve(pkg):
    need = {0: (50, 70), 1: (10**9, 80)}
    opt = pkg.PdhgOptions(max_iterations=1_000)
    x0s = [np.array([0.0]), np.array([1.0])]
    y0s = [np.array([-0.0]), np.array([-1.0])]
    for budget in (0, 1_000, 5_000):
        e = FakeEngine(pkg, need)
        rs = pkg.warmstart.solve_family_with_fallback(e, [0, 1], opt, x0s, y0s, budget=budget)
        assert [r.iterations for r in rs] == [50, 1_000] and len(e.calls) == 1
    e = FakeEngine(pkg, need)
    rs = pkg.warmstart.solve_family_with_fallback(e, [0, 1], opt, None, None, budget=10)
    assert [r.iterations for r in rs] == [70, 80] and e.calls[0][2] is False
