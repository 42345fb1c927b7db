"""The bootstrap's draws solved together (batched slots) reach the same decisions as the same
draws solved one at a time through the Session (the reference's loop)."""
import numpy as np
import pytest

from rumb import RUM
from rumb import bootstrap as BS
from rumb.instances import panel_instance

pytestmark = pytest.mark.gpu


def test_batched_and_sequential_bootstrap_agree():
    n = 10
    panel, (m, a, p) = panel_instance(n, 0.3, 80, 8, 5, seed=7)
    rum = RUM(m, a, p, num_alternatives=n)
    b1 = rum.bootstrap(panel=panel, B=24, weights="multinomial", seed=1, method="bm_admm",
                       method_args={"dtype": "float64"})
    r1 = b1.p_value()
    b2 = rum.bootstrap(panel=panel, B=24, weights="multinomial", seed=1, method="bm_admm",
                       method_args={"dtype": "float64"})
    b2._certify()
    b2._screen()
    todo = np.flatnonzero((BS.decide(b2.L, b2.U, *b2.tau) == BS.UNDECIDED))
    tau_lo, tau_hi = b2.tau
    P = BS.perturb(b2.p_hat, b2.draws.rows(todo), b2.r_n, b2.eps_n)
    for j, b in enumerate(todo):
        r = b2.session.solve(P[j], abs_tol=b2.abs_tol, rel_tol=b2.rel_tol, warm=True, below=tau_lo, above=tau_hi)
        b2.L[b], b2.U[b] = max(b2.L[b], r.lb), min(b2.U[b], r.ub)
    d1 = BS.decide(b1.L, b1.U, *b1.tau)
    d2 = BS.decide(b2.L, b2.U, *b2.tau)
    assert np.array_equal(d1, d2)
    assert r1.n_solved == todo.size
    # every bracket of the batch contains the one-at-a-time bracket's distance
    assert np.all(b1.L <= b2.U + 1e-9) and np.all(b2.L <= b1.U + 1e-9)


def test_distance_and_confidence_intervals():
    """distance_interval needs only the screen's norms (equal to the host's); confidence_interval
    solves to tolerance every draw left in the final quantile band, and the lower end from every
    draw solved lies in its reported bracket."""
    n = 10
    panel, (m, a, p) = panel_instance(n, 0.3, 80, 8, 5, seed=7)
    rum = RUM(m, a, p, num_alternatives=n)
    b = rum.bootstrap(panel=panel, B=24, weights="multinomial", seed=1, method="bm_admm",
                      method_args={"dtype": "float64"})
    alpha = 0.1
    di = b.distance_interval(alpha)
    rows = b.draws.rows(np.arange(24))
    dev = np.sqrt(np.einsum("ij,ij->i", rows - b.p_hat, rows - b.p_hat))
    np.testing.assert_allclose(b.dev, dev, rtol=1e-12, atol=0)
    c = float(np.quantile(b.dev, 1 - alpha))
    assert di.half_width == c and di.lower == max(0.0, b.L0 - c) and di.upper == b.U0 + c
    ci = b.confidence_interval(alpha)
    assert ci.lower <= ci.lower_bracket[1] and ci.upper == np.inf
    q_l, q_u = BS.quantile_band(b.L, b.U, alpha)
    hot = (b.U >= q_l) & (b.L <= q_u)
    assert np.all(b.tol_full[hot] <= b.abs_tol)
    # every draw solved to tolerance: the lower end then lies in the bracket
    b.solve_draws(np.arange(24), stops=False)
    low, high, _ = BS.ci_lower(b.L0, b.U0, b.L, b.U, alpha, b.r_n, b.eps_n)
    assert ci.lower - 1e-9 <= low <= ci.lower_bracket[1] + 1e-9


def test_p_value_stop_when_decided():
    """Stopping once the decision is locked gives the full run's decision with no more solves."""
    n = 10
    panel, (m, a, p) = panel_instance(n, 0.3, 80, 8, 5, seed=7)
    rum = RUM(m, a, p, num_alternatives=n)
    kw = dict(panel=panel, B=24, weights="multinomial", seed=1, method="bm_admm", method_args={"dtype": "float64"})
    full = rum.bootstrap(**kw).p_value(0.1)
    early = rum.bootstrap(**kw).p_value(0.1, stop_when_decided=True)
    assert early.reject == full.reject and early.n_solved <= full.n_solved
    assert early.T == (early.dist_hat[0] * np.sqrt(80), early.dist_hat[1] * np.sqrt(80))


@pytest.mark.parametrize("source", ["poisson", "mammen", "exponential", "replies"])
def test_bootstrap_weight_schemes_and_replies(source):
    """Every weight scheme and the replies table run the whole test: integer weights through the
    GPU draws, real weights and replies through the host blocks; the screen's bounds are real
    distances (U_b >= the certified lower bound of a solved draw)."""
    from rumb import cells_from_panel
    n = 10
    panel, _ = panel_instance(n, 0.3, 80, 8, 5, seed=7)
    if source == "replies":
        table = dict(menu=panel["menu"], chosen=panel["chosen"])
        rum = RUM(*cells_from_panel(table, n), num_alternatives=n)
        b = rum.bootstrap(replies=table, B=16, seed=1, method="bm_admm", method_args={"dtype": "float64"})
    else:
        rum = RUM(*cells_from_panel(panel, n), num_alternatives=n)
        b = rum.bootstrap(panel=panel, B=16, weights=source, seed=1, method="bm_admm",
                          method_args={"dtype": "float64"})
    pv = b.p_value(0.1)
    assert 0.0 <= pv.p <= 1.0 and pv.B == 16
    assert b.draws.integer_weights == (source == "poisson")
    P = b._draw_rows().rows(np.arange(16), b.eps_n * b.r_n)
    np.testing.assert_array_equal(P, BS.perturb(b.p_hat, b.draws.rows(np.arange(16)), b.r_n, b.eps_n))
    solved = np.flatnonzero(b.solved)
    assert np.all(b.L[solved] <= b.U[solved] + 1e-9)
