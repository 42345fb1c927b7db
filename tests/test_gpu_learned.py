"""The learned warm start on a DSR-shaped bootstrap (alternative 0 observed on 60 menus of 10
alternatives): the network trained on the first draws' fits predicts later draws' fitted cells
far better than the fit of p_hat that the method without it uses for every draw, and the draws
it seeds keep certified brackets that agree with the plain solves."""
import numpy as np
import pytest

from rumb import RUM
from rumb import bootstrap as BS
from rumb.instances import dsr_instance

pytestmark = pytest.mark.gpu


def test_learned_warm_start_predicts_fits_and_keeps_brackets():
    panel, (m, a, p) = dsr_instance(10, 60, 520, 40, seed=1)
    rum = RUM(m, a, p, num_alternatives=10)
    ntr, nte = 96, 32
    boot = rum.bootstrap(panel=panel, B=ntr + nte, weights="multinomial_reject", seed=0, method="bm_admm",
                         method_args={"dtype": "float64"}, learned=True, train_draws=ntr, mlp_epochs=300)
    plain = rum.bootstrap(panel=panel, B=ntr + nte, weights="multinomial_reject", seed=0, method="bm_admm",
                          method_args={"dtype": "float64"})
    for b in (boot, plain):
        b._certify()
    idx = np.arange(ntr + nte)
    boot.solve_draws(idx, stops=False)          # trains on the first ntr, seeds the rest
    plain.solve_draws(idx, stops=False)
    assert boot.learned_info["n_train"] == ntr
    te = idx[ntr:]
    # every bracket is certified and agrees with the plain solve of the same draw
    assert np.all(boot.L[te] <= plain.U[te] + 1e-9) and np.all(plain.L[te] <= boot.U[te] + 1e-9)
    assert np.all(boot.U[te] - boot.L[te] <= boot.abs_tol + 1e-12)
    # the gain: the predicted fit of an unseen draw against its certified fit, versus p_hat's fit
    from rumb.rum_solver import context
    g = rum._geom
    ctx = context()
    P = BS.perturb(boot.p_hat, boot.draws.rows(te), boot.r_n, boot.eps_n)
    prob = ctx.bm_problem(10, g.menu.astype(np.uint32), g.alternative.astype(np.int32), boot.p_hat)
    a_ = boot.session._args
    par = ctx.bm_params(a_["beta"], abs_tol=boot.abs_tol, rel_tol=None, dtype="float64")
    res, _ = ctx.bm_solve_batch(prob, par, P, warm=boot.session._kept, want_fit=True)
    fits = np.stack([r["p_fit"] for r in res])
    err_net = np.linalg.norm(boot.predict_fit(P) - fits, axis=1).mean()
    err_hat = np.linalg.norm(boot.session.fit - fits, axis=1).mean()
    assert err_net < 0.25 * err_hat, (err_net, err_hat)
    # the seeded draws take no more iterations than the plain ones
    assert boot.iters[te].sum() <= plain.iters[te].sum()
