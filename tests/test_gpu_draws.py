"""Bootstrap draws on the GPU (rumb_draws_*): every draw's rows equal the host builder's
(Draws.rows, the count-list builder) bit for bit, raw and perturbed, and the screen's norms
equal numpy's to rounding."""
import numpy as np
import pytest

from rumb import _lib
from rumb import bootstrap as BS
from rumb.instances import config_instance, panel_instance

pytestmark = pytest.mark.gpu


def _cases():
    panel, (m, a, p) = panel_instance(10, 0.3, 80, 8, 5, seed=7)
    yield "n10_panel80", panel, m, a, p, 40, "multinomial"
    yield "n10_panel80_reject", panel, m, a, p, 40, "multinomial_reject"
    panel, (m, a, p) = panel_instance(10, 0.3, 7000, 8, 5, seed=8)       # weights above 48 KB of shared memory
    yield "n10_panel7000", panel, m, a, p, 16, "multinomial"
    n, m, a, p, panel = config_instance("n20_d1pct_panel520")
    yield "n20_d1pct_panel520", panel, m, a, p, 48, "multinomial"


CASES = list(_cases())


@pytest.mark.parametrize("name,panel,m,a,p,B,weights", CASES, ids=[c[0] for c in CASES])
def test_draw_rows_and_screen_match_host(ctx, name, panel, m, a, p, B, weights):
    d = BS.Draws(panel, m, a, p, B=B, weights=weights, seed=3)
    g = _lib.DrawRows(ctx, d.W, d.lists, d.p_hat)
    r_n, eps_n, _ = BS.scaling(d.R)
    scale = eps_n * r_n
    idx = np.array([B - 1, 0, 7, 7, 3], dtype=np.int64)
    host = d.rows(idx)
    np.testing.assert_array_equal(g.rows(idx), host)
    np.testing.assert_array_equal(g.rows(idx, scale), BS.perturb(d.p_hat, host, r_n, eps_n))
    # the screen against numpy, for every draw
    fit = np.clip(d.p_hat + 0.01 * np.sin(np.arange(d.M)), 0.0, 1.0)
    dev, ub = g.screen(fit, scale)
    all_rows = d.rows(np.arange(B))
    P = BS.perturb(d.p_hat, all_rows, r_n, eps_n)
    np.testing.assert_allclose(dev, np.sqrt(np.einsum("ij,ij->i", all_rows - d.p_hat, all_rows - d.p_hat)),
                               rtol=1e-12, atol=0)
    np.testing.assert_allclose(ub, np.sqrt(np.einsum("ij,ij->i", P - fit, P - fit)), rtol=1e-12, atol=0)
    dev2, ub2 = g.screen(None, scale)
    assert ub2 is None and np.array_equal(dev2, dev)
    with pytest.raises(_lib.RumbError):
        g.rows(np.array([B], dtype=np.int64))
    g.close()


def test_gpu_rows_match_reference_golden(ctx):
    """The GPU rows equal the reference's own draws (tests/golden/draws.npz) bit for bit."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "draws.npz"))
    panel = dict(respondent=g["panel_respondent"], menu=g["panel_menu"], chosen=g["panel_chosen"])
    for w in ("multinomial", "multinomial_reject"):
        d = BS.Draws(panel, g["menu"], g["alternative"], g["p_hat"], B=12, weights=w, seed=5)
        gd = _lib.DrawRows(ctx, d.W, d.lists, d.p_hat)
        np.testing.assert_array_equal(gd.rows(np.arange(12)), g["rows_" + w])
        gd.close()


def test_draws_reject_bad_input(ctx):
    """Bad panels are refused on the host with an error, before anything reaches the GPU."""
    import copy
    panel, (m, a, p) = panel_instance(8, 0.4, 20, 4, 3, seed=2)
    d = BS.Draws(panel, m, a, p, B=4, weights="multinomial", seed=0)
    with pytest.raises(_lib.RumbError):                     # a row's menu out of range
        bad = copy.copy(d.lists)
        bad.row_menu = d.lists.row_menu.copy()
        bad.row_menu[0] = d.lists.n_menus
        _lib.DrawRows(ctx, d.W, bad, d.p_hat)
    with pytest.raises(_lib.RumbError):                     # a respondent beyond R
        bad = copy.copy(d.lists)
        bad.menu_resp = d.lists.menu_resp.copy()
        bad.menu_resp[0] = d.R
        _lib.DrawRows(ctx, d.W, bad, d.p_hat)
    g = _lib.DrawRows(ctx, d.W, d.lists, d.p_hat)
    with pytest.raises(_lib.RumbError):                     # a draw index out of range
        g.rows(np.array([-1], dtype=np.int64))
    assert g.rows(np.zeros(0, dtype=np.int64)).shape == (0, d.M)
    g.close()
