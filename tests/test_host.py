"""Host logic without a GPU: input checks and messages of the RUM class, planning with a fake
device-memory query (the reference's stub-profile pattern, tests/test_cpu.py:215-279), the
Flow-CG master pieces against the reference's golden vectors, and the seeded generators."""
import json
import math
import os

import numpy as np
import pytest

from rumb import rum_solver, flow_cg, defaults
from rumb.instances import config_instance, mixture_instance, panel_instance, dsr_instance

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture
def fake_gpu(monkeypatch):
    monkeypatch.setattr(rum_solver, "gpu_free_bytes", lambda device=0: 150 * 2 ** 30)


def test_input_errors():
    R = rum_solver.RUM
    with pytest.raises(ValueError, match="no observations"):
        R([], [], [])
    with pytest.raises(ValueError, match="empty menu"):
        R([0, 3], [0, 1], [0.5, 0.5])
    with pytest.raises(ValueError, match="not in its menu"):
        R([3, 3], [0, 2], [0.5, 0.5])
    with pytest.raises(ValueError, match="appears more than once"):
        R([3, 3], [0, 0], [0.5, 0.5])
    with pytest.raises(ValueError, match="outside"):
        R([3, 3], [0, 1], [0.5, 1.5])
    with pytest.raises(ValueError, match="must hold integers"):
        R([3.5, 3], [0, 1], [0.5, 0.5])
    with pytest.raises(ValueError, match="num_alternatives"):
        R([3, 3], [0, 1], [0.5, 0.5], num_alternatives=1)
    with pytest.warns(UserWarning, match="summing to more than 1"):
        R([3, 3], [0, 1], [0.7, 0.7])


def test_method_args_and_planning(fake_gpu):
    n, m, a, p = config_instance("n10_all_k20")
    rum = rum_solver.RUM(m, a, p)
    with pytest.raises(ValueError, match="unknown method_args"):
        rum._plan("bm_admm", {"bogus": 1})
    with pytest.raises(ValueError, match="needs a named method"):
        rum._plan(None, {"check": 10})
    with pytest.raises(ValueError, match="unknown method"):
        rum._plan("ip_cg", None)
    name, _, args = rum._plan("bm_admm", {"check": 25})
    assert name == "bm_admm" and args["check"] == 25 and args["dtype"] == "float64"
    assert args["beta"] == pytest.approx(2.534415507522252)
    name, _, args = rum._plan("flow_cg", {"pricing": "stream_u16"})
    assert args["_engine"] == "u16" and args["pricing"] == "stream"
    with pytest.raises(ValueError, match="contradicts"):
        rum._plan("flow_cg", {"pricing": "stream_u16", "dtype": "uint24"})
    with pytest.raises(ValueError, match="mask pricing stores float32"):
        rum._plan("flow_cg", {"pricing": "mask", "dtype": "uint16"})
    with pytest.raises(ValueError):
        rum._plan("bm_admm", {"dtype": "float16"})


def test_choose_method_density_rule(fake_gpu):
    assert rum_solver.choose_method(10, 5110)[0] == "flow_cg"
    assert rum_solver.choose_method(18, 23650)[0] == "bm_admm"          # 1 % >= 0.5 %
    assert rum_solver.choose_method(18, 5000)[0] == "flow_cg"           # 0.2 %
    assert rum_solver.choose_method(12, 20000)[0] == "bm_admm"


def test_planner_memory_refusal(monkeypatch):
    monkeypatch.setattr(rum_solver, "gpu_free_bytes", lambda device=0: 2 ** 30)
    with pytest.raises(RuntimeError, match="needs .* GB of GPU memory"):
        rum_solver._plan_bm_admm(24, 1000, dict(defaults.METHOD_ARGS["bm_admm"]))
    # the automatic choice falls back to flow_cg
    assert rum_solver.choose_method(24, 4 * 10 ** 6)[0] == "flow_cg"


def test_races_and_weights_refused():
    n, m, a, p = config_instance("n10_all_k20")
    rum = rum_solver.RUM(m, a, p)
    with pytest.raises(ValueError, match="races"):
        rum.calculate_distance(opt=1.0)
    with pytest.raises(RuntimeError, match="unweighted"):
        rum.calculate_distance(vcov=2 * np.eye(p.size))


def test_threshold_on_rest_rows():
    assert rum_solver._on_rest(None, 0.3, True) is None
    assert rum_solver._on_rest(0.5, 0.3, True) == 0.0
    assert rum_solver._on_rest(0.5, 0.3, False) is None
    assert rum_solver._on_rest(1.0, 0.36, True) == pytest.approx(0.8)
    with pytest.raises(ValueError):
        rum_solver._on_rest(math.inf, 0.0, True)


def test_master_pieces_against_reference():
    g = np.load(os.path.join(GOLD, "qp.npz"))
    for t in range(4):
        lam, A = flow_cg.solve_qp_native(g["Q_%d" % t], g["h_%d" % t])
        np.testing.assert_allclose(lam, g["lam_%d" % t], atol=1e-12)
        np.testing.assert_array_equal(flow_cg.project_simplex(g["ps_y_%d" % t]), g["ps_x_%d" % t])
    c = np.load(os.path.join(GOLD, "columns.npz"))
    for t in range(5):
        col = flow_cg.ranking_column(c["menus"].astype(np.uint64), c["alts"], c["rank_%d" % t], 18)
        np.testing.assert_array_equal(col, c["col_%d" % t])


def test_gram_and_pout_maintainers():
    rng = np.random.default_rng(1)
    M = 300
    ph = rng.random(M)
    g = flow_cg.GramMaintainer(M, ph, max_K=10)
    po = flow_cg.PoutMaintainer(M)
    cols = [(rng.random(M) < 0.4).astype(np.uint8) for _ in range(6)]
    for c in cols:
        g.add_column(c.astype(np.float64))
        po.add_column(c)
    V = np.stack(cols, axis=1).astype(np.float64)
    Q, h = g.view()
    np.testing.assert_array_equal(Q, V.T @ V)
    np.testing.assert_allclose(h, V.T @ ph, rtol=1e-14)
    lam = rng.dirichlet(np.ones(6))
    po.apply_delta(lam)
    np.testing.assert_allclose(po.p_out, V @ lam, atol=1e-14)


def test_draws_match_reference_golden():
    """The bootstrap's draws equal the reference's own (tests/golden/make_draws_golden.py) bit for
    bit: every weight scheme's weights and rows, a replies table's draws and cells, the cells of one
    alternative, and the refusals' messages."""
    from rumb import draws as D
    g = np.load(os.path.join(GOLD, "draws.npz"))
    panel = dict(respondent=g["panel_respondent"], menu=g["panel_menu"], chosen=g["panel_chosen"])
    for w in D.WEIGHTS:
        d = D.Draws(panel, g["menu"], g["alternative"], g["p_hat"], B=12, weights=w, seed=5)
        np.testing.assert_array_equal(d.W, g["W_" + w])
        if w in D.INTEGER_WEIGHTS:          # exact integer sums: bit for bit
            np.testing.assert_array_equal(d.rows(np.arange(12)), g["rows_" + w])
        else:                               # real weights: float64 sums in another order
            np.testing.assert_allclose(d.rows(np.arange(12)), g["rows_" + w], rtol=1e-14, atol=1e-15)
        np.testing.assert_array_equal(d.rows(np.array([11, 0, 5])), d.rows(np.arange(12))[[11, 0, 5]])
    replies = dict(menu=g["panel_menu"], chosen=g["panel_chosen"])
    rm, ra, rp = D.cells_from_panel(replies, 8)
    np.testing.assert_array_equal(rm, g["rep_menu"])
    np.testing.assert_array_equal(ra, g["rep_alt"])
    np.testing.assert_array_equal(rp, g["rep_p"])
    md = D.MenuDraws(replies, rm, ra, rp, B=12, seed=5)
    np.testing.assert_array_equal(md.rows(np.arange(12)), g["rows_replies"])
    am, aa, ap = D.cells_from_panel(panel, 8, alternatives=[0])
    np.testing.assert_array_equal(am, g["alt0_menu"])
    np.testing.assert_array_equal(ap, g["alt0_p"])
    m, a, p = g["menu"], g["alternative"], g["p_hat"]
    bad = (lambda: D.Draws(panel, m, a, p + 0.01, B=2),
           lambda: D.Draws(dict(respondent=g["panel_respondent"], menu=g["panel_menu"]), m, a, p, B=2),
           lambda: D.Draws(panel, np.r_[m, 255], np.r_[a, 0], np.r_[p, 0.5], B=2))
    for f, msg in zip(bad, g["errors"]):
        with pytest.raises(ValueError) as e:
            f()
        assert str(e.value) == str(msg)


def test_interval_formulas_match_reference_golden():
    from rumb import bootstrap as BS
    g = np.load(os.path.join(GOLD, "draws.npz"))
    for j, alpha in enumerate((0.05, 0.1, 0.5)):
        low, high, q = BS.ci_lower(1.2, 1.3, g["hl_L"], g["hl_U"], alpha, 22.8, 0.124)
        np.testing.assert_array_equal([low, high, q[0], q[1]], g["hl_ci_%d" % j])
        np.testing.assert_array_equal(BS.distance_interval(1.2, 1.3, g["hl_dev"], alpha), g["hl_di_%d" % j])
        np.testing.assert_array_equal(BS.quantile_band(g["hl_L"], g["hl_U"], alpha), g["hl_band_%d" % j])
    for (a_, o_, b_, al), want in zip(g["hl_locked_in"], g["hl_locked"]):
        assert BS.locked(int(a_), int(o_), int(b_), al) == bool(want)
    with pytest.raises(ValueError):
        BS.check_alpha(1.0)


def test_flow_cg_lower_bound_layout():
    """The reference's choice of the final lower bound's form by device memory: the float64 slab,
    else two float64 lattice layers, else the pricing bound."""
    assert flow_cg.lb_layout(18, 23568, 180e9) == "slab"
    slab = 16 * (30 << 29) + 16 * (1 << 30)
    two = flow_cg.sweep_max64_bytes(30, 10 ** 5)
    assert two < slab
    assert flow_cg.lb_layout(30, 10 ** 5, slab) == "slab"
    assert flow_cg.lb_layout(30, 10 ** 5, slab - 1) == "two layers"
    assert flow_cg.lb_layout(30, 10 ** 5, two - 1) == "pricing sweep"
    assert flow_cg.sweep_max64_bytes(33, 0) == 2 * 8 * math.comb(33, 16) + 8 * 34 * 35 + 4096


def test_gram_maintainer_growth():
    """Q and h stay V'V and V'p_hat while the storage doubles (256 -> 512 columns)."""
    rng = np.random.default_rng(4)
    M = 200
    ph = rng.random(M)
    g = flow_cg.GramMaintainer(M, ph, max_K=600)
    cols = [(rng.random(M) < 0.3).astype(np.uint8) for _ in range(300)]
    for c in cols:
        g.add_column(c.astype(np.float64))
    V = np.stack(cols, axis=1).astype(np.float64)
    Q, h = g.view()
    assert g.cap == 512
    np.testing.assert_array_equal(Q, V.T @ V)
    np.testing.assert_allclose(h, V.T @ ph, rtol=1e-13)


def test_qp_memo_is_bit_identical():
    """The master's reuse of the previous call's last active-set solve changes no bit of lambda or
    the support over a CG-like sequence of growing Gram matrices."""
    rng = np.random.default_rng(5)
    M, K = 400, 120
    ph = rng.dirichlet(np.ones(M)) * 30
    g = flow_cg.GramMaintainer(M, ph, max_K=K)
    A_plain = A_memo = [0]
    memo = {}
    hits = 0
    for k in range(K):
        g.add_column((rng.random(M) < 0.35).astype(np.float64))
        Q, h = g.view()
        hits += memo.get("key") == tuple(A_memo)
        lam1, A_plain = flow_cg.solve_qp_native(Q, h, A_init=A_plain)
        lam2, A_memo = flow_cg.solve_qp_native(Q, h, A_init=A_memo, memo=memo)
        np.testing.assert_array_equal(lam1, lam2)
        assert A_plain == A_memo
    assert hits > K // 2


def test_cg_loop_matches_oracle_with_a_scripted_pricer():
    """The host CG loop (with its master pieces and the QP memo) and the oracle's CG loop, driven by
    the same scripted pricer, take the same columns and reach the same bounds bit for bit."""
    import oracle as O
    n = 9
    m, a, p = mixture_instance(n, 0.5, K=8, N=60, seed=3)

    def scripted(scores, menus, alts):
        s = np.bincount(alts, weights=scores.astype(np.float64), minlength=n)
        order = np.argsort(-s, kind="stable")
        rank = np.empty(n, dtype=np.int32)
        rank[order] = np.arange(n, dtype=np.int32)
        col = O.ranking_column(n, menus, alts, rank)
        return float(scores.astype(np.float64)[col > 0].sum()), rank, 0.0

    class Prob:
        pass

    prob = Prob()
    prob.n = n
    prob.menus, prob.alts, _, _, prob.perm = flow_cg.prepare_choice_data(m, a, p, n)

    class Pricer:
        def price(self, scores):
            return scripted(scores, prob.menus, prob.alts)

    prob.pricer = Pricer()
    mine = flow_cg.solve_cg(prob, p, max_iters=60, gap_abs_tol=1e-9, record_columns=True)
    ref = O.cg_solve(n, m, a, p, max_iters=60, gap_abs_tol=1e-9,
                     pricer=lambda sc: scripted(sc, prob.menus, prob.alts))
    assert len(mine["picked"]) == len(ref["columns"])
    for x, y in zip(mine["picked"], ref["columns"]):
        np.testing.assert_array_equal(x, y)
    assert mine["distance"] == ref["ub"] and mine["lb"] == ref["lb"]


def test_generators_shapes_and_determinism():
    n, m, a, p = config_instance("n10_all_k20")
    assert np.unique(m).size == 1013 and m.size == 5110
    sums = np.bincount(np.unique(m, return_inverse=True)[1], weights=p)
    np.testing.assert_allclose(sums, 1.0)
    m1, a1, p1 = mixture_instance(12, 0.2, 5, 100, seed=4)
    m2, a2, p2 = mixture_instance(12, 0.2, 5, 100, seed=4)
    assert np.array_equal(m1, m2) and np.array_equal(p1, p2)
    panel, (mm, aa, pp) = panel_instance(12, 0.1, 40, 5, 4, seed=1)
    assert panel["menu"].size == 200 and set(np.unique(panel["respondent"])) == set(range(40))
    panel, (mm, aa, pp) = dsr_instance(10, 20, 30, 4, seed=1)
    assert mm.size == 20 and (aa == 0).all() and ((mm & 1) == 1).all()


def test_bootstrap_draws_and_formulas():
    from rumb import bootstrap as BS
    from rumb.instances import panel_instance
    panel, (m, a, p) = panel_instance(10, 0.2, 60, 6, 4, seed=3)
    d = BS.Draws(panel, m, a, p, B=20, weights="multinomial", seed=0)
    rows = d.rows(np.arange(20))
    assert rows.shape == (20, p.size)
    # a draw with every respondent weighted once reproduces p_hat
    d.W[0] = 1.0
    d._held = None                              # the weights changed under the kept block
    np.testing.assert_allclose(d.rows([0])[0], p, atol=1e-12)
    # shares stay shares
    sums = np.zeros((20, np.unique(m).size))
    inv = np.unique(m, return_inverse=True)[1]
    for k in range(20):
        sums[k] = np.bincount(inv, weights=rows[k])
    np.testing.assert_allclose(sums, 1.0, atol=1e-12)
    r_n, eps_n, s = BS.scaling(520)
    assert r_n == pytest.approx(math.sqrt(520)) and eps_n == pytest.approx(520 ** (-1 / 3))
    dec = BS.decide([0.0, 3.0, 1.0], [0.5, 4.0, 2.5], 1.0, 2.0)
    assert list(dec) == [BS.BELOW, BS.ABOVE, BS.UNDECIDED]


def test_bootstrap_record_checkpoint_and_resume(fake_gpu, tmp_path):
    """The record's layout (the reference's, solver/inference/bootstrap.py:356-400), an atomic
    checkpoint, a resume that restores every draw, and a refusal to resume another run's file."""
    from rumb import bootstrap as BS
    from rumb.rum_solver import RUM
    panel, (m, a, p) = panel_instance(10, 0.2, 60, 6, 4, seed=3)
    rum = RUM(m, a, p, num_alternatives=10)
    path = str(tmp_path / "boot.json")
    b = rum.bootstrap(panel=panel, B=12, weights="multinomial", seed=0, method="bm_admm", checkpoint=path)
    b.L0, b.U0 = 0.5, 0.6
    b.L[:4], b.U[:4] = [0.1, 0.2, 0.3, 0.4], [0.15, 0.25, 0.35, 0.45]
    b.flag[:4] = [1, 1, 5, -2]
    b.tol_stop[:4] = 5e-4
    b.screened, b.n_screened = True, 3
    b.save(path)
    rec = json.load(open(path))
    assert set(rec) >= {"version", "settings", "fingerprints", "plan", "p_hat", "tau", "scaling", "screen", "panel",
                        "draws", "results", "time", "when"}
    assert rec["draws"]["exit_flag"][:5] == [1, 1, 5, -2, BS.NEVER] and rec["draws"]["ub"][5] == float("inf")
    r = rum.bootstrap(panel=panel, B=12, weights="multinomial", seed=0, method="bm_admm", checkpoint=path)
    np.testing.assert_array_equal(r.L, b.L)
    np.testing.assert_array_equal(r.U, b.U)
    np.testing.assert_array_equal(r.flag, b.flag)
    assert (r.L0, r.U0) == (0.5, 0.6) and r.screened and r.solved.sum() == 4
    with pytest.raises(ValueError, match="belongs to another run"):
        rum.bootstrap(panel=panel, B=12, weights="multinomial", seed=1, method="bm_admm", checkpoint=path)


def test_bootstrap_inputs_refused(fake_gpu):
    """The bootstrap's constructor refuses what the reference refuses: both tables or neither,
    weights with replies, tolerances that cannot stop, an n that the replies cannot give."""
    from rumb import cells_from_panel
    panel, _ = panel_instance(8, 0.4, 30, 5, 3, seed=4)
    replies = dict(menu=panel["menu"], chosen=panel["chosen"])
    rum = rum_solver.RUM(*cells_from_panel(panel, 8), num_alternatives=8)
    with pytest.raises(ValueError, match="give the choices behind p_hat once"):
        rum.bootstrap(panel=panel, replies=replies, B=4)
    with pytest.raises(ValueError, match="give the choices behind p_hat once"):
        rum.bootstrap(B=4)
    with pytest.raises(ValueError, match="not both 0"):
        rum.bootstrap(panel=panel, B=4, abs_tol=0.0, rel_tol=0.0)
    with pytest.raises(ValueError, match="n = 7, but the panel has 30 respondents"):
        rum.bootstrap(panel=panel, B=4, n=7)
    rr = rum_solver.RUM(*cells_from_panel(replies, 8), num_alternatives=8)
    with pytest.raises(ValueError, match="is for panel="):
        rr.bootstrap(replies=replies, B=4, weights="poisson")
    b = rr.bootstrap(replies=replies, B=4)
    assert b.settings["input"] == "replies" and b.n == b.draws.default_n
    assert set(b.record()) >= {"replies", "p_hat", "draws", "results"}
    with pytest.raises(ValueError, match="replies per menu"):
        rr.bootstrap(replies=replies, B=4, n=10 ** 6)


_RECORDS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "records.json")


@pytest.mark.skipif(not os.path.exists(_RECORDS), reason="reference records not recorded")
def test_records_byte_compatible_with_the_reference(fake_gpu):
    """Result.to_dict() and Bootstrap.record() give the JSON text the reference's own writers gave
    for the same values and inputs (tests/golden/make_record_golden.py; solver/rum_solver.py:143-149,
    solver/inference/bootstrap.py:356-370), byte for byte: field names, order and values."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_record_golden as MRG
    from rumb import cells_from_panel
    g = json.load(open(_RECORDS))
    assert json.dumps(rum_solver.Result(**MRG.RESULT_FIELDS).to_dict()) == g["result_to_dict"]
    panel, m, a, p = MRG.panel_case()
    rec = rum_solver.RUM(m, a, p, num_alternatives=8).bootstrap(panel=panel, B=12, weights="multinomial",
                                                               seed=5).record()
    rec.pop("when")
    assert json.dumps(rec, indent=1) == g["bootstrap_panel_record"]
    replies = dict(menu=panel["menu"], chosen=panel["chosen"])
    rec = rum_solver.RUM(*cells_from_panel(replies, 8), num_alternatives=8).bootstrap(replies=replies, B=6,
                                                                                      seed=3).record()
    rec.pop("when")
    assert json.dumps(rec, indent=1) == g["bootstrap_replies_record"]


def test_prox_profile_records_match_the_built_source():
    """bench.py reads the prox's DRAM traffic from the committed ncu summary whose source digest is
    the digest of csrc/prox.cu + prox.cuh as built, and reports null otherwise: every prox form the
    tuner picks at the bench's workload (one or two threads per menu) has a record for this source."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for kernel in ("prox_pair<f64>", "prox_tau2<f64>"):
        traffic, src = bench.kernel_traffic(kernel)
        assert traffic is not None and src is not None, kernel
        assert 55e6 < traffic < 70e6, (kernel, traffic)
