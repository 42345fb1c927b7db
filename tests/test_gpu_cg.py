"""Flow-CG pricing on the GPU through the C ABI: bit-exact against the oracle (values, rankings,
quantization steps) in every storage mode, and column-for-column equal CG trajectories."""
import os

import numpy as np
import pytest

import oracle as O
import paper_instances as PI
from rumb import _lib
from rumb.instances import config_instance

pytestmark = pytest.mark.gpu


def _cases():
    yield "pair6", PI.gen_pairwise(6)[0], 6
    yield "pair8", PI.gen_pairwise(8)[0], 8
    yield "med12", PI.gen_medium(12, mult=3)[0], 12
    yield "pair16", PI.gen_pairwise(16)[0], 16
    yield "med16", PI.gen_medium(16, mult=2)[0], 16
    n, m, a, p = config_instance("n18_d05pct_k50")
    yield "n18_d05pct", np.column_stack([m, a, p]).astype(np.float64), n


CASES = list(_cases())


@pytest.mark.parametrize("name,cd,n", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("mode", ["mask", "f32", "f32_stream", "u16", "u24"])
def test_pricer_bit_exact_against_oracle(ctx, name, cd, n, mode):
    """f32 stores the lattice by mask where it fits; f32_stream keeps the two rank-indexed layers."""
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    stream = mode == "f32_stream"
    mode = "f32" if stream else mode
    pr = _lib.Pricer(ctx, n, menus, offsets, mode=mode, stream=stream)
    rng = np.random.RandomState(7)
    trials = 2 if n >= 16 else 3
    for trial in range(trials):
        scores = (rng.randn(menus.size) * (2.0 if trial == 0 else 0.05)).astype(np.float32)
        if trial == trials - 1:
            scores = (p32 - p32.mean()).astype(np.float32)      # residual-like scores
        if mode == "mask":
            v_ref, r_ref = O.price_mask(n, menus, scores, offsets)
            m_ref = 0.0
        else:
            v_ref, r_ref, m_ref, steps_ref = O.price_stream(n, menus, scores, offsets, mode=mode)
        v, r, m, steps = pr.price(scores, want_steps=True)
        assert v == v_ref, (trial, v, v_ref)
        np.testing.assert_array_equal(r, r_ref)
        if mode in ("u16", "u24"):
            np.testing.assert_array_equal(steps, steps_ref)
            assert m == m_ref
    pr.close()


def _cover_entries(menus, n):
    pc = np.array([bin(int(v)).count("1") for v in menus])
    return int(np.sum(np.ldexp(1.0, n - pc)))


@pytest.mark.parametrize("name,cd,n", CASES, ids=[c[0] for c in CASES])
def test_cover_lists_equal_row_scan(ctx, name, cd, n):
    """The cover-list sweep and the row-scan sweep give the same bits in every storage mode (the
    scan itself is pinned to the oracle above and by the recorded reference kernels)."""
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    rng = np.random.RandomState(11)
    scores = [rng.randn(menus.size).astype(np.float32), (p32 - p32.mean()).astype(np.float32),
              np.round(rng.randn(menus.size) * 4).astype(np.float32)]       # many exact ties
    for mode, stream in (("mask", False), ("f32", False), ("f32", True), ("u16", False), ("u24", False)):
        a = _lib.Pricer(ctx, n, menus, offsets, mode=mode, stream=stream)
        b = _lib.Pricer(ctx, n, menus, offsets, mode=mode, lists=False, stream=stream)
        assert a.list_entries == _cover_entries(menus, n) and b.list_entries == -1
        for s in scores:
            va, ra, ma, sa = a.price(s, want_steps=True)
            vb, rb, mb, sb = b.price(s, want_steps=True)
            assert va == vb and ma == mb, (mode, va, vb)
            np.testing.assert_array_equal(ra, rb)
            np.testing.assert_array_equal(sa, sb)
        a.close()
        b.close()


def test_cover_lists_wide_alternative(ctx):
    """An alternative with more than 65536 rows (32-bit list entries): n = 18, alternative 0 observed
    in every menu of 9 or more that holds it (89,846 rows), the others in a sparse random set."""
    n = 18
    rng = np.random.RandomState(5)
    all_m = np.arange(1, 1 << n, dtype=np.int64)
    pc = np.array([bin(int(v)).count("1") for v in all_m])
    wide = all_m[((all_m & 1) == 1) & (pc >= 9)]
    rest = all_m[(pc >= 2) & (rng.rand(all_m.size) < 0.01)]
    rest_a = [[x for x in range(1, n) if (int(m) >> x) & 1] for m in rest]
    rows_m = np.concatenate([wide, np.repeat(rest, [len(r) for r in rest_a])])
    rows_a = np.concatenate([np.zeros(wide.size, dtype=np.int64), np.concatenate(rest_a).astype(np.int64)])
    menus, alts, p32, offsets, _ = O.cg_layout(n, rows_m, rows_a, np.ones(rows_m.size))
    assert offsets[1] - offsets[0] > 65536
    s = (rng.randn(menus.size) * 0.01).astype(np.float32)
    for mode in ("mask", "u24"):
        a = _lib.Pricer(ctx, n, menus, offsets, mode=mode)
        b = _lib.Pricer(ctx, n, menus, offsets, mode=mode, lists=False)
        assert a.list_entries == _cover_entries(menus, n)
        va, ra, ma = a.price(s)
        vb, rb, mb = b.price(s)
        assert va == vb and ma == mb
        np.testing.assert_array_equal(ra, rb)
        a.close()
        b.close()


@pytest.mark.parametrize("name,cd,n", CASES, ids=[c[0] for c in CASES])
def test_max64_sweep_bit_exact(ctx, monkeypatch, name, cd, n):
    """The float64 max sweep (rumb_cg_pricer_max64: the layer kernels over cover lists or scanning
    rows, and from n = 12 the group form) equals the oracle's and the reference's own
    bf_stream_max64 kernel bit for bit."""
    import ref_replay
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    rng = np.random.RandomState(13)
    for lists, form in ((True, "layer"), (False, "layer"), (False, "group")):
        monkeypatch.setenv("RUMB_STREAM_FORM", form)
        pr = _lib.Pricer(ctx, n, menus, offsets, mode="u24", lists=lists)
        for trial in range(2):
            s = rng.randn(menus.size) * (1.0 if trial == 0 else 1e-3)
            v = pr.max64(s)
            assert v == O.sweep_max64(n, menus, s, offsets)
            if ref_replay.available() and "max64" in ref_replay._mods():
                assert v == ref_replay.sweep_max64(menus, s, offsets, n)
        pr.close()


def test_two_layer_bound_equals_slab_bound(ctx):
    """fw_lb_stream64 through the max sweep and the slab-based float64 bound (rumb_fw_lb64) agree."""
    from rumb import flow_cg
    cd, mp = PI.gen_medium(14, mult=3)
    n = 14
    prob = flow_cg.CGProblem(ctx, n, cd[:, 0], cd[:, 1], "u24")
    rng = np.random.RandomState(2)
    p = cd[:, 2]
    for _ in range(3):
        y = np.clip(p + 0.05 * rng.randn(p.size), 0.0, 1.0)
        a = flow_cg.fw_lb_stream64(prob, y, p)
        b = ctx.fw_lb64(n, cd[:, 0].astype(np.uint32), cd[:, 1].astype(np.int32), y, p)
        assert abs(a - b) <= 1e-11 * max(1.0, b)
        assert a == O.fw_lb_stream64(n, cd[:, 0], cd[:, 1], y, p)


def test_master_and_max64_reject_bad_input(ctx):
    """The CG master and the float64 sweep refuse bad arguments with an error."""
    n = 8
    cd, mp = PI.gen_medium(n, mult=2)
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    pr = _lib.Pricer(ctx, n, menus, offsets, mode="mask")
    with pytest.raises(ValueError):
        pr.max64(np.zeros(menus.size + 1))
    with pytest.raises(_lib.RumbError):                     # an alternative out of range
        bad = alts.copy()
        bad[0] = n
        _lib.CgMaster(pr, bad, p32.astype(np.float64), 4)
    m = _lib.CgMaster(pr, alts, p32.astype(np.float64), 2)
    with pytest.raises(_lib.RumbError):                     # not a permutation
        m.add_column(rank_pos=np.zeros(n, dtype=np.int32))
    k, bits, row = m.add_column(rank_pos=np.arange(n, dtype=np.int32))
    assert k == 0 and row[0] == float(np.unpackbits(bits.view(np.uint8)).sum())
    with pytest.raises(_lib.RumbError):                     # a column the master does not hold
        m.apply(np.array([1]), np.array([0.5]))
    m.add_column(rank_pos=np.arange(n, dtype=np.int32)[::-1].copy())
    with pytest.raises(_lib.RumbError):                     # columns not increasing
        m.apply(np.array([1, 0]), np.array([0.5, 0.5]))
    with pytest.raises(_lib.RumbError):                     # beyond max_cols
        m.add_column(rank_pos=np.arange(n, dtype=np.int32))
    m.close()
    pr.close()


def test_mask_and_f32_stream_identical(ctx):
    cd, mp = PI.gen_medium(14, mult=4)
    menus, alts, p32, offsets, _ = O.cg_layout(14, cd[:, 0], cd[:, 1], cd[:, 2])
    a = _lib.Pricer(ctx, 14, menus, offsets, mode="mask")
    b = _lib.Pricer(ctx, 14, menus, offsets, mode="f32", k_pred=6, stream=True)
    rng = np.random.RandomState(3)
    for _ in range(4):
        s = rng.randn(menus.size).astype(np.float32)
        va, ra, _ = a.price(s)
        vb, rb, _ = b.price(s)
        assert va == vb and np.array_equal(ra, rb)


@pytest.mark.parametrize("mode", ["u24", "u16", "f32"])
def test_cg_trajectory_matches_oracle(ctx, mode):
    from rumb import flow_cg
    cd, mp = PI.gen_medium(12, mult=4)
    n = 12
    prob = flow_cg.CGProblem(ctx, n, cd[:, 0], cd[:, 1], mode)
    mine = flow_cg.solve_cg(prob, cd[:, 2], max_iters=120, gap_abs_tol=1e-6, record_columns=True)
    ref = O.cg_solve(n, cd[:, 0], cd[:, 1], cd[:, 2], mode=mode, max_iters=120, gap_abs_tol=1e-6)
    assert len(mine["picked"]) == len(ref["columns"])
    for i, (a, b) in enumerate(zip(mine["picked"], ref["columns"])):
        assert np.array_equal(a, b), "column %d differs" % i
    assert mine["distance"] == ref["ub"] and mine["lb"] == ref["lb"]


@pytest.mark.parametrize("mode", ["mask", "u24"])
def test_device_master_equals_host_master(ctx, mode):
    """The column bookkeeping on the GPU (rumb_cg_master_*) and the reference's host maintainers give
    the same run bit for bit: every column, lambda, p_out and the bounds (n = 14, warm restart too)."""
    from rumb import flow_cg
    cd, mp = PI.gen_medium(14, mult=3)
    n = 14

    class HostPricer:                      # not a _lib.Pricer: the loop keeps its books on the host
        def __init__(self, inner):
            self.inner = inner

        def price(self, s):
            return self.inner.price(s)

    prob = flow_cg.CGProblem(ctx, n, cd[:, 0], cd[:, 1], mode)
    dev = flow_cg.solve_cg(prob, cd[:, 2], max_iters=150, gap_abs_tol=1e-7, record_columns=True)
    inner = prob.pricer
    prob.pricer = HostPricer(inner)
    host = flow_cg.solve_cg(prob, cd[:, 2], max_iters=150, gap_abs_tol=1e-7, record_columns=True)
    assert dev["n_cols"] == host["n_cols"] and len(dev["picked"]) == len(host["picked"])
    for a, b in zip(dev["picked"], host["picked"]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(dev["columns"], host["columns"]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(dev["lam"], host["lam"])
    np.testing.assert_array_equal(dev["p_out"], host["p_out"])
    assert dev["distance"] == host["distance"] and dev["lb"] == host["lb"]
    # a warm restart from the kept columns
    prob.pricer = inner
    kw = dict(init_columns=dev["columns"], init_lambda=dev["lam"], max_iters=20, gap_abs_tol=1e-9)
    dev2 = flow_cg.solve_cg(prob, cd[:, 2], **kw)
    prob.pricer = HostPricer(inner)
    host2 = flow_cg.solve_cg(prob, cd[:, 2], **kw)
    np.testing.assert_array_equal(dev2["p_out"], host2["p_out"])
    np.testing.assert_array_equal(dev2["lam"], host2["lam"])


def test_cg_columns_on_config3_residuals(ctx):
    """n = 18, 0.5 % density: the GPU loop's residual scores at several iterations, priced again by
    the oracle, give the same columns."""
    from rumb import flow_cg
    n, m, a, p = config_instance("n18_d05pct_k50")
    for mode in ("u24", "u16"):
        prob = flow_cg.CGProblem(ctx, n, m, a, mode)
        seen = []

        class Spy:
            def __init__(self, inner):
                self.inner = inner

            def price(self, s):
                out = self.inner.price(s)
                if len(seen) in (0, 5, 20):
                    seen.append((s.copy(), out))
                else:
                    seen.append(None)
                return out

        prob.pricer = Spy(prob.pricer)
        flow_cg.solve_cg(prob, p, max_iters=25, gap_abs_tol=1e-9)
        menus, alts, p32, offsets, _ = O.cg_layout(n, m, a, p)
        for item in seen:
            if item is None:
                continue
            s, (v, r, mg) = item
            v_ref, r_ref, m_ref, _ = O.price_stream(n, menus, s, offsets, mode=mode)
            assert v == v_ref and np.array_equal(r, r_ref) and mg == m_ref


def test_pricer_rejects_bad_rows(ctx):
    with pytest.raises(_lib.RumbError):
        _lib.Pricer(ctx, 4, np.array([3, 4], dtype=np.uint64), np.array([0, 1, 2, 2, 2]), mode="u24")


_REPLAY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pricer_replay.npz")


@pytest.mark.skipif(not os.path.exists(_REPLAY), reason="reference kernel outputs not recorded")
def test_pricer_matches_recorded_reference_kernels(ctx):
    """Every stream mode and the mask sweep against the outputs the reference's own kernels gave
    (tests/golden/make_replay_golden.py), bit for bit, n = 8 .. 18."""
    import make_replay_golden as MR
    g = np.load(_REPLAY)
    for name, n, m, a, p in MR.cases():
        menus, alts, p32, offsets, _ = O.cg_layout(n, m, a, p)
        for mode in ("f32", "f32_stream", "u16", "u24") + (("mask",) if n <= 16 else ()):
            stream = mode == "f32_stream"
            mode = "f32" if stream else mode
            pr = _lib.Pricer(ctx, n, menus, offsets, mode=mode, stream=stream)
            for trial in range(2):
                key = "%s_t%d" % (name, trial)
                s = g[key + "_scores"]
                if mode == "mask":
                    v, r, _ = pr.price(s)
                    assert np.float32(v) == g[key + "_mask_vmax"]
                    np.testing.assert_array_equal(r, g[key + "_mask_rank"])
                    continue
                v, r, mg, steps = pr.price(s, want_steps=True)
                assert np.float32(v) == g["%s_%s_vmax" % (key, mode)], (key, mode)
                np.testing.assert_array_equal(r, g["%s_%s_rank" % (key, mode)])
                np.testing.assert_array_equal(np.asarray(steps, np.float32), g["%s_%s_steps" % (key, mode)])
                assert abs(mg - float(g["%s_%s_margin" % (key, mode)])) <= 1e-6 * max(1.0, mg)
            pr.close()


_CG3 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cg_config3.npz")


@pytest.mark.skipif(not os.path.exists(_CG3), reason="the n18_d05pct_k50 column sequence is not recorded")
@pytest.mark.parametrize("mode", ["u24", "u16"])
def test_config3_column_sequence_matches_recorded_reference(ctx, mode):
    """Flow-CG at n = 18, 0.5 % menus (the n18_d05pct_k50 workload) to abs 1e-5 (uint16: 1,000 columns,
    whose quantization margin keeps the bound above abs 1e-5): every CG iteration's column
    is the recorded one, which the reference's own pricing kernels picked on the same residual
    (tests/golden/make_cg_golden.py), and the bracket is the recorded bracket."""
    from rumb import flow_cg
    g = np.load(_CG3)
    n, m, a, p = config_instance("n18_d05pct_k50")
    prob = flow_cg.CGProblem(ctx, n, m, a, mode)
    res = flow_cg.solve_cg(prob, p, max_iters=4000 if mode == "u24" else 1000, gap_abs_tol=1e-5,
                           record_columns=True)
    np.testing.assert_array_equal(np.array(res["picked"]), g["picked_" + mode])
    assert [res["lb"], res["distance"]] == g["bracket_" + mode].tolist()


def _mask_pricer(ctx, monkeypatch, form, n, menus, offsets, **kw):
    monkeypatch.setenv("RUMB_MASK_FORM", form)
    pr = _lib.Pricer(ctx, n, menus, offsets, mode="mask", **kw)
    monkeypatch.delenv("RUMB_MASK_FORM")
    return pr


MASK_CASES = [c for c in CASES if c[2] >= 9]


@pytest.mark.parametrize("name,cd,n", MASK_CASES, ids=[c[0] for c in MASK_CASES])
@pytest.mark.parametrize("lists", [True, False], ids=["lists", "scan"])
def test_mask_tile_sweep_bit_exact(ctx, monkeypatch, name, cd, n, lists):
    """The tile sweep of the mask storage (one warp per 256 masks, launches by the popcount of the
    high part) against the oracle and against the layer kernels: value and ranking bit for bit on
    random, tie-heavy (integer) and residual-like scores."""
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    pt = _mask_pricer(ctx, monkeypatch, "tile", n, menus, offsets, lists=lists)
    pl = _mask_pricer(ctx, monkeypatch, "layer", n, menus, offsets, lists=lists)
    rng = np.random.RandomState(17)
    for scores in (rng.randn(menus.size).astype(np.float32),
                   np.round(rng.randn(menus.size) * 3).astype(np.float32),
                   (p32 - p32.mean()).astype(np.float32)):
        v_ref, r_ref = O.price_mask(n, menus, scores, offsets)
        for pr in (pt, pl):
            v, r, m = pr.price(scores)
            assert v == v_ref and m == 0.0
            np.testing.assert_array_equal(r, r_ref)
    pt.close()
    pl.close()


def test_mask_pricer_at_n28_equals_float32_stream(ctx, monkeypatch):
    """The mask pricer at n = 28 (2^28 float32 values, 1 GiB) gives the float32 stream pricer's
    value and ranking bit for bit (the reference's own check, validation/feasibility/
    test_stream_pricer.py:56-84, at the large-n end), in both mask forms."""
    n = 28
    cd, _ = PI.gen_pairwise(n)
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    scores = (np.random.RandomState(29).randn(menus.size)).astype(np.float32)
    pt = _mask_pricer(ctx, monkeypatch, "tile", n, menus, offsets)
    pl = _mask_pricer(ctx, monkeypatch, "layer", n, menus, offsets)
    ps = _lib.Pricer(ctx, n, menus, offsets, mode="f32", stream=True)
    vs, rs, _ = ps.price(scores)
    for pm in (pt, pl):
        vm, rm, _ = pm.price(scores)
        assert vm == vs and np.array_equal(rm, rs)
        pm.close()
    ps.close()


def test_mask_pricer_at_n32_equals_float32_stream(ctx):
    """Mask storage at n = 32 (2^32 values: 16 GiB of float32 and 4 GiB of predecessors, the tile
    sweep) against the float32 stream pricer on the pairwise instance."""
    n = 32
    cd, _ = PI.gen_pairwise(n)
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    scores = (np.random.RandomState(32).randn(menus.size)).astype(np.float32)
    pm = _lib.Pricer(ctx, n, menus, offsets, mode="mask")
    vm, rm, _ = pm.price(scores)
    pm.close()
    ps = _lib.Pricer(ctx, n, menus, offsets, mode="f32", stream=True)
    vs, rs, _ = ps.price(scores)
    ps.close()
    assert vm == vs and np.array_equal(rm, rs)


STREAM_CASES = [c for c in CASES if c[2] >= 12]


def _stream_pricer(ctx, monkeypatch, form, n, menus, offsets, mode, **kw):
    monkeypatch.setenv("RUMB_STREAM_FORM", form)
    stream = mode == "f32_stream"
    pr = _lib.Pricer(ctx, n, menus, offsets, mode="f32" if stream else mode, stream=stream, **kw)
    monkeypatch.delenv("RUMB_STREAM_FORM")
    return pr


@pytest.mark.parametrize("name,cd,n", STREAM_CASES, ids=[c[0] for c in STREAM_CASES])
@pytest.mark.parametrize("mode", ["f32_stream", "u16", "u24"])
def test_stream_group_sweep_bit_exact(ctx, monkeypatch, name, cd, n, mode):
    """The group sweep of the rank-indexed storage (one warp per set of subsets sharing their
    elements >= 10) against the oracle and the layer kernels: value, ranking, per-layer steps and
    margin bit for bit, with cover lists and with rows scanned."""
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    omode = "f32" if mode == "f32_stream" else mode
    rng = np.random.RandomState(23)
    scores = [rng.randn(menus.size).astype(np.float32), np.round(rng.randn(menus.size) * 3).astype(np.float32),
              (p32 - p32.mean()).astype(np.float32)]
    for lists in (True, False):
        pg = _stream_pricer(ctx, monkeypatch, "group", n, menus, offsets, mode, lists=lists)
        pl = _stream_pricer(ctx, monkeypatch, "layer", n, menus, offsets, mode, lists=lists)
        for s in scores:
            v_ref, r_ref, m_ref, steps_ref = O.price_stream(n, menus, s, offsets, mode=omode)
            for pr in (pg, pl):
                v, r, m, steps = pr.price(s, want_steps=True)
                assert v == v_ref, (lists, v, v_ref)
                np.testing.assert_array_equal(r, r_ref)
                np.testing.assert_array_equal(steps, steps_ref)
                assert m == m_ref
        pg.close()
        pl.close()


@pytest.mark.parametrize("mode", ["f32_stream", "u16", "u24"])
def test_sublattice_by_tile_sweep(ctx, mode):
    """Sub-lattices of 12 elements and more (k_pred >= 12) are solved by a tile sweep over the
    restricted rows; the value and ranking equal the oracle's with the same k_pred. In float32
    storage the ranking is also the one of the default k_pred (whose sub-lattice one CTA solves);
    quantized storages descend through predecessors chosen on decoded values, so theirs may move
    with k_pred."""
    omode = "f32" if mode == "f32_stream" else mode
    for name, cd, n in [c for c in CASES if c[2] >= 16]:
        menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
        s = np.random.RandomState(n).randn(menus.size).astype(np.float32)
        v0, r0, m0 = _lib.Pricer(ctx, n, menus, offsets, mode=omode, stream=True).price(s)
        for kp in (12, 14, n - 1):
            pr = _lib.Pricer(ctx, n, menus, offsets, mode=omode, stream=True, k_pred=kp)
            v_ref, r_ref, m_ref, _ = O.price_stream(n, menus, s, offsets, mode=omode, k_pred=kp)
            v, r, m = pr.price(s)
            pr.close()
            assert v == v_ref == v0 and m == m_ref
            np.testing.assert_array_equal(r, r_ref)
            if omode == "f32":
                np.testing.assert_array_equal(r, r0)


def test_stream_pricers_at_n33(ctx):
    """n = 33 (pairwise): the float32 stream (two rank-indexed layers, 9 GB; its 23-element
    sub-lattice by the tile sweep) equals the mask storage (40 GB) bit for bit, and the uint16
    stream's value lies within its margin of the exact one (validation/feasibility/
    test_stream_pricer.py:56-84)."""
    n = 33
    cd, _ = PI.gen_pairwise(n)
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    scores = (np.random.RandomState(33).randn(menus.size)).astype(np.float32)
    pm = _lib.Pricer(ctx, n, menus, offsets, mode="mask")
    vm, rm, _ = pm.price(scores)
    pm.close()
    ps = _lib.Pricer(ctx, n, menus, offsets, mode="f32", stream=True)
    vs, rs, _ = ps.price(scores)
    ps.close()
    assert vm == vs and np.array_equal(rm, rs)
    pu = _lib.Pricer(ctx, n, menus, offsets, mode="u16")
    vu, ru, mu = pu.price(scores)
    pu.close()
    assert mu > 0 and abs(vu - vm) <= mu + 1e-5 + 1e-6 * abs(vm)
    assert sorted(ru.tolist()) == list(range(n))
