"""Flow-CG: column generation whose pricing (the Bellman-Ford longest path over the subset
lattice) runs in librumb.so, with the restricted master on the host.

The host side follows the reference step for step, so that with bit-identical pricing the column
picked at every iteration is the reference's:

    CGData layout          rows stably sorted by alternative, p_hat as float32
                           (solver/flow_cg/cg_core.py:135-145)
    ranking -> column      the alternative is the best-ranked member of its menu
                           (solver/flow_cg/cg_core.py:63-80)
    Gram maintainer        Q = V'V by popcount of packed 0/1 columns, h = V'p_hat
                           (solver/flow_cg/qp_bitset_incremental.py:36-83)
    p_out maintainer       p_out = V lam, updated by the change in lam (:99-141)
    master                 active set + Cholesky on the simplex QP (solver/common/qp_native.py:20-99)
    CG loop                solve_cgbfqp_cholbitset (solver/flow_cg/solver.py:28-279)
    certified runner       _run_flow_cg (solver/rum_solver.py:941-1016): float64 ub and lb for the
                           true p, one retry with tightened tolerances
"""
import math
import time

import numpy as np
from scipy.linalg import cho_factor, cho_solve


# ------------------------------------------------------------------ layout and columns
def prepare_choice_data(menu, alt, p, n):
    """x-major rows: (menus uint64, alternatives int32, p float32, offsets int64[n+1], perm)."""
    menu = np.asarray(menu, dtype=np.int64).astype(np.uint64)
    alt = np.asarray(alt, dtype=np.int32)
    perm = np.argsort(alt, kind="stable")
    counts = np.bincount(alt, minlength=n)
    offsets = np.concatenate(([0], np.cumsum(counts))).astype(np.int64)
    return menu[perm], alt[perm], np.asarray(p, dtype=np.float64)[perm].astype(np.float32), offsets, perm


def ranking_column(menus, alts, rank_pos, n):
    """0/1 column: row s is 1 when alts[s] is the best-ranked member of menus[s] (alternatives
    visited best first; a row's winner is the first of them in its menu)."""
    rank_pos = np.asarray(rank_pos, dtype=np.int64)
    left = np.ones(menus.size, dtype=bool)
    col = np.zeros(menus.size, dtype=np.uint8)
    for x in np.argsort(rank_pos, kind="stable"):
        hit = left & ((menus & np.uint64(1 << int(x))) != 0)
        col[hit & (alts == x)] = 1
        left &= ~hit
    return col


def _popcount64(x):
    return np.bitwise_count(np.asarray(x, dtype=np.uint64))


def _pack(col):
    M = len(col)
    w = (M + 63) // 64
    padded = np.zeros(w * 64, dtype=np.uint8)
    padded[:M] = (col > 0.5).astype(np.uint8)
    return np.packbits(padded, bitorder="little").view(np.uint64)


class GramMaintainer:
    """Q = V'V (popcount of packed columns) and h = V'p_hat, one column at a time."""

    def __init__(self, M, phat, max_K):
        self.M, self.W = int(M), (int(M) + 63) // 64
        self.phat = np.asarray(phat, dtype=np.float64)
        self.K, self.max_K = 0, int(max_K)
        self._grow(min(self.max_K, 256))

    def _grow(self, cap):
        """Storage for cap columns (doubled as columns arrive, so Q's rows stay close together)."""
        bits, Q, h = np.zeros((cap, self.W), dtype=np.uint64), np.zeros((cap, cap)), np.zeros(cap)
        if self.K:
            k = self.K
            bits[:k], Q[:k, :k], h[:k] = self.bits[:k], self.Q[:k, :k], self.h[:k]
        self.bits, self.Q, self.h, self.cap = bits, Q, h, cap

    def add_column(self, col):
        k = self.K
        if k >= self.max_K:
            raise RuntimeError("max_K=%d exceeded" % self.max_K)
        if k >= self.cap:
            self._grow(min(self.max_K, 2 * self.cap))
        b = _pack(col)
        self.bits[k] = b
        if k > 0:
            counts = _popcount64(self.bits[:k] & b).sum(axis=1, dtype=np.int64).astype(np.float64)
            self.Q[k, :k] = counts
            self.Q[:k, k] = counts
        self.Q[k, k] = float(_popcount64(b).sum())
        self.h[k] = float(self.phat[np.where(col > 0.5)[0]].sum())
        self.K += 1
        return k

    def view(self):
        return self.Q[:self.K, :self.K], self.h[:self.K]


class PoutMaintainer:
    """p_out = sum_a lam_a V[:, a], updated by the change in lam."""

    def __init__(self, M):
        self.p_out = np.zeros(M)
        self.pos = []

    def add_column(self, col):
        self.pos.append(np.where(col.astype(bool))[0].astype(np.int64))

    def apply_delta(self, delta):
        # np.add.at adds in index order, one element at a time: the same float64 sums as the
        # reference's fancy-index += (a column's positions are distinct), without its temporaries
        for a in np.where(np.abs(delta) > 1e-12)[0]:
            np.add.at(self.p_out, self.pos[int(a)], float(delta[a]))


class _HostMaster:
    """Column bookkeeping on the host (the reference's maintainers): for pricers that are not the
    library's (scripted pricers in tests)."""

    def __init__(self, prob, p_obs, max_K):
        self.prob, self.p_obs = prob, p_obs
        self.gram = GramMaintainer(p_obs.size, p_obs, max_K)
        self.pout = PoutMaintainer(p_obs.size)

    def add_ranking(self, rank_pos):
        return self.add_col(ranking_column(self.prob.menus, self.prob.alts, rank_pos, self.prob.n))

    def add_col(self, col):
        self.gram.add_column(col.astype(np.float64))
        self.pout.add_column(col)
        return col

    def view(self):
        return self.gram.view()

    def apply_delta(self, delta):
        self.pout.apply_delta(delta)

    def price(self):
        return self.prob.pricer.price((self.p_obs - self.pout.p_out).astype(np.float32))

    def p_out(self):
        return self.pout.p_out.copy()


class _DeviceMaster:
    """Column bookkeeping on the pricer's GPU (rumb_cg_master_*): the column of a ranking, its Gram
    row, p_out and the float32 residual stay on the device, bit for bit the host maintainers'
    values; Q and h = V'p_obs (numpy's sum, as the reference) are kept here for the QP."""

    def __init__(self, prob, p_obs, max_K):
        from . import _lib
        self.dev = _lib.CgMaster(prob.pricer, prob.alts, p_obs, max_K)
        self.gram = GramMaintainer(p_obs.size, p_obs, max_K)
        self.M = p_obs.size

    def _store(self, k, bits, row):
        g = self.gram
        if k >= g.cap:
            g._grow(min(g.max_K, 2 * g.cap))
        col = np.unpackbits(bits.view(np.uint8), bitorder="little")[:self.M]
        g.bits[k] = bits
        g.Q[k, :k] = row[:k]
        g.Q[:k, k] = row[:k]
        g.Q[k, k] = row[k]
        g.h[k] = float(g.phat[np.where(col > 0.5)[0]].sum())
        g.K = k + 1
        return col

    def add_ranking(self, rank_pos):
        return self._store(*self.dev.add_column(rank_pos=rank_pos))

    def add_col(self, col):
        return self._store(*self.dev.add_column(bits=_pack(col)))

    def view(self):
        return self.gram.view()

    def apply_delta(self, delta):
        a = np.where(np.abs(delta) > 1e-12)[0]
        self.dev.apply(a, delta[a])

    def price(self):
        return self.dev.price()

    def p_out(self):
        return self.dev.p_out()


def project_simplex(y):
    n = y.size
    u = np.sort(y)[::-1]
    css = np.cumsum(u) - 1.0
    cond = u - css / np.arange(1, n + 1) > 0
    if not cond.any():
        return np.ones(n) / n
    rho = int(np.where(cond)[0][-1] + 1)
    return np.maximum(y - css[rho - 1] / rho, 0.0)


def solve_qp_native(Q, h, A_init=None, max_outer=200, tol=1e-10, reg=1e-12, memo=None):
    """Active set + Cholesky for min 1/2 lam'Q lam - h'lam over the simplex; (lam, support).

    memo: a dict kept across the calls of one CG run. Q's and h's entries never change once a
    column is in (columns are only appended), so the solve for an active set seen in the previous
    call's last step (the warm start's set, as a rule) is that step's result, bit for bit; it is
    reused instead of factorized again."""
    K = len(h)
    A = [int(i) for i in (A_init if A_init is not None else []) if 0 <= i < K] or [int(np.argmax(h))]
    lam_A, A_arr = None, None
    for _ in range(max_outer):
        A_arr = np.asarray(A, dtype=np.int64)
        k = len(A)
        key = tuple(A)
        if memo is not None and memo.get("key") == key:
            lam_A, mu = memo["lam_A"], memo["mu"]
        else:
            ones_A = np.ones(k)
            Q_AA = Q[np.ix_(A_arr, A_arr)]
            Q_AA[np.diag_indices(k)] += reg       # = Q_AA + reg * I bit for bit (the entries are >= 0)
            h_A = h[A_arr]
            try:
                cf = cho_factor(Q_AA, lower=True, check_finite=False)
                sol = cho_solve(cf, np.column_stack([h_A, ones_A]), check_finite=False)
                Q_inv_h, Q_inv_e = sol[:, 0], sol[:, 1]
            except np.linalg.LinAlgError:
                Q_inv_h = np.linalg.lstsq(Q_AA, h_A, rcond=None)[0]
                Q_inv_e = np.linalg.lstsq(Q_AA, ones_A, rcond=None)[0]
            eQe = float(ones_A @ Q_inv_e)
            eQh = float(ones_A @ Q_inv_h)
            mu = (eQh - 1.0) / eQe if abs(eQe) > 1e-30 else 0.0
            lam_A = Q_inv_h - mu * Q_inv_e
            if memo is not None:
                memo.update(key=key, lam_A=lam_A, mu=mu)
        if k > 0 and float(lam_A.min()) < -tol:
            del A[int(np.argmin(lam_A))]
            continue
        if K > k:
            mask = np.ones(K, dtype=bool)
            mask[A_arr] = False
            inactive = np.where(mask)[0]
            grad = Q[np.ix_(inactive, A_arr)] @ lam_A + mu - h[inactive]
            i_min = int(np.argmin(grad))
            if grad[i_min] < -tol:
                A.append(int(inactive[i_min]))
                continue
        break
    lam = np.zeros(K)
    lam[A_arr] = lam_A
    lam = project_simplex(lam)
    return lam, [int(i) for i in A if lam[i] > 1e-9]


# ------------------------------------------------------------------ the CG engine
class CGProblem:
    """The x-major rows of one geometry and its GPU pricer (built once, reused across solves)."""

    def __init__(self, ctx, n, menu, alt, mode, k_pred=None):
        from . import _lib
        self.n = int(n)
        self.menus, self.alts, _, self.offsets, self.perm = prepare_choice_data(menu, alt, np.zeros(len(menu)), n)
        self.mode = mode
        self.pricer = _lib.Pricer(ctx, n, self.menus, self.offsets, mode=mode, k_pred=k_pred)


def _one_blas_thread():
    """The master's matrices are at most a few hundred wide: a multithreaded BLAS spends more on
    waking threads than on the factorizations, so the CG loop runs with one BLAS thread."""
    try:
        from threadpoolctl import threadpool_limits
    except ImportError:
        import contextlib
        return contextlib.nullcontext()
    return threadpool_limits(1, user_api="blas")


def solve_cg(prob, p, **kw):
    """solve_cgbfqp_cholbitset on a CGProblem with row probabilities p (input row order)."""
    with _one_blas_thread():
        return _solve_cg(prob, p, **kw)


def _solve_cg(prob, p, rc_tol=0.0, max_iters=4000, time_limit_s=0.0, seed=0, phi_ub_target=None, gap_rel_tol=None,
              gap_abs_tol=None, init_columns=None, init_lambda=None, early_ub_check=False, lb_stop=None,
              record_columns=False, on_price=None):
    """on_price(it, scores, vmax, rank_pos, margin), when given, sees every pricing call with the
    float32 residual it priced (x-major rows; read back from the master, so it costs a copy)."""
    n = prob.n
    t_setup = time.perf_counter()
    p_obs = np.asarray(p, dtype=np.float64)[prob.perm].astype(np.float32).astype(np.float64)
    M = p_obs.size
    p_sq = float(p_obs @ p_obs)
    lb_best, gap_rel = 0.0, math.inf
    n_init = len(init_columns) if init_columns is not None else 0
    from . import _lib
    master = (_DeviceMaster if isinstance(prob.pricer, _lib.Pricer) else _HostMaster)(prob, p_obs,
                                                                                      max_iters + 2 + n_init)
    if n_init:
        cols = [np.ascontiguousarray(np.asarray(c, dtype=np.uint8)) for c in init_columns]
        for c in cols:
            master.add_col(c)
        K = n_init
        lam = (np.asarray(init_lambda, dtype=np.float64).copy() if init_lambda is not None else np.full(K, 1.0 / K))
        lam = np.maximum(lam, 0.0)
        lam /= lam.sum()
        master.apply_delta(lam)
        A_warm = [int(i) for i in np.where(lam > 1e-12)[0]] or [0]
        keys = [bytes(c) for c in cols]
    else:
        perm0 = np.random.RandomState(seed).permutation(n)
        col0 = master.add_ranking(perm0)
        K, lam, A_warm = 1, np.array([1.0]), [0]
        master.apply_delta(np.array([1.0]))
        keys = [bytes(col0)]
    setup_s = time.perf_counter() - t_setup
    qp_s = price_s = 0.0
    qp_memo = {}
    UB, rc_final, stop, margins, trace, picked = math.inf, math.nan, "max_iters", [], [], []
    t_total = time.perf_counter()
    it = 0
    for it in range(1, max_iters + 1):
        if time_limit_s > 0 and (time.perf_counter() - t_total) > time_limit_s:
            stop = "time_limit"
            break
        t = time.perf_counter()
        Qv, hv = master.view()
        lam_new, A_warm = solve_qp_native(Qv, hv, A_init=A_warm, memo=qp_memo)
        master.apply_delta(lam_new - lam)
        lam = lam_new
        QL = Qv @ lam
        lql = float(lam @ QL)
        hl = float(hv @ lam)
        err2 = lql - 2.0 * hl + p_sq
        inner = hl - lql
        if early_ub_check and phi_ub_target is not None:
            UB = float(np.sqrt(max(0.0, err2)))
            if UB <= phi_ub_target:
                stop = "phi_ub"
                break
        qp_s += time.perf_counter() - t
        t = time.perf_counter()
        vmax, rank_pos, margin = master.price()      # the float32 residual p_obs - p_out
        price_s += time.perf_counter() - t
        margins.append(margin)
        if record_columns:
            picked.append(rank_pos.copy())
        if on_price is not None:
            on_price(it, (p_obs - master.p_out()).astype(np.float32), vmax, rank_pos, margin)
        fw_gap = (vmax + margin) - inner
        rc_final = fw_gap
        UB = float(np.sqrt(max(0.0, err2)))
        lb_best = max(lb_best, float(np.sqrt(max(0.0, err2 - 2.0 * fw_gap))))
        gap_rel = (UB - lb_best) / lb_best if lb_best > 0 else math.inf
        trace.append((it, time.perf_counter() - t_total, UB, lb_best, K))
        if phi_ub_target is not None and UB <= phi_ub_target:
            stop = "phi_ub"
            break
        if lb_stop is not None and lb_best >= lb_stop:
            stop = "lb_stop"
            break
        if gap_rel_tol is not None and gap_rel <= gap_rel_tol:
            stop = "gap_rel"
            break
        if gap_abs_tol is not None and (UB - lb_best) <= gap_abs_tol:
            stop = "gap_abs"
            break
        if fw_gap < rc_tol:
            stop = "rc"
            break
        col = master.add_ranking(rank_pos)
        keys.append(bytes(col))
        K += 1
        lam = np.concatenate([lam, [0.0]])
    wall_s = time.perf_counter() - t_total
    return dict(wall_s=wall_s, setup_s=setup_s, trace=trace, margins=margins, iters=it, n_cols=K, lam=lam,
                p_out=master.p_out(), columns=[np.frombuffer(k, dtype=np.uint8).copy() for k in keys],
                rc_final=rc_final, distance=UB, lb=lb_best, gap_rel=gap_rel, stop_reason=stop, qp_s=qp_s,
                price_s=price_s, picked=picked)


# ------------------------------------------------------------------ certified runner
def sweep_max64_bytes(n, rows):
    """Device bytes of the float64 max sweep: two float64 layers of C(n, n//2) ranks, the rows
    (menu + score) and the tables (solver/flow_cg/pricing_stream.py:228-231)."""
    return 2 * 8 * math.comb(n, n // 2) + 16 * int(rows) + 8 * (n + 1) * (n + 2) + 4096


def fw_lb_stream64(prob, y, phat):
    """fw_lb_stream64 (solver/common/transforms.py:117-129) on a CGProblem's pricer: the float64
    Frank-Wolfe bound at the point y (rows in input order) through the two-layer max sweep."""
    y = np.asarray(y, dtype=np.float64)
    r = np.asarray(phat, dtype=np.float64) - y
    vmax = prob.pricer.max64(r[prob.perm])
    rc = vmax - float(r @ y)
    return float(np.sqrt(max(0.0, float(r @ r) - 2.0 * rc)))


def lb_layout(n, rows, budget):
    """_flow_cg_lb's choice (solver/rum_solver.py:926-938): the float64 bound from its slab when
    the slab fits, else two lattice layers at a time, else the pricing bound lowered by delta."""
    if 16 * (n << (n - 1)) + 16 * (1 << n) <= budget:
        return "slab"
    if sweep_max64_bytes(n, rows) <= budget:
        return "two layers"
    return "pricing sweep"


def _cg_stops(below, above, margin):
    kw = {}
    if below is not None:
        kw.update(phi_ub_target=max(below - margin, 0.0), early_ub_check=True)
    if above is not None:
        kw["lb_stop"] = above + margin
    return kw


def run_flow_cg(t, ctx):
    """The reference's _run_flow_cg: the engine solves for float32-rounded p; ub = the exact
    distance of the fitted mixture for the true p; lb = the float64 Frank-Wolfe bound at that
    mixture (on the GPU); one retry with tolerances tightened by the float64 excess."""
    from .rum_solver import _TimeUp  # noqa: F401
    g, a, st = t.geom, t.args, t.state
    n = g.num_alternatives
    engine = a["_engine"]
    key = (engine,)
    if g.pricer is None or g.pricer[0] != key:
        g.pricer = (key, CGProblem(ctx, n, g.menu, g.alternative, engine))
    prob = g.pricer[1]
    delta = float(np.linalg.norm(t.p - t.p.astype(np.float32).astype(np.float64)))
    rel, abs_e = t.rel_tol, max(t.abs_tol - 2 * delta, 0.0)
    below, above, kept = getattr(t, "below", None), getattr(t, "above", None), getattr(t, "warm", None)
    warm = {} if kept is None else dict(init_columns=kept["columns"], init_lambda=kept["lam"])
    stops = _cg_stops(below, above, 2 * delta)
    r = None
    for attempt in range(2):
        remaining = t.deadline - time.perf_counter()
        if remaining <= 0:
            return "time"
        t_call = time.perf_counter()
        kw = dict(gap_rel_tol=rel, gap_abs_tol=abs_e or None, time_limit_s=remaining, max_iters=int(a["max_iters"]),
                  seed=t.seed)
        kw.update(warm)
        kw.update(stops)
        r = solve_cg(prob, t.p, **kw)
        p_fit = np.empty(g.M)
        p_fit[prob.perm] = r["p_out"]
        st["p_fit"] = p_fit
        st["ub"] = float(np.linalg.norm(p_fit - t.p))
        lb_prev = st["lb"]
        from . import defaults
        from .rum_solver import gpu_free_bytes
        layout = lb_layout(n, g.M, defaults.AUTO["gpu_memory_fraction"] * gpu_free_bytes())
        if below is not None and st["ub"] < below:
            lb = lb_prev
        elif layout == "slab":
            lb = ctx.fw_lb64(n, g.menu.astype(np.uint32), g.alternative.astype(np.int32), p_fit, t.p)
        elif layout == "two layers":
            lb = fw_lb_stream64(prob, p_fit, t.p)
        else:
            lb = float(r["lb"]) - delta
        st["lb"] = max(lb_prev, lb)
        st["iterations"] = int(r["n_cols"])
        st["setup"] += float(r["setup_s"])
        off = t_call - t.t0 + float(r["setup_s"])
        st["trace"] += [(k, off + w, ub, max(lb_prev, lbv - delta)) for _it, w, ub, lbv, k in r["trace"]]
        if st["trace"]:
            st["trace"][-1] = st["trace"][-1][:2] + (st["ub"], st["lb"])
        st["info"].update(pricing=engine, p_float32_shift=delta,
                          pricing_margin=max(r["margins"]) if r["margins"] else 0.0, restarts=attempt,
                          lb_dtype=a["dtype"] if layout == "pricing sweep" else "float64", lb_layout=layout,
                          lb_rigorous=layout != "pricing sweep", qp_s=round(r["qp_s"], 3), price_s=round(r["price_s"], 3))
        if getattr(t, "keep", False):
            st["keep"] = dict(columns=r["columns"], lam=r["lam"])
        if (below is not None and st["ub"] < below) or (above is not None and st["lb"] >= above):
            return "threshold"
        gap = st["ub"] - st["lb"]
        if (attempt or r["stop_reason"] not in ("gap_rel", "gap_abs", "phi_ub", "lb_stop") or gap <= t.abs_tol
                or gap <= t.rel_tol * st["lb"]):
            break
        excess = 1.5 * max(gap - (float(r["distance"]) - float(r["lb"])), 2 * delta)
        rel = max(t.rel_tol - excess / st["lb"], 0.0) if st["lb"] > 0 else 0.0
        abs_e = max(t.abs_tol - 2 * delta - excess, 0.0)
        if rel <= 0 and abs_e <= 0 and not stops:
            break
        stops = _cg_stops(below, above, 2 * delta + excess)
        warm = dict(init_columns=r["columns"], init_lambda=r["lam"])
    return {"gap_rel": "tol", "gap_abs": "tol", "rc": "tol", "time_limit": "time",
            "max_iters": "iters"}.get(r["stop_reason"], "stalled")
