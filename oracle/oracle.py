"""CPU oracle for the CUDA library -- TEST INFRASTRUCTURE ONLY.

A restatement of the reference's two hot paths (mingxiz/rum-testing-gpu) on the host: the C
pieces in rum_oracle.c (built into liboracle.so by the Makefile here) plus the host loops around
them. Only tests/, the smoke check and bench.py's CPU-baseline leg import this module; the
library under rum-testing-gpu_b200/ never does, and its product path fails loudly when its own
CUDA extension is missing.

Reference behaviour followed (file:line in the reference project):
  BMOracle.__init__    solve_kadmm_v2 setup         solver/bm_admm/solver.py:184-238
  BMOracle.iterate     one_iter                     solver/bm_admm/solver.py:240-254
  BMOracle.solve       check loop + runner hooks    solver/bm_admm/solver.py:308-367,
                                                    solver/rum_solver.py:869-911
  push_ub64            push_to_ub64                 solver/common/transforms.py:94-98
  fw_lb64              fw_lb_rows_gpu               solver/common/transforms.py:101-114
  price_stream         StreamPricer.price           solver/flow_cg/pricing_stream.py:267-412
  price_mask           bf_update sweep + backtrace  solver/flow_cg/solver.py:169-200
  cg_solve             solve_cgbfqp_cholbitset      solver/flow_cg/solver.py:28-279
  qp_native            solve_qp_native              solver/common/qp_native.py:37-99
"""
import ctypes
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_llp = ctypes.POINTER(ctypes.c_longlong)
_ullp = ctypes.POINTER(ctypes.c_ulonglong)
_ip = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_ubyte)


def build():
    """Compile liboracle.so with the Makefile next to this file."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.ora_slab_index.argtypes = [ctypes.c_int, ctypes.c_longlong, _ullp, _llp, _llp]
        L.ora_bfly_f64.argtypes = [ctypes.c_int, _dp] + [ctypes.c_double] * 4
        L.ora_bfly_f32.argtypes = [ctypes.c_int, _fp] + [ctypes.c_float] * 4
        L.ora_prox_f64.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double]
        L.ora_prox_f32.argtypes = [ctypes.c_int, _fp, _fp, _fp, _fp, ctypes.c_float]
        L.ora_admm_iter_f64.argtypes = ([ctypes.c_int] + [_dp] * 7 + [_dp] + [ctypes.c_double] * 6
                                        + [_dp, ctypes.c_int])
        L.ora_admm_iter_f32.argtypes = ([ctypes.c_int] + [_fp] * 7 + [_dp] + [ctypes.c_float] * 6
                                        + [_fp, ctypes.c_int])
        L.ora_make_feasible64.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double]
        L.ora_longest_path64.argtypes = [ctypes.c_int, _dp]
        L.ora_longest_path64.restype = ctypes.c_double
        L.ora_layers.argtypes = [ctypes.c_int, _llp, _llp]
        L.ora_colex_rank.argtypes = [ctypes.c_ulonglong]
        L.ora_colex_rank.restype = ctypes.c_ulonglong
        L.ora_price_mask.argtypes = [ctypes.c_int, _ullp, _fp, _llp, _ip]
        L.ora_price_mask.restype = ctypes.c_float
        L.ora_price_stream.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ullp, _fp,
                                       _llp, _dp, _ip, _dp, _fp]
        L.ora_ranking_column.argtypes = [ctypes.c_int, ctypes.c_longlong, _ullp, _ip, _ip, _u8p]
        L.ora_sweep_max64.argtypes = [ctypes.c_int, _ullp, _dp, _llp]
        L.ora_sweep_max64.restype = ctypes.c_double
        L.ora_set_threads.argtypes = [ctypes.c_int]
        L.ora_get_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def set_threads(t):
    """Threads of the oracle's parallel loops (0 = every core); results do not depend on it."""
    lib().ora_set_threads(int(t))
    return lib().ora_get_threads()


def _ptr(a, t):
    return a.ctypes.data_as(t)


# ------------------------------------------------------------------ lattice primitives
def slab_index(n, menu, alt):
    menu = np.ascontiguousarray(menu, dtype=np.uint64)
    alt = np.ascontiguousarray(alt, dtype=np.int64)
    out = np.empty(menu.size, dtype=np.int64)
    lib().ora_slab_index(n, menu.size, _ptr(menu, _ullp), _ptr(alt, _llp), _ptr(out, _llp))
    return out


def butterfly(n, v, a, b, c, d):
    """New array: the (a,b,c,d) butterfly over the rest bits, ascending, in v's dtype."""
    v = np.array(v, copy=True)
    if v.dtype == np.float64:
        lib().ora_bfly_f64(n, _ptr(v, _dp), a, b, c, d)
    elif v.dtype == np.float32:
        f = np.float32
        lib().ora_bfly_f32(n, _ptr(v, _fp), f(a), f(b), f(c), f(d))
    else:
        raise TypeError(v.dtype)
    return v


def prox(n, v, xhat, wmask, beta2):
    v = np.ascontiguousarray(v)
    out = np.zeros_like(v)
    xhat = np.ascontiguousarray(xhat, dtype=v.dtype)
    wmask = np.ascontiguousarray(wmask, dtype=v.dtype)
    if v.dtype == np.float64:
        lib().ora_prox_f64(n, _ptr(v, _dp), _ptr(out, _dp), _ptr(xhat, _dp), _ptr(wmask, _dp), float(beta2))
    else:
        lib().ora_prox_f32(n, _ptr(v, _fp), _ptr(out, _fp), _ptr(xhat, _fp), _ptr(wmask, _fp),
                           np.float32(beta2))
    return out


def layers(n):
    order = np.empty(1 << n, dtype=np.int64)
    bounds = np.empty(n + 2, dtype=np.int64)
    lib().ora_layers(n, _ptr(order, _llp), _ptr(bounds, _llp))
    return order, bounds


def make_feasible64(n, q, eps=1e-12):
    q = np.ascontiguousarray(q, dtype=np.float64)
    rf = np.empty_like(q)
    lib().ora_make_feasible64(n, _ptr(q, _dp), _ptr(rf, _dp), eps)
    return rf


def longest_path64(n, R):
    R = np.ascontiguousarray(R, dtype=np.float64)
    return float(lib().ora_longest_path64(n, _ptr(R, _dp)))


def push_ub64(n, x, obs_idx, p):
    """(ub, x_ub slab): Mobius -> exact unit flow -> zeta, in float64."""
    q = butterfly(n, np.asarray(x, dtype=np.float64), 1.0, -1.0, 0.0, 1.0)
    x_ub = butterfly(n, make_feasible64(n, q), 1.0, 1.0, 0.0, 1.0)
    d = x_ub[obs_idx] - p
    return float(np.sqrt(np.sum(d * d))), x_ub


def fw_lb64(n, obs_idx, y, p):
    """Frank-Wolfe lower bound at the point with values y at the observed positions."""
    r = np.asarray(p, dtype=np.float64) - np.asarray(y, dtype=np.float64)
    f = float(r @ r)
    g = np.zeros(n << (n - 1))
    g[obs_idx] = r
    g = butterfly(n, g, 1.0, 0.0, 1.0, 1.0)
    rc = longest_path64(n, g) - float(r @ y)
    return float(np.sqrt(max(0.0, f - 2.0 * rc)))


def eigen_data(n, precond_p, gamma):
    """(Qt, Q, inv_gl[Nloc] float64) of the per-bit matrix [[1,-1],[-1,1+p^2]]."""
    p = float(precond_p)
    G = np.array([[1.0, -1.0], [-1.0, 1.0 + p * p]])
    evals, Q = np.linalg.eigh(G)
    Nloc = 1 << (n - 1)
    lam = np.ones(Nloc)
    for bit in range(n - 1):
        b1s = ((np.arange(Nloc) >> bit) & 1).astype(np.float64)
        lam *= np.where(b1s > 0, evals[1], evals[0])
    return Q.T.copy(), Q, 1.0 / (gamma + lam)


def beta_default(mp):
    """Penalty from the number of observed cells (solver/params.py:52-54)."""
    return float(min(100.0, max(0.3, 10 ** -1.48 * float(mp) ** 0.508)))


class BMOracle:
    """The BM-ADMM engine on host slabs, one instance per (problem, dtype)."""

    def __init__(self, n, menu, alt, p, beta=None, alpha=1.95, precond_p=math.sqrt(2.0), dtype=np.float64):
        self.n = int(n)
        self.dt = np.dtype(dtype)
        dt = self.dt
        self.Nloc = 1 << (n - 1)
        self.m2 = n * self.Nloc
        self.menu = np.asarray(menu, dtype=np.uint64)
        self.alt = np.asarray(alt, dtype=np.int64)
        self.p = np.asarray(p, dtype=np.float64)
        self.obs = slab_index(n, self.menu, self.alt)
        beta = beta_default(self.p.size) if beta is None else float(beta)
        self.beta = beta
        self.xhat = np.zeros(self.m2, dt)
        self.wmask = np.zeros(self.m2, dt)
        self.xhat[self.obs] = self.p.astype(dt)
        self.wmask[self.obs] = 1
        Qt, Q, inv_gl = eigen_data(n, precond_p, 1.0)
        self.co = np.ascontiguousarray(np.concatenate([Qt.reshape(-1), Q.reshape(-1)]))
        self.inv_gl = inv_gl.astype(dt)
        self.b1 = dt.type(beta)
        self.b2 = dt.type(beta)
        self.ib1 = dt.type(1.0 / beta)
        self.ib2 = dt.type(1.0 / beta)
        self.alpha = dt.type(alpha)
        self.pp = dt.type(precond_p)
        self.scratch = np.zeros(6 * self.m2, dt)
        self.x2 = prox(n, self.xhat, self.xhat, self.wmask, self.b2)      # cold start: prox of xhat
        self.s = np.zeros(self.m2, dt)
        self.y = np.zeros(self.m2, dt)
        self.z = np.zeros(self.m2, dt)

    def state(self):
        return dict(x2=self.x2.copy(), s=self.s.copy(), y=self.y.copy(), z=self.z.copy())

    def set_state(self, st):
        for k in ("x2", "s", "y", "z"):
            setattr(self, k, np.ascontiguousarray(st[k], dtype=self.dt).copy())

    def iterate(self, iters=1):
        L = lib()
        if self.dt == np.float64:
            P = lambda a: _ptr(a, _dp)
            L.ora_admm_iter_f64(self.n, P(self.x2), P(self.s), P(self.y), P(self.z), P(self.xhat),
                                P(self.wmask), P(self.inv_gl), _ptr(self.co, _dp), self.b1, self.b2,
                                self.ib1, self.ib2, self.alpha, self.pp, P(self.scratch), int(iters))
        else:
            P = lambda a: _ptr(a, _fp)
            L.ora_admm_iter_f32(self.n, P(self.x2), P(self.s), P(self.y), P(self.z), P(self.xhat),
                                P(self.wmask), P(self.inv_gl), _ptr(self.co, _dp), self.b1, self.b2,
                                self.ib1, self.ib2, self.alpha, self.pp, P(self.scratch), int(iters))

    def phi(self):
        d = self.x2[self.obs].astype(np.float64) - self.p
        return float(np.sqrt(np.sum(d * d)))

    def solve(self, check=50, lb_every=1, max_iter=10 ** 7, abs_tol=1e-5, rel_tol=1e-4, time_limit=None,
              ub_target=None, lb_target=None):
        """The certified loop of the runner: push every check (running min), lower bound every
        lb_every checks (running max), stop on the gap, a threshold, max_iter or time."""
        t0 = time.perf_counter()
        it, checks = 0, 0
        ub, lb, p_fit, stop, trace = math.inf, 0.0, None, "max_iter", []
        while it < max_iter:
            self.iterate(check)
            it += check
            if time_limit is not None and time.perf_counter() - t0 > time_limit:
                stop = "time_limit"
                break
            u, x_ub = push_ub64(self.n, self.x2, self.obs, self.p)
            checks += 1
            if u < ub:
                ub, p_fit = u, x_ub[self.obs].copy()
            if ub_target is not None and ub <= ub_target:
                stop = "ub_target"
                break
            if (checks - 1) % lb_every == 0:
                lb = max(lb, fw_lb64(self.n, self.obs, self.x2[self.obs].astype(np.float64), self.p))
            trace.append((it, time.perf_counter() - t0, ub, lb))
            if lb_target is not None and lb >= lb_target:
                stop = "lb_target"
                break
            gap = ub - lb
            if abs_tol is not None and gap <= abs_tol:
                stop = "gap_abs"
                break
            if rel_tol is not None and lb > 0 and gap / lb <= rel_tol:
                stop = "gap_rel"
                break
        return dict(ub=ub, lb=lb, iters=it, stop=stop, p_fit=p_fit, trace=trace,
                    wall_s=time.perf_counter() - t0)


# ------------------------------------------------------------------ Flow-CG pricing
def cg_layout(n, menu, alt, p):
    """x-major rows (stable sort by alternative), p as float32, offsets[n+1]
    (solver/flow_cg/cg_core.py:135-145)."""
    menu = np.asarray(menu, dtype=np.int64).astype(np.uint64)
    alt = np.asarray(alt, dtype=np.int32)
    perm = np.argsort(alt, kind="stable")
    counts = np.bincount(alt, minlength=n)
    offsets = np.concatenate(([0], np.cumsum(counts))).astype(np.int64)
    return menu[perm], alt[perm], np.asarray(p, dtype=np.float64)[perm].astype(np.float32), offsets, perm


MODES = {"f32": 0, "u16": 1, "u24": 2}


def price_stream(n, menus, scores, offsets, mode="u24", k_pred=None, fma_decode=True):
    """(vmax, rank_pos int32[n], margin, layer_step float32[n+1])."""
    k_pred = n - 10 if k_pred is None else int(k_pred)
    k_pred = max(1, min(k_pred, n))
    menus = np.ascontiguousarray(menus, dtype=np.uint64)
    scores = np.ascontiguousarray(scores, dtype=np.float32)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    vmax = ctypes.c_double()
    margin = ctypes.c_double()
    rank = np.zeros(n, dtype=np.int32)
    steps = np.zeros(n + 1, dtype=np.float32)
    lib().ora_price_stream(MODES[mode], int(bool(fma_decode)), n, k_pred, _ptr(menus, _ullp),
                           _ptr(scores, _fp), _ptr(offsets, _llp), ctypes.byref(vmax), _ptr(rank, _ip),
                           ctypes.byref(margin), _ptr(steps, _fp))
    return vmax.value, rank, margin.value, steps


def sweep_max64(n, menus, scores, offsets):
    """V[full] of the float64 max sweep (solver/flow_cg/pricing_stream.py:236-249); x-major rows."""
    menus = np.ascontiguousarray(menus, dtype=np.uint64)
    scores = np.ascontiguousarray(scores, dtype=np.float64)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    return float(lib().ora_sweep_max64(int(n), _ptr(menus, _ullp), _ptr(scores, _dp), _ptr(offsets, _llp)))


def fw_lb_stream64(n, menu, alt, y, phat):
    """fw_lb_stream64 (solver/common/transforms.py:117-129): the float64 Frank-Wolfe bound at the
    point y through the two-layer max sweep; rows in any order."""
    alt = np.asarray(alt, dtype=np.int64)
    y = np.asarray(y, dtype=np.float64)
    r = np.asarray(phat, dtype=np.float64) - y
    perm = np.argsort(alt, kind="stable")
    offsets = np.concatenate(([0], np.cumsum(np.bincount(alt, minlength=n)))).astype(np.int64)
    vmax = sweep_max64(n, np.asarray(menu, dtype=np.uint64)[perm], r[perm], offsets)
    rc = vmax - float(r @ y)
    return float(np.sqrt(max(0.0, float(r @ r) - 2.0 * rc)))


def price_mask(n, menus, scores, offsets):
    """(vmax float32 as float, rank_pos) of the mask-indexed sweep."""
    menus = np.ascontiguousarray(menus, dtype=np.uint64)
    scores = np.ascontiguousarray(scores, dtype=np.float32)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    rank = np.zeros(n, dtype=np.int32)
    v = lib().ora_price_mask(n, _ptr(menus, _ullp), _ptr(scores, _fp), _ptr(offsets, _llp), _ptr(rank, _ip))
    return float(v), rank


def ranking_column(n, menus, alts, rank_pos):
    menus = np.ascontiguousarray(menus, dtype=np.uint64)
    alts = np.ascontiguousarray(alts, dtype=np.int32)
    rank_pos = np.ascontiguousarray(rank_pos, dtype=np.int32)
    out = np.empty(menus.size, dtype=np.uint8)
    lib().ora_ranking_column(n, menus.size, _ptr(menus, _ullp), _ptr(alts, _ip), _ptr(rank_pos, _ip),
                             _ptr(out, _u8p))
    return out


def project_simplex(y):
    n = y.size
    u = np.sort(y)[::-1]
    css = np.cumsum(u) - 1.0
    cond = u - css / np.arange(1, n + 1) > 0
    if not cond.any():
        return np.ones(n) / n
    rho = int(np.where(cond)[0][-1] + 1)
    return np.maximum(y - css[rho - 1] / rho, 0.0)


def qp_native(Q, h, A_init=None, max_outer=200, tol=1e-10, reg=1e-12):
    """Active-set + Cholesky on the simplex QP min 1/2 l'Ql - h'l."""
    from scipy.linalg import cho_factor, cho_solve
    K = len(h)
    A = [int(i) for i in (A_init or []) if 0 <= i < K] or [int(np.argmax(h))]
    lam_A, A_arr = None, None
    for _ in range(max_outer):
        A_arr = np.asarray(A, dtype=np.int64)
        k = len(A)
        ones_A = np.ones(k)
        Q_AA = Q[np.ix_(A_arr, A_arr)] + reg * np.eye(k)
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


def cg_solve(n, menu, alt, p, mode="u24", k_pred=None, max_iters=200, gap_abs_tol=1e-5, gap_rel_tol=None,
             seed=0, pricer=None):
    """Column generation with this oracle's pricer (or `pricer(scores) -> (vmax, rank_pos,
    margin)`): returns dict(columns=[rank_pos per iteration], ub, lb, iters, stop). The master
    keeps Q = V'V and h = V'p exactly (float64 counts), as the bitset maintainer does."""
    menus, alts, p32, offsets, _perm = cg_layout(n, menu, alt, p)
    p_obs = p32.astype(np.float64)
    p_sq = float(p_obs @ p_obs)
    if pricer is None:
        if mode == "mask":
            pricer = lambda sc: price_mask(n, menus, sc, offsets) + (0.0,)
        else:
            pricer = lambda sc: price_stream(n, menus, sc, offsets, mode=mode, k_pred=k_pred)[:3]
    # the first column: a seeded permutation read directly as rank positions
    # (solver/flow_cg/solver.py:87-88)
    perm0 = np.random.RandomState(seed).permutation(n).astype(np.int32)
    cols = [ranking_column(n, menus, alts, perm0)]
    Qm = np.zeros((max_iters + 2, max_iters + 2))
    h = np.zeros(max_iters + 2)
    V = [cols[0].astype(np.float64)]
    Qm[0, 0] = float(cols[0].sum())
    h[0] = float(p_obs[cols[0] > 0].sum())
    K, lam, A = 1, np.array([1.0]), [0]
    p_out = V[0].copy()
    lb_best, ub, stop, picked = 0.0, math.inf, "max_iters", []
    for it in range(1, max_iters + 1):
        lam_new, A = qp_native(Qm[:K, :K], h[:K], A_init=A)
        delta = lam_new - lam
        for a in np.where(np.abs(delta) > 1e-12)[0]:
            p_out[V[a] > 0] += float(delta[a])
        lam = lam_new
        QL = Qm[:K, :K] @ lam
        lql = float(lam @ QL)
        hl = float(h[:K] @ lam)
        err2 = lql - 2.0 * hl + p_sq
        inner = hl - lql
        residual = p_obs - p_out
        vmax, rank_pos, margin = pricer(residual.astype(np.float32))
        picked.append(np.asarray(rank_pos, dtype=np.int32).copy())
        fw_gap = (vmax + margin) - inner
        ub = float(np.sqrt(max(0.0, err2)))
        lb_best = max(lb_best, float(np.sqrt(max(0.0, err2 - 2.0 * fw_gap))))
        gap_rel = (ub - lb_best) / lb_best if lb_best > 0 else math.inf
        if gap_rel_tol is not None and gap_rel <= gap_rel_tol:
            stop = "gap_rel"
            break
        if gap_abs_tol is not None and ub - lb_best <= gap_abs_tol:
            stop = "gap_abs"
            break
        col = ranking_column(n, menus, alts, rank_pos)
        v = col.astype(np.float64)
        for j in range(K):
            Qm[K, j] = Qm[j, K] = float(np.dot(V[j], v))
        Qm[K, K] = float(v.sum())
        h[K] = float(p_obs[col > 0].sum())
        V.append(v)
        K += 1
        lam = np.concatenate([lam, [0.0]])
    return dict(columns=picked, ub=ub, lb=lb_best, iters=len(picked), stop=stop)
