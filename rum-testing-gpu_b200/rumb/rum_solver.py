"""The RUM class: the distance from observed choice probabilities to the random utility model,
with a certified bracket lb <= dist <= ub -- the reference's public interface
(solver/rum_solver.py:1-330, 522-658), for the two GPU methods this library implements.

    from rumb import RUM
    rum = RUM(menu, alternative, choice_probability)
    res = rum.calculate_distance(method="bm_admm", method_args={"dtype": "float64", "check": 50})
    res = rum.calculate_distance(method="flow_cg", method_args={"dtype": "uint24", "pricing": "stream"})

Input rows: menu[i] is the bitmask of the offered menu, alternative[i] the chosen alternative
(0-based), choice_probability[i] its observed probability. Rows of singleton menus are taken out
before solving (their probability must be 1) and added back as a constant.

A call stops when ub - lb <= abs_tol or (ub - lb) / lb <= rel_tol, when max_time runs out (setup
included), or on the method's own limits; whatever the reason, lb <= dist <= ub and distance = ub.

    exit_flag   1 abs_tol met    2 rel_tol met    3 both met    5 threshold reached (Session)
                0 time limit    -1 iteration limit    -2 stalled    -3 out of memory
               -4 interrupted   -5 solver error (message says which)

Methods: "bm_admm" (Block-Marschak ADMM) and "flow_cg" (column generation with Bellman-Ford
pricing), both on the GPU through librumb.so. The reference's CPU/Gurobi methods and its paper
races are not part of this library and raise.
"""
import math
import time
import types
import warnings
from dataclasses import dataclass, field, fields

import numpy as np

from . import defaults, params

METHODS = ("bm_admm", "flow_cg")
ALIASES = {"cgbfqp": "flow_cg", "cgbf": "flow_cg"}
STATUS = {5: "threshold reached", 3: "abs_tol and rel_tol met", 1: "abs_tol met", 2: "rel_tol met",
          0: "time limit", -1: "iteration limit", -2: "stalled", -3: "out of memory", -4: "interrupted",
          -5: "solver error"}
_FLAG = {"threshold": 5, "time": 0, "iters": -1, "stalled": -2, "oom": -3, "interrupted": -4, "error": -5}
_UNIT = {"bm_admm": "ADMM iterations", "flow_cg": "columns"}


@dataclass
class Result:
    exit_flag: int
    status: str
    message: str
    distance: float
    lb: float
    ub: float
    abs_gap: float
    rel_gap: float
    abs_tol: float
    rel_tol: float
    met_abs: bool
    met_rel: bool
    method: str
    auto_reason: str
    method_args: dict
    iterations: int
    iteration_unit: str
    time: float
    time_setup: float
    time_solve: float
    seed: object
    p_fit: np.ndarray = None
    trace: list = field(default_factory=list)
    machine: str = ""
    info: dict = field(default_factory=dict)
    mode: str = "certificate"
    # the reference's race fields (solver/rum_solver.py:109-112); a certified distance leaves them None
    opt: float = None
    target: float = None
    abs_to_opt: float = None
    rel_to_opt: float = None

    def __repr__(self):
        rows = [("exit_flag", "%d (%s)" % (self.exit_flag, self.status)), ("distance", "%.10g" % self.distance),
                ("lb, ub", "%.10g, %.10g" % (self.lb, self.ub)),
                ("abs_gap", "%.3g (abs_tol %.3g, %s)" % (self.abs_gap, self.abs_tol, "met" if self.met_abs else "not met")),
                ("rel_gap", "%.3g (rel_tol %.3g, %s)" % (self.rel_gap, self.rel_tol, "met" if self.met_rel else "not met")),
                ("method", self.method + ("  [%s]" % self.auto_reason if self.auto_reason else "")),
                ("iterations", "%d %s" % (self.iterations, self.iteration_unit)),
                ("time", "%.3f s (setup %.3f s, solve %.3f s)" % (self.time, self.time_setup, self.time_solve)),
                ("seed", str(self.seed))]
        if self.message:
            rows.append(("message", self.message))
        rows.append(("method_args", str(self.method_args)))
        rows.append(("p_fit", "None" if self.p_fit is None else "array of %d" % len(self.p_fit)))
        rows.append(("trace", "%d entries" % len(self.trace)))
        rows.append(("machine", self.machine))
        if self.info:
            rows.append(("info", str(self.info)))
        w = max(len(k) for k, _ in rows)
        return "\n".join("%s : %s" % (k.rjust(w), v) for k, v in rows)

    def to_dict(self, p_fit=False):
        """The fields as plain Python values, ready for json.dump; p_fit only when asked."""
        d = {f.name: getattr(self, f.name) for f in fields(self) if f.name != "p_fit"}
        d["trace"] = [list(row) for row in self.trace]
        if p_fit:
            d["p_fit"] = None if self.p_fit is None else self.p_fit.tolist()
        return d


class _TimeUp(Exception):
    pass


class _Geometry:
    """The non-singleton rows."""

    def __init__(self, menu, alternative, n):
        self.menu = np.asarray(menu, dtype=np.uint64)
        self.alternative = np.asarray(alternative, dtype=np.int64)
        self.num_alternatives = int(n)
        self.M = int(self.menu.size)
        self.pricer = None          # flow_cg: the device pricer, reused across calls


# ---------------------------------------------------------------------- the GPU context
_CTX = {}


def context(device=0):
    """The process-wide library context of a GPU (created on first use)."""
    from . import _lib
    if device not in _CTX:
        _CTX[device] = _lib.Context(device)
    return _CTX[device]


def gpu_free_bytes(device=0):
    """Free device memory (the library's mem_info; replaces the reference's machine query)."""
    return context(device).mem_info()[0]


class RUM:
    def __init__(self, menu, alternative, choice_probability, num_alternatives=None):
        menu = _as_int(menu, "menu")
        alternative = _as_int(alternative, "alternative")
        if menu.ndim != 1 or alternative.shape != menu.shape:
            raise ValueError("menu and alternative must be 1-D arrays of the same length")
        if menu.size == 0:
            raise ValueError("no observations")
        if (menu <= 0).any():
            raise ValueError("row %d: empty menu" % int(np.flatnonzero(menu <= 0)[0]))
        if (alternative < 0).any():
            raise ValueError("row %d: negative alternative" % int(np.flatnonzero(alternative < 0)[0]))
        need = max(int(menu.max()).bit_length(), int(alternative.max()) + 1)
        n = need if num_alternatives is None else int(num_alternatives)
        if n < need:
            raise ValueError("num_alternatives = %d, but the data use alternatives up to %d" % (n, need - 1))
        if n > 62:
            raise ValueError("menus are 64-bit masks: at most 62 alternatives")
        off = ((menu >> alternative) & 1) == 0
        if off.any():
            i = int(np.flatnonzero(off)[0])
            raise ValueError("row %d: alternative %d is not in its menu (mask %d)" % (i, alternative[i], menu[i]))
        _, first, counts = np.unique(np.column_stack([menu, alternative]), axis=0, return_index=True,
                                     return_counts=True)
        if (counts > 1).any():
            i = int(first[np.flatnonzero(counts > 1)[0]])
            raise ValueError("row %d: (menu %d, alternative %d) appears more than once" % (i, menu[i], alternative[i]))
        self.n = n
        self.M = int(menu.size)
        self.menu = menu
        self.alternative = alternative
        self.singleton = (menu & (menu - 1)) == 0
        self._rest = np.flatnonzero(~self.singleton)
        self._single = np.flatnonzero(self.singleton)
        self._geom = _Geometry(menu[self._rest], alternative[self._rest], n)
        self._menu_of_row = np.unique(menu, return_inverse=True)[1]
        self.choice_probability = self._check_p(choice_probability)

    @classmethod
    def from_rows(cls, rows, num_alternatives=None):
        rows = np.asarray(rows)
        if rows.ndim != 2 or rows.shape[1] != 3:
            raise ValueError("rows must be an (M, 3) array: menu, alternative, choice probability")
        return cls(rows[:, 0], rows[:, 1], rows[:, 2], num_alternatives=num_alternatives)

    def __repr__(self):
        return "RUM(n=%d, %d rows, %d menus, %d singleton rows)" % (
            self.n, self.M, np.unique(self.menu).size, self._single.size)

    # ------------------------------------------------------------------ distance
    def calculate_distance(self, abs_tol=None, rel_tol=None, method=None, method_args=None, max_time=None, p=None,
                           vcov=None, seed=0, verbose=False, machine=None, opt=None, opt_rel_tol=None, opt_floor=None):
        """dist(p) with a certified bracket; see the module docstring. vcov (a weight matrix) and opt
        (the paper's races) belong to methods outside this library and raise."""
        if opt is not None or opt_rel_tol is not None or opt_floor is not None:
            raise ValueError("races to a known optimum (opt=...) are not part of this library; "
                             "leave opt out for a certified distance")
        if vcov is not None and not _is_identity(vcov):
            raise RuntimeError("bm_admm and flow_cg compute the unweighted distance only (vcov None or identity)")
        t0 = time.perf_counter()
        abs_tol = float(defaults.ABS_TOL if abs_tol is None else abs_tol)
        rel_tol = float(defaults.REL_TOL if rel_tol is None else rel_tol)
        max_time = float(defaults.MAX_TIME if max_time is None else max_time)
        if abs_tol < 0 or rel_tol < 0 or not max_time > 0:
            raise ValueError("abs_tol and rel_tol must be >= 0 and max_time > 0")
        if seed is None:
            seed = int(np.random.SeedSequence().entropy % (2 ** 31))
        p = self.choice_probability if p is None else self._check_p(p)
        const = self._const(p)
        geom, pr = self._geom, p[self._rest]
        if geom.M == 0:
            d = math.sqrt(const)
            return self._result(t0, t0, "none", "only singleton menus", {}, abs_tol, rel_tol, seed,
                                dict(lb=d, ub=d, p_fit=np.zeros(0), iterations=0, trace=[], info={}, setup=0.0),
                                "tol", "", 0.0)
        name, reason, args = self._plan(method, method_args)
        st = dict(lb=0.0, ub=math.inf, p_fit=None, iterations=0, trace=[], info={}, setup=0.0)
        task = types.SimpleNamespace(geom=geom, p=pr, args=args, abs_tol=abs_tol, rel_tol=rel_tol,
                                     deadline=t0 + max_time, seed=seed, verbose=verbose, t0=t0, state=st,
                                     const=const)
        t_run = time.perf_counter()
        message = ""
        try:
            stop = _RUN[name](task)
        except _TimeUp:
            stop = "time"
        except KeyboardInterrupt:
            stop, message = "interrupted", "interrupted by the user"
        except Exception as e:                # noqa: BLE001 -- reported through exit_flag
            stop = "oom" if _is_oom(e) else "error"
            message = "%s: %s" % (type(e).__name__, e)
        return self._result(t0, t_run, name, reason, args, abs_tol, rel_tol, seed, st, stop, message, const)

    def session(self, method=None, method_args=None, vcov=None, machine=None, seed=0):
        """A Session: one plan, many solves at any finite p, with threshold stops and warm starts."""
        return Session(self, method, method_args, vcov, machine, seed)

    def bootstrap(self, *a, **k):
        from .bootstrap import Bootstrap
        return Bootstrap(self, *a, **k)

    # ------------------------------------------------------------------ helpers
    def _check_p(self, p):
        p = np.asarray(p, dtype=np.float64)
        if p.shape != (self.M,):
            raise ValueError("choice probabilities: expected %d values, got shape %s" % (self.M, p.shape))
        if not np.isfinite(p).all():
            raise ValueError("choice probabilities must be finite")
        if (p < -1e-12).any() or (p > 1 + 1e-12).any():
            i = int(np.flatnonzero((p < -1e-12) | (p > 1 + 1e-12))[0])
            raise ValueError("row %d: probability %.6g is outside [0, 1]" % (i, p[i]))
        sums = np.bincount(self._menu_of_row, weights=p)
        if (sums > 1 + 1e-9).any():
            warnings.warn("%d menus have observed probabilities summing to more than 1 (largest %.6g)"
                          % (int((sums > 1 + 1e-9).sum()), sums.max()))
        return p

    def _finite_p(self, p):
        p = np.asarray(p, dtype=np.float64)
        if p.shape != (self.M,):
            raise ValueError("p: expected %d values, got shape %s" % (self.M, p.shape))
        if not np.isfinite(p).all():
            raise ValueError("p must be finite")
        return p

    def _const(self, p):
        r_s = 1.0 - p[self._single]
        return float(r_s @ r_s)

    def _plan(self, method, method_args):
        n, mp = self.n, self._geom.M
        if method is None:
            if method_args:
                raise ValueError("method_args needs a named method")
            name, reason = choose_method(n, mp)
        else:
            name, reason = _method_name(method), ""
        args = dict(defaults.METHOD_ARGS[name])
        bad = set(method_args or {}) - set(args)
        if bad:
            raise ValueError("unknown method_args for %s: %s; allowed: %s" % (name, sorted(bad), sorted(args)))
        args.update(method_args or {})
        return name, reason, _PLAN[name](n, mp, args)

    def _result(self, t0, t_run, name, reason, args, abs_tol, rel_tol, seed, st, stop, message, const):
        lb = math.sqrt(max(st["lb"], 0.0) ** 2 + const)
        ub = math.sqrt(st["ub"] ** 2 + const) if math.isfinite(st["ub"]) else math.inf
        abs_gap = ub - lb
        rel_gap = abs_gap / lb if lb > 0 else math.inf
        met_abs, met_rel = abs_gap <= abs_tol, lb > 0 and rel_gap <= rel_tol
        flag = 3 if (met_abs and met_rel) else 1 if met_abs else 2 if met_rel else _FLAG.get(stop, -2)
        message = message or st.get("message", "")
        if flag == -2 and not message:
            message = ("the method stopped on its own test, but the bracket does not meet the tolerances"
                       if stop == "tol" else "the method stopped without meeting the tolerances")
        elif flag == 0 and not message:
            message = "max_time reached"
        elif flag == -1 and not message:
            message = "the method's iteration limit was reached (see method_args)"
        info, met = st["info"], flag in (1, 2, 3)
        if name == "bm_admm" and args.get("dtype") == "float32" and not met:
            message = "; ".join(([message] if message else []) + [
                "a float32 state's pushed upper bound usually stalls above the tolerances; dtype='float64' "
                "or 'mixed' certifies"])
        p_fit = None
        if st["p_fit"] is not None:
            p_fit = np.ones(self.M)
            p_fit[self._rest] = st["p_fit"]
        t_end = time.perf_counter()
        setup = (t_run - t0) + st["setup"]
        return Result(exit_flag=flag, status=STATUS[flag], message=message, distance=ub, lb=lb, ub=ub,
                      abs_gap=abs_gap, rel_gap=rel_gap, abs_tol=abs_tol, rel_tol=rel_tol, met_abs=bool(met_abs),
                      met_rel=bool(met_rel), method=name, auto_reason=reason,
                      method_args={k: v for k, v in args.items() if not k.startswith("_")},
                      iterations=int(st["iterations"]), iteration_unit=_UNIT.get(name, ""), time=t_end - t0,
                      time_setup=setup, time_solve=(t_end - t0) - setup, seed=seed, p_fit=p_fit, trace=st["trace"],
                      machine=_machine_line(), info=info)


class Session:
    """One plan, many solves (the bootstrap's solver): the method and its storage format are
    planned once; solve() takes any finite p, with early stops (below: ub < below; above:
    lb >= above; exit_flag 5) and warm starts from a kept solve (bm_admm: its ADMM state on the
    device; flow_cg: its columns and weights)."""

    def __init__(self, rum, method=None, method_args=None, vcov=None, machine=None, seed=0):
        t0 = time.perf_counter()
        if vcov is not None and not _is_identity(vcov):
            raise RuntimeError("bm_admm and flow_cg compute the unweighted distance only")
        self.rum, self.seed = rum, seed
        self.method, self.auto_reason, self._args = rum._plan(method, method_args)
        self.method_args = {k: v for k, v in self._args.items() if not k.startswith("_")}
        self.fit = None
        self._kept = None
        self.time_plan = time.perf_counter() - t0

    def solve(self, p, abs_tol=None, rel_tol=None, max_time=None, below=None, above=None, warm=False, keep=False,
              verbose=False):
        rum, t0 = self.rum, time.perf_counter()
        abs_tol = float(defaults.ABS_TOL if abs_tol is None else abs_tol)
        rel_tol = float(defaults.REL_TOL if rel_tol is None else rel_tol)
        max_time = float(defaults.MAX_TIME if max_time is None else max_time)
        if abs_tol < 0 or rel_tol < 0 or not max_time > 0:
            raise ValueError("abs_tol and rel_tol must be >= 0 and max_time > 0")
        if warm and self._kept is None:
            raise ValueError("warm=True starts from a kept solve: call solve(..., keep=True) first")
        p = rum._finite_p(p)
        const = rum._const(p)
        geom, pr = rum._geom, p[rum._rest]
        if geom.M == 0:
            d = math.sqrt(const)
            return rum._result(t0, t0, "none", "only singleton menus", {}, abs_tol, rel_tol, self.seed,
                               dict(lb=d, ub=d, p_fit=np.zeros(0), iterations=0, trace=[], info={}, setup=0.0),
                               "tol", "", 0.0)
        st = dict(lb=0.0, ub=math.inf, p_fit=None, iterations=0, trace=[], info={}, setup=0.0)
        task = types.SimpleNamespace(geom=geom, p=pr, args=self._args, abs_tol=abs_tol, rel_tol=rel_tol,
                                     deadline=t0 + max_time, seed=self.seed, verbose=verbose, t0=t0, state=st,
                                     const=const, below=_on_rest(below, const, False), above=_on_rest(above, const, True),
                                     warm=self._kept if warm else None, keep=bool(keep))
        t_run = time.perf_counter()
        message = ""
        try:
            stop = _RUN[self.method](task)
        except _TimeUp:
            stop = "time"
        except KeyboardInterrupt:
            stop, message = "interrupted", "interrupted by the user"
        except Exception as e:                # noqa: BLE001
            stop = "oom" if _is_oom(e) else "error"
            message = "%s: %s" % (type(e).__name__, e)
        kept = st.pop("keep", None)
        res = rum._result(t0, t_run, self.method, self.auto_reason, self._args, abs_tol, rel_tol, self.seed, st,
                          stop, message, const)
        if keep:
            self._kept, self.fit = kept, res.p_fit
        return res

    def close(self):
        self._kept = self.fit = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __repr__(self):
        return "Session(%s, %s; kept state: %s)" % (self.method, self.method_args,
                                                    "no" if self._kept is None else "yes")


def _on_rest(tau, const, above):
    """A threshold on dist as one on the non-singleton rows (dist^2 = rest^2 + const)."""
    if tau is None:
        return None
    tau = float(tau)
    if not math.isfinite(tau):
        raise ValueError("below and above must be finite")
    if tau * tau <= const:
        return 0.0 if above else None
    return math.sqrt(tau * tau - const)


# ---------------------------------------------------------------------- choosing and planning
def bm_admm_min_density(n):
    steps = [d for n0, d in sorted(defaults.AUTO["bm_admm_min_density"].items()) if n >= n0]
    return steps[-1] if steps else None


def choose_method(n, mp):
    """bm_admm from the density set for this n, flow_cg below it and whenever bm_admm does not fit
    the GPU (solver/rum_solver.py:675-711, GPU branch)."""
    density = mp / (n << (n - 1))
    why = ["n = %d, %d rows, density %.3g%%" % (n, mp, 100 * density)]
    d_min = bm_admm_min_density(n)
    if d_min is None:
        why.append("n <= %d -> flow_cg at any density" % (min(defaults.AUTO["bm_admm_min_density"]) - 1))
    elif density < d_min:
        why.append("density < %.2g%% at n = %d -> flow_cg" % (100 * d_min, n))
    else:
        try:
            _plan_bm_admm(n, mp, dict(defaults.METHOD_ARGS["bm_admm"]))
            return "bm_admm", "; ".join(why + ["density >= %.2g%% at n = %d -> bm_admm" % (100 * d_min, n)])
        except RuntimeError as e:
            why.append(str(e))
    _plan_flow_cg(n, mp, dict(defaults.METHOD_ARGS["flow_cg"]))
    return "flow_cg", "; ".join(why)


# Device bytes of one BM-ADMM solve in this library (rumb_bm_plan: the buffers the solve allocates,
# both state dtypes for "mixed"), plus 10 % as the reference's planner keeps
# (solver/rum_solver.py:735-737).
def _bm_admm_bytes(n, dtype, mp=1):
    from . import _lib
    return int(1.1 * _lib.bm_plan(n, mp, dtype))


def _plan_bm_admm(n, mp, a):
    if not 2 <= n <= 30:
        raise RuntimeError("bm_admm handles 2 <= n <= 30")
    for k in ("check", "lb_every", "max_iter"):
        if int(a[k]) < 1:
            raise ValueError("bm_admm %s must be >= 1" % k)
    if a["dtype"] not in ("auto", "float64", "float32", "mixed"):
        raise ValueError("bm_admm dtype must be 'auto', 'float64', 'float32' or 'mixed'")
    dt = "float64" if a["dtype"] == "auto" else a["dtype"]
    budget = defaults.AUTO["gpu_memory_fraction"] * gpu_free_bytes()
    need = _bm_admm_bytes(n, dt, mp)
    if need > budget:
        raise RuntimeError("bm_admm at n = %d in %s needs %.1f GB of GPU memory; %.1f GB may be used. Use flow_cg"
                           % (n, dt, need / 2 ** 30, budget / 2 ** 30))
    a.update(dtype=dt, use_graph=True if a["use_graph"] == "auto" else bool(a["use_graph"]), _gpu_bytes=need)
    a["beta"] = params.bm_beta_default(mp) if a["beta"] is None else float(a["beta"])
    return a


_CG_ENGINE = {("mask", "float32"): "mask", ("stream", "float32"): "f32", ("stream", "uint24"): "u24",
              ("stream", "uint16"): "u16"}
_CG_OLD = {"stream_f32": ("stream", "float32"), "stream_u24": ("stream", "uint24"), "stream_u16": ("stream", "uint16")}


def _flow_cg_bytes(n, engine):
    cap = math.comb(n, n // 2)
    if engine == "mask":
        return 5 * (1 << n)
    k_pred = max(1, n - 10)
    item = {"f32": 4, "u24": 3, "u16": 2}[engine]
    return 2 * cap * item + sum(math.comb(n, k) for k in range(k_pred, n + 1)) + 5 * (1 << k_pred)


def _plan_flow_cg(n, mp, a):
    layout, dt = a["pricing"], a["dtype"]
    if layout in _CG_OLD:
        if dt not in ("auto", _CG_OLD[layout][1]):
            raise ValueError("pricing=%r is %s storage; it contradicts dtype=%r" % (layout, _CG_OLD[layout][1], dt))
        layout, dt = _CG_OLD[layout]
    if layout not in ("auto", "mask", "stream"):
        raise ValueError("flow_cg pricing must be 'auto', 'mask' or 'stream' (old names: stream_f32, stream_u24, "
                         "stream_u16)")
    if dt not in ("auto", "float32", "uint24", "uint16"):
        raise ValueError("flow_cg dtype must be 'auto', 'float32', 'uint24' or 'uint16'")
    if layout == "mask" and dt not in ("auto", "float32"):
        raise ValueError("mask pricing stores float32 only; dtype=%r needs pricing='stream' or 'auto'" % dt)
    if n > 39:
        raise RuntimeError("flow_cg handles n <= 39")
    budget = defaults.AUTO["gpu_memory_fraction"] * gpu_free_bytes()
    tried = []
    for (lay, d), engine in _CG_ENGINE.items():
        if layout not in ("auto", lay) or dt not in ("auto", d) or (lay == "mask" and n > 34):
            continue
        need = _flow_cg_bytes(n, engine)
        if need <= budget:
            a.update(pricing=lay, dtype=d, _engine=engine, _gpu_bytes=need)
            return a
        tried.append("%s %s %.1f GB" % (lay, d, need / 2 ** 30))
    raise RuntimeError("flow_cg at n = %d does not fit the GPU (%s)" % (n, "; ".join(tried) or "mask needs n <= 34"))


_PLAN = {"bm_admm": _plan_bm_admm, "flow_cg": _plan_flow_cg}


# ---------------------------------------------------------------------- runners
def _run_bm_admm(t):
    """The certified BM-ADMM solve (solver/rum_solver.py:869-925): running-min float64 push,
    float64 lower bound every lb_every checks, threshold stops and warm start for a Session."""
    from . import _lib
    g, a, st = t.geom, t.args, t.state
    n = g.num_alternatives
    ctx = context()
    remaining = t.deadline - time.perf_counter()
    if remaining <= 0:
        raise _TimeUp
    below, above, warm = getattr(t, "below", None), getattr(t, "above", None), getattr(t, "warm", None)
    par = ctx.bm_params(a["beta"], alpha=a["alpha"], precond_p=a["precond_p"], check=a["check"],
                        lb_every=a["lb_every"], max_iter=a["max_iter"], abs_tol=t.abs_tol, rel_tol=t.rel_tol,
                        time_limit=max(remaining, 1e-3), ub_target=below if below is not None and below > 0 else None,
                        lb_target=above, dtype=a["dtype"], use_graph=a["use_graph"])
    prob = ctx.bm_problem(n, g.menu.astype(np.uint32), g.alternative.astype(np.int32), t.p)
    st["info"].update(gpu_bytes_planned=a["_gpu_bytes"], lb_dtype="float64", lb_layout="slab", lb_rigorous=True)
    t_call = time.perf_counter()
    rows = []
    try:
        r, fit, kept = ctx.bm_solve(prob, par, warm=warm, keep=getattr(t, "keep", False), trace=rows)
    except _lib.RumbError as e:
        if e.code == _lib.E_CANCEL:
            raise KeyboardInterrupt from e
        raise
    off = t_call - t.t0
    st["trace"] = [(it, off + w, ub, lb) for it, w, _phi, ub, lb in rows]
    st["iterations"] = int(r["iters"])
    st["setup"] = float(r["setup_s"])
    if math.isfinite(r["ub"]):
        st["ub"], st["p_fit"] = float(r["ub"]), fit
    st["lb"] = max(st["lb"], float(r["lb"]))
    st["info"].update(per_iter_ms=round(r["per_iter_ms"], 4), push_s=round(r["push_s"], 3),
                      iters_float32=int(r["iters_f32"]), device_ms=round(r["device_ms"], 3))
    if getattr(t, "keep", False):
        st["keep"] = kept
    stop = r["stop_reason"]
    if stop == "cancel":
        raise KeyboardInterrupt
    return {"gap_abs": "tol", "gap_rel": "tol", "time_limit": "time", "max_iter": "iters", "ub_target": "threshold",
            "lb_target": "threshold"}.get(stop, "stalled")


def _run_flow_cg(t):
    from .flow_cg import run_flow_cg
    return run_flow_cg(t, context())


_RUN = {"bm_admm": _run_bm_admm, "flow_cg": _run_flow_cg}


# ---------------------------------------------------------------------- small helpers
def _method_name(method):
    name = str(method).strip().lower().replace("-", "_")
    name = ALIASES.get(name, name)
    if name not in METHODS:
        raise ValueError("unknown method %r; this library implements %s" % (method, METHODS))
    return name


def _as_int(x, what):
    a = np.asarray(x)
    if a.dtype.kind == "f":
        if not np.all(np.isfinite(a)) or not np.all(a == np.floor(a)):
            raise ValueError("%s must hold integers" % what)
    elif a.dtype.kind not in "iu":
        raise ValueError("%s must hold integers" % what)
    return a.astype(np.int64)


def _is_identity(V):
    try:
        import scipy.sparse as sp
        if sp.issparse(V):
            return (V - sp.identity(V.shape[0], dtype=V.dtype, format="csr")).count_nonzero() == 0
    except ImportError:
        pass
    V = np.asarray(V)
    return V.ndim == 2 and V.shape[0] == V.shape[1] and np.array_equal(V, np.eye(V.shape[0]))


def _is_oom(e):
    return isinstance(e, MemoryError) or "OutOfMemory" in type(e).__name__ or "out of memory" in str(e).lower()


def _machine_line():
    try:
        free, total = context().mem_info()
        return "GPU 0 (%.0f GB, librumb %d)" % (total / 1e9, __import__("rumb._lib")._lib.load().rumb_version())
    except Exception:
        return "no GPU"
