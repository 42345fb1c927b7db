"""Hong and Li's bootstrap on the RUM distance, with the draws solved many at a time on the GPU.

    from rumb import RUM, cells_from_panel
    menu, alt, p_hat = cells_from_panel(panel, n)             # panel: respondent, menu, chosen
    boot = RUM(menu, alt, p_hat, num_alternatives=n).bootstrap(panel=panel, B=10000)
    print(boot.p_value(), boot.confidence_interval(), boot.distance_interval())

The reference's pipeline (solver/inference/bootstrap.py:182-335, solver/inference/hong_li.py,
solver/inference/draws.py:161-290), with its formulas and decisions:

    certify   p_hat with a Session (one plan for every solve), keeping its state and fit:
              dist(p_hat) in [L0, U0]; the band tau = s [L0, U0], s = 1 + eps_n r_n
    screen    every draw P_b = p_hat + eps_n r_n (p_hat_b - p_hat): ||p_fit - P_b|| bounds dist(P_b)
              (on the GPU for integer weights, rumb_draws_*; with the reference's host blocks for
              real weights and replies)
    solve     the draws still open, warm from p_hat's state, each stopping once it clears the band
              (ub < tau_lo: below; lb >= tau_hi: above). bm_admm solves them together with
              rumb_bm_solve_batch (slots admitted by device memory, retired as they finish);
              flow_cg one at a time through the Session, as the reference does. A float32 session
              solves the batch in float32; draws whose bracket stalls undecided are solved again in
              float64 (a mixed session batches in float64)
    learned   (learned=True, bm_admm) the first train_draws solved draws train a small BF16 network
              on the tensor cores (rumb_mlp_*) to map a draw's cells to its fitted cells; every
              later draw starts from the prediction: its bracket from the Frank-Wolfe lower bound
              at the prediction (certified whatever the prediction); y0_state=True also moves the
              start state's fitted cells there. A poor prediction costs iterations, never
              correctness
    p-value   p = (#above + #undecided) / B (stop_when_decided: stop once the decision is locked)
    intervals confidence_interval (draws solved to tolerance while they overlap the quantile band)
              and distance_interval (p_hat's bracket widened by the quantile of ||p_b - p_hat||)

The draws (rumb.draws, solver/inference/draws.py): a panel's respondents resampled with the
weights multinomial_reject, multinomial, exponential, poisson or mammen, or a replies table's
menus resampled one by one, drawn in the reference's order from its seeds.
"""
import hashlib
import json
import math
import os
import time
from dataclasses import asdict, dataclass

import numpy as np
import scipy.sparse as sp

from . import defaults
from .draws import Draws, MenuDraws, cells_from_panel  # noqa: F401  (re-exported)

BELOW, ABOVE, UNDECIDED = 0, 1, 2
ZERO = 1e-9
VERSION = 1                      # the record format's version (solver/inference/bootstrap.py:48)
NEVER = 127                      # exit_flag of a draw that was never solved
# a batched draw's stop reason as the Session's exit flag (1 tol, 5 threshold, 0 time, -1 iters,
# -2 stalled)
_STOP_FLAG = {"gap_abs": 1, "gap_rel": 2, "ub_target": 5, "lb_target": 5, "time_limit": 0, "max_iter": -1,
              "stall": -2, "cancel": -4}


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def _plain(x):
    if isinstance(x, np.generic):
        return x.item()
    if isinstance(x, np.ndarray):
        return x.tolist()
    raise TypeError("not JSON serializable: %r" % type(x))


def scaling(n, r_n=None, eps_n=None):
    """(r_n, eps_n, s): sqrt(n), n^(-1/3) and 1 + eps_n r_n (solver/inference/hong_li.py:33-45)."""
    if int(n) != n or n < 1:
        raise ValueError("n, the sample size, must be a positive integer; got %r" % (n,))
    r_n = math.sqrt(n) if r_n is None else float(r_n)
    eps_n = n ** (-1.0 / 3.0) if eps_n is None else float(eps_n)
    return r_n, eps_n, 1.0 + eps_n * r_n


def perturb(p_hat, p_b, r_n, eps_n):
    return p_hat + (eps_n * r_n) * (p_b - p_hat)


def decide(L, U, tau_lo, tau_hi):
    d = np.full(np.shape(U), UNDECIDED, dtype=np.int8)
    d[np.asarray(L) >= tau_hi] = ABOVE
    d[np.asarray(U) < tau_lo] = BELOW
    return d


def check_alpha(alpha):
    alpha = float(alpha)
    if not 0.0 < alpha < 1.0:
        raise ValueError("alpha must lie in (0, 1); got %r" % alpha)
    return alpha


def locked(n_above, n_open, B, alpha):
    """Whether the decision at alpha can no longer change while n_open draws are undecided or
    unsolved (solver/inference/hong_li.py:74-78): counting all of them above still rejects, or the
    draws certified above already exceed alpha."""
    return (n_above + n_open) / B <= alpha or n_above / B > alpha


def quantile_band(L, U, alpha):
    """(Q(L), Q(U)): the (1 - alpha)-quantile of the draws' distances lies between these
    (solver/inference/hong_li.py:102-107); only a draw whose bracket overlaps it moves either end."""
    return (float(np.quantile(np.asarray(L, dtype=np.float64), 1.0 - alpha)),
            float(np.quantile(np.asarray(U, dtype=np.float64), 1.0 - alpha)))


def ci_lower(L0, U0, L, U, alpha, r_n, eps_n):
    """The one-sided interval's lower end as (value, the upper end of its bracket, (q_lo, q_hi))
    (solver/inference/hong_li.py:81-90): value = L0 - q_hi / r_n with q_hi the (1 - alpha)-quantile
    of (U_b - L0) / eps_n, and the exact end lies below U0 - q_lo / r_n, q_lo the same quantile of
    (L_b - U0) / eps_n (the end grows with dist(p_hat) and falls with every dist(P_b))."""
    q_hi = float(np.quantile((np.asarray(U, dtype=np.float64) - L0) / eps_n, 1.0 - alpha))
    q_lo = float(np.quantile((np.asarray(L, dtype=np.float64) - U0) / eps_n, 1.0 - alpha))
    return L0 - q_hi / r_n, U0 - q_lo / r_n, (q_lo, q_hi)


def distance_interval(L0, U0, dev, alpha):
    """The two-sided interval (lower, upper, c) with c the (1 - alpha)-quantile of ||p_b - p_hat||
    (solver/inference/hong_li.py:93-99): dist is 1-Lipschitz, so [max(0, L0 - c), U0 + c] needs no
    draw solved."""
    c = float(np.quantile(np.asarray(dev, dtype=np.float64), 1.0 - alpha))
    return max(0.0, L0 - c), U0 + c, c


@dataclass
class PValue:
    p: float
    p_lo: float
    p_hi: float
    alpha: float
    reject: bool
    certain: bool
    n_below: int
    n_above: int
    n_undecided: int
    n_screened: int
    n_solved: int
    B: int
    tau: tuple
    dist_hat: tuple
    time: float
    draws_per_s: float
    T: tuple = ()               # (r_n L0, r_n U0): the test statistic's bracket
    stopped_early: bool = False # stop_when_decided ended the solves with draws still open


@dataclass
class Interval:
    """The one-sided (1 - alpha) interval [lower, inf) (solver/inference/bootstrap.py's Interval)."""
    lower: float
    lower_bracket: tuple
    lower_clipped: float
    upper: float
    alpha: float
    q: tuple
    reject: bool
    n_solved: int
    time: float


@dataclass
class DistanceInterval:
    """The two-sided (1 - alpha) interval [max(0, L0 - c), U0 + c] (solver/inference/bootstrap.py:108-118)."""
    lower: float
    upper: float
    alpha: float
    half_width: float
    dist_hat: tuple
    reject: bool
    time: float


class _HostDrawRows:
    """rows / screen of the GPU draws, computed block by block on the host as the reference does."""

    def __init__(self, draws, p_hat):
        self.d, self.p_hat = draws, np.asarray(p_hat, dtype=np.float64)

    def rows(self, idx, scale=None):
        rows = self.d.rows(idx)
        return rows if scale is None else self.p_hat + scale * (rows - self.p_hat)

    def screen(self, fit, scale):
        dev = np.empty(self.d.B)
        ub = None if fit is None else np.empty(self.d.B)
        for lo, hi, block in self.d.blocks():
            D = block - self.p_hat
            dev[lo:hi] = np.sqrt(np.einsum("ij,ij->i", D, D))
            if fit is not None:
                E = (self.p_hat + scale * (block - self.p_hat)) - fit
                ub[lo:hi] = np.sqrt(np.einsum("ij,ij->i", E, E))
        return dev, ub


def _dist(group):
    """(rank, world, group) of the process group the draws are sharded over (1 rank without one)."""
    try:
        import torch.distributed as dist
    except ImportError:
        return 0, 1, None
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return 0, 1, None
    return dist.get_rank(group), dist.get_world_size(group), group


def _device_for(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _broadcast_band(L0, U0, group):
    import torch
    import torch.distributed as dist
    t = torch.tensor([L0, U0], dtype=torch.float64, device=_device_for(group))
    dist.broadcast(t, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    return float(t[0]), float(t[1])


def _gather_record(L, U, solved, flag, tol_stop, tol_full, group):
    """Every rank's per-draw record combined: a draw's bounds are the tightest any rank found, its
    tolerances the tightest any rank reached, and its exit flag the one of a rank that solved it
    (NEVER when none did)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    t = torch.from_numpy(np.stack([L, U, solved.astype(np.float64), flag.astype(np.float64), tol_stop,
                                   tol_full])).to(_device_for(group))
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    allr = torch.stack(parts).cpu().numpy()
    flags = allr[:, 3]
    have = flags != NEVER
    first = np.argmax(have, axis=0)                       # the lowest rank that solved the draw
    cols = np.arange(flags.shape[1])
    flag_all = np.where(have.any(axis=0), flags[first, cols], NEVER).astype(np.int8)
    return (allr[:, 0].max(axis=0), allr[:, 1].min(axis=0), allr[:, 2].max(axis=0) > 0, flag_all,
            allr[:, 4].min(axis=0), allr[:, 5].min(axis=0))


class Bootstrap:
    def __init__(self, rum, n=None, panel=None, replies=None, B=None, weights=None, seed=None, r_n=None, eps_n=None,
                 method=None, method_args=None, abs_tol=None, rel_tol=None, refine=None, max_time=None,
                 draw_time=None, batch_slots=0, verbose=False, learned=False, train_draws=512,
                 mlp_hidden=(1024, 1024, 1024), mlp_epochs=100, mlp_batch=128, mlp_lr=1e-3, y0_state=False,
                 seed_net=0, checkpoint=None):
        d = defaults.BOOTSTRAP
        pick = lambda value, key: d[key] if value is None else value      # noqa: E731
        self.rum, self.p_hat = rum, rum.choice_probability
        self.B = int(pick(B, "B"))
        self.abs_tol, self.rel_tol = float(pick(abs_tol, "abs_tol")), float(pick(rel_tol, "rel_tol"))
        self.refine = int(pick(refine, "refine"))
        self.max_time = float(pick(max_time, "max_time"))
        self.draw_time = float(pick(draw_time, "draw_time"))
        if self.abs_tol < 0 or self.rel_tol < 0 or self.abs_tol + self.rel_tol == 0 or self.refine < 0:
            raise ValueError("abs_tol and rel_tol must be >= 0 and not both 0, and refine >= 0")
        if (panel is None) == (replies is None):
            raise ValueError("give the choices behind p_hat once: panel= (respondent, menu, chosen; respondents are "
                             "resampled) or replies= (menu, chosen; each menu's replies are resampled)")
        if panel is not None:
            self.draws = Draws(panel, rum.menu, rum.alternative, self.p_hat, self.B, pick(weights, "weights"),
                               pick(seed, "seed"))
        elif weights not in (None, MenuDraws.weights):
            raise ValueError("weights = %r is for panel=; replies= are resampled menu by menu" % (weights,))
        else:
            self.draws = MenuDraws(replies, rum.menu, rum.alternative, self.p_hat, self.B, pick(seed, "seed"))
        self.n = int(self.draws.default_n if n is None else n)
        self.r_n, self.eps_n, self.s = scaling(self.n, r_n, eps_n)
        self.draws.check_n(self.n)
        self._session, self._session_args = None, dict(method=method, method_args=method_args)
        self.batch_slots = batch_slots
        self.L, self.U = np.zeros(self.B), np.full(self.B, np.inf)
        self.solved = np.zeros(self.B, dtype=bool)
        self.n_refined = 0          # float32 draws that stalled undecided and finished in float64
        self.iters = np.zeros(self.B, dtype=np.int64)
        self.slot_iters = 0         # iterations the batched solves ran, summed over draws
        # learned warm start: a network trained on solved draws predicts a draw's fitted cells
        self.learned, self.train_draws = bool(learned), int(train_draws)
        self.mlp_hidden, self.mlp_epochs, self.mlp_batch = tuple(mlp_hidden), int(mlp_epochs), int(mlp_batch)
        self.mlp_lr, self.y0_state, self.seed_net = float(mlp_lr), bool(y0_state), int(seed_net)
        self.net, self.learned_info = None, None
        # the record (solver/inference/bootstrap.py:159-180,356-400): settings, fingerprints and
        # per draw the bracket, the tightest tolerances asked and the last exit flag
        self.method, self.method_args = method, method_args
        self.settings = dict(n=self.n, input=self.draws.input, B=self.B, weights=self.draws.weights,
                             seed=self.draws.seed, r_n=self.r_n, eps_n=self.eps_n, method=method,
                             method_args=method_args, abs_tol=self.abs_tol, rel_tol=self.rel_tol, refine=self.refine,
                             max_time=self.max_time, draw_time=self.draw_time, weighted=False)
        self.fingerprints = {"data": _sha(np.column_stack([np.asarray(rum.menu, dtype=np.float64),
                                                           np.asarray(rum.alternative, dtype=np.float64),
                                                           self.p_hat])),
                             self.draws.input: self.draws.input_fingerprint, "draws": None}
        self.certificates = []      # every certification of p_hat, as the reference records them
        self.tol_stop = np.full(self.B, np.inf)
        self.tol_full = np.full(self.B, np.inf)
        self.flag = np.full(self.B, NEVER, dtype=np.int8)
        self.results = {"p_value": {}, "confidence_interval": {}, "distance_interval": {}}
        self.screened = False
        self.n_screened = 0
        self.checkpoint = checkpoint
        self.L0 = self.U0 = None
        self.verbose = verbose
        self.time = dict(certificate=0.0, screen=0.0, solve=0.0)
        if checkpoint and os.path.exists(checkpoint):
            self._resume(checkpoint)

    @property
    def tau(self):
        return (self.s * self.L0, self.s * self.U0)

    @property
    def session(self):
        """The Session every solve of this bootstrap goes through, opened on first use as the
        reference opens its own (solver/inference/bootstrap.py:261-266): the record's plan stays
        None until a solve has run."""
        if self._session is None:
            self._session = self.rum.session(**self._session_args)
        return self._session

    @session.setter
    def session(self, s):
        self._session = s

    def _certify(self):
        """p_hat's bracket at the current tolerances (a later, tighter one only narrows it)."""
        t0 = time.perf_counter()
        r = self.session.solve(self.p_hat, abs_tol=self.abs_tol, rel_tol=self.rel_tol, max_time=self.max_time,
                               keep=True)
        if not math.isfinite(r.ub):
            raise RuntimeError("p_hat could not be certified: %s (%s)" % (r.status, r.message))
        self.certificates.append(dict(abs_tol=self.abs_tol, rel_tol=self.rel_tol, lb=r.lb, ub=r.ub,
                                      exit_flag=r.exit_flag, status=r.status, message=r.message,
                                      iterations=r.iterations, time=r.time, method=r.method,
                                      method_args=r.method_args, machine=r.machine))
        self.L0 = r.lb if self.L0 is None else max(self.L0, r.lb)
        self.U0 = r.ub if self.U0 is None else min(self.U0, r.ub)
        self.time["certificate"] += time.perf_counter() - t0

    def _start(self):
        """p_hat certified and every draw screened (once)."""
        if self.L0 is None:
            self._certify()
        if not self.screened:
            if self.session.fit is None:          # resumed before the screen: certify again
                self._certify()
            self._screen()

    def _draw_rows(self):
        """The draws' rows and the screen's norms (built on first use): on the GPU for integer panel
        weights, whose counts are exact in any order; on the host (rumb.draws, block by block) for
        real weights and replies."""
        if getattr(self, "_gdraws", None) is None:
            d = self.draws
            if getattr(d, "integer_weights", False):
                from . import _lib
                from .rum_solver import context
                self._gdraws = _lib.DrawRows(context(), d.W, d.lists, d.p_hat)
            else:
                self._gdraws = _HostDrawRows(d, self.p_hat)
        return self._gdraws

    def _screen(self):
        """dev_b = ||p_b - p_hat|| and U_b = min(U_b, ||perturb(p_b) - p_fit||) for every draw, on the
        GPU (the rows are the host's bit for bit; the norms agree to rounding)."""
        t0, fit = time.perf_counter(), self.session.fit
        self.dev, ub = self._draw_rows().screen(fit, self.eps_n * self.r_n)
        if ub is not None:
            self.U = np.minimum(self.U, ub)
        self.fingerprints["draws"] = self.draws.fingerprint      # set by a host pass over the blocks
        self.n_screened = int((self.U < self.tau[0]).sum())
        self.screened = True
        self.time["screen"] += time.perf_counter() - t0

    def _batch(self, ctx, prob, par, P, below, above, y0=None, want_fit=False):
        """One batched solve of the rows P; a float32 batch's draws whose bracket stalls undecided
        are solved again in float64. The result dicts, in P's order."""
        s = self.session
        res, info = ctx.bm_solve_batch(prob, par, P, below=below, above=above, warm=s._kept, slots=self.batch_slots,
                                       draw_time=self.draw_time, y0=y0, y0_state=self.y0_state and y0 is not None,
                                       want_fit=want_fit)
        self.last_batch = info
        self.slot_iters += int(info["total_iters"])
        if par.dtype == 1:
            lo = -np.inf if below is None else below
            hi = np.inf if above is None else above
            L = np.array([r["lb"] for r in res])
            U = np.array([r["ub"] for r in res])
            dec = decide(L, U, lo, hi)
            redo = [j for j in range(len(res)) if res[j]["stop_reason"] == "stall" and
                    (below is None or dec[j] == UNDECIDED)]
            if redo:
                par.dtype = 0
                res2, info2 = ctx.bm_solve_batch(prob, par, P[redo], below=below, above=above, warm=s._kept,
                                                 slots=self.batch_slots, draw_time=self.draw_time,
                                                 y0=None if y0 is None else y0[redo],
                                                 y0_state=self.y0_state and y0 is not None, want_fit=want_fit)
                par.dtype = 1
                self.slot_iters += int(info2["total_iters"])
                for j, r in zip(redo, res2):
                    r["lb"], r["ub"] = max(r["lb"], res[j]["lb"]), min(r["ub"], res[j]["ub"])
                    res[j] = r
                self.n_refined += len(redo)
                self.last_batch_f64 = info2
        return res

    def _train_net(self, P, fits):
        """Fits the network on solved draws: (P_b - p_hat) -> (p_fit_b - p_fit(p_hat)), scaled."""
        from . import _lib
        from .rum_solver import context
        X = P - self.p_hat
        Y = fits - self.session.fit
        self.x_scale = float(np.std(X)) or 1.0
        self.y_scale = float(np.std(Y)) or 1.0
        mp = P.shape[1]
        if mp > 16384:
            raise ValueError("the learned warm start takes at most 16384 observed cells; got %d" % mp)
        self.net = _lib.MLP(context(), [mp] + list(self.mlp_hidden) + [mp], seed=self.seed_net)
        loss = self.net.train(X / self.x_scale, Y / self.y_scale, epochs=self.mlp_epochs, batch=self.mlp_batch,
                              lr=self.mlp_lr, seed=self.seed_net)
        self.learned_info = dict(n_train=int(P.shape[0]), train_loss=loss)

    def predict_fit(self, P):
        """The network's predicted fitted cells for the draws' rows P."""
        return self.session.fit + self.y_scale * self.net.forward((P - self.p_hat) / self.x_scale)

    def solve_draws(self, idx, stops=True):
        """Solve the draws idx: bm_admm all together (batched), flow_cg one at a time. With learned=True
        the first train_draws draws solved train the network, and every later draw starts from its
        prediction (a certified lower-bound seed and, with y0_state, the start state's fitted cells)."""
        t0 = time.perf_counter()
        idx = np.asarray(idx, dtype=np.int64)
        if idx.size == 0:
            return
        tau_lo, tau_hi = self.tau
        P = self._draw_rows().rows(idx, self.eps_n * self.r_n)       # = perturb(p_hat, draws.rows(idx), ...)
        rum, s = self.rum, self.session
        if s.method == "bm_admm" and rum.n >= 8 and rum._single.size == 0:
            from .rum_solver import context
            if s._kept is None:                    # a resumed run: p_hat's state again, for the warm starts
                s.solve(self.p_hat, abs_tol=self.abs_tol, rel_tol=self.rel_tol, max_time=self.max_time, keep=True)
            ctx = context()
            a = s._args
            g = rum._geom
            prob = ctx.bm_problem(rum.n, g.menu.astype(np.uint32), g.alternative.astype(np.int32), self.p_hat)
            # a float32 batch only for a float32 session: a mixed session's draws would mostly stall
            # above the tolerance in float32 (the bootstrap's abs 5e-4 is far below the float32
            # floor at the distances of its panels) and be solved again from the start
            dt = "float32" if a["dtype"] == "float32" else "float64"
            par = ctx.bm_params(a["beta"], alpha=a["alpha"], precond_p=a["precond_p"], check=a["check"],
                                lb_every=a["lb_every"], max_iter=a["max_iter"], abs_tol=self.abs_tol,
                                rel_tol=self.rel_tol if self.rel_tol > 0 else None, dtype=dt)
            below, above = (tau_lo, tau_hi) if stops else (None, None)
            res = [None] * idx.size
            todo = np.arange(idx.size)
            if self.learned and self.net is None:
                ntr = min(self.train_draws, idx.size)
                part = self._batch(ctx, prob, par, P[:ntr], below, above, want_fit=True)
                res[:ntr] = part
                self._train_net(P[:ntr], np.stack([r["p_fit"] for r in part]))
                todo = todo[ntr:]
            if todo.size:
                y0 = self.predict_fit(P[todo]) if self.net is not None else None
                part = self._batch(ctx, prob, par, P[todo], below, above, y0=y0)
                for j, r in zip(todo, part):
                    res[j] = r
            for j, b in enumerate(idx):
                self.L[b] = max(self.L[b], res[j]["lb"])
                self.U[b] = min(self.U[b], res[j]["ub"])
                self.iters[b] = res[j]["iters"]
                self.flag[b] = _STOP_FLAG.get(res[j]["stop_reason"], -5)
        else:
            for j, b in enumerate(idx):
                r = s.solve(P[j], abs_tol=self.abs_tol, rel_tol=self.rel_tol, max_time=self.draw_time, warm=True,
                            below=tau_lo if stops else None, above=tau_hi if stops else None)
                self.L[b], self.U[b] = max(self.L[b], r.lb), min(self.U[b], r.ub)
                self.iters[b] = r.iterations
                self.flag[b] = r.exit_flag
        self.tol_stop[idx] = np.minimum(self.tol_stop[idx], self.abs_tol)
        if not stops:
            self.tol_full[idx] = np.minimum(self.tol_full[idx], self.abs_tol)
        self.solved[idx] = True
        self._save_checkpoint()
        self.time["solve"] += time.perf_counter() - t0

    # ------------------------------------------------------------------ record, checkpoint
    def record(self):
        """Everything needed to report or resume the run, as plain Python values, in the reference's
        record layout (solver/inference/bootstrap.py:356-370)."""
        s = self._session
        return dict(version=VERSION, settings=self.settings, fingerprints=self.fingerprints,
                    plan=None if s is None else dict(method=s.method, method_args=s.method_args,
                                                    auto_reason=s.auto_reason),
                    p_hat=dict(lb=self.L0, ub=self.U0, certificates=getattr(self, "certificates", [])),
                    tau=None if self.L0 is None else list(self.tau),
                    scaling=dict(r_n=self.r_n, eps_n=self.eps_n, s=self.s),
                    screen=dict(done=self.screened, n_below=self.n_screened),
                    **{self.draws.input: self.draws.summary()},
                    draws=dict(lb=self.L.tolist(), ub=self.U.tolist(), tol_stop=self.tol_stop.tolist(),
                               tol_full=self.tol_full.tolist(), exit_flag=self.flag.tolist()),
                    results=self.results, time=self.time, when=time.strftime("%Y-%m-%d %H:%M:%S"))

    def save(self, path):
        """record() as JSON (infinite bounds as Infinity), written atomically."""
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.record(), f, indent=1, default=_plain)
        os.replace(tmp, path)

    def _save_checkpoint(self):
        """The record written to the checkpoint path; under torch.distributed by rank 0 alone (every
        rank holds the same gathered record, and one writer keeps the file whole)."""
        if self.checkpoint and _dist(getattr(self, "_group", None))[0] == 0:
            self.save(self.checkpoint)

    def _resume(self, path):
        rec = json.load(open(path))
        same = dict(version=rec.get("version") == VERSION,
                    settings=json.loads(json.dumps(self.settings, default=_plain)) == rec.get("settings"),
                    data=rec.get("fingerprints", {}).get("data") == self.fingerprints["data"],
                    **{self.draws.input: rec.get("fingerprints", {}).get(self.draws.input)
                       == self.fingerprints[self.draws.input]})
        if not all(same.values()):
            raise ValueError("checkpoint %s belongs to another run (differs in: %s); delete it or pass another path"
                             % (path, ", ".join(k for k, v in same.items() if not v)))
        dr = rec["draws"]
        self.L, self.U = np.array(dr["lb"], dtype=np.float64), np.array(dr["ub"], dtype=np.float64)
        self.tol_stop = np.array(dr["tol_stop"], dtype=np.float64)
        self.tol_full = np.array(dr["tol_full"], dtype=np.float64)
        self.flag = np.array(dr["exit_flag"], dtype=np.int8)
        self.solved = self.flag != NEVER
        self.L0, self.U0 = rec["p_hat"]["lb"], rec["p_hat"]["ub"]
        self.screened, self.n_screened = rec["screen"]["done"], rec["screen"]["n_below"]
        self.results, self.time = rec["results"], rec["time"]
        self.certificates = rec["p_hat"].get("certificates", [])

    def confidence_interval(self, alpha=0.05):
        """The certified one-sided interval [lower, inf) (solver/inference/bootstrap.py:212-240):
        draws are solved to tolerance, largest upper bound first, only while their bracket overlaps
        the band [Q(L), Q(U)] of the quantile; up to `refine` rounds tighten the tolerances ten-fold
        (p_hat certified again) while the lower end's bracket is wider than 2 abs_tol."""
        alpha, t0 = check_alpha(alpha), time.perf_counter()
        self._start()
        n0 = int(np.isfinite(self.tol_full).sum())
        batch = max(1, math.ceil(alpha * self.B / 4))
        saved = (self.abs_tol, self.rel_tol)
        tol_a, tol_r = saved
        try:
            for rnd in range(self.refine + 1):
                if rnd:
                    low, high, _ = ci_lower(self.L0, self.U0, self.L, self.U, alpha, self.r_n, self.eps_n)
                    if high - low <= 2 * saved[0]:
                        break
                    tol_a, tol_r = tol_a / 10, tol_r / 10
                    self.abs_tol, self.rel_tol = tol_a, tol_r
                    if self.U0 - self.L0 > tol_a:
                        self._certify()
                while True:
                    q_l, q_u = quantile_band(self.L, self.U, alpha)
                    hot = np.flatnonzero((self.U >= q_l) & (self.L <= q_u) & (self.tol_full > tol_a))
                    if hot.size == 0:
                        break
                    self.solve_draws(np.sort(hot[np.argsort(-self.U[hot], kind="stable")[:batch]]), stops=False)
        finally:
            self.abs_tol, self.rel_tol = saved
        low, high, q = ci_lower(self.L0, self.U0, self.L, self.U, alpha, self.r_n, self.eps_n)
        res = Interval(lower=low, lower_bracket=(low, high), lower_clipped=max(0.0, low), upper=math.inf,
                       alpha=alpha, q=q, reject=low > 0, n_solved=int(np.isfinite(self.tol_full).sum()) - n0,
                       time=time.perf_counter() - t0)
        self.results["confidence_interval"][repr(alpha)] = asdict(res)
        self._save_checkpoint()
        return res

    def distance_interval(self, alpha=0.05):
        """The certified two-sided interval [max(0, L0 - c), U0 + c], c the (1 - alpha)-quantile of
        ||p_b - p_hat|| (solver/inference/bootstrap.py:242-255): p_hat's certificate and the screen's
        pass over the draws (on the GPU), no draw solved."""
        alpha, t0 = check_alpha(alpha), time.perf_counter()
        self._start()
        if getattr(self, "dev", None) is None:
            self.dev, _ = self._draw_rows().screen(None, self.eps_n * self.r_n)
        lower, upper, c = distance_interval(self.L0, self.U0, self.dev, alpha)
        res = DistanceInterval(lower=lower, upper=upper, alpha=alpha, half_width=c, dist_hat=(self.L0, self.U0),
                               reject=lower > 0, time=time.perf_counter() - t0)
        self.results["distance_interval"][repr(alpha)] = asdict(res)
        self._save_checkpoint()
        return res

    def p_value(self, alpha=0.05, stop_when_decided=False, max_draws=None, group=None):
        """The test's p-value. stop_when_decided: solve the open draws in chunks and stop once the
        decision at alpha is locked (the remaining draws cannot change it; one process only).
        Under torch.distributed (group: a process group, or the default one when it is initialized)
        every rank certifies p_hat on its own GPU, takes rank 0's band, solves every world-th open
        draw starting at its rank, and one all_gather of the per-draw record (L, U, solved, exit flag,
        tolerances) gives every rank the whole record; draws are independent, so nothing else is
        exchanged. Rank 0 alone writes the checkpoint."""
        alpha = check_alpha(alpha)
        t0 = time.perf_counter()
        rank, world, group = _dist(group)
        if self.L0 is None:
            self._certify()
            if world > 1:
                self.L0, self.U0 = _broadcast_band(self.L0, self.U0, group)
        self._start()
        if self.U0 > ZERO:
            dec = decide(self.L, self.U, *self.tau)
            todo = np.flatnonzero((dec == UNDECIDED) & ~self.solved)
            if max_draws is not None:
                todo = todo[:max_draws]
            mine = todo[rank::world] if world > 1 else todo
            if stop_when_decided and world == 1:
                chunk = max(64, int(self.batch_slots or 0))
                for lo in range(0, mine.size, chunk):
                    dec = decide(self.L, self.U, *self.tau)
                    if locked(int((dec == ABOVE).sum()), int((dec == UNDECIDED).sum()), self.B, alpha):
                        break
                    self.solve_draws(mine[lo:lo + chunk])
            elif mine.size:
                self.solve_draws(mine)
            if world > 1:
                (self.L, self.U, self.solved, self.flag, self.tol_stop,
                 self.tol_full) = _gather_record(self.L, self.U, self.solved, self.flag, self.tol_stop,
                                                 self.tol_full, group)
        self._group = group
        dec = decide(self.L, self.U, *self.tau)
        above = int((dec == ABOVE).sum())
        und = int((dec == UNDECIDED).sum())
        p_lo, p_hi = above / self.B, (above + und) / self.B
        solved = int(self.solved.sum())
        res = PValue(p=p_hi, p_lo=p_lo, p_hi=p_hi, alpha=alpha, reject=p_hi <= alpha,
                      certain=p_hi <= alpha or p_lo > alpha, n_below=int((dec == BELOW).sum()), n_above=above,
                      n_undecided=und, n_screened=self.n_screened, n_solved=solved, B=self.B, tau=self.tau,
                      dist_hat=(self.L0, self.U0), time=time.perf_counter() - t0,
                      draws_per_s=solved / self.time["solve"] if self.time["solve"] > 0 else float("nan"),
                      T=(self.r_n * self.L0, self.r_n * self.U0),
                      stopped_early=bool(stop_when_decided and und > 0 and locked(above, und, self.B, alpha)))
        self.results.setdefault("p_value", {})[repr(alpha)] = asdict(res)
        self._save_checkpoint()
        return res
