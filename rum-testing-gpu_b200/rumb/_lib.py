"""ctypes binding of librumb.so (include/rumb.h).

The library is the product path: there is no fallback. Loading fails loudly, with the reason,
when librumb.so is missing or cannot be loaded; every call raises RumbError on a nonzero status.
"""
import ctypes
import math
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "librumb.so")

OK, E_INVAL, E_OOM, E_CUDA, E_TIMEOUT, E_CANCEL, E_NODEV, E_INTERNAL = range(8)
F64, F32, MIXED = 0, 1, 2
STOP = {1: "gap_abs", 2: "gap_rel", 3: "time_limit", 4: "max_iter", 5: "ub_target", 6: "lb_target", 7: "cancel",
        8: "stall"}
DTYPES = {"float64": F64, "float32": F32, "mixed": MIXED}


class RumbError(RuntimeError):
    """A nonzero status from librumb; .code is the RUMB_E_* value."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class OutOfMemory(RumbError, MemoryError):
    pass


class BMProblem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("mp", ctypes.c_longlong), ("menu", ctypes.c_void_p),
                ("alt", ctypes.c_void_p), ("p", ctypes.c_void_p), ("on_device", ctypes.c_int)]


class BMParams(ctypes.Structure):
    _fields_ = [("beta", ctypes.c_double), ("alpha", ctypes.c_double), ("precond_p", ctypes.c_double),
                ("check", ctypes.c_int), ("lb_every", ctypes.c_int), ("max_iter", ctypes.c_longlong),
                ("abs_tol", ctypes.c_double), ("rel_tol", ctypes.c_double), ("time_limit", ctypes.c_double),
                ("ub_target", ctypes.c_double), ("lb_target", ctypes.c_double), ("dtype", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("stall_checks", ctypes.c_int), ("stall_rtol", ctypes.c_double),
                ("overlap_check", ctypes.c_int)]


class BMResult(ctypes.Structure):
    _fields_ = [("lb", ctypes.c_double), ("ub", ctypes.c_double), ("phi", ctypes.c_double),
                ("iters", ctypes.c_longlong), ("iters_f32", ctypes.c_longlong), ("stop", ctypes.c_int),
                ("n_push", ctypes.c_int), ("n_lb", ctypes.c_int), ("setup_s", ctypes.c_double),
                ("solve_s", ctypes.c_double), ("push_s", ctypes.c_double), ("per_iter_ms", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("launches", ctypes.c_longlong)]


class BatchParams(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("mem_fraction", ctypes.c_double), ("draw_time", ctypes.c_double),
                ("y0", ctypes.c_void_p), ("y0_state", ctypes.c_int), ("p_fit", ctypes.c_void_p)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("bytes_per_slot", ctypes.c_double), ("total_iters", ctypes.c_longlong),
                ("setup_s", ctypes.c_double), ("solve_s", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("lo_bits", ctypes.c_int), ("launches", ctypes.c_longlong)]


class KernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 64), ("launches", ctypes.c_longlong), ("total_ms", ctypes.c_double),
                ("bytes_per_launch", ctypes.c_double), ("graph", ctypes.c_int)]


TRACE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_double,
                            ctypes.c_double, ctypes.c_double)

_vp = ctypes.c_void_p
_SIGS = {
    "rumb_version": ([], ctypes.c_int),
    "rumb_gemm_bf16": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp], ctypes.c_int),
    "rumb_mlp_create": ([_vp, ctypes.c_int, _vp, ctypes.c_ulonglong, ctypes.POINTER(_vp)], ctypes.c_int),
    "rumb_mlp_destroy": ([_vp], ctypes.c_int),
    "rumb_mlp_num_params": ([_vp, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "rumb_mlp_get_params": ([_vp, _vp], ctypes.c_int),
    "rumb_mlp_set_params": ([_vp, _vp], ctypes.c_int),
    "rumb_mlp_forward": ([_vp, _vp, ctypes.c_longlong, _vp], ctypes.c_int),
    "rumb_mlp_loss_grad": ([_vp, _vp, _vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double), _vp], ctypes.c_int),
    "rumb_mlp_train": ([_vp, _vp, _vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                        ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "rumb_last_error": ([ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    "rumb_ctx_create": ([ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
    "rumb_ctx_destroy": ([_vp], ctypes.c_int),
    "rumb_ctx_set_stream": ([_vp, _vp], ctypes.c_int),
    "rumb_ctx_sync": ([_vp], ctypes.c_int),
    "rumb_mem_info": ([_vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "rumb_cancel": ([_vp], ctypes.c_int),
    "rumb_butterfly": ([_vp, ctypes.c_int, ctypes.c_int, _vp, _vp] + [ctypes.c_double] * 4, ctypes.c_int),
    "rumb_butterfly_noalloc": ([_vp, ctypes.c_int, ctypes.c_int, _vp, _vp] + [ctypes.c_double] * 4, ctypes.c_int),
    "rumb_prox": ([_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_double, _vp], ctypes.c_int),
    "rumb_push_ub64": ([_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_longlong, _vp, _vp, _vp,
                        ctypes.POINTER(ctypes.c_double), _vp], ctypes.c_int),
    "rumb_fw_lb64": ([_vp, ctypes.c_int, ctypes.c_longlong, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_double)],
                     ctypes.c_int),
    "rumb_bm_solve": ([_vp, ctypes.POINTER(BMProblem), ctypes.POINTER(BMParams), _vp, ctypes.POINTER(_vp),
                       ctypes.POINTER(BMResult), _vp, TRACE_FN, _vp], ctypes.c_int),
    "rumb_bm_state_destroy": ([_vp], ctypes.c_int),
    "rumb_bm_solve_batch": ([_vp, ctypes.POINTER(BMProblem), ctypes.POINTER(BMParams), ctypes.POINTER(BatchParams),
                             ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.POINTER(BMResult), ctypes.POINTER(BatchInfo)],
                            ctypes.c_int),
    "rumb_bm_profile": ([_vp, ctypes.POINTER(BMProblem), ctypes.POINTER(BMParams), ctypes.c_int, ctypes.c_int,
                         ctypes.POINTER(KernelStat), ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "rumb_cg_pricer_create": ([_vp, ctypes.c_int, ctypes.c_longlong, _vp, _vp, ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
    "rumb_cg_price": ([_vp, _vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _vp,
                       ctypes.POINTER(ctypes.c_double), _vp], ctypes.c_int),
    "rumb_cg_pricer_destroy": ([_vp], ctypes.c_int),
    "rumb_cg_master_create": ([_vp, _vp, _vp, ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
    "rumb_cg_master_add_column": ([_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "rumb_cg_master_apply": ([_vp, _vp, _vp, ctypes.c_int], ctypes.c_int),
    "rumb_cg_master_price": ([_vp, ctypes.POINTER(ctypes.c_double), _vp, ctypes.POINTER(ctypes.c_double)],
                             ctypes.c_int),
    "rumb_cg_master_p_out": ([_vp, _vp], ctypes.c_int),
    "rumb_cg_master_destroy": ([_vp], ctypes.c_int),
    "rumb_draws_create": ([_vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_longlong, ctypes.c_int, _vp, _vp, _vp, _vp,
                           _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)], ctypes.c_int),
    "rumb_draws_rows": ([_vp, _vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_double, _vp], ctypes.c_int),
    "rumb_draws_screen": ([_vp, _vp, ctypes.c_double, _vp, _vp], ctypes.c_int),
    "rumb_draws_destroy": ([_vp], ctypes.c_int),
    "rumb_cg_pricer_info": ([_vp, _vp, _vp], ctypes.c_int),
    "rumb_cg_pricer_max64": ([_vp, _vp, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "rumb_bm_iterate": ([_vp, ctypes.POINTER(BMProblem), ctypes.POINTER(BMParams), _vp, _vp, _vp, _vp,
                         ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "rumb_bm_plan": ([_vp, ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)],
                     ctypes.c_int),
}

_lib = None
_lock = threading.Lock()


def load():
    """The loaded librumb.so (raises with the reason when it is missing or fails to load)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError("librumb.so is not built (%s); run rum-testing-gpu_b200/build.py" % LIB_PATH)
            L = ctypes.CDLL(LIB_PATH)
            for name, (args, res) in _SIGS.items():
                f = getattr(L, name)
                f.argtypes = args
                f.restype = res
            _lib = L
    return _lib


def bm_plan(n, mp, dtype):
    """Device bytes one rumb_bm_solve of (n, mp, dtype) allocates (rumb_bm_plan; no GPU needed).
    dtype: "float64", "float32" or "mixed"."""
    out = ctypes.c_size_t()
    check(load().rumb_bm_plan(None, int(n), int(mp), DTYPES[dtype], ctypes.byref(out)))
    return int(out.value)


def exported_symbols():
    return sorted(_SIGS)


def last_error():
    buf = ctypes.create_string_buffer(4096)
    load().rumb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status):
    if status != OK:
        msg = last_error()
        if status == E_OOM:
            raise OutOfMemory(status, "out of memory: " + msg)
        raise RumbError(status, msg)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """One GPU's library context (device memory, stream, graphs, cached tables)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check(load().rumb_ctx_create(int(device), ctypes.byref(h)))
        self.h = h
        self.device = int(device)

    def close(self):
        if self.h:
            load().rumb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        check(load().rumb_ctx_set_stream(self.h, ctypes.c_void_p(int(stream_handle) if stream_handle else 0)))

    def sync(self):
        check(load().rumb_ctx_sync(self.h))

    def mem_info(self):
        f, t = ctypes.c_size_t(), ctypes.c_size_t()
        check(load().rumb_mem_info(self.h, ctypes.byref(f), ctypes.byref(t)))
        return f.value, t.value

    def cancel(self):
        load().rumb_cancel(self.h)

    # -------------------------------------------------------------- primitives
    def butterfly(self, n, v, a, b, c, d):
        v = np.ascontiguousarray(v)
        dt = {np.dtype(np.float64): F64, np.dtype(np.float32): F32}[v.dtype]
        if v.size != n << (n - 1):
            raise ValueError("slab of n * 2^(n-1) values expected")
        out = np.empty_like(v)
        check(load().rumb_butterfly(self.h, n, dt, _p(v), _p(out), a, b, c, d))
        return out

    def butterfly_noalloc(self, n, v, a, b, c, d):
        """butterfly() staged in the library's static device array: no device allocation, n <= 16."""
        v = np.ascontiguousarray(v)
        dt = {np.dtype(np.float64): F64, np.dtype(np.float32): F32}[v.dtype]
        if v.size != n << (n - 1):
            raise ValueError("slab of n * 2^(n-1) values expected")
        out = np.empty_like(v)
        check(load().rumb_butterfly_noalloc(self.h, n, dt, _p(v), _p(out), a, b, c, d))
        return out

    def prox(self, n, v, xhat, wmask, beta2):
        v = np.ascontiguousarray(v)
        dt = {np.dtype(np.float64): F64, np.dtype(np.float32): F32}[v.dtype]
        xhat = np.ascontiguousarray(xhat, dtype=v.dtype)
        wmask = np.ascontiguousarray(wmask, dtype=v.dtype)
        out = np.empty_like(v)
        check(load().rumb_prox(self.h, n, dt, _p(v), _p(xhat), _p(wmask), float(beta2), _p(out)))
        return out

    def push_ub64(self, n, x, menu, alt, p, want_fit=True):
        x = np.ascontiguousarray(x)
        dt = {np.dtype(np.float64): F64, np.dtype(np.float32): F32}[x.dtype]
        menu = np.ascontiguousarray(menu, dtype=np.uint32)
        alt = np.ascontiguousarray(alt, dtype=np.int32)
        p = np.ascontiguousarray(p, dtype=np.float64)
        ub = ctypes.c_double()
        fit = np.empty(p.size) if want_fit else None
        check(load().rumb_push_ub64(self.h, n, dt, _p(x), p.size, _p(menu), _p(alt), _p(p), ctypes.byref(ub),
                                    _p(fit) if want_fit else None))
        return ub.value, fit

    def fw_lb64(self, n, menu, alt, y, p):
        menu = np.ascontiguousarray(menu, dtype=np.uint32)
        alt = np.ascontiguousarray(alt, dtype=np.int32)
        y = np.ascontiguousarray(y, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        lb = ctypes.c_double()
        check(load().rumb_fw_lb64(self.h, n, p.size, _p(menu), _p(alt), _p(y), _p(p), ctypes.byref(lb)))
        return lb.value

    # -------------------------------------------------------------- BM-ADMM
    @staticmethod
    def bm_params(beta, alpha=1.95, precond_p=math.sqrt(2.0), check=50, lb_every=1, max_iter=10 ** 7,
                  abs_tol=1e-5, rel_tol=1e-4, time_limit=0.0, ub_target=None, lb_target=None, dtype="float64",
                  use_graph=True, stall_checks=20, stall_rtol=0.05, overlap_check=False):
        P = BMParams()
        P.beta, P.alpha, P.precond_p = float(beta), float(alpha), float(precond_p)
        P.check, P.lb_every, P.max_iter = int(check), int(lb_every), int(max_iter)
        P.abs_tol = -1.0 if abs_tol is None else float(abs_tol)
        P.rel_tol = -1.0 if rel_tol is None else float(rel_tol)
        P.time_limit = float(time_limit or 0.0)
        P.ub_target = math.nan if ub_target is None else float(ub_target)
        P.lb_target = math.nan if lb_target is None else float(lb_target)
        P.dtype = DTYPES[dtype] if isinstance(dtype, str) else int(dtype)
        P.use_graph = int(bool(use_graph))
        P.stall_checks, P.stall_rtol = int(stall_checks), float(stall_rtol)
        P.overlap_check = int(bool(overlap_check))
        return P

    @staticmethod
    def bm_problem(n, menu, alt, p):
        """(BMProblem, keep-alive arrays) from host rows."""
        menu = np.ascontiguousarray(menu, dtype=np.uint32)
        alt = np.ascontiguousarray(alt, dtype=np.int32)
        p = np.ascontiguousarray(p, dtype=np.float64)
        pr = BMProblem(int(n), p.size, _p(menu), _p(alt), _p(p), 0)
        return pr, (menu, alt, p)

    def bm_solve(self, problem, params, warm=None, keep=False, want_fit=True, trace=None):
        """(result dict, p_fit or None, kept state handle or None)."""
        pr, _alive = problem if isinstance(problem, tuple) else (problem, None)
        res = BMResult()
        fit = np.empty(pr.mp) if want_fit else None
        kept = ctypes.c_void_p()
        rows = []
        if trace is not None:
            def cb(_u, it, wall, phi, ub, lb):
                rows.append((int(it), float(wall), float(phi), float(ub), float(lb)))
            fn = TRACE_FN(cb)
        else:
            fn = TRACE_FN()
        st = load().rumb_bm_solve(self.h, ctypes.byref(pr), ctypes.byref(params), warm.h if warm else None,
                                  ctypes.byref(kept) if keep else None, ctypes.byref(res),
                                  _p(fit) if want_fit else None, fn, None)
        check(st)
        out = {f: getattr(res, f) for f, _ in BMResult._fields_}
        out["stop_reason"] = STOP.get(res.stop, "unknown")
        if trace is not None:
            trace.extend(rows)
        return out, fit, (BMState(kept) if keep and kept.value else None)

    def bm_solve_batch(self, problem, params, P, below=None, above=None, warm=None, slots=0, mem_fraction=0.8,
                       draw_time=0.0, y0=None, y0_state=False, want_fit=False):
        """Solves the rows of P (B x mp) together; (list of result dicts, info dict). y0 (B x mp):
        predicted fits, whose Frank-Wolfe lower bounds seed the brackets (y0_state: and the start
        states); want_fit: each result dict gets its draw's "p_fit" row."""
        pr, _alive = problem if isinstance(problem, tuple) else (problem, None)
        P = np.ascontiguousarray(P, dtype=np.float64)
        if P.ndim != 2 or P.shape[1] != pr.mp:
            raise ValueError("P must be (B, %d)" % pr.mp)
        B = P.shape[0]
        lo = None if below is None else np.ascontiguousarray(np.broadcast_to(below, (B,)), dtype=np.float64)
        hi = None if above is None else np.ascontiguousarray(np.broadcast_to(above, (B,)), dtype=np.float64)
        res = (BMResult * B)()
        info = BatchInfo()
        yy = None if y0 is None else np.ascontiguousarray(y0, dtype=np.float64)
        if yy is not None and yy.shape != P.shape:
            raise ValueError("y0 must have P's shape")
        fits = np.zeros(P.shape, dtype=np.float64) if want_fit else None
        bp = BatchParams(int(slots), float(mem_fraction), float(draw_time), _p(yy) if yy is not None else None,
                         int(bool(y0_state)), _p(fits) if fits is not None else None)
        check(load().rumb_bm_solve_batch(self.h, ctypes.byref(pr), ctypes.byref(params), ctypes.byref(bp), B, _p(P),
                                         _p(lo) if lo is not None else None, _p(hi) if hi is not None else None,
                                         warm.h if warm else None, res, ctypes.byref(info)))
        out = []
        for b, r in enumerate(res):
            d = {f: getattr(r, f) for f, _ in BMResult._fields_}
            d["stop_reason"] = STOP.get(r.stop, "unknown")
            if fits is not None:
                d["p_fit"] = fits[b]
            out.append(d)
        return out, {f: getattr(info, f) for f, _ in BatchInfo._fields_}

    def bm_profile(self, problem, params, iters=20, warmup=3):
        """[dict(name, launches, total_ms, bytes_per_launch)] over `iters` eager iterations."""
        pr, _alive = problem if isinstance(problem, tuple) else (problem, None)
        cap = 64
        arr = (KernelStat * cap)()
        cnt = ctypes.c_int()
        check(load().rumb_bm_profile(self.h, ctypes.byref(pr), ctypes.byref(params), int(warmup), int(iters), arr, cap,
                                     ctypes.byref(cnt)))
        return [dict(name=arr[i].name.decode(), launches=arr[i].launches, total_ms=arr[i].total_ms,
                     bytes_per_launch=arr[i].bytes_per_launch, graph=bool(arr[i].graph)) for i in range(cnt.value)]

    def bm_iterate(self, problem, params, state, iters, cold_start=False):
        pr, _alive = problem if isinstance(problem, tuple) else (problem, None)
        dt = np.float64 if params.dtype == F64 else np.float32
        m2 = pr.n << (pr.n - 1)
        st = {}
        for k in ("x2", "s", "y", "z"):
            st[k] = np.ascontiguousarray(state[k], dtype=dt).copy() if state is not None else np.zeros(m2, dt)
        check(load().rumb_bm_iterate(self.h, ctypes.byref(pr), ctypes.byref(params), _p(st["x2"]), _p(st["s"]),
                                     _p(st["y"]), _p(st["z"]), int(iters), int(bool(cold_start))))
        return st


PRICE_MODES = {"mask": 0, "f32": 1, "u16": 2, "u24": 3}
PRICE_SCAN = 16
PRICE_STREAM = 32


def to_bf16_bits(x):
    """float32 -> bfloat16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def gemm_bf16(ctx, A_bits, B_bits):
    """C = A . B^T on the tensor cores (A [M x K], B [N x K] bfloat16 bit patterns): float32 C."""
    A = np.ascontiguousarray(A_bits, dtype=np.uint16)
    B = np.ascontiguousarray(B_bits, dtype=np.uint16)
    (M, K), (N, K2) = A.shape, B.shape
    if K != K2:
        raise ValueError("A and B must share K")
    C = np.empty((M, N), dtype=np.float32)
    check(load().rumb_gemm_bf16(ctx.h, M, N, K, _p(A), _p(B), _p(C)))
    return C


class MLP:
    """The tensor-core MLP (rumb_mlp_*): widths dims[0] -> ... -> dims[-1], GELU between layers."""

    def __init__(self, ctx, dims, seed=0):
        self.ctx, self.dims = ctx, [int(d) for d in dims]
        d = np.asarray(self.dims, dtype=np.int32)
        h = ctypes.c_void_p()
        check(load().rumb_mlp_create(ctx.h, len(self.dims) - 1, _p(d), int(seed), ctypes.byref(h)))
        self.h = h
        n = ctypes.c_longlong()
        check(load().rumb_mlp_num_params(self.h, ctypes.byref(n)))
        self.num_params = int(n.value)

    def close(self):
        if getattr(self, "h", None):
            load().rumb_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        out = np.empty(self.num_params, dtype=np.float32)
        check(load().rumb_mlp_get_params(self.h, _p(out)))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError("expected %d parameters" % self.num_params)
        check(load().rumb_mlp_set_params(self.h, _p(p)))

    def forward(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.empty((X.shape[0], self.dims[-1]), dtype=np.float32)
        check(load().rumb_mlp_forward(self.h, _p(X), X.shape[0], _p(Y)))
        return Y

    def loss_grad(self, X, T, want_grad=True):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = ctypes.c_double()
        g = np.empty(self.num_params, dtype=np.float32) if want_grad else None
        check(load().rumb_mlp_loss_grad(self.h, _p(X), _p(T), X.shape[0], ctypes.byref(loss),
                                        _p(g) if g is not None else None))
        return loss.value, g

    def train(self, X, T, epochs=20, batch=256, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = ctypes.c_double()
        check(load().rumb_mlp_train(self.h, _p(X), _p(T), X.shape[0], int(epochs), int(batch), float(lr), int(seed),
                                    ctypes.byref(loss)))
        return loss.value


class CgMaster:
    """The CG master's column bookkeeping on a pricer's GPU (see rumb_cg_master_create)."""

    def __init__(self, pricer, alts, p_obs, max_cols):
        alts = np.ascontiguousarray(alts, dtype=np.int32)
        p_obs = np.ascontiguousarray(p_obs, dtype=np.float64)
        self.M, self.n, self.W = int(p_obs.size), pricer.n, (int(p_obs.size) + 63) // 64
        h = ctypes.c_void_p()
        check(load().rumb_cg_master_create(pricer.h, _p(alts), _p(p_obs), int(max_cols), ctypes.byref(h)))
        self.h, self.pricer, self.K = h, pricer, 0

    def add_column(self, rank_pos=None, bits=None):
        """(index, packed column bits uint64[W], Gram row float64[index + 1])."""
        out = np.empty(self.W, dtype=np.uint64)
        row = np.empty(self.K + 1)
        k = ctypes.c_int()
        rp = None if rank_pos is None else np.ascontiguousarray(rank_pos, dtype=np.int32)
        b = None if bits is None else np.ascontiguousarray(bits, dtype=np.uint64)
        check(load().rumb_cg_master_add_column(self.h, None if rp is None else _p(rp), None if b is None else _p(b),
                                               _p(out), _p(row), ctypes.byref(k)))
        self.K += 1
        return k.value, out, row

    def apply(self, cols, delta):
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        delta = np.ascontiguousarray(delta, dtype=np.float64)
        check(load().rumb_cg_master_apply(self.h, _p(cols), _p(delta), int(cols.size)))

    def price(self):
        vmax, margin = ctypes.c_double(), ctypes.c_double()
        rank = np.zeros(self.n, dtype=np.int32)
        check(load().rumb_cg_master_price(self.h, ctypes.byref(vmax), _p(rank), ctypes.byref(margin)))
        return vmax.value, rank, margin.value

    def p_out(self):
        out = np.empty(self.M)
        check(load().rumb_cg_master_p_out(self.h, _p(out)))
        return out

    def close(self):
        if self.h:
            load().rumb_cg_master_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DrawRows:
    """Bootstrap draws on one GPU (see rumb_draws_create): W is the B x R respondent weights and
    lists the panel's count lists (rumb.draws.CountLists: per menu the respondents offered it, per
    row the respondents who chose it, each with its count, and every row's menu)."""

    def __init__(self, ctx, W, lists, p_hat):
        W = np.ascontiguousarray(W, dtype=np.float64)
        B, R = W.shape
        optr = np.ascontiguousarray(lists.menu_ptr, dtype=np.int64)
        oresp = np.ascontiguousarray(lists.menu_resp, dtype=np.int32)
        ocnt = np.ascontiguousarray(lists.menu_cnt, dtype=np.float64)
        cptr = np.ascontiguousarray(lists.row_ptr, dtype=np.int64)
        cresp = np.ascontiguousarray(lists.row_resp, dtype=np.int32)
        ccnt = np.ascontiguousarray(lists.row_cnt, dtype=np.float64)
        row_menu = np.ascontiguousarray(lists.row_menu, dtype=np.int32)
        p_hat = np.ascontiguousarray(p_hat, dtype=np.float64)
        self.B, self.R, self.M = int(B), int(R), int(p_hat.size)
        h = ctypes.c_void_p()
        check(load().rumb_draws_create(ctx.h, self.B, self.R, self.M, int(optr.size - 1), _p(W), _p(optr), _p(oresp),
                                       _p(ocnt), _p(cptr), _p(cresp), _p(ccnt), _p(row_menu), _p(p_hat),
                                       ctypes.byref(h)))
        self.h, self.ctx = h, ctx

    def rows(self, idx, scale=None):
        """Draws idx as rows (len(idx) x M): the shares, or with scale p_hat + scale (p_b - p_hat)."""
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        out = np.empty((idx.size, self.M))
        check(load().rumb_draws_rows(self.h, _p(idx), idx.size, 0 if scale is None else 1,
                                     0.0 if scale is None else float(scale), _p(out)))
        return out

    def screen(self, fit, scale):
        """(dev, ub) over all draws: ||p_b - p_hat|| and ||p_hat + scale (p_b - p_hat) - fit||."""
        dev, ub = np.empty(self.B), np.empty(self.B)
        f = None if fit is None else np.ascontiguousarray(fit, dtype=np.float64)
        check(load().rumb_draws_screen(self.h, None if f is None else _p(f), float(scale), _p(dev),
                                       None if f is None else _p(ub)))
        return dev, (ub if f is not None else None)

    def close(self):
        if self.h:
            load().rumb_draws_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pricer:
    """Flow-CG pricer on one GPU (rows in x-major order; see rumb_cg_pricer_create)."""

    def __init__(self, ctx, n, menus, offsets, mode="u24", k_pred=None, fma_decode=True, lists=True, stream=False):
        """lists=False: scan x's rows in every sweep instead of walking the cover lists.
        stream=True (float32 storage): keep the two rank-indexed layers even when the lattice would
        fit by mask."""
        menus = np.ascontiguousarray(menus, dtype=np.uint64)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        h = ctypes.c_void_p()
        code = PRICE_MODES[mode] | (0 if lists else PRICE_SCAN) | (PRICE_STREAM if stream else 0)
        check(load().rumb_cg_pricer_create(ctx.h, int(n), menus.size, _p(menus), _p(offsets), code,
                                           0 if k_pred is None else int(k_pred), int(bool(fma_decode)),
                                           ctypes.byref(h)))
        self.h, self.n, self.mp, self.mode, self.ctx = h, int(n), menus.size, mode, ctx

    def max64(self, scores):
        """V[full] of the float64 max sweep over float64 scores in the pricer's row order."""
        scores = np.ascontiguousarray(scores, dtype=np.float64)
        if scores.size != self.mp:
            raise ValueError("expected %d scores" % self.mp)
        v = ctypes.c_double()
        check(load().rumb_cg_pricer_max64(self.h, _p(scores), ctypes.byref(v)))
        return v.value

    @property
    def list_entries(self):
        """Cover-list entries (-1 when the pricer scans rows)."""
        e = ctypes.c_longlong()
        check(load().rumb_cg_pricer_info(self.h, ctypes.byref(e), None))
        return e.value

    def price(self, scores, want_steps=False):
        """(vmax, rank_pos int32[n], margin[, layer_step float32[n+1]]) for float32 scores."""
        scores = np.ascontiguousarray(scores, dtype=np.float32)
        if scores.size != self.mp:
            raise ValueError("expected %d scores" % self.mp)
        vmax, margin = ctypes.c_double(), ctypes.c_double()
        rank = np.zeros(self.n, dtype=np.int32)
        steps = np.zeros(self.n + 1, dtype=np.float32)
        check(load().rumb_cg_price(self.h, _p(scores), 0, ctypes.byref(vmax), _p(rank), ctypes.byref(margin),
                                   _p(steps)))
        if want_steps:
            return vmax.value, rank, margin.value, steps
        return vmax.value, rank, margin.value

    def price_device(self, scores_ptr):
        vmax, margin = ctypes.c_double(), ctypes.c_double()
        rank = np.zeros(self.n, dtype=np.int32)
        check(load().rumb_cg_price(self.h, ctypes.c_void_p(int(scores_ptr)), 1, ctypes.byref(vmax), _p(rank),
                                   ctypes.byref(margin), None))
        return vmax.value, rank, margin.value

    def close(self):
        if self.h:
            load().rumb_cg_pricer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BMState:
    """A kept ADMM state on the device (freed with the object)."""

    def __init__(self, h):
        self.h = h

    def close(self):
        if self.h:
            load().rumb_bm_state_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
