"""The reference's own kernels, JIT-compiled and replayed on the GPU: the comparison side of the
parity tests and of bench.py's reference-kernel timing (never the product).

baseline/build_ref.py writes the reference's CUDA source strings to baseline/_ref/*.cu. This module
compiles them with NVRTC (through cuda-python, the same compiler CuPy drives, default options:
fmad on, IEEE division) and replays the reference's host sequence with them:

  price_stream / price_mask   StreamPricer.price and the mask sweep + backtrace
                              (solver/flow_cg/pricing_stream.py:302-412, solver/flow_cg/solver.py:169-200)
  BMReplay                    solve_kadmm_v2's float64 iteration (solver/bm_admm/solver.py:240-254)
                              with Bfly2's calibrated stage plan (solver/bm_admm/butterfly2.py:160-230),
                              replayed as a CUDA graph like the reference's use_graph path, its
                              float64 check (push_to_ub64 + fw_lb_rows_gpu) and the runner's certified
                              loop: the reference side of the iterate and bracket parity tests, and
                              of bench.py's reference-kernel timing
  time_pricing                the reference's pricing kernels on one sweep's layers (bf_stream_u24 /
                              bf_stream_u16 per layer, bf_update for the mask storage)

Device buffers are torch tensors (plumbing); kernels launch through the CUDA driver API on the
current torch stream. Only tests/ and bench.py's comparison legs use this module.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")


def available():
    return all(os.path.exists(os.path.join(REF, f)) for f in ("ref_bm_f64.cu", "ref_cert64.cu", "ref_pricing.cu"))


def _check(res):
    err = res[0] if isinstance(res, tuple) else res
    if int(err) != 0:
        raise RuntimeError("CUDA driver / NVRTC error %s" % (err,))
    return res[1:] if isinstance(res, tuple) and len(res) > 1 else None


class _Module:
    def __init__(self, path, options=()):
        from cuda.bindings import driver, nvrtc
        import torch
        torch.zeros(1, device="cuda")                      # make torch's primary context current
        src = open(path).read().encode()
        major = torch.cuda.get_device_capability()[0]
        minor = torch.cuda.get_device_capability()[1]
        err, prog = nvrtc.nvrtcCreateProgram(src, os.path.basename(path).encode(), 0, [], [])
        _check((err,))
        opts = [("--gpu-architecture=sm_%d%d" % (major, minor)).encode()] + [o.encode() for o in options]
        err = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)[0]
        if int(err) != 0:
            _, n = nvrtc.nvrtcGetProgramLogSize(prog)
            log = b" " * n
            nvrtc.nvrtcGetProgramLog(prog, log)
            raise RuntimeError("NVRTC failed on %s:\n%s" % (path, log.decode(errors="replace")))
        _, size = nvrtc.nvrtcGetCUBINSize(prog)
        cubin = b" " * size
        _check(nvrtc.nvrtcGetCUBIN(prog, cubin))
        err, self.mod = driver.cuModuleLoadData(cubin)
        _check((err,))
        self.driver = driver
        self.fns = {}

    def fn(self, name):
        if name not in self.fns:
            err, f = self.driver.cuModuleGetFunction(self.mod, name.encode())
            _check((err,))
            self.fns[name] = f
        return self.fns[name]


class _Launcher:
    """launch(name, grid, block, args, shmem): args are (ctypes type, value) pairs; a torch
    tensor stands for its device pointer."""

    def __init__(self, *modules):
        self.modules = modules
        from cuda.bindings import driver
        self.driver = driver

    def _fn(self, name):
        for m in self.modules:
            try:
                return m.fn(name)
            except RuntimeError:
                continue
        raise KeyError(name)

    def launch(self, name, grid, block, args, shmem=0):
        import torch
        vals = []
        for a in args:
            if isinstance(a, torch.Tensor):
                vals.append(ctypes.c_void_p(a.data_ptr()))
            elif isinstance(a, tuple):
                vals.append(a[0](a[1]))
            else:
                raise TypeError(a)
        arr = (ctypes.c_void_p * len(vals))(*[ctypes.addressof(v) for v in vals])
        f = self._fn(name)
        if shmem > 48 * 1024:
            self.driver.cuFuncSetAttribute(
                f, self.driver.CUfunction_attribute.CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, shmem)
        st = torch.cuda.current_stream().cuda_stream
        _check(self.driver.cuLaunchKernel(f, int(grid), 1, 1, int(block), 1, 1, int(shmem), st,
                                          ctypes.addressof(arr), 0))
        self._keep = (vals, arr)


_I, _LL, _ULL, _D, _F = ctypes.c_int, ctypes.c_longlong, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_float
_MODS = {}


def _mods():
    if not _MODS:
        _MODS["bm"] = _Module(os.path.join(REF, "ref_bm_f64.cu"))
        _MODS["cert"] = _Module(os.path.join(REF, "ref_cert64.cu"))
        _MODS["pricing"] = _Module(os.path.join(REF, "ref_pricing.cu"), options=("--std=c++11",))
        if os.path.exists(os.path.join(REF, "ref_max64.cu")):
            _MODS["max64"] = _Module(os.path.join(REF, "ref_max64.cu"), options=("--std=c++11",))
    return _MODS


# ------------------------------------------------------------------ pricing
def _binom(n):
    t = np.zeros((n + 1) * (n + 1), dtype=np.uint64)
    for b in range(n + 1):
        for k in range(b + 1):
            t[b * (n + 1) + k] = math.comb(b, k)
    return t


def _colex_rank(mask):
    r, t, b = 0, 0, 0
    while mask:
        if mask & 1:
            t += 1
            r += math.comb(b, t)
        mask >>= 1
        b += 1
    return r


def _layers(n):
    """The masks of popcount k in ascending order, k = 0 .. n (the reference's layer tables)."""
    m = np.arange(1 << n, dtype=np.uint32)
    x = m - ((m >> np.uint32(1)) & np.uint32(0x55555555))
    x = (x & np.uint32(0x33333333)) + ((x >> np.uint32(2)) & np.uint32(0x33333333))
    x = (x + (x >> np.uint32(4))) & np.uint32(0x0F0F0F0F)
    pc = ((x * np.uint32(0x01010101)) >> np.uint32(24)).astype(np.uint8)
    del x
    order = np.argsort(pc, kind="stable").astype(np.int32)
    bounds = np.concatenate(([0], np.cumsum(np.bincount(pc, minlength=n + 1))))
    return [order[bounds[k]:bounds[k + 1]] for k in range(n + 1)]



def price_mask_sub(L, masks_u32, scores_f32, offs_u64, K):
    """The mask sweep with bf_update on a K-bit lattice: (V[full] float32, rank_pos over 0..K-1)."""
    import torch
    V = torch.zeros(1 << K, dtype=torch.float32, device="cuda")
    pred = torch.zeros(1 << K, dtype=torch.uint8, device="cuda")
    gm = torch.from_numpy(np.ascontiguousarray(masks_u32).view(np.int32)).cuda()
    gs = torch.from_numpy(np.ascontiguousarray(scores_f32)).cuda()
    go = torch.from_numpy(np.ascontiguousarray(offs_u64).view(np.int64)).cuda()
    lay = _layers(K)
    for c in range(1, K + 1):
        st = torch.from_numpy(np.ascontiguousarray(lay[c])).cuda()
        ns = st.numel()
        L.launch("bf_update", (ns + 255) // 256, 256, [V, pred, gm, gs, go, st, (_I, ns)])
    torch.cuda.synchronize()
    ph = pred.cpu().numpy()
    D = (1 << K) - 1
    vfull = float(V[D].item())
    order = np.zeros(K, dtype=np.int32)
    for i in range(K):
        x = int(ph[D])
        order[x] = i
        D ^= 1 << x
    return vfull, order


def price_mask(menus, scores, offsets, n):
    """solver/flow_cg/solver.py:169-200 with the reference's bf_update: (vmax, rank_pos)."""
    L = _Launcher(_mods()["pricing"])
    v, order = price_mask_sub(L, np.asarray(menus, dtype=np.uint64).astype(np.uint32),
                              np.asarray(scores, dtype=np.float32), np.asarray(offsets, dtype=np.uint64), n)
    return v, order


def price_stream(menus, alts, scores, offsets, n, mode="u24", k_pred=None):
    """StreamPricer.price with the reference's kernels: (vmax, rank_pos, margin, layer_step)."""
    import torch
    L = _Launcher(_mods()["pricing"])
    k_pred = n - 10 if k_pred is None else int(k_pred)
    k_pred = max(1, min(k_pred, n))
    menus = np.ascontiguousarray(menus, dtype=np.uint64)
    alts = np.asarray(alts, dtype=np.int32)
    scores = np.ascontiguousarray(scores, dtype=np.float32)
    counts = [math.comb(n, k) for k in range(n + 1)]
    cap = max(counts)
    nblk = (cap + 1023) // 1024
    vt = torch.float32 if mode == "f32" else torch.int16
    vbuf = [torch.zeros(cap, dtype=vt, device="cuda") for _ in range(2)]
    lbuf = [torch.zeros(cap, dtype=torch.uint8, device="cuda") for _ in range(2)]
    mbuf = [torch.zeros(nblk, dtype=torch.float32, device="cuda") for _ in range(2)]
    ebuf = [torch.zeros(nblk, dtype=torch.float32, device="cuda") for _ in range(2)]
    pred = {k: torch.zeros(counts[k], dtype=torch.uint8, device="cuda") for k in range(k_pred, n + 1)}
    dummy = torch.zeros(1, dtype=torch.uint8, device="cuda")
    binom = torch.from_numpy(_binom(n).view(np.int64)).cuda()
    gm = torch.from_numpy(menus.view(np.int64)).cuda()
    gs = torch.from_numpy(scores).cuda()
    go = torch.from_numpy(np.asarray(offsets, dtype=np.uint64).view(np.int64)).cuda()
    layer_step = np.zeros(n + 1, dtype=np.float32)
    kernel = {"f32": "bf_stream_f32", "u16": "bf_stream_u16", "u24": "bf_stream_u24"}[mode]
    cur, prev = 0, 1
    for k in range(1, n + 1):
        count = counts[k]
        grid = (count + 1023) // 1024
        store = 1 if k >= k_pred else 0
        pk = pred[k] if store else dummy
        if mode == "u24":
            args = [binom, (_I, n), (_I, k), (_ULL, count), vbuf[prev], lbuf[prev], mbuf[prev], ebuf[prev],
                    vbuf[cur], lbuf[cur], mbuf[cur], ebuf[cur], pk, (_I, store), gm, gs, go]
        else:
            args = [binom, (_I, n), (_I, k), (_ULL, count), vbuf[prev], mbuf[prev], ebuf[prev],
                    vbuf[cur], mbuf[cur], ebuf[cur], pk, (_I, store), gm, gs, go]
        L.launch(kernel, grid, 256, args)
        if mode != "f32":
            layer_step[k] = float(ebuf[cur][:grid].max().item())
        cur, prev = prev, cur
    torch.cuda.synchronize()
    if mode == "f32":
        vmax = float(vbuf[prev][0].item())
        margin = 0.0
    else:
        q = int(vbuf[prev][0].item()) & 0xFFFF
        if mode == "u24":
            q = (q << 8) | int(lbuf[prev][0].item())
        vmax = float(mbuf[prev][0].item()) + q * float(ebuf[prev][0].item())
        s = float(np.sum(layer_step[1:n + 1], dtype=np.float32))
        margin = 0.5 * s if mode == "u16" else s
    # backtrace (pricing_stream.py:348-370) and the sub-lattice (:372-405)
    rank_pos = np.zeros(n, dtype=np.int32)
    D = (1 << n) - 1
    pos = 0
    for k in range(n, k_pred, -1):
        x = int(pred[k][_colex_rank(D)].item())
        rank_pos[x] = pos
        pos += 1
        D ^= 1 << x
    elems = [b for b in range(n) if (D >> b) & 1]
    emask = 0
    for e in elems:
        emask |= 1 << e
    inside = (menus & np.uint64(emask)) == menus
    idx = np.nonzero(inside)[0]
    sub_masks = np.zeros(idx.size, dtype=np.uint32)
    for j, e in enumerate(elems):
        sub_masks |= (((menus[idx] >> np.uint64(e)) & np.uint64(1)).astype(np.uint32) << np.uint32(j))
    pos_of = {e: j for j, e in enumerate(elems)}
    sub_alts = np.array([pos_of[int(a)] for a in alts[idx]], dtype=np.int32)
    sub_scores = scores[idx]
    perm = np.argsort(sub_alts, kind="stable")
    sub_masks, sub_alts, sub_scores = sub_masks[perm], sub_alts[perm], sub_scores[perm]
    K = len(elems)
    offs = np.concatenate(([0], np.cumsum(np.bincount(sub_alts, minlength=K)))).astype(np.uint64)
    _, order = price_mask_sub(L, sub_masks, sub_scores, offs, K)
    for j, e in enumerate(elems):
        rank_pos[e] = pos + int(order[j])
    return vmax, rank_pos, margin, layer_step


def sweep_max64(menus, scores, offsets, n):
    """sweep_max64 (solver/flow_cg/pricing_stream.py:236-249) with the reference's bf_stream_max64:
    V[full] in float64 with two live layers; rows x-major, scores float64."""
    import torch
    L = _Launcher(_mods()["max64"])
    counts = [math.comb(n, k) for k in range(n + 1)]
    buf = [torch.zeros(max(counts), dtype=torch.float64, device="cuda") for _ in range(2)]
    gm = torch.from_numpy(np.ascontiguousarray(menus, dtype=np.uint64).view(np.int64)).cuda()
    gs = torch.from_numpy(np.ascontiguousarray(scores, dtype=np.float64)).cuda()
    go = torch.from_numpy(np.asarray(offsets, dtype=np.uint64).view(np.int64)).cuda()
    binom = torch.from_numpy(_binom(n).view(np.int64)).cuda()
    prev, cur = 0, 1
    for k in range(1, n + 1):
        L.launch("bf_stream_max64", (counts[k] + 255) // 256, 256,
                 [binom, (_I, n), (_I, k), (_ULL, counts[k]), buf[prev], buf[cur], gm, gs, go])
        prev, cur = cur, prev
    torch.cuda.synchronize()
    return float(buf[prev][0].item())


# ------------------------------------------------------------------ BM-ADMM timing replay
class BMReplay:
    """solve_kadmm_v2's float64 iteration and float64 check with the reference's kernels: its
    state after any number of iterations (state, iterate), its certified bracket (solve), and the
    timings t_iter (graph replay of one_iter, like use_graph=True) and t_check (push_to_ub64 +
    fw_lb_rows_gpu, eager launches as the reference issues them)."""

    def __init__(self, n, menu, alt, p, beta, alpha=1.95, precond_p=math.sqrt(2.0)):
        import torch
        self.L = _Launcher(_mods()["bm"], _mods()["cert"])
        self.n, self.Nloc = n, 1 << (n - 1)
        self.m2 = n * self.Nloc
        dev = "cuda"
        f64 = torch.float64
        m2 = self.m2
        self.xhat = torch.zeros(m2, dtype=f64, device=dev)
        self.wmask = torch.zeros(m2, dtype=f64, device=dev)
        om = torch.from_numpy(np.asarray(menu, dtype=np.uint32).view(np.int32)).cuda()
        ox = torch.from_numpy(np.asarray(alt, dtype=np.int32)).cuda()
        ph = torch.from_numpy(np.asarray(p, dtype=np.float64)).cuda()
        M = ph.numel()
        g = (M + 255) // 256
        self.L.launch("scatter_obs", g, 256, [ox, om, ph, self.xhat, (_I, M), (_I, self.Nloc)])
        self.L.launch("scatter_obs", g, 256, [ox, om, torch.ones(M, dtype=f64, device=dev), self.wmask, (_I, M),
                                              (_I, self.Nloc)])
        obs = np.asarray(alt, dtype=np.int64) * self.Nloc
        mm = np.asarray(menu, dtype=np.int64) & ~(1 << np.asarray(alt, dtype=np.int64))
        x = np.asarray(alt, dtype=np.int64)
        obs = obs + ((mm & ((1 << x) - 1)) | ((mm >> (x + 1)) << x))
        self.obs = torch.from_numpy(obs).cuda()
        self.p = ph
        pp = float(precond_p)
        G = np.array([[1.0, -1.0], [-1.0, 1.0 + pp * pp]])
        evals, Q = np.linalg.eigh(G)
        lam = np.ones(self.Nloc)
        for bit in range(n - 1):
            b1s = ((np.arange(self.Nloc) >> bit) & 1).astype(np.float64)
            lam *= np.where(b1s > 0, evals[1], evals[0])
        self.inv_gl = torch.from_numpy(1.0 / (1.0 + lam)).cuda()
        self.Q, self.Qt, self.p_ = Q, Q.T, pp
        masks = np.concatenate(_layers(n)[1:])
        self.all_masks = torch.from_numpy(masks).cuda()
        self.n_menus = masks.size
        self.b1 = self.b2 = float(beta)
        self.ib1 = self.ib2 = 1.0 / float(beta)
        self.alpha = float(alpha)
        z = lambda: torch.zeros(m2, dtype=f64, device=dev)
        self.x2, self.s, self.y, self.z = z(), z(), z(), z()
        self.w, self.AT, self.rhs, self.x, self.Ax, self.xk, self.x2n = z(), z(), z(), z(), z(), z(), z()
        self.plan = self._calibrate()
        # cold start: prox of xhat
        self._prox(self.xhat, self.x2)
        torch.cuda.synchronize()

    # Bfly2 (butterfly2.py:124-195): feasible shapes, timed stage costs, shortest-path DP
    @staticmethod
    def _feasible(kind, s, B, nbits, isize=8):
        if B < 1 or s + B > nbits:
            return False
        if kind == "co":
            return s >= 5 and B >= 5 and (1 << B) * 32 * isize <= (1 << 16)
        if kind == "blk":
            return B <= 10 and (1 << B) * isize <= (1 << 16)
        return B <= 11 and (1 << B) * isize <= (1 << 16)

    def _stage(self, kind, s, B, src, out, co):
        n, Nloc, nbits = self.n, self.Nloc, self.n - 1
        a, b, c, d = (float(v) for v in co)
        if kind == "co":
            nlowblk = (1 << s) >> 5
            nhigh = 1 << (nbits - s - B)
            self.L.launch("bfly_co", n * nhigh * nlowblk, 1024,
                          [src, out, (_LL, Nloc), (_I, s), (_I, B), (_LL, nlowblk), (_LL, nhigh), (_D, a), (_D, b),
                           (_D, c), (_D, d)], shmem=(1 << B) * 32 * 8)
        else:
            blk = (1 << B) if kind == "blk" else (1 << (B - 1))
            self.L.launch("bfly_" + kind, n * (Nloc >> B), blk,
                          [src, out, (_LL, Nloc), (_I, s), (_I, B), (_D, a), (_D, b), (_D, c), (_D, d)],
                          shmem=(1 << B) * 8)

    def _calibrate(self, reps=5, warmup=3):
        import torch
        nbits = self.n - 1
        co = (0.5, 0.8660254037844386, -0.8660254037844386, 0.5)
        src, out = self.AT, self.rhs
        src.fill_(1.0)
        tab = {}
        for kind in ("blk", "blk2", "co"):
            for B in range(min(4, nbits), 12):
                for strided in (0, 1):
                    s = 0 if strided == 0 else max(5, (nbits - B) // 2)
                    if not self._feasible(kind, s, B, nbits):
                        continue
                    inp = src if strided == 0 else out
                    for _ in range(warmup):
                        self._stage(kind, s, B, inp, out, co)
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(reps):
                        self._stage(kind, s, B, inp, out, co)
                    e1.record()
                    e1.synchronize()
                    tab[(kind, strided, B)] = e0.elapsed_time(e1) / reps
        INF = float("inf")
        best = [INF] * (nbits + 1)
        back = [None] * (nbits + 1)
        best[0] = 0.0
        for s in range(nbits):
            if best[s] == INF:
                continue
            for kind in ("blk", "blk2", "co"):
                for B in range(1, 12):
                    if not self._feasible(kind, s, B, nbits):
                        continue
                    c = tab.get((kind, 0 if s == 0 else 1, B))
                    if c is None:
                        continue
                    if best[s] + c < best[s + B]:
                        best[s + B] = best[s] + c
                        back[s + B] = (kind, s, B)
        plan, s = [], nbits
        while s > 0:
            plan.append(back[s])
            s -= back[s][2]
        return list(reversed(plan))

    def _bfly(self, src, out, co):
        cur = src
        for kind, s, B in self.plan:
            self._stage(kind, s, B, cur, out, co)
            cur = out

    def _ew(self, name, args):
        self.L.launch(name, (self.m2 + 255) // 256, 256, args + [(_LL, self.m2)])

    def _prox(self, src, out):
        self.L.launch("prox_all", (self.n_menus + 255) // 256, 256,
                      [src, out, self.xhat, self.wmask, self.all_masks, (_LL, self.Nloc), (_D, self.b2),
                       (_I, self.n_menus)])

    def one_iter(self):
        p = self.p_
        self._ew("fuse_w", [self.y, self.s, (_D, self.b1), self.w])
        self._bfly(self.w, self.AT, (1.0, 0.0, -1.0, p))
        self._ew("fuse_rhs", [self.AT, self.z, self.x2, (_D, self.b2), (_D, self.ib1), self.rhs])
        self._bfly(self.rhs, self.x, tuple(self.Qt.reshape(-1)))
        self._ew("diag_mul", [self.inv_gl, (_LL, self.Nloc), self.x])
        self._bfly(self.x, self.x, tuple(self.Q.reshape(-1)))
        self._bfly(self.x, self.Ax, (1.0, -1.0, 0.0, p))
        self._ew("fuse_xk", [self.x, self.x2, self.z, (_D, self.alpha), (_D, self.ib2), self.xk])
        self._prox(self.xk, self.x2n)
        self._ew("fuse_z", [self.x, self.x2, self.x2n, (_D, self.alpha), (_D, self.b2), self.z])
        self._ew("fuse_sy", [self.Ax, (_D, self.alpha), (_D, self.b1), (_D, self.ib1), self.s, self.y])
        self.x2.copy_(self.x2n)

    def state(self):
        """The ADMM state {x2, s, y, z} as float64 host arrays."""
        return {k: getattr(self, k).cpu().numpy().copy() for k in ("x2", "s", "y", "z")}

    def _graph(self):
        """one_iter captured as a CUDA graph, the state left as it was (the reference's use_graph
        path: a warm-up iteration before capture, then the snapshot restored,
        solver/bm_admm/solver.py:273-292)."""
        import torch
        if getattr(self, "_g", None) is None:
            snap = [t.clone() for t in (self.x2, self.s, self.y, self.z)]
            st = torch.cuda.Stream()
            torch.cuda.synchronize()
            with torch.cuda.stream(st):
                self.one_iter()
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=st):
                    self.one_iter()
            torch.cuda.synchronize()
            for t, v in zip((self.x2, self.s, self.y, self.z), snap):
                t.copy_(v)
            torch.cuda.synchronize()
            self._g = g
        return self._g

    def iterate(self, iters, graph=False):
        """`iters` float64 iterations from the current state (eager launches, or graph replays)."""
        import torch
        g = self._graph() if graph else None
        for _ in range(iters):
            if g is not None:
                g.replay()
            else:
                self.one_iter()
        torch.cuda.synchronize()

    def solve(self, abs_tol=1e-5, check=50, lb_every=1, max_iter=10 ** 7, time_limit=3600.0):
        """The reference's certified float64 solve with the runner's hooks: `check` graph-replayed
        iterations, then the float64 push (upper bound, the best one kept) and every `lb_every`
        checks the Frank-Wolfe lower bound (the best one kept), until ub - lb <= abs_tol
        (solver/bm_admm/solver.py:308-352 with ub_arm_immediately, ub_running_min and gap_abs_tol
        as solver/rum_solver.py:879-905 sets them). Returns the bracket, the iterations, the checks
        and the wall time of the loop (device synchronized at each check, as the reference's host
        reads are)."""
        import time
        import torch
        g = self._graph()
        torch.cuda.synchronize()
        ub, lb, it, checks, stop = float("nan"), 0.0, 0, 0, "max_iter"
        t_iter = t_check = 0.0
        t0 = time.perf_counter()
        while it < max_iter:
            a = time.perf_counter()
            for _ in range(check):
                g.replay()
            torch.cuda.synchronize()
            b = time.perf_counter()
            it += check
            u, l = self.check_once(with_lb=(checks % lb_every == 0))
            checks += 1
            t_iter += b - a
            t_check += time.perf_counter() - b
            ub = u if math.isnan(ub) else min(ub, u)
            if l is not None:
                lb = max(lb, l)
            if ub - lb <= abs_tol:
                stop = "gap_abs"
                break
            if time.perf_counter() - t0 > time_limit:
                stop = "time_limit"
                break
        wall = time.perf_counter() - t0
        return {"ub": ub, "lb": lb, "iters": it, "checks": checks, "stop_reason": stop, "wall_s": wall,
                "iter_s": t_iter, "check_s": t_check}

    def time_iterations(self, iters=50, graph=True):
        """milliseconds per iteration (CUDA events), replaying a captured one_iter when graph."""
        import torch
        self.one_iter()
        torch.cuda.synchronize()
        g = None
        if graph:
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                self.one_iter()
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=st):
                    self.one_iter()
            torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            if g is not None:
                g.replay()
            else:
                self.one_iter()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / iters

    # butterfly_fast (solver/common/butterfly.py:381-422): the certificate's transforms
    def _bfly_fast(self, r, co):
        import torch
        n, Nloc, nbits = self.n, self.Nloc, self.n - 1
        R = torch.empty_like(r)
        Bmax, Bco = 9, 8
        src, s, first = r, 0, True
        a, b, c, d = co
        while s < nbits:
            rem = nbits - s
            if first:
                B, use_co, first = min(Bmax, rem), False, False
            else:
                B = rem if rem <= Bco else (rem - 5 if rem - Bco < 5 else Bco)
                use_co = B >= 5 and s >= 5
            if use_co:
                nlowblk = (1 << s) >> 5
                nhigh = 1 << (nbits - s - B)
                self.L.launch("bfly_co", n * nhigh * nlowblk, 1024,
                              [src, R, (_LL, Nloc), (_I, s), (_I, B), (_LL, nlowblk), (_LL, nhigh), (_D, a), (_D, b),
                               (_D, c), (_D, d)], shmem=(1 << B) * 32 * 8)
            else:
                self.L.launch("bfly_blk", n * (Nloc >> B), 1 << B,
                              [src, R, (_LL, Nloc), (_I, s), (_I, B), (_D, a), (_D, b), (_D, c), (_D, d)],
                              shmem=(1 << B) * 8)
            src = R
            s += B
        return R

    def check_once(self, with_lb=True):
        """push_to_ub64 + fw_lb_rows_gpu on the current iterate: (ub, lb); lb is None without
        with_lb."""
        import torch
        n, Nloc, N = self.n, self.Nloc, 1 << self.n
        q = self._bfly_fast(self.x2.clone(), (1.0, -1.0, 0.0, 1.0))
        w = torch.clamp(q, min=0.0) + 1e-12
        outw = torch.empty(N, dtype=torch.float64, device="cuda")
        self.L.launch("outwt64", (N + 255) // 256, 256, [w, outw, (_I, n), (_LL, Nloc)])
        mass = torch.zeros(N, dtype=torch.float64, device="cuda")
        mass[0] = 1.0
        if not hasattr(self, "_layers"):
            order = np.argsort(np.array([bin(v).count("1") for v in range(N)]), kind="stable")
            bounds = np.searchsorted(np.array([bin(v).count("1") for v in order]), np.arange(n + 2))
            self._layers = (torch.from_numpy(order.astype(np.int64)).cuda(), bounds)
        layers, bounds = self._layers
        for cc in range(1, n + 1):
            lo, hi = int(bounds[cc]), int(bounds[cc + 1])
            self.L.launch("massg64", (hi - lo + 255) // 256, 256,
                          [w, outw, mass, layers[lo:hi], (_LL, hi - lo), (_I, n), (_LL, Nloc)])
        rf = torch.empty_like(w)
        self.L.launch("extract64", (self.m2 + 255) // 256, 256, [w, outw, mass, rf, (_I, n), (_LL, Nloc)])
        xub = self._bfly_fast(rf, (1.0, 1.0, 0.0, 1.0))
        ub = float(torch.sqrt(torch.sum((xub[self.obs] - self.p) ** 2)).item())
        if not with_lb:
            return ub, None
        y = self.x2[self.obs]
        r = self.p - y
        f = float((r @ r).item())
        g = torch.zeros(self.m2, dtype=torch.float64, device="cuda")
        g[self.obs] = r
        g = self._bfly_fast(g, (1.0, 0.0, 1.0, 1.0))
        dp = torch.empty(N, dtype=torch.float64, device="cuda")
        dp[0] = 0.0
        for cc in range(1, n + 1):
            lo, hi = int(bounds[cc]), int(bounds[cc + 1])
            self.L.launch("lpath64", (hi - lo + 255) // 256, 256,
                          [g, dp, layers[lo:hi], (_LL, hi - lo), (_I, n), (_LL, Nloc)])
        rc = float(dp[N - 1].item()) - float((r @ y).item())
        return ub, math.sqrt(max(0.0, f - 2.0 * rc))

    def time_check(self, reps=5):
        import torch
        self.check_once()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            self.check_once()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps


# ------------------------------------------------------------------ pricing timing
def time_pricing(menus, offsets, scores, n, reps=10):
    """Milliseconds per sweep of the reference's pricing kernels on one sweep's layers, CUDA events
    around the layer launches only (no host reads between layers, no backtrace): a lower bound of
    its sweep. Stream storage: bf_stream_u24 / bf_stream_u16 (one 256-thread CTA per 1024 ranks,
    x-major rows scanned per rank, solver/flow_cg/pricing_stream.py:61-181); mask storage:
    bf_update (a thread per subset, solver/flow_cg/bf_pricing.py:8-47). Rows x-major."""
    import torch
    L = _Launcher(_mods()["pricing"])
    counts = [math.comb(n, k) for k in range(n + 1)]
    cap, k_pred = max(counts), n - 10
    nblk = (cap + 1023) // 1024
    binom = torch.from_numpy(_binom(n).view(np.int64)).cuda()
    gm = torch.from_numpy(np.ascontiguousarray(menus, dtype=np.uint64).view(np.int64)).cuda()
    gs = torch.from_numpy(np.ascontiguousarray(scores, dtype=np.float32)).cuda()
    go = torch.from_numpy(np.asarray(offsets, dtype=np.uint64).view(np.int64)).cuda()
    out = {}

    def timed(sweep):
        for _ in range(2):
            sweep()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            sweep()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    for mode in ("u24", "u16"):
        vbuf = [torch.zeros(cap, dtype=torch.int16, device="cuda") for _ in range(2)]
        lbuf = [torch.zeros(cap, dtype=torch.uint8, device="cuda") for _ in range(2)]
        mbuf = [torch.zeros(nblk, dtype=torch.float32, device="cuda") for _ in range(2)]
        ebuf = [torch.zeros(nblk, dtype=torch.float32, device="cuda") for _ in range(2)]
        pred = {k: torch.zeros(counts[k], dtype=torch.uint8, device="cuda") for k in range(max(k_pred, 1), n + 1)}
        dummy = torch.zeros(1, dtype=torch.uint8, device="cuda")

        def sweep(mode=mode, vbuf=vbuf, lbuf=lbuf, mbuf=mbuf, ebuf=ebuf, pred=pred, dummy=dummy):
            cur, prev = 0, 1
            for k in range(1, n + 1):
                store = 1 if k >= k_pred else 0
                pk = pred[k] if store else dummy
                if mode == "u24":
                    args = [binom, (_I, n), (_I, k), (_ULL, counts[k]), vbuf[prev], lbuf[prev], mbuf[prev], ebuf[prev],
                            vbuf[cur], lbuf[cur], mbuf[cur], ebuf[cur], pk, (_I, store), gm, gs, go]
                else:
                    args = [binom, (_I, n), (_I, k), (_ULL, counts[k]), vbuf[prev], mbuf[prev], ebuf[prev],
                            vbuf[cur], mbuf[cur], ebuf[cur], pk, (_I, store), gm, gs, go]
                L.launch("bf_stream_" + mode, (counts[k] + 1023) // 1024, 256, args)
                cur, prev = prev, cur

        out[mode + "_layers_ms"] = timed(sweep)
    V = torch.zeros(1 << n, dtype=torch.float32, device="cuda")
    P = torch.zeros(1 << n, dtype=torch.uint8, device="cuda")
    gm32 = torch.from_numpy(np.asarray(menus, dtype=np.uint64).astype(np.uint32).view(np.int32)).cuda()
    states = [torch.from_numpy(np.ascontiguousarray(t)).cuda() for t in _layers(n)]

    def mask_sweep():
        for c in range(1, n + 1):
            ns = states[c].numel()
            L.launch("bf_update", (ns + 255) // 256, 256, [V, P, gm32, gs, go, states[c], (_I, ns)])

    out["mask_layers_ms"] = timed(mask_sweep)
    return out
