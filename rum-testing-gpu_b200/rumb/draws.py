"""Bootstrap draws of p_hat, built from the choices behind it (the reference's
solver/inference/draws.py interface: the same tables, weight schemes, seeds and draws).

Input tables hold one row per choice, as a DataFrame or a dict of equal-length columns:

    panel     respondent, menu, chosen   respondents answered several menus and are resampled as a
                                         whole (Draws)
    replies   menu, chosen               independent replies, resampled menu by menu (MenuDraws)

A menu is a bitmask of offered alternatives; `chosen` is one of its members. rum's rows are the
table's shares, p_hat(D, a) = #(menu D, chose a) / #(menu D) (cells_from_panel builds them).

How a panel draw is built here. The panel is reduced once to two count lists in compressed form,
respondents ascending within each list:

    menu lists   for each of rum's menus D: the respondents offered D and how many times
    row lists    for each of rum's rows (D, a): the respondents who chose a from D and how many times

A draw gives respondent i a weight w_i, and its row (D, a) is the share
    sum over a's list of w_i count_i  /  sum over D's list of w_i count_i,
p_hat where the denominator is 0 (a menu the draw left unseen). These are the lists the GPU
kernel walks (rumb_draws_*, csrc/draws.cu); the host walks them with segment sums in list order.
With integer weights (multinomial, multinomial_reject, poisson) every sum is an exact integer, so
host, GPU and the reference agree bit for bit whatever the order. With real weights (exponential,
mammen) the float64 sums depend on their order: here they run in list order, the reference's in
its BLAS product's, and the rows agree to rounding (1e-15 relative).

Weights, drawn in the reference's order so that a seed gives the reference's draws:
    multinomial_reject   respondent counts of R picks with replacement (rng.multinomial); weight
                         rows that leave one of rum's menus unseen are drawn again, up to
                         REDRAW_ROUNDS rounds (the default scheme)
    multinomial          the same without the redraw: an unseen menu keeps p_hat
    exponential          Exp(1) multipliers
    poisson              Poisson(1) multipliers
    mammen               the wild bootstrap's two-point weights; the row is
                         clip(p_hat + sum_i w_i (chose_i - offered_i p_hat) / N_D, 0, 1)
Replies draws: menu D's reply counts ~ Multinomial(N_D, its shares), menus in increasing mask
order, block k of draws from numpy.random.default_rng([seed, k]); the block size (BLOCK_BYTES of
float64 draws) is therefore part of the stream.
"""
import hashlib

import numpy as np

WEIGHTS = ("multinomial_reject", "multinomial", "exponential", "poisson", "mammen")
INTEGER_WEIGHTS = ("multinomial_reject", "multinomial", "poisson")
COLUMNS = ("respondent", "menu", "chosen")
P_HAT_TOL = 1e-9                # rum's p_hat against the table's counts
BLOCK_BYTES = 1 << 27           # float64 draws built per block (fixes the replies draws' streams)
REDRAW_ROUNDS = 10000           # multinomial_reject gives up after this many rounds
_MAX_MENU = 1 << 62             # menus are sets of at most 62 alternatives
_WORK_BYTES = 1 << 27           # scratch of one segment-sum pass over weight rows


# ------------------------------------------------------------------ reading a table
def _as_int(values, table, column):
    """A column of whole numbers as int64; floats must be finite and integral."""
    kind = values.dtype.kind
    if kind in "iu":
        return values.astype(np.int64)
    if kind != "f":
        raise ValueError("the %s's %s column must hold integers" % (table, column))
    nan = ~np.isfinite(values)
    if nan.any():
        raise ValueError("%s row %d: missing %s" % (table, int(np.argmax(nan)), column))
    off = values != np.floor(values)
    if off.any():
        j = int(np.argmax(off))
        raise ValueError("%s row %d: %s %r is not an integer" % (table, j, column, values[j]))
    return values.astype(np.int64)


def _first(mask):
    return int(np.argmax(mask))


class _Choices:
    """The checked columns of a choice table: menu and chosen (int64) and, for a panel, the
    respondent codes 0..R-1 in sorted id order."""

    def __init__(self, table, name, num_alternatives=None, panel=False):
        cols = COLUMNS if panel else COLUMNS[1:]
        absent = [c for c in cols if c not in table]
        if absent:
            raise ValueError("the %s needs the columns %s and %s; missing: %s"
                             % (name, ", ".join(cols[:-1]), cols[-1], ", ".join(absent)))
        raw = {c: np.asarray(table[c]) for c in cols}
        sizes = {a.size for a in raw.values()}
        if len(sizes) != 1 or any(a.ndim != 1 for a in raw.values()):
            raise ValueError("the %s's columns must be 1-D and of equal length" % name)
        if sizes.pop() == 0:
            raise ValueError("the %s has no rows" % name)
        menu = _as_int(raw["menu"], name, "menu")
        chosen = _as_int(raw["chosen"], name, "chosen")
        bad = (menu <= 0) | (menu >= _MAX_MENU)
        if bad.any():
            j = _first(bad)
            raise ValueError("%s row %d: menu mask %d is not a nonempty set of at most 62 alternatives"
                             % (name, j, menu[j]))
        bad = (chosen < 0) | (chosen > 61)
        if bad.any():
            j = _first(bad)
            raise ValueError("%s row %d: chosen %d is not an alternative (0 to 61)" % (name, j, chosen[j]))
        bad = ((menu >> chosen) & 1) == 0
        if bad.any():
            j = _first(bad)
            raise ValueError("%s row %d: chosen %d is not in its menu (mask %d)" % (name, j, chosen[j], menu[j]))
        if num_alternatives is not None:
            bad = menu >= 1 << int(num_alternatives)
            if bad.any():
                j = _first(bad)
                raise ValueError("%s row %d: menu mask %d has alternatives beyond num_alternatives = %d"
                                 % (name, j, menu[j], num_alternatives))
        self.menu, self.chosen = menu, chosen
        self.codes, self.R = None, 0
        if panel:
            self.codes, self.R = self._respondents(raw["respondent"])

    @staticmethod
    def _respondents(ids):
        if ids.dtype.kind == "f":
            nan = ~np.isfinite(ids)
            if nan.any():
                raise ValueError("panel row %d: missing respondent" % _first(nan))
        elif ids.dtype.kind == "O":
            for j, v in enumerate(ids):
                if v is None or v != v:
                    raise ValueError("panel row %d: missing respondent" % j)
        try:
            uniq, codes = np.unique(ids, return_inverse=True)
        except TypeError:
            raise ValueError("respondent ids must be all numbers or all strings") from None
        return codes.astype(np.int64).ravel(), int(uniq.size)


def read_panel(panel, num_alternatives=None):
    """(respondent codes 0..R-1 in sorted id order, R, menu, chosen) of a panel, checked."""
    t = _Choices(panel, "panel", num_alternatives, panel=True)
    return t.codes, t.R, t.menu, t.chosen


def cells_from_panel(table, num_alternatives=None, alternatives=None):
    """rum's rows (menu, alternative, p_hat) counted from a panel or a replies table (a table with a
    respondent column is read as a panel): every menu of the table, increasing, with each member
    alternative (or each of `alternatives` it offers), increasing; p_hat is the share of the
    menu's rows that chose the alternative, 0 when none did."""
    if COLUMNS[0] in table:
        t = _Choices(table, "panel", num_alternatives, panel=True)
    else:
        t = _Choices(table, "replies table", num_alternatives)
    n = (int(num_alternatives) if num_alternatives is not None
         else max(int(t.menu.max()).bit_length(), int(t.chosen.max()) + 1))
    if alternatives is None:
        keep = np.arange(n)
    else:
        keep = np.unique(np.asarray(alternatives, dtype=np.int64))
    if keep.size == 0 or keep[0] < 0 or keep[-1] >= n:
        raise ValueError("alternatives must be a nonempty list of alternatives from 0 to %d" % (n - 1))
    menus, inv, offered = np.unique(t.menu, return_inverse=True, return_counts=True)
    # replies per (menu, chosen): keys menu index * 64 + chosen, counted once
    pairs, chose = np.unique(inv.ravel().astype(np.int64) * 64 + t.chosen, return_counts=True)
    wanted = np.zeros(64, dtype=bool)
    wanted[keep] = True
    offers = ((menus[:, None] >> np.arange(64)[None, :]) & 1).astype(bool) & wanted[None, :]
    mi, ai = np.nonzero(offers)                  # menu-major, alternatives increasing
    if mi.size == 0:
        raise ValueError("no menu of the table offers any of the alternatives %s" % keep.tolist())
    key = mi.astype(np.int64) * 64 + ai
    at = np.minimum(np.searchsorted(pairs, key), pairs.size - 1)
    num = np.where(pairs[at] == key, chose[at], 0)
    return menus[mi], ai.astype(np.int64), num / offered[mi]


# ------------------------------------------------------------------ count lists
def _rum_rows(menu, alternative):
    """rum's menus (sorted), each row's menu index, and a lookup (menu index, alternative) -> row."""
    menu, alternative = np.asarray(menu, dtype=np.int64), np.asarray(alternative, dtype=np.int64)
    menus, row_menu = np.unique(menu, return_inverse=True)
    keys = row_menu.astype(np.int64) * 64 + alternative
    order = np.argsort(keys, kind="stable")
    return menus, row_menu.astype(np.int64), keys[order], order


def _menu_index(menus, table_menu):
    """The index of each table menu among rum's menus, and which table rows have one."""
    j = np.searchsorted(menus, table_menu)
    jc = np.minimum(j, menus.size - 1)
    return jc, menus[jc] == table_menu


def _lists(seg, who, nseg, nwho):
    """CSR lists from (segment, member) pairs with repeats: ptr [nseg + 1], members ascending
    within a segment (int32) and how often each pair occurred (float64)."""
    key, cnt = np.unique(seg.astype(np.int64) * nwho + who.astype(np.int64), return_counts=True)
    s = key // nwho
    ptr = np.zeros(nseg + 1, dtype=np.int64)
    np.add.at(ptr, s + 1, 1)
    return np.cumsum(ptr), (key % nwho).astype(np.int32), cnt.astype(np.float64)


class CountLists:
    """A panel reduced to what its draws are made from (the inputs of rumb_draws_create):
    menu_ptr / menu_resp / menu_cnt   per rum menu, the respondents offered it and how often
    row_ptr / row_resp / row_cnt      per rum row, the respondents who chose it and how often
    row_menu                          each rum row's menu index"""

    def __init__(self, menu_ptr, menu_resp, menu_cnt, row_ptr, row_resp, row_cnt, row_menu, R):
        self.menu_ptr, self.menu_resp, self.menu_cnt = menu_ptr, menu_resp, menu_cnt
        self.row_ptr, self.row_resp, self.row_cnt = row_ptr, row_resp, row_cnt
        self.row_menu = row_menu
        self.R = int(R)
        self.n_menus = menu_ptr.size - 1
        self.M = row_ptr.size - 1

    def menu_sums(self, W):
        """(rows of W) x (rum menus): sum over each menu's list of w_i count_i."""
        return _segment_sums(W, self.menu_ptr, self.menu_resp, self.menu_cnt)

    def row_sums(self, W):
        """(rows of W) x (rum rows): sum over each row's list of w_i count_i."""
        return _segment_sums(W, self.row_ptr, self.row_resp, self.row_cnt)


def _segment_sums(W, ptr, who, cnt):
    """out[b, j] = sum over k in [ptr[j], ptr[j+1]) of W[b, who[k]] cnt[k], added in list order;
    0 for an empty list. W rows are processed in chunks of at most _WORK_BYTES of products."""
    W = np.atleast_2d(W)
    nseg = ptr.size - 1
    out = np.zeros((W.shape[0], nseg))
    full = np.flatnonzero(ptr[1:] > ptr[:-1])
    if full.size == 0:
        return out
    step = max(1, _WORK_BYTES // (8 * max(1, who.size)))
    for lo in range(0, W.shape[0], step):
        prod = W[lo:lo + step][:, who] * cnt
        out[lo:lo + step, full] = np.add.reduceat(prod, ptr[full], axis=1)
    return out


# ------------------------------------------------------------------ draws in blocks
class _BlockedDraws:
    """B draws of M rows made block by block (at most BLOCK_BYTES of float64 per block; the last
    block made is kept). A subclass gives make_block(k) -> (rows, draws that left a menu unseen)."""

    def _setup_blocks(self, width):
        self.rows_per_block = max(1, min(self.B, BLOCK_BYTES // (8 * width)))
        self.n_blocks = -(-self.B // self.rows_per_block)
        self._held = None
        self.n_empty = None
        self.fingerprint = None

    def block(self, k):
        if self._held is None or self._held[0] != k:
            rows, empty = self.make_block(k)
            self._held = (k, rows, empty)
        return self._held[1]

    def blocks(self):
        """(first, last + 1, rows) for every block. A full pass sets `fingerprint` (the first 16
        hex digits of the sha256 of all B x M float64 draws in order) and `n_empty`."""
        digest, empty = hashlib.sha256(), 0
        for k in range(self.n_blocks):
            rows = self.block(k)
            empty += self._held[2]
            digest.update(np.ascontiguousarray(rows).tobytes())
            lo = k * self.rows_per_block
            yield lo, lo + rows.shape[0], rows
        self.fingerprint, self.n_empty = digest.hexdigest()[:16], empty

    def rows(self, idx):
        """The draws idx as a (len(idx), M) array."""
        idx = np.asarray(idx, dtype=np.int64)
        out = np.empty((idx.size, self.M))
        blk = idx // self.rows_per_block
        for k in np.unique(blk):
            at = np.flatnonzero(blk == k)
            out[at] = self.block(int(k))[idx[at] - k * self.rows_per_block]
        return out


class Draws(_BlockedDraws):
    """B draws of p_hat for rum's rows (menu, alternative, p_hat), made from a respondent panel."""

    input = "panel"

    def __init__(self, panel, menu, alternative, p_hat, B=10000, weights="multinomial_reject", seed=0):
        if weights not in WEIGHTS:
            raise ValueError("unknown weights %r; choose from %s" % (weights, WEIGHTS))
        if int(B) != B or B < 1:
            raise ValueError("B must be a positive integer")
        t = _Choices(panel, "panel", panel=True)
        codes, R = t.codes, t.R
        self.input_fingerprint = hashlib.sha256(codes.tobytes() + t.menu.tobytes()
                                                + t.chosen.tobytes()).hexdigest()[:16]
        menu, alternative = np.asarray(menu, dtype=np.int64), np.asarray(alternative, dtype=np.int64)
        self.p_hat = p_hat = np.asarray(p_hat, dtype=np.float64)
        M = menu.size
        menus, row_menu, sorted_keys, sorted_rows = _rum_rows(menu, alternative)
        j, on_rum = _menu_index(menus, t.menu)
        # the panel rows whose (menu, chosen) is one of rum's rows, and which row
        want = j * 64 + t.chosen
        at = np.minimum(np.searchsorted(sorted_keys, want), M - 1)
        is_row = on_rum & (sorted_keys[at] == want)
        mptr, mresp, mcnt = _lists(j[on_rum], codes[on_rum], menus.size, R)
        rptr, rresp, rcnt = _lists(sorted_rows[at[is_row]], codes[is_row], M, R)
        self.lists = CountLists(mptr, mresp, mcnt, rptr, rresp, rcnt, row_menu.astype(np.int32), R)
        N = self.lists.menu_sums(np.ones((1, R)))[0][row_menu]        # panel rows per row's menu
        if (N == 0).any():
            k = _first(N == 0)
            raise ValueError("rum row %d (menu %d): the menu is not in the panel" % (k, menu[k]))
        c = self.lists.row_sums(np.ones((1, R)))[0]
        gap = np.abs(c / N - p_hat)
        if gap.max() > P_HAT_TOL:
            k = int(np.argmax(gap))
            raise ValueError("rum row %d (menu %d, alternative %d): p_hat = %.6g, but the panel gives %.6g (%d of %d "
                             "rows); build rum with cells_from_panel(panel, ...)"
                             % (k, menu[k], alternative[k], p_hat[k], c[k] / N[k], c[k], N[k]))
        self.N = N
        self.B, self.R, self.M, self.weights, self.seed = int(B), R, M, weights, seed
        self.rows_unused = int((~on_rum).sum())          # panel rows on menus that have no rum row
        self.n_redraws = self.n_reject_rounds = 0
        self._setup_blocks(M)
        self.W = self._draw_weights(np.random.default_rng(seed))

    @property
    def row_menu(self):
        return self.lists.row_menu

    @property
    def integer_weights(self):
        return self.weights in INTEGER_WEIGHTS

    @property
    def default_n(self):
        return self.R

    def check_n(self, n):
        if self.R != n:
            raise ValueError("n = %d, but the panel has %d respondents" % (n, self.R))

    def summary(self):
        return dict(respondents=self.R, rows_unused=self.rows_unused, redraws=self.n_redraws,
                    emptied_menu_draws=self.n_empty)

    def _multinomial(self, rng, count):
        R = self.R
        return rng.multinomial(R, np.full(R, 1.0 / R), size=count).astype(np.float64)

    def _draw_weights(self, rng):
        """The B x R weight matrix, drawn as the reference draws it for this scheme and seed."""
        shape = (self.B, self.R)
        if self.weights == "exponential":
            return rng.exponential(1.0, size=shape)
        if self.weights == "poisson":
            return rng.poisson(1.0, size=shape).astype(np.float64)
        if self.weights == "mammen":
            r5 = np.sqrt(5.0)
            low = rng.random(shape) < (r5 + 1.0) / (2.0 * r5)
            return np.where(low, -(r5 - 1.0) / 2.0, (r5 + 1.0) / 2.0)
        W = self._multinomial(rng, self.B)
        if self.weights == "multinomial_reject":
            # a row that saw every menu keeps its weights, so each round tests only the rows just
            # drawn again (the same rows, in the same order, as testing all of W would find)
            todo = np.flatnonzero(self.leaves_menu_unseen(W))
            for _ in range(REDRAW_ROUNDS):
                if todo.size == 0:
                    break
                self.n_redraws += int(todo.size)
                self.n_reject_rounds += 1
                W[todo] = self._multinomial(rng, int(todo.size))
                todo = todo[self.leaves_menu_unseen(W[todo])]
        return W

    def leaves_menu_unseen(self, W):
        """For each weight row: does some rum menu get total weight 0?"""
        return np.any(self.lists.menu_sums(W) <= 0, axis=1)

    def make_block(self, k):
        Wb = self.W[k * self.rows_per_block:(k + 1) * self.rows_per_block]
        L = self.lists
        seen = L.menu_sums(Wb)[:, L.row_menu]
        chose = L.row_sums(Wb)
        if self.weights == "mammen":
            return np.clip(self.p_hat + (chose - seen * self.p_hat) / np.maximum(self.N, 1.0), 0.0, 1.0), 0
        empty = seen <= 0
        rows = np.where(empty, self.p_hat, chose / np.where(empty, 1.0, seen))
        return rows, int(empty.any(axis=1).sum())


class MenuDraws(_BlockedDraws):
    """B draws of p_hat for rum's rows made from a replies table: each menu's replies resampled on
    their own, menu D's counts ~ Multinomial(N_D, the shares of D's replies). Block k comes from
    numpy.random.default_rng([seed, k]), menus in increasing mask order, so a block rebuilds alone."""

    input, weights = "replies", "multinomial"
    integer_weights = False

    def __init__(self, replies, menu, alternative, p_hat, B=10000, seed=0):
        if int(B) != B or B < 1:
            raise ValueError("B must be a positive integer")
        t = _Choices(replies, "replies table")
        self.input_fingerprint = hashlib.sha256(t.menu.tobytes() + t.chosen.tobytes()).hexdigest()[:16]
        menu, alternative = np.asarray(menu, dtype=np.int64), np.asarray(alternative, dtype=np.int64)
        self.p_hat = p_hat = np.asarray(p_hat, dtype=np.float64)
        M = menu.size
        menus, row_menu, _, _ = _rum_rows(menu, alternative)
        j, on_rum = _menu_index(menus, t.menu)
        N = np.bincount(j[on_rum], minlength=menus.size)
        if (N[row_menu] == 0).any():
            k = _first(N[row_menu] == 0)
            raise ValueError("rum row %d (menu %d): the menu is not in the replies" % (k, menu[k]))
        # the (menu, alternative) pairs chosen at least once, menu-major, and their counts: the
        # categories of each menu's multinomial, in the order the draws consume them
        cat, cnt = np.unique(j[on_rum] * 64 + t.chosen[on_rum], return_counts=True)
        cat_menu = cat // 64
        key = row_menu * 64 + alternative
        at = np.minimum(np.searchsorted(cat, key), cat.size - 1)
        found = cat[at] == key
        c = np.where(found, cnt[at], 0)
        den = N[row_menu]
        gap = np.abs(c / den - p_hat)
        if gap.max() > P_HAT_TOL:
            k = int(np.argmax(gap))
            raise ValueError("rum row %d (menu %d, alternative %d): p_hat = %.6g, but the replies give %.6g (%d of "
                             "%d rows); build rum with cells_from_panel(replies, ...)"
                             % (k, menu[k], alternative[k], p_hat[k], c[k] / den[k], c[k], den[k]))
        self.N = N
        self._cat_share = cnt / N[cat_menu]
        self._cat_start = np.searchsorted(cat_menu, np.arange(N.size + 1))
        self._row_cat = np.where(found, at, -1)
        self._den = den.astype(np.float64)
        self.B, self.M, self.seed = int(B), M, seed
        self.rows_unused = int((~on_rum).sum())
        self.n_redraws = 0
        self._setup_blocks(max(M, cat.size))

    @property
    def default_n(self):
        return int(self.N.max())

    def check_n(self, n):
        if not self.N.min() <= n <= self.N.max():
            raise ValueError("n = %d, but the menus have %d to %d replies; with replies, n is the number of replies "
                             "per menu" % (n, self.N.min(), self.N.max()))

    def summary(self):
        return dict(replies=int(self.N.sum()), replies_per_menu=[int(self.N.min()), int(self.N.max())],
                    rows_unused=self.rows_unused)

    def make_block(self, k):
        first = k * self.rows_per_block
        count = min(self.rows_per_block, self.B - first)
        rng = np.random.default_rng([self.seed, k])
        tally = np.empty((count, self._cat_share.size))
        for d in range(self.N.size):
            a, b = self._cat_start[d], self._cat_start[d + 1]
            tally[:, a:b] = rng.multinomial(self.N[d], self._cat_share[a:b], size=count)
        got = tally[:, np.maximum(self._row_cat, 0)]
        return np.where(self._row_cat >= 0, got, 0.0) / self._den, 0
