"""Default parameters of the two methods and the one rule that varies with the instance: the
BM-ADMM penalty (the reference's solver/params.py:1-80, same constants and rule).

    alpha = 1.95        over-relaxation
    p     = sqrt(2)     per-bit diagonal preconditioner of the inequality block
    beta  = f(mp)       penalty, 10^-1.48 * mp^0.508 clipped to [0.3, 100]
"""
import math

BM_ALPHA = 1.95
BM_PRECOND_P = math.sqrt(2.0)
BM_CHECK_EVERY = 50
BM_BETA_COEF, BM_BETA_EXP = 10 ** -1.48, 0.508
BM_BETA_MIN, BM_BETA_MAX = 0.3, 100.0
PROBE_ITERS = 300

CB_DEFAULTS = dict(rc_tol=0.0, max_iters=4000)


def bm_beta_default(mp):
    """Penalty from the number of observed (menu, alternative) cells."""
    return float(min(BM_BETA_MAX, max(BM_BETA_MIN, BM_BETA_COEF * float(mp) ** BM_BETA_EXP)))
