"""Default settings of the RUM class (rumb.rum_solver), with the reference's names and values
(solver/defaults.py:19-108). method_args may only use the names listed for the method; anything
else is an error.

Storage: bm_admm takes dtype "float64" (auto), "float32" or "mixed" (float32 iterations until the
pushed upper bound stalls, then float64 to the end; the bounds are float64 in every mode);
flow_cg takes "float32", "uint24" or "uint16" pricing values.
"""
import math

ABS_TOL = 1e-5
REL_TOL = 1e-4
MAX_TIME = 3600.0
SEED = 0

METHOD_ARGS = {
    "bm_admm": dict(
        beta=None,              # penalty; None = params.bm_beta_default(mp)
        alpha=1.95,             # over-relaxation
        precond_p=math.sqrt(2.0),
        check=50,               # iterations between upper bounds (feasibility push)
        lb_every=1,             # upper-bound checks between lower bounds
        dtype="auto",           # "float64" (auto), "float32" or "mixed"
        use_graph="auto",       # replay each check interval as a CUDA graph; auto = on
        max_iter=10 ** 7,
    ),
    "flow_cg": dict(
        dtype="auto",           # pricing values "float32", "uint24" or "uint16"; auto = the first that fits
        pricing="auto",         # "mask" (one value per subset, n <= 34) or "stream" (two live layers)
        layers="auto",          # accepted for compatibility; the lattice layers are implicit here
        max_iters=4000,         # columns
    ),
}

AUTO = dict(
    bm_admm_min_density={11: 0.02, 14: 0.01, 18: 0.005},
    gpu_memory_fraction=0.9,
)

BOOTSTRAP = dict(
    B=10000,
    weights="multinomial_reject",
    seed=0,
    abs_tol=5e-4,
    rel_tol=0.0,
    refine=2,
    max_time=3600.0,
    draw_time=120.0,
    checkpoint_every=60.0,
)
