"""The binding a maintainer of the reference would add to its solver package, written against
module objects so that a test can install it: it routes the reference's RUM runner and planner
tables for bm_admm and flow_cg (solver/rum_solver.py:858,1186-1187) to rumb's."""


def install(ref, rumb_solver):
    """Route bm_admm and flow_cg of the reference's solver.rum_solver (module `ref`) to rumb."""

    def run(name):
        impl = rumb_solver._RUN[name]

        def runner(task):
            try:
                return impl(task)
            except rumb_solver._TimeUp:
                raise ref._TimeUp
        return runner

    ref._RUN["bm_admm"] = run("bm_admm")
    ref._RUN["flow_cg"] = run("flow_cg")
    # the planners must produce rumb's private keys too (_gpu_bytes, _engine, use_graph)
    ref._PLAN["bm_admm"] = lambda n, mp, w, prof, a: rumb_solver._plan_bm_admm(n, mp, a)
    ref._PLAN["flow_cg"] = lambda n, mp, w, prof, a: rumb_solver._plan_flow_cg(n, mp, a)
