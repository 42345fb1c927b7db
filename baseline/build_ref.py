"""Extracts the reference's own CUDA kernel sources into baseline/_ref/ (the comparison side of
the parity tests and of bench.py's reference-kernel timing; never the product).

    python baseline/build_ref.py [reference root]     # default: $RUM_REFERENCE_ROOT, else DEFAULT_ROOT

The reference (mingxiz/rum-testing-gpu) keeps its GPU kernels as CUDA C source strings inside
Python modules and JIT-compiles them with NVRTC through CuPy. CuPy is not installed here, so this
script reads those string constants with `ast` (the source text only, never a binary) and writes
them as .cu files under baseline/_ref/, which is git-ignored and travels to the GPU box. There
baseline/ref_replay.py compiles them with NVRTC (the compiler CuPy uses, default options) and
replays the reference's host sequence, for two purposes:
  * pinning the pricer's bit-exactness against the reference's compiled kernels, and
  * timing the reference's float64 BM-ADMM iteration on the same GPU.

Files written:
  ref_bm_f64.cu     scatter_obs, the fused elementwise kernels of solve_kadmm_v2 (as _mk_ew
                    wraps them), prox_all, bfly_blk, bfly_co, bfly_blk2 with `typedef double real`
  ref_cert64.cu     outwt64, massg64, extract64, lpath64
  ref_max64.cu      bf_stream_max64 (solver/flow_cg/pricing_stream.py _SRC64: the float64 max sweep)
  ref_pricing.cu    bf_stream_f32 / bf_stream_u16 / bf_stream_u24 (BLOCK etc. substituted as the
                    module does) and bf_update
"""
import ast
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# where this recipe finds the reference's source tree unless RUM_REFERENCE_ROOT says otherwise
DEFAULT_ROOT = "/root/reference"


def reference_root():
    """The reference's source tree, or None when it is not present on this machine."""
    root = os.environ.get("RUM_REFERENCE_ROOT", DEFAULT_ROOT)
    return root if os.path.isdir(os.path.join(root, "solver")) else None


def _module(root, rel):
    path = os.path.join(root, rel)
    return ast.parse(open(path).read(), filename=path)


def _assigned(tree, name):
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id == name for t in node.targets):
            return node.value
    raise KeyError(name)


def _string(node):
    return ast.literal_eval(node)


def _call_arg(tree, name):
    """first positional argument (a string) of the call assigned to name"""
    v = _assigned(tree, name)
    assert isinstance(v, ast.Call), name
    return _string(v.args[0])


def extract(root):
    os.makedirs(OUT, exist_ok=True)
    solver = _module(root, "solver/bm_admm/solver.py")
    kernels = _module(root, "solver/bm_admm/kernels.py")
    bfly = _module(root, "solver/common/butterfly.py")
    bfly2 = _module(root, "solver/bm_admm/butterfly2.py")
    arc = _module(root, "solver/common/arcflow_kernels.py")
    stream = _module(root, "solver/flow_cg/pricing_stream.py")
    bfp = _module(root, "solver/flow_cg/bf_pricing.py")

    ew = _string(_assigned(solver, "_EW_SRC"))
    parts = ["typedef double real;"]
    # the wrapper _mk_ew puts around each (args, body) pair (solver/bm_admm/solver.py:57-63)
    for name, (args, body) in ew.items():
        parts.append('extern "C" __global__ void %s(%s, long long m2){\n'
                     "  long long i = blockIdx.x*(long long)blockDim.x + threadIdx.x;\n"
                     "  if (i >= m2) return;\n  %s\n}" % (name, args, body))
    parts.append(_string(_assigned(solver, "_PROX1_SRC")))
    parts.append(_call_arg(kernels, "_SCATTER_DT"))
    parts.append(_string(_assigned(bfly, "_BLK_SRC")))
    parts.append(_string(_assigned(bfly, "_CO_SRC")))
    parts.append(_string(_assigned(bfly2, "_BLK2_SRC")))
    open(os.path.join(OUT, "ref_bm_f64.cu"), "w").write("\n\n".join(parts) + "\n")

    cert = [_call_arg(arc, nm) for nm in ("_OUTWT64", "_MASSG64", "_EXTRACT64", "_LPATH64")]
    open(os.path.join(OUT, "ref_cert64.cu"), "w").write("\n\n".join(cert) + "\n")

    consts = {}
    for nm in ("BLOCK", "THREADS", "MAXN"):
        consts[nm] = ast.literal_eval(_assigned(stream, nm))
    consts["VPT"] = consts["BLOCK"] // consts["THREADS"]
    consts["LOG2BLOCK"] = int(math.log2(consts["BLOCK"]))
    src = _assigned(stream, "_SRC")
    assert isinstance(src, ast.BinOp) and isinstance(src.op, ast.Mod)
    pricing = _string(src.left) % consts
    pricing += "\n\n" + _string(_assigned(bfp, "_BF_UPDATE_SRC"))
    open(os.path.join(OUT, "ref_pricing.cu"), "w").write(pricing + "\n")
    open(os.path.join(OUT, "ref_max64.cu"), "w").write(_string(_assigned(stream, "_SRC64")) + "\n")
    open(os.path.join(OUT, "consts.txt"), "w").write(repr(consts) + "\n")
    return OUT


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    if root is None:
        raise SystemExit("the reference's source tree was not found (set RUM_REFERENCE_ROOT)")
    print(extract(root))
