"""The bootstrap's draws sharded over two gloo ranks on the CPU: the band comes from rank 0, each
rank solves its share of the open draws, and the gathered record and p-value equal a single
process's. The solver is a stand-in (no GPU); what is tested is the host-side sharding."""
import os
import socket
import types

import numpy as np
import pytest
import torch.multiprocessing as mp

from rumb import bootstrap as BS

B = 41


def _fake(rank_u0=None):
    b = object.__new__(BS.Bootstrap)
    b.B, b.s, b.r_n, b.n_screened = B, 2.0, 4.0, 0
    b.L, b.U = np.zeros(B), np.full(B, np.inf)
    b.solved = np.zeros(B, dtype=bool)
    b.L0 = b.U0 = None
    b.screened = False
    b.session = types.SimpleNamespace(fit=np.zeros(1))
    b.time = dict(certificate=0.0, screen=0.0, solve=0.0)
    b.results, b.checkpoint = {"p_value": {}}, None
    b.seen = []
    b.flag = np.full(B, BS.NEVER, dtype=np.int8)
    b.tol_stop, b.tol_full = np.full(B, np.inf), np.full(B, np.inf)
    b.saves = []

    def certify():
        b.L0, b.U0 = 1.0, (1.2 if rank_u0 is None else rank_u0)

    def screen():
        k = np.arange(B)
        b.U = np.minimum(b.U, np.where(k % 3 == 0, 0.5, 10.0))       # every third draw screened below
        b.n_screened = int((b.U < b.tau[0]).sum())
        b.screened = True

    def solve(idx, stops=True):
        idx = np.asarray(idx)
        b.seen.extend(idx.tolist())
        b.L[idx] = 0.1 * idx                                           # above for idx >= 25
        b.U[idx] = 0.1 * idx + 0.05
        b.solved[idx] = True
        b.flag[idx] = 1
        b.tol_stop[idx] = b.tol_full[idx] = 1e-5
        b.time["solve"] += 1e-3

    def save(path):                                   # the record's per-draw part, as a checkpoint
        b.saves.append(path)
        np.savez(path, L=b.L, U=b.U, flag=b.flag, tol_stop=b.tol_stop, tol_full=b.tol_full)

    b._certify, b._screen, b.solve_draws, b.save = certify, screen, solve, save
    return b


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = _fake(rank_u0=1.2 if rank == 0 else 7.0)     # rank 1's own band must be overridden
        b.checkpoint = os.path.join(out, "checkpoint.npz")
        pv = b.p_value()
        np.savez(os.path.join(out, "r%d.npz" % rank), L=b.L, U=b.U, solved=b.solved, seen=np.array(b.seen),
                 p=pv.p, tau=np.array(pv.tau), flag=b.flag, tol_stop=b.tol_stop, tol_full=b.tol_full,
                 saves=len(b.saves))
    finally:
        dist.destroy_process_group()


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_sharded_bootstrap_matches_one_process(tmp_path):
    one = _fake()
    pv1 = one.p_value()
    mp.start_processes(_worker, args=(2, _port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r = [np.load(os.path.join(tmp_path, "r%d.npz" % k)) for k in range(2)]
    for k in range(2):
        np.testing.assert_array_equal(r[k]["L"], one.L)
        np.testing.assert_array_equal(r[k]["U"], one.U)
        np.testing.assert_array_equal(r[k]["solved"], one.solved)
        assert float(r[k]["p"]) == pytest.approx(pv1.p)
        np.testing.assert_array_equal(r[k]["tau"], np.array(pv1.tau))
        # the exit flags and tolerances travel with the bounds
        np.testing.assert_array_equal(r[k]["flag"], one.flag)
        np.testing.assert_array_equal(r[k]["tol_stop"], one.tol_stop)
        np.testing.assert_array_equal(r[k]["tol_full"], one.tol_full)
    # the open draws were split, each solved exactly once
    s0, s1 = set(r[0]["seen"].tolist()), set(r[1]["seen"].tolist())
    assert not (s0 & s1) and s0 | s1 == set(one.seen) and s0 and s1
    # rank 0 alone wrote the checkpoint, and it holds the whole record: a resume from it counts
    # every draw either rank solved as solved (flag != NEVER), so none is solved again
    assert int(r[0]["saves"]) == 1 and int(r[1]["saves"]) == 0
    ck = np.load(os.path.join(tmp_path, "checkpoint.npz"))
    np.testing.assert_array_equal(ck["flag"], one.flag)
    np.testing.assert_array_equal(ck["flag"] != BS.NEVER, one.solved)
    np.testing.assert_array_equal(ck["L"], one.L)
    np.testing.assert_array_equal(ck["tol_full"], one.tol_full)
