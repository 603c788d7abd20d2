"""World-size-2 CPU (gloo) test of the replica timing harness used by bench.py
for N > 1 GPUs: each rank owns independent solves, ranks meet only for the
barrier and the max of the elapsed times."""
import multiprocessing as mp
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from chidg_b200 import replicas
    from oracle import oracle as O
    from chidg_b200 import mesh
    r, w, local, dist = replicas.init_from_env(backend="gloo", timeout_s=60)
    mine = list(replicas.split_work(5, r, w))
    # each rank solves its own independent systems with the CPU oracle
    done = 0
    for item in mine:
        pat = mesh.box_pattern(2, 2, 2, 5, 1)
        A = O.OracleMatrix(pat)
        A.set_values(mesh.synth_values(pat, seed=item))
        b = mesh.synth_vector(A.n, seed=100 + item)
        _, res = O.fgmres(A, O.OraclePrecon(A, "ilu0"), b,
                          O.default_opts(tol=0.0, rtol=1e-10, nkrylov=20, inner_fgmres=0, nmax=100))
        assert res["residual_norm"] <= 1e-9 * res["r0norm_initial"]
        done += 1
    replicas.barrier(dist)
    elapsed = 1.0 + r          # rank-dependent stand-in for a measured time
    emax = replicas.allmax(dist, elapsed)
    counts = [None] * w
    dist.all_gather_object(counts, done)
    q.put((r, mine, emax, replicas.aggregate_throughput(counts, emax)))
    dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [list(o[1]) for o in out] == [[0, 1, 2], [3, 4]]
    assert out[0][2] == out[1][2] == 2.0             # max over ranks
    assert out[0][3] == pytest.approx(5 / 2.0)       # all units / slowest rank


def test_split_work_covers_everything():
    from chidg_b200 import replicas
    for n in (0, 1, 7, 64):
        for w in (1, 2, 3, 8):
            got = [i for r in range(w) for i in replicas.split_work(n, r, w)]
            assert got == list(range(n))
