"""The multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py runs one independent dot per GPU (replicas); its only collectives
are the barrier and the max over ranks of the timed step.  Here two
processes reduce different values and both must see the larger one, and the
reference arm prints only on rank 0.  The line's per-iteration byte
accounting is checked against its definition.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        got = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 2.5), (1, 2.5)]


def test_reference_arm_is_silent_off_rank_zero():
    sys.path.insert(0, ROOT)
    import bench
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(None, rank=1, world=2)
    assert buf.getvalue() == ""


def test_per_iteration_bytes():
    """The bench line's per-iteration accounting: algorithmic bytes are
    B_SpMV + one vector per atom, the bytes the two-kernel design moves are
    B_H + six vectors per atom, and the fractions divide by the time per
    first-pass iteration and the measured copy bandwidth."""
    import bench
    pk = bench.peaks()[0]["hbm_gbs"]
    natoms, its, solve_ms = 1000000, 1000, 1000.0  # 1 ms per iteration
    for bits, vec, alg_atom, moved_atom in ((32, 160, 1256 + 160, 936 + 6 * 160),
                                            (64, 320, 2504 + 320, 1864 + 6 * 320)):
        r = bench.per_iteration(bits, natoms, {"solve_ms": solve_ms}, {"iterations": its})
        assert r["ms"] == 1.0
        assert abs(r["algorithmic_gb"] - alg_atom * natoms / 1e9) < 1e-12
        assert abs(r["moved_gb"] - moved_atom * natoms / 1e9) < 1e-12
        assert abs(r["algorithmic_frac"] - alg_atom * natoms / 1e-3 / 1e9 / pk) < 1e-12
        assert abs(r["moved_frac"] - moved_atom * natoms / 1e-3 / 1e9 / pk) < 1e-12
