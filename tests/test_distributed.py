"""Multi-process host logic of the sharded evaluation: world_size-2 gloo process groups on CPU.
The per-rank partial sums come from the oracle (the GPU evaluators plug in the same way)."""
import os
import socket
from fractions import Fraction

import numpy as np
import pytest

from mertens_bound_b200 import distributed


def test_shard_range_partitions():
    for n in (0, 1, 7, 1000, 2_325_572):
        for world in (1, 2, 3, 8):
            parts = [distributed.shard_range(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            assert max(e - s for s, e in parts) - min(e - s for s, e in parts) <= 1
    with pytest.raises(ValueError):
        distributed.shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from mertens_bound_b200 import distributed as D, synth
    from oracle.oracle import Oracle
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        data = synth.make_table(800, seed=31)
        cands = synth.make_candidates(5, seed=32)
        O = Oracle()

        def ev_value(j0, j1):
            sub = synth.ZeroTableData(data.G3[j0:j1], data.gamma[j0:j1], data.c_re[j0:j1], data.c_im[j0:j1], 0)
            hi, lo = O.k2(cands, sub, 3e-9, j1 - j0)
            return hi

        def ev_interval(j0, j1):
            v = ev_value(j0, j1)[:, 0]
            return v - 1e-13, v + 1e-13

        tot = D.zero_sharded_value(ev_value, data.n)
        ivs = D.zero_sharded_certified(ev_interval, data.n)
        lo_c, hi_c = distributed.shard_range(cands.n, world, rank)
        gathered = D.gather_candidates(np.arange(lo_c, hi_c, dtype=np.float64) * 10.0)
        q.put((rank, tot, [(float(a), float(b)) for a, b in ivs], gathered.tolist()))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:             # report, do not hang the parent
        q.put((rank, repr(e), None, None))


def test_zero_sharded_sums_match_single_process(oracle):
    import multiprocessing as mp
    from mertens_bound_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
    for r in res:
        assert not isinstance(r[1], str), r[1]
    data = synth.make_table(800, seed=31)
    cands = synth.make_candidates(5, seed=32)
    full, _ = oracle.k2(cands, data, 3e-9, data.n)
    for rank, tot, ivs, gathered in res:
        assert np.max(np.abs(tot - full)) < 1e-13 * np.max(np.abs(full))
        for p, (a, b) in enumerate(ivs):
            assert a <= full[p, 0] <= b and b - a < 1e-12
        assert gathered == [0.0, 10.0, 20.0, 30.0, 40.0]
