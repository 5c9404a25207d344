"""World-size-2 test of the replicas form on CPU (gloo): each rank runs its own
system (oracle restatement, distinct seed), the timing is reduced with MAX and
the whole-job rate is identical on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import time
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from new_arch_b200.replicas import gather_ints, reduce_max, replica_seed, whole_job_rate
    from new_arch_b200.spec import diblock_melt
    from oracle.oracle import OracleSystem
    spec = diblock_melt(100 + 20 * rank, 16, 0.5, (6, 6, 6), 15.0, 50.0, seed=replica_seed(7, rank))
    o = OracleSystem(spec)
    o.init_coords()
    o.reset_density()
    o.update_omega()
    dist.barrier()
    t0 = time.perf_counter()
    o.step(5)
    el = time.perf_counter() - t0
    el_max = reduce_max(el, dist)
    beads = gather_ints(spec.n_beads, dist)
    rate = whole_job_rate(beads, 5, el_max)
    out[rank] = (el, el_max, beads, rate, o.counts().sum(), o.coords()[:4].copy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (e0, m0, b0, r0, c0, x0), (e1, m1, b1, r1, c1, x1) = out[0], out[1]
    assert m0 == m1 == max(e0, e1)
    assert b0 == b1 == [100 * 16, 120 * 16]
    assert r0 == r1 == pytest.approx(sum(b0) * 5 / m0)
    assert c0 == b0[0] and c1 == b0[1]
    assert not np.array_equal(x0, x1)   # distinct seeds, distinct chains
