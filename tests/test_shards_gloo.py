"""World-size-2 test of the chain-shard form on CPU (gloo).

Each rank takes its shard of one system (the library's own partition,
scmf_shard_chains), runs the shard in the oracle with the chains' whole-system
random-stream ids and the whole system's field scaling, and sums the shard
counts over the ranks with an all-reduce before every field step, which is
the per-sweep sequence a ShardedSystem runs over NCCL.  Every rank's positions
equal its slice of the whole system run in one process, bit for bit, and the
summed counts and omega equal the whole system's.
"""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _spec():
    from new_arch_b200.spec import Arch, SystemSpec, cell_units, interaction_matrix
    k, sig = cell_units()
    return SystemSpec(2, 8, 6, 5, 8.0, 6.0, 5.0, interaction_matrix(2, 15.0, 40.0), 16, k, 0.3, seed=19,
                      archs=[Arch(16, 23, [0] * 6 + [1] * 10, [[i, i + 1] for i in range(15)], sig),
                             Arch(12, 9, [1] * 12, [[i, i + 1] for i in range(11)], sig)])


SWEEPS = 4


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import copy
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from new_arch_b200.shard import shard_chains
    from oracle.oracle import OracleSystem
    spec = _spec()
    first, count = shard_chains(spec, rank, world)
    mine = copy.deepcopy(spec)
    for a, c in zip(mine.archs, count):
        a.n_chains = c
    o = OracleSystem(mine)
    bases, base = [], 0
    for a, f in zip(spec.archs, first):
        bases.append(base + f)
        base += a.n_chains
    o.set_shard(bases, spec.n_beads)

    def summed():
        t = torch.from_numpy(o.counts().astype(np.int64))
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t.numpy().astype(np.uint32)

    o.init_coords()
    o.reset_density()
    o.field_from(summed())
    for _ in range(SWEEPS):
        o.smc_move(1)
        o.reset_density()
        total = summed()
        o.field_from(total)
    out[rank] = (first, count, o.coords().copy(), total.copy(), o.omega().copy(), o.stats()["total_accepts"])
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_shards_equal_whole_system():
    from oracle.oracle import OracleSystem
    spec = _spec()
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
    whole = OracleSystem(spec)
    whole.init_coords()
    whole.reset_density()
    whole.update_omega()
    whole.step(SWEEPS)
    w_xyz = whole.coords()
    # the shards cover every chain exactly once, in order
    for a, arch in enumerate(spec.archs):
        assert out[0][0][a] == 0 and out[0][1][a] + out[1][1][a] == arch.n_chains
        assert out[1][0][a] == out[0][1][a]
    # positions: per architecture, rank 0's run then rank 1's
    pieces, starts, bead_base = [], [0, 0], 0
    for a, arch in enumerate(spec.archs):
        for r in range(2):
            n = out[r][1][a] * arch.length
            piece = out[r][2][starts[r]:starts[r] + n]
            assert np.array_equal(piece.view(np.uint32), w_xyz[bead_base:bead_base + n].view(np.uint32)), (a, r)
            starts[r] += n
            bead_base += n
    for r in range(2):
        assert np.array_equal(out[r][3], whole.counts())
        assert np.array_equal(out[r][4].view(np.uint32), whole.omega().view(np.uint32))
    assert out[0][5] + out[1][5] == whole.stats()["total_accepts"]
