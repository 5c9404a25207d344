"""Chain shards against the whole system, on one GPU.

Three shards of one system live in this process and share one stream; the
sum over shards that NCCL does between GPUs is a plain device sum here.  After
initialisation and several sweeps, every bead position (gathered in the whole
system's chain order), the summed counts and each shard's omega are
bit-identical to the same system run whole, accepted moves add up to the whole
system's, and the field energy of every shard is the whole system's.
"""
import numpy as np
import pytest

from tests._util import assert_close, assert_coords_equal, assert_counts_equal

pytestmark = pytest.mark.gpu


def _specs():
    from new_arch_b200.spec import Arch, SystemSpec, cell_units, diblock_melt, interaction_matrix
    k, sig = cell_units()
    blend = SystemSpec(2, 16, 16, 8, 16.0, 16.0, 8.0, interaction_matrix(2, 15.0, 40.0), 64, k, 0.5, seed=77,
                       archs=[Arch(64, 101, [0] * 64, [[i, i + 1] for i in range(63)], sig),
                              Arch(64, 77, [1] * 64, [[i, i + 1] for i in range(63)], sig),
                              Arch(32, 45, [0] * 16 + [1] * 16, [[i, i + 1] for i in range(31)], sig)])
    return {"blend power-of-two grid": blend,
            "diblocks N=48 on 20x18x12": diblock_melt(1300, 48, 0.4, (20, 18, 12), 22.0, 50.0, seed=5)}


@pytest.mark.parametrize("name", list(_specs()))
def test_shards_equal_whole_system(name):
    import torch
    import new_arch_b200 as nb
    from new_arch_b200.shard import Shard, shard_chains
    spec = _specs()[name]
    n_shards, sweeps = 3, 6
    stream = torch.cuda.Stream()   # a real stream: handle 0 would give each shard a private one
    with nb.System(spec, stream=stream.cuda_stream) as whole:
        whole.init_coords()
        whole.step(sweeps)
        w_xyz, w_cnt, w_om, w_st = whole.coords(), whole.counts(), whole.omega(), whole.stats()
    shards = [Shard(spec, s, n_shards, stream.cuda_stream) for s in range(n_shards)]
    words = shards[0].count_words
    with torch.cuda.stream(stream):
        part = [torch.zeros(words, dtype=torch.int32, device="cuda") for _ in shards]
        total = torch.zeros(words, dtype=torch.int32, device="cuda")

    def summed():
        with torch.cuda.stream(stream):
            total.copy_(part[0])
            for p in part[1:]:
                total.add_(p)

    for sh, p in zip(shards, part):
        sh.init_coords(p.data_ptr())
    summed()
    for sh in shards:
        sh.field(total.data_ptr(), close_sweep=False)
    for _ in range(sweeps):
        for sh, p in zip(shards, part):
            sh.move(p.data_ptr())
        summed()
        for sh in shards:
            sh.field(total.data_ptr(), close_sweep=True)
    stream.synchronize()
    # positions in the whole system's order: per architecture, the shards' runs in shard order
    pieces, starts = [], [0] * n_shards
    for a, arch in enumerate(spec.archs):
        for s, sh in enumerate(shards):
            first, count = shard_chains(spec, s, n_shards)
            xyz = sh.coords()
            n = count[a] * arch.length
            pieces.append(xyz[starts[s]:starts[s] + n])
            starts[s] += n
    assert_coords_equal(np.concatenate(pieces), w_xyz, f"{name}: shard positions")
    with torch.cuda.stream(stream):
        tot = total.cpu().numpy().view(np.uint32)
    assert_counts_equal(tot, w_cnt, f"{name}: summed counts")
    acc = 0
    for sh in shards:
        assert np.array_equal(sh.omega().view(np.uint32), w_om.view(np.uint32)), f"{name}: shard omega"
        st = sh.stats()
        assert st["step"] == sweeps
        assert_close([st["e_field"]], [w_st["e_field"]], what=f"{name}: shard field energy")
        acc += st["total_accepts"]
    assert acc == w_st["total_accepts"]
    assert_close([sum(sh.stats()["e_bond"] for sh in shards)], [w_st["e_bond"]], what=f"{name}: bond energy")
    # a shard refuses the whole-system calls
    with pytest.raises(nb.ScmfError) as e:
        nb._lib.check(nb.lib().scmf_step(shards[0]._h, 1))
    assert e.value.code == -6
    for sh in shards:
        sh.close()


def test_single_process_sharded_system_equals_whole():
    """ShardedSystem without a process group holds the one shard of the
    system; its summed counts after init and sweeps are the whole system's."""
    import new_arch_b200 as nb
    from new_arch_b200.shard import ShardedSystem
    from new_arch_b200.spec import diblock_melt
    spec = diblock_melt(2500, 32, 0.3, (16, 16, 16), 25.0, 50.0, seed=3)
    with nb.System(spec) as whole:
        whole.init_coords()
        whole.step(4)
        want = whole.counts()
    sh = ShardedSystem(spec)
    sh.init_coords()
    sh.step(4)
    assert_counts_equal(sh.counts(), want, "one-shard system")
    sh.close()
