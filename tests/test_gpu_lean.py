"""The single-system lean move kernel (k_sweep_lean) against the oracle.

It runs for one system whose chains are linear with an even length L <= 64
and L/2 dividing 32, on a grid of power-of-two axes.  These cases cover what
it does differently from the general register kernel: chain ends replaced by
the bead itself (L = 2, where both ends are one pair, up to L = 64, one chain
per warp), lanes past a tile's last chain (chain counts that leave partial
iterations), several architectures in one system, 16-bit counts, the
move-only reference call sequence, and a one-system batch.  Positions and
counts must be bit-identical, omega and energies within 1e-6.
"""
import pytest

from tests._util import compare_state, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import new_arch_b200
    return new_arch_b200


@pytest.mark.parametrize("n,chains,grid", [(2, 3001, (16, 8, 8)), (4, 1503, (8, 8, 8)), (8, 777, (16, 16, 8)),
                                           (16, 1001, (16, 16, 16)), (32, 333, (8, 16, 8)), (64, 131, (16, 8, 16))])
def test_lean_chain_lengths_and_partial_tiles(nb, n, chains, grid):
    spec = nb.spec.diblock_melt(chains, n, 0.4, grid, 22.0, 50.0, seed=100 + n)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(7)
        orc.step(7)
        compare_state(s, orc, f"lean N={n}")


def test_lean_small_steps_accept_often(nb):
    """A small smart-MC step (most trials accepted): every lane moves beads and
    counts across cells, so the count moves under the warp vote run often."""
    spec = nb.spec.diblock_melt(900, 32, 0.5, (16, 16, 16), 18.0, 50.0, seed=7, smc_a=0.02)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(10)
        orc.step(10)
        compare_state(s, orc, "lean A=0.02")
        assert s.stats()["total_accepts"] > 0.3 * 10 * spec.n_beads


def test_lean_mixed_architectures_and_16_bit_counts(nb):
    from new_arch_b200.spec import Arch, SystemSpec, cell_units, interaction_matrix
    k, sig = cell_units()
    archs = [Arch(64, 40, [0] * 64, [[i, i + 1] for i in range(63)], sig),
             Arch(32, 70, [0] * 10 + [1] * 22, [[i, i + 1] for i in range(31)], sig),
             Arch(8, 101, [1] * 8, [[i, i + 1] for i in range(7)], sig)]
    spec = SystemSpec(2, 16, 8, 16, 16.0, 8.0, 16.0, interaction_matrix(2, 15.0, 40.0), 64, k, 0.5, seed=21,
                      count_bits=16, archs=archs)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(6)
        orc.step(6)
        compare_state(s, orc, "lean mixed architectures")


def test_lean_reference_shaped_calls(nb):
    """smc_move (move only) -> reset_density_fields -> update_omega_fields_scmf0."""
    spec = nb.spec.diblock_melt(500, 16, 0.5, (8, 8, 8), 15.0, 50.0, seed=3, field_rule=0)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        for step in range(1, 13):
            s.smc_move(1)
            orc.smc_move(1)
            s.reset_density_fields()
            orc.reset_density()
            if step % 10:
                s.update_omega_fields_scmf0()
                orc.update_omega()
            compare_state(s, orc, f"lean reference step {step}", energies=False)


def test_lean_one_system_batch_with_explicit_tiles(nb):
    spec = nb.spec.diblock_melt(2000, 32, 0.3, (16, 16, 16), 25.0, 50.0, seed=9)
    with nb.System(spec) as s:
        s.init_coords()
        b = nb.Batch([s], tune={"threads_move": 256, "beads_per_tile": 1024})
        b.step(5)
        b.close()
        orc = oracle_for(spec)
        orc.step(5)
        compare_state(s, orc, "lean one-system batch")


@pytest.mark.parametrize("seeds", ["one", "same_high_word", "distinct_high_words"])
def test_leanm_batches_and_grids(nb, seeds):
    """The multi-system lean kernel (k_sweep_leanm): systems of even,
    warp-filling lengths on grids with and without power-of-two axes, batched
    with each Philox key mode, plus a lone system on a grid that k_sweep_lean
    does not take; a partial last iteration in every tile kind."""
    specs = [nb.spec.diblock_melt(301, 16, 0.3, (10, 12, 7), 18.0, 50.0),
             nb.spec.diblock_melt(157, 32, 0.6, (16, 16, 8), 25.0, 50.0),
             nb.spec.diblock_melt(61, 64, 0.5, (9, 8, 11), 12.0, 50.0)]
    for i, sp in enumerate(specs):
        sp.seed = {"one": 5, "same_high_word": 5 + i, "distinct_high_words": 5 + (i << 33)}[seeds]
    systems = [nb.System(sp) for sp in specs]
    for s in systems:
        s.init_coords()
    b = nb.Batch(systems, tune={"threads_move": 64, "beads_per_tile": 1024})
    b.step(5)
    b.close()
    for i, (sp, s) in enumerate(zip(specs, systems)):
        orc = oracle_for(sp)
        orc.step(5)
        compare_state(s, orc, f"leanm {seeds} member {i}")
        s.close()
    # alone: one system, a grid without power-of-two axes
    sp = nb.spec.diblock_melt(700, 32, 0.4, (12, 10, 14), 20.0, 50.0, seed=8)
    with nb.System(sp) as s:
        s.init_coords()
        orc = oracle_for(sp)
        s.step(6)
        orc.step(6)
        compare_state(s, orc, "leanm alone")
