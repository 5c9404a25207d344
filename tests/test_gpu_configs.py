"""Parity at the benchmark configurations themselves.

* The plain system exactly as specified (1,000 AB diblocks of N=32, f_A=0.5,
  16^3 cells, chiN=20, kappaN=50, 16-bit counts, seed 42, 1,000 sweeps with the
  field updated every sweep): positions and counts bit-exact against the
  oracle after all 1,000 sweeps.
* Systems drawn from the 256-system batched mix, at full size, advanced 100
  sweeps in one batch: each bit-exact against the oracle run of that system
  alone.
"""
import numpy as np
import pytest

from tests._util import assert_close, assert_coords_equal, assert_counts_equal, compare_state, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import new_arch_b200
    return new_arch_b200


def test_plain_config_1000_sweeps(nb):
    from oracle.oracle import set_threads
    import os
    spec = nb.spec.plain_system(seed=42)
    assert spec.count_bits == 16 and spec.n_beads == 32000 and spec.n_cells == 4096
    set_threads(os.cpu_count() or 1)
    try:
        with nb.System(spec) as s:
            s.init_coords()
            orc = oracle_for(spec)
            for chunk in (1, 99, 900):
                s.step(chunk)
                orc.step(chunk)
            compare_state(s, orc, "plain config, 1000 sweeps")
            st = s.stats()
            assert st["step"] == 1000 and st["total_moves"] == 1000 * spec.n_beads
            assert int(s.counts().sum()) == spec.n_beads
    finally:
        set_threads(1)


def test_batched_mix_members_match_oracle(nb):
    from oracle.oracle import set_threads
    import os
    specs = nb.spec.batched_mix(256)
    rng = np.random.default_rng(3)
    pick = sorted(rng.choice(256, 6, replace=False).tolist())
    chosen = [specs[i] for i in pick]
    systems = [nb.System(sp) for sp in chosen]
    for x in systems:
        x.init_coords()
    b = nb.Batch(systems, tune={"chains_per_tile": 48, "threads_move": 128})
    b.step(100)
    set_threads(os.cpu_count() or 1)
    try:
        for i, (sp, x) in zip(pick, zip(chosen, systems)):
            orc = oracle_for(sp)
            orc.step(100)
            compare_state(x, orc, f"mix system {i}")
    finally:
        set_threads(1)
        b.close()
        for x in systems:
            x.close()
