"""The move kernels reject a trial before reading omega when its bonded energy
change minus the span of omega (published by every field step) already fails
the Metropolis bound.  That must give the oracle's outcome for any omega:

* right after scmf_set_omega the span is unknown (+inf), so every trial reads
  omega;
* the reference field rule keeps omega through a sweep whose step is a
  multiple of 10, and the field step of that sweep computes the span from the
  kept values: large finite spikes (a wide span), NaN cells (skipped by the
  span; a trial that reads one is rejected, as the oracle's NaN energy is) and
  infinite cells (no bound).

Each case runs through the lean kernel (N=32 on a power-of-two grid), the
multi-system lean kernel (N=32 on other grids), the register kernel (odd N)
and the long-chain kernel (N=80), with positions, counts and accepted moves
compared bit for bit after every sweep."""
import numpy as np
import pytest

from tests._util import assert_coords_equal, assert_counts_equal, oracle_for

pytestmark = pytest.mark.gpu

KERNELS = {
    "lean": (32, (16, 16, 16)),
    "lean_multi": (32, (20, 18, 12)),
    "register": (33, (16, 16, 16)),
    "long_chains": (80, (16, 16, 16)),
}


def _odd_omega(w, case, rng):
    w = w.copy()
    idx = rng.choice(w.size, size=max(8, w.size // 50), replace=False)
    if case == "spikes":
        w[idx] += rng.choice([-40.0, 40.0], size=idx.size).astype(np.float32)
    elif case == "nan":
        w[idx] = np.nan
    else:
        w[idx[: idx.size // 2]] = np.inf
        w[idx[idx.size // 2:]] = -np.inf
    return w


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("case", ["spikes", "nan", "inf"])
def test_span_rejection_matches_oracle_for_any_omega(kernel, case):
    import new_arch_b200 as nb
    from new_arch_b200.spec import diblock_melt

    n, grid = KERNELS[kernel]
    chains = int(round(7.8 * grid[0] * grid[1] * grid[2] / n))
    spec = diblock_melt(chains, n, 0.3, grid, 25.0, 50.0, seed=21, field_rule=nb.FIELD_REFERENCE)
    rng = np.random.default_rng(3)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(3)
        orc.step(3)
        s.set_step(9)       # the next sweep is sweep 10: its field step keeps omega
        orc.set_step(9)
        w = _odd_omega(s.omega(), case, rng)
        s.set_omega(w)      # span unknown for sweep 10
        orc.set_omega(w)
        for k in range(5):  # sweep 11 runs with the span of the kept, odd omega
            s.step(1)
            orc.step(1)
            what = f"{kernel}/{case}, sweep {10 + k}"
            assert_coords_equal(s.coords(), orc.coords(), what + " coords")
            assert_counts_equal(s.counts(), orc.counts(), what + " counts")
            gs, os_ = s.stats(), orc.stats()
            assert gs["total_accepts"] == os_["total_accepts"], f"{what}: accepts"
            if k == 0:
                kept = s.omega()
                assert np.array_equal(kept.view(np.uint32), w.view(np.uint32)), f"{what}: omega not kept"
        assert np.all(np.isfinite(s.omega())), "the field steps after sweep 10 recompute omega from the counts"
