"""Bit-exact trajectories at the benchmark's full sizes.

* The large single system (1.6M AB diblocks of N=32, 51.2M beads, 128^3 cells,
  chiN=25, kappaN=50, seed 7) and the blend (2M chains: A and B homopolymers
  of N=64 with 10 % AB diblocks of N=32, 121.6M beads, 256x256x64 cells,
  chiN=15 at N_ref=64, kappaN=40, seed 11): after random-walk initialisation
  and after three sweeps on the GPU, positions (every bit), counts and
  accepted moves equal the OpenMP oracle's run of the same system from the
  same seed; omega and energies agree within 1e-6.  These are the kernel
  instances and launch shapes the benchmark times (one seed per launch, so the
  Philox round keys come from the kernel parameters; tiles of 4,096 beads).
* Served requests at the largest edge of the served stream (128 cells), run
  side by side in the server for 50 sweeps: counts bit-exact, accepted moves
  equal, energies within 1e-6 against the oracle run of each request alone.
  One has a cubic power-of-two grid and N=48 (chains across warps), the other
  128 x 101 x 77 cells (multiply-high fold) and N=64.

The oracle runs on all host threads (bit-identical to its single-threaded
form).
"""
import os

import numpy as np
import pytest

from tests._util import assert_close, assert_counts_equal, compare_state, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import new_arch_b200
    return new_arch_b200


@pytest.fixture()
def all_threads():
    from oracle.oracle import set_threads
    set_threads(os.cpu_count() or 1)
    yield
    set_threads(1)


@pytest.mark.parametrize("which", ["large", "blend"])
def test_full_size_trajectory_matches_oracle(nb, all_threads, which):
    from new_arch_b200.spec import blend_system, large_system
    spec = large_system(seed=7) if which == "large" else blend_system(seed=11)
    assert spec.n_beads == (51_200_000 if which == "large" else 121_600_000)
    sweeps = 3
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        compare_state(s, orc, f"{which} init")
        s.step(sweeps)
        orc.step(sweeps)
        compare_state(s, orc, f"{which}, {sweeps} sweeps")
        st = s.stats()
        assert st["step"] == sweeps and st["total_moves"] == sweeps * spec.n_beads
        assert st["total_accepts"] > 0


def test_served_edge_128_requests_match_oracle(nb, all_threads):
    from new_arch_b200.server import Server
    from new_arch_b200.spec import diblock_melt

    def request(edges, n, f_a, chi, seed):
        cells = edges[0] * edges[1] * edges[2]
        return diblock_melt(int(round(7.8 * cells / n)), n, f_a, edges, chi, 50.0, seed)

    reqs = [request((128, 128, 128), 48, 0.35, 22.0, 50_123), request((128, 101, 77), 64, 0.6, 14.0, 50_456)]
    K = 50
    with Server(150 * 10**9) as srv:
        ids = {srv.submit(sp, K): i for i, sp in enumerate(reqs)}
        res = []
        while len(res) < len(reqs):
            res += srv.poll(8, 1000)
    assert sorted(ids) == sorted(r["id"] for r in res)
    for r in res:
        sp = reqs[ids[r["id"]]]
        assert r["status"] == 0 and r["sweeps_done"] == K
        orc = oracle_for(sp)
        orc.step(K)
        ost = orc.stats()
        what = f"served {sp.nx}x{sp.ny}x{sp.nz} N={sp.archs[0].length}"
        assert_counts_equal(r["counts"], orc.counts(), what + " counts")
        assert r["accepts"] == ost["total_accepts"], what + " accepts"
        assert_close([r["e_field"]], [ost["e_field"]], what=what + " e_field")
        assert_close([r["e_bond"]], [ost["e_bond"]], what=what + " e_bond")
        assert int(np.asarray(r["counts"]).sum()) == sp.n_beads
