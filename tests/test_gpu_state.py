"""GPU tests of the state around the hot path, against the oracle: the
time-averaged density accumulated inside the fused sweep (bit-exact sums), its
file, exact resume from a binary checkpoint, and the chain observables."""
import os

import numpy as np
import pytest

from tests._util import assert_close, compare_state, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import new_arch_b200
    return new_arch_b200


# (grid, count bits): vector field path (32-bit counts, cells % 4 == 0) and the
# scalar paths (16-bit counts; odd cell count)
CASES = [((8, 8, 6), 32), ((6, 5, 4), 16), ((5, 5, 5), 32)]


@pytest.mark.parametrize("grid,bits", CASES)
def test_average_density_matches_oracle(nb, grid, bits):
    from new_arch_b200.spec import diblock_melt
    spec = diblock_melt(int(7.8 * np.prod(grid) / 16), 16, 0.4, grid, 22.0, 50.0, seed=31, count_bits=bits)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.average_start(3)
        orc.average_start(3)
        s.step(11)
        orc.step(11)
        g, gn = s.average()
        o, on = orc.average()
        assert gn == on == 3
        assert np.array_equal(g, o)
        s.average_sample()
        orc.average_sample()
        g, gn = s.average()
        o, on = orc.average()
        assert gn == on == 4 and np.array_equal(g, o)
        compare_state(s, orc, "after averaging")
        s.average_start(0)
        with pytest.raises(nb.ScmfError):
            s.average()


def test_average_density_file(nb, tmp_path):
    from new_arch_b200.spec import diblock_melt
    spec = diblock_melt(240, 16, 0.5, (6, 5, 4), 20.0, 50.0, seed=4)
    with nb.System(spec) as s:
        s.init_coords()
        with pytest.raises(nb.ScmfError):
            s.io_out_aver_density(0, str(tmp_path / "x.dat"))   # not started
        s.average_start(1)
        s.step(4)
        s.io_out_aver_density(4, str(tmp_path / "density_aver_4.dat"))
        sums, n = s.average()
        om = s.omega()
    lines = (tmp_path / "density_aver_4.dat").read_text().splitlines()
    assert lines[0] == "Nx=6, Ny=5, Nz=4" and lines[1] == "dx=1, dy=1, dz=1"
    vals = np.array([[float(v) for v in l.split()] for l in lines[2:]])
    nc = spec.n_cells
    want = sums.reshape(2, -1).T.astype(np.float64) / n * (nc / spec.n_beads)
    assert np.allclose(vals[:, :2], want, rtol=1e-5)
    assert np.allclose(vals[:, 2:], om.reshape(2, -1).T, rtol=1e-5, atol=1e-6)
    # mean phi summed over cells and types is the cell count (conservation)
    assert abs(vals[:, :2].sum() - nc) < 1e-3 * nc


@pytest.mark.parametrize("split", [10, 15])
def test_checkpoint_resumes_exactly(nb, tmp_path, split):
    """The reference field rule skips omega at multiples of 10, so a resume at
    step 10 is exact only if omega itself is restored; at 15 the stored
    averaging state must carry on."""
    from new_arch_b200.spec import diblock_melt
    spec = diblock_melt(300, 16, 0.35, (8, 6, 6), 24.0, 50.0, seed=12, field_rule=nb.FIELD_REFERENCE)
    path = str(tmp_path / "ck.bin")
    with nb.System(spec) as a:
        a.init_coords()
        a.average_start(2)
        a.step(split)
        a.checkpoint_write(path)
        a.step(25 - split)
        want = (a.coords(), a.counts(), a.omega(), a.stats(), a.average())
    info = nb.checkpoint_info(path)
    assert info["step"] == split and info["avg_every"] == 2 and info["avg_samples"] == split // 2
    with nb.System(spec) as b:
        b.init_coords()
        b.step(3)                                   # state to be overwritten
        b.checkpoint_read(path)
        assert b.sweep_stats()["step"] == split
        b.step(25 - split)
        got = (b.coords(), b.counts(), b.omega(), b.stats(), b.average())
    assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32))
    assert np.array_equal(got[1], want[1])
    assert np.array_equal(got[2].view(np.uint32), want[2].view(np.uint32))
    for k in ("step", "total_accepts", "total_moves", "last_accepts"):
        assert got[3][k] == want[3][k], k
    assert got[3]["e_field"] == want[3]["e_field"] and got[3]["e_bond"] == want[3]["e_bond"]
    assert got[4][1] == want[4][1] and np.array_equal(got[4][0], want[4][0])


def test_checkpoint_refuses_another_system(nb, tmp_path):
    from new_arch_b200.spec import diblock_melt
    spec = diblock_melt(100, 16, 0.5, (6, 6, 6), 20.0, 50.0, seed=5)
    path = str(tmp_path / "ck.bin")
    with nb.System(spec) as a:
        a.init_coords()
        a.step(2)
        a.checkpoint_write(path)
    for other in (diblock_melt(100, 16, 0.5, (6, 6, 6), 21.0, 50.0, seed=5),    # another chiN
                  diblock_melt(100, 16, 0.5, (6, 6, 6), 20.0, 50.0, seed=6),    # another seed
                  diblock_melt(101, 16, 0.5, (6, 6, 6), 20.0, 50.0, seed=5)):   # another size
        with nb.System(other) as b:
            with pytest.raises(nb.ScmfError) as e:
                b.checkpoint_read(path)
            assert e.value.code == -1


def test_observables_match_oracle(nb):
    from new_arch_b200.spec import blend_system
    spec = blend_system(seed=9, n_chains=3000, grid=(16, 16, 8))
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(3)
        orc.step(3)
        got0 = s.analyze()
        assert all(np.all(np.isnan(g["msd"])) for g in got0)
        s.analysis_reference()
        orc.analysis_reference()
        s.step(6)
        orc.step(6)
        compare_state(s, orc, "observables run")
        got = s.analyze()
        st = s.stats()
    assert len(got) == len(spec.archs)
    for ai, g in enumerate(got):
        o = orc.analyze(ai)
        a = spec.archs[ai]
        assert g["n_chains"] == a.n_chains and g["n_beads"] == a.n_chains * a.length
        assert g["n_bonds"] == a.n_chains * len(a.bonds)
        for k in ("re2", "rg2", "bond2", "msd", "msd_com"):
            np.testing.assert_allclose(g[k][:3], o[k], rtol=1e-9, err_msg=f"arch {ai} {k}")
            assert abs(g[k][3] - g[k][:3].sum()) <= 1e-12 * abs(g[k][3])
        assert g["acc_ratio"] == st["last_accepts"] / spec.n_beads


# ------------------------------------------------------------ validation
def test_validate_clean_and_stale_counts(nb):
    from new_arch_b200.spec import diblock_melt
    for bits, grid in ((32, (8, 8, 8)), (16, (6, 5, 4))):
        spec = diblock_melt(int(7.8 * np.prod(grid) / 16), 16, 0.4, grid, 20.0, 50.0, seed=2, count_bits=bits)
        with nb.System(spec) as s:
            s.init_coords()
            s.step(3)
            v = s.validate()
            assert v["ok"] and v["count_mismatch_words"] == 0 and v["count_sum_error"] == 0
            s.smc_move(1)                       # counts now lag the positions
            v = s.validate(raise_on_error=False)
            assert not v["ok"] and v["count_mismatch_words"] > 0 and v["count_sum_error"] == 0
            s.reset_density_fields()
            assert s.validate()["ok"]
            s.step(2)                           # validation left the idle counts buffer clear
            orc = oracle_for(spec)
            orc.step(3)
            orc.smc_move(1)
            orc.reset_density()
            orc.step(2)
            compare_state(s, orc, f"after validation ({bits}-bit counts)")


def test_validate_reports_bad_positions(nb):
    """Host-made bad input: one non-finite coordinate and one far outside the
    exact fold range.  The fold keeps every cell index inside the grid, so the
    state stays usable; the check reports both beads and nothing else."""
    from new_arch_b200.spec import diblock_melt
    for grid in ((8, 8, 8), (6, 5, 7)):
        spec = diblock_melt(40, 16, 0.5, grid, 20.0, 50.0, seed=3)
        with nb.System(spec) as s:
            s.init_coords()
            xyz = s.coords().copy()
            xyz[5, 1] = np.nan
            xyz[17, 2] = 3.0e8
            s.set_coords(xyz)
            v = s.validate(raise_on_error=False)
            assert not v["ok"]
            assert v["nonfinite_positions"] == 1 and v["positions_out_of_range"] == 1
            assert v["count_sum_error"] == 0 and v["count_mismatch_words"] == 0
            with pytest.raises(nb.ScmfError) as e:
                s.validate()
            assert e.value.code == -8


def test_step_stats_async_matches_blocking_read(nb):
    """scmf_step_stats_async copies each sweep's statistics into page-locked
    host memory without waiting; after scmf_synchronize they equal what the
    blocking scmf_step_stats returns for the same sweeps of an identical system."""
    import ctypes
    import torch
    from new_arch_b200 import _lib
    spec = nb.spec.diblock_melt(2000, 32, 0.4, (12, 12, 12), 22.0, 50.0, seed=31)
    size = ctypes.sizeof(_lib.Stats)
    host = torch.zeros(size * 4, dtype=torch.uint8, pin_memory=True)
    with nb.System(spec) as a, nb.System(spec) as b:
        a.init_coords()
        b.init_coords()
        for k in range(4):
            a.step_stats_async(k + 1, host.data_ptr() + k * size)
        a.synchronize()
        for k in range(4):
            got, want = nb.System.stats_at(host.data_ptr() + k * size), b.step_stats(k + 1)
            for key in ("step", "last_accepts", "total_accepts", "total_moves", "e_field", "error_word"):
                assert got[key] == want[key], (k, key, got[key], want[key])
            assert np.isnan(got["e_bond"]) and np.isnan(want["e_bond"])
        assert np.array_equal(a.counts(), b.counts())
