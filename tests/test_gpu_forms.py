"""GPU tests of the served form, the reference file outputs / CLI, and
size-independent properties at the full benchmark sizes."""
import filecmp
import os
import shutil
import subprocess
import time

import numpy as np
import pytest

from tests._util import assert_close, assert_coords_equal, assert_counts_equal, compare_state, oracle_for

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def nb():
    import new_arch_b200
    return new_arch_b200


# ------------------------------------------------------------------ serving
def _alone(nb, spec, k):
    with nb.System(spec) as s:
        s.init_coords()
        s.step(k)
        st = s.stats()
        return s.counts(), st


def test_served_results_equal_alone(nb):
    """Requests that overlap on the device give the same counts (bit-exact) and
    energies (1e-6) as the same request run alone."""
    from new_arch_b200.server import Server
    from new_arch_b200.spec import served_request
    rng = np.random.default_rng(77)
    reqs = [served_request(rng, seed=900 + i, edge_lo=8, edge_hi=24) for i in range(12)]
    reqs = [(sp, k // 10) for sp, k in reqs]           # 5 / 10 / 50 sweeps keep the test short
    with Server(8 * 10**9, sweeps_per_round=3) as srv:
        ids = {}
        for i, (sp, k) in enumerate(reqs):
            ids[srv.submit(sp, k)] = i
            if i % 4 == 3:
                time.sleep(0.01)                        # later requests join running rounds
        res = []
        while len(res) < len(reqs):
            res += srv.poll(64, 500)
    assert sorted(ids) == sorted(r["id"] for r in res)
    for r in res:
        assert r["status"] == 0
        sp, k = reqs[ids[r["id"]]]
        cnt, st = _alone(nb, sp, k)
        assert_counts_equal(r["counts"], cnt, "served counts")
        assert r["accepts"] == st["total_accepts"]
        assert_close([r["e_field"]], [st["e_field"]], what="served e_field")
        assert_close([r["e_bond"]], [st["e_bond"]], what="served e_bond")
        assert r["t_submit"] <= r["t_admit"] <= r["t_done"]


def test_server_admission_under_budget(nb):
    """A budget that holds one request at a time serialises the work; a request
    larger than the budget is refused at submission."""
    from new_arch_b200.server import Server
    from new_arch_b200.spec import diblock_melt
    sp = diblock_melt(2000, 16, 0.5, (16, 16, 16), 20.0, 50.0, seed=5)
    budget = int(sp.device_bytes() * 1.5)
    with Server(budget, sweeps_per_round=2) as srv:
        for _ in range(3):
            srv.submit(sp, 4)
        peak_active = 0
        res = []
        while len(res) < 3:
            _, active, used = srv.pending()
            peak_active = max(peak_active, active)
            assert used <= budget
            res += srv.poll(8, 20)
        assert peak_active <= 1
        big = diblock_melt(200000, 32, 0.5, (64, 64, 64), 20.0, 50.0)
        with pytest.raises(nb.ScmfError) as e:
            srv.submit(big, 1)
        assert e.value.code == -3
    # the three identical requests give identical results
    assert all(np.array_equal(r["counts"], res[0]["counts"]) for r in res)


# ---------------------------------------------------------- file surface
def test_density_and_coord_files(nb, tmp_path):
    spec = nb.spec.diblock_melt(200, 16, 0.5, (6, 5, 4), 20.0, 50.0, seed=3)
    with nb.System(spec) as s:
        s.init_coords()
        s.step(3)
        s.io_out_density(3, str(tmp_path / "density_3.dat"))
        s.io_out_coord(str(tmp_path / "coord.dat"))
        cnt, om, xyz = s.counts(), s.omega(), s.coords()
    lines = (tmp_path / "density_3.dat").read_text().splitlines()
    assert lines[0] == "Nx=6, Ny=5, Nz=4"
    assert lines[1] == "dx=1, dy=1, dz=1"
    vals = np.array([[float(v) for v in l.split()] for l in lines[2:]])
    assert vals.shape == (120, 4)
    scale = 120 / spec.n_beads
    assert np.allclose(vals[:, :2], cnt.reshape(2, -1).T * scale, rtol=1e-5)
    assert np.allclose(vals[:, 2:], om.reshape(2, -1).T, rtol=1e-5, atol=1e-6)
    back = nb.read_coords_file(str(tmp_path / "coord.dat"), spec.n_beads)
    assert np.allclose(back, xyz, rtol=1e-5, atol=1e-4)


def test_cli_end_to_end_on_reference_inputs(nb, tmp_path):
    """The drop-in executable on the reference's configuration.dat / polymer.dat:
    density_<step>.dat every Check_T steps, coord.dat, the timing line; the
    density files convert with the reference VTK rules, and a restart from
    coord.dat (read_file=1) continues."""
    shutil.copy(os.path.join(GOLDEN, "configuration.dat"), tmp_path)
    shutil.copy(os.path.join(GOLDEN, "polymer.dat"), tmp_path)
    exe = os.path.join(ROOT, "new_arch_b200", "_lib", "scmf")
    r = subprocess.run([exe, "-Steps_N=20", "-Check_T=10", "-seed=5"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "step 10 end to end dis" in r.stdout and "step 20 end to end dis" in r.stdout
    assert "time =" in r.stdout
    for step in (10, 20):
        lines = (tmp_path / f"density_{step}.dat").read_text().splitlines()
        assert lines[0] == "Nx=24, Ny=24, Nz=24" and lines[1] == "dx=0.166667, dy=0.166667, dz=0.166667"
        phi = np.array([[float(v) for v in l.split()[:2]] for l in lines[2:]])
        counts = phi * 409600 / 13824
        assert np.allclose(counts, np.round(counts), atol=1e-3)
        assert int(np.round(counts).sum()) == 409600
    assert sum(1 for _ in open(tmp_path / "coord.dat")) == 409600
    nb.vtk_convert(str(tmp_path / "density_20.dat"), str(tmp_path / "out.vtk"), 0)
    r2 = subprocess.run([exe, "-Steps_N=10", "-Check_T=10", "-Start_time=20", "-read_file=1", "-seed=5"],
                        cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r2.returncode == 0, r2.stderr
    assert "step 30 end to end dis" in r2.stdout


def test_reference_run_matches_oracle(nb):
    """The reference's own input files (12,800 chains of 32 beads, 24^3 cells,
    R_e units, SCMF0, omega skipped every tenth step) through the library, against
    the oracle: bit-exact positions and counts."""
    spec = nb.SystemSpec.from_files(os.path.join(GOLDEN, "configuration.dat"), os.path.join(GOLDEN, "polymer.dat"), 2024)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        compare_state(s, orc, "reference init")
        s.step(12)
        orc.step(12)
        compare_state(s, orc, "reference 12 steps")


# ------------------------------------------------ properties at full size
@pytest.mark.parametrize("which", ["large", "blend"])
def test_full_size_properties(nb, which):
    """At the benchmark sizes: counts are conserved, equal a recount of the
    final positions by the oracle's gridding, and omega equals the oracle's
    field of those counts."""
    from oracle.oracle import OracleSystem, set_threads
    from new_arch_b200.spec import blend_system, large_system
    spec = large_system() if which == "large" else blend_system()
    with nb.System(spec) as s:
        s.init_coords()
        s.step(4)
        cnt, om, xyz = s.counts(), s.omega(), s.coords()
        st = s.stats()
    assert int(cnt.sum()) == spec.n_beads
    assert st["step"] == 4 and st["total_moves"] == 4 * spec.n_beads
    # the cheap per-sweep read agrees on everything the sweep itself produced
    with nb.System(spec) as s2:
        s2.init_coords()
        s2.step(2)
        a, b = s2.sweep_stats(), s2.stats()
        assert a["step"] == b["step"] == 2 and a["total_accepts"] == b["total_accepts"]
        assert a["e_field"] == b["e_field"] and np.isnan(a["e_bond"]) and b["e_bond"] > 0
        assert s2.sweep_stats()["e_bond"] == b["e_bond"]
    set_threads(os.cpu_count() or 1)
    o = OracleSystem(spec)
    o.set_coords(xyz)
    o.set_step(4)
    o.reset_density()
    o.update_omega()
    set_threads(1)
    assert_counts_equal(cnt, o.counts(), which + " recount")
    assert_close(om, o.omega(), what=which + " omega")


def test_cli_checkpoint_resume_and_average(nb, tmp_path):
    """-checkpoint=1 then -read_file=2 continues exactly: coord.dat after 10 + 10
    steps equals coord.dat after 20 uninterrupted steps (byte for byte), and
    -Aver_T writes density_aver_<step>.dat beside each density file."""
    exe = os.path.join(ROOT, "new_arch_b200", "_lib", "scmf")
    a, b = tmp_path / "split", tmp_path / "whole"
    for d in (a, b):
        d.mkdir()
        shutil.copy(os.path.join(GOLDEN, "configuration.dat"), d)
        shutil.copy(os.path.join(GOLDEN, "polymer.dat"), d)
    run = lambda d, *args: subprocess.run([exe, "-seed=5", "-Check_T=10", *args], cwd=d, capture_output=True,
                                          text=True, timeout=300)
    r = run(a, "-Steps_N=10", "-checkpoint=1", "-Aver_T=2")
    assert r.returncode == 0, r.stderr
    assert (a / "checkpoint.bin").exists() and (a / "density_aver_10.dat").exists()
    info = nb.checkpoint_info(str(a / "checkpoint.bin"))
    assert info["step"] == 10 and info["avg_every"] == 2 and info["avg_samples"] == 5
    r = run(a, "-Steps_N=10", "-read_file=2", "-Aver_T=2")
    assert r.returncode == 0, r.stderr
    assert "step 20 end to end dis" in r.stdout
    r = run(b, "-Steps_N=20", "-Aver_T=2")
    assert r.returncode == 0, r.stderr
    assert filecmp.cmp(a / "coord.dat", b / "coord.dat", shallow=False)
    assert filecmp.cmp(a / "density_20.dat", b / "density_20.dat", shallow=False)
    assert filecmp.cmp(a / "density_aver_20.dat", b / "density_aver_20.dat", shallow=False)
    # the end-to-end line is the device reduction of the same positions
    line_a = [l for l in r.stdout.splitlines() if l.startswith("step 20 end")]
    assert line_a


def test_server_cancel_and_drain(nb):
    """A cancelled queued request never runs; a cancelled running one stops at
    a round boundary with its sweeps so far; the others finish as if alone;
    a drain with a tiny limit times out while work remains, then succeeds."""
    from new_arch_b200.server import Server
    from new_arch_b200.spec import diblock_melt
    sp = diblock_melt(3000, 16, 0.5, (16, 16, 16), 20.0, 50.0, seed=8)
    budget = int(sp.device_bytes() * 2.5)             # two systems at a time
    K = 5000
    with Server(budget, sweeps_per_round=2) as srv:
        ids = [srv.submit(sp, K) for _ in range(4)]
        srv.cancel(ids[3])                             # still queued: the budget holds two
        t0 = time.time()
        while srv.pending()[1] < 1 and time.time() - t0 < 30:
            time.sleep(0.001)
        srv.cancel(ids[0])                             # admitted first, so running now
        with pytest.raises(nb.ScmfError) as e:
            srv.drain(1)
        assert e.value.code == -7
        with pytest.raises(nb.ScmfError) as e:
            srv.cancel(12345)
        assert e.value.code == -1
        srv.drain(120_000)
        res = {r["id"]: r for r in srv.poll(16, 1000)}
    assert sorted(res) == sorted(ids)
    assert res[ids[3]]["status"] == -9 and res[ids[3]]["sweeps_done"] == 0 and res[ids[3]]["t_admit"] == 0
    assert res[ids[0]]["status"] == -9 and 0 <= res[ids[0]]["sweeps_done"] < K and res[ids[0]]["t_admit"] > 0
    cnt, st = _alone(nb, sp, K)
    for i in ids[1:3]:
        r = res[i]
        assert r["status"] == 0 and r["sweeps_done"] == K
        assert_counts_equal(r["counts"], cnt, "served counts after cancellations")
        assert r["accepts"] == st["total_accepts"]


def test_server_destroy_cancels_outstanding_work(nb):
    """Closing a server with requests queued and running returns at the next
    round boundary instead of finishing them all."""
    from new_arch_b200.server import Server
    from new_arch_b200.spec import diblock_melt
    sp = diblock_melt(3000, 16, 0.5, (16, 16, 16), 20.0, 50.0, seed=9)
    srv = Server(int(sp.device_bytes() * 2.5), sweeps_per_round=2)
    for _ in range(20):
        srv.submit(sp, 200_000)                      # hours of work if it all ran
    t0 = time.time()
    while srv.pending()[1] < 1 and time.time() - t0 < 30:
        time.sleep(0.001)
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 10


def test_bench_line_contract():
    """A short plain-form bench run prints one JSON line with every key of the
    benchmark contract, a roofline of the move kernel and sampled clocks."""
    import json
    import sys
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--forms", "plain", "--steps", "3", "--warmup",
                        "3", "--no-cpu-baseline"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "clocks", "gpu_launches"):
        assert k in d, k
    assert d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0 and d["gpu_launches"] == 6
    rf = d["roofline"]
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s" and 0 < rf["frac"] < 1.5
    assert abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-9
    assert d["e2e"]["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    import bench
    from new_arch_b200.spec import large_system
    assert d["config"] == bench.workload_config(large_system(seed=7))   # what the reference arm prints
