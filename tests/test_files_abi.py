"""CPU tests of the library's host side: every C-ABI symbol is exported, the
reference's input files parse to the reference's derived constants, the VTK
converter reproduces the reference's vtk.c byte for byte, coord.dat round trips,
and malformed inputs fail with an error code (no GPU needed)."""
import ctypes as C
import filecmp
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import new_arch_b200 as nb
from new_arch_b200 import _lib
from new_arch_b200.spec import SystemSpec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
from oracle.oracle import reference_dir

REF = reference_dir() or ""
HAS_GPU = False
try:
    import torch
    HAS_GPU = torch.cuda.is_available()
except Exception:
    pass


def header_symbols():
    text = open(os.path.join(ROOT, "include", "scmf.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(scmf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) > 40
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    # and the Python binding declares a signature for each
    assert not [s for s in syms if s not in _lib.SIGNATURES], [s for s in syms if s not in _lib.SIGNATURES]


def test_version_string():
    assert b"sm_100a" in _lib.lib().scmf_version()


def test_parse_reference_inputs():
    spec = SystemSpec.from_files(os.path.join(GOLDEN, "configuration.dat"), os.path.join(GOLDEN, "polymer.dat"), 1)
    assert (spec.n_types, spec.nx, spec.ny, spec.nz) == (2, 24, 24, 24)
    assert (spec.lx, spec.ly, spec.lz) == (4.0, 4.0, 4.0)
    assert spec.xn == [50.0, 30.0, 30.0, 50.0]
    assert spec.nref == 32
    # harmonic_normb = 1/(2 sigma^2), sigma = 1/sqrt(3(N_ref-1)) (init_config.cu:480-484)
    assert spec.harmonic_normb == pytest.approx(3 * 31 / 2)
    # A = dt*N/xi / N_ref (init_config.cu:807)
    assert spec.smc_a == pytest.approx(0.17 / 32)
    assert spec.field_rule == nb.FIELD_REFERENCE and spec.hamiltonian == nb.HAM_SCMF0
    (a,) = spec.archs
    assert (a.length, a.n_chains) == (32, 12800)
    assert list(a.mono_type) == [1] * 16 + [0] * 16
    assert sorted(map(tuple, a.bonds)) == [(i, i + 1) for i in range(31)]
    assert a.init_sigma == pytest.approx(1 / np.sqrt(3 * 31))
    assert spec.n_beads == 409600


def test_parse_three_type_configuration():
    spec = SystemSpec.from_files(os.path.join(GOLDEN, "configuration_3types.dat"), os.path.join(GOLDEN, "polymer.dat"), 1)
    assert spec.n_types == 3
    assert spec.xn == [50.0, 30.0, 30.0, 30.0, 50.0, 30.0, 30.0, 30.0, 50.0]


def test_parse_errors(tmp_path):
    good_cfg = open(os.path.join(GOLDEN, "configuration.dat")).read()
    good_poly = open(os.path.join(GOLDEN, "polymer.dat")).read()
    cases = {
        "cfg_missing_box": (good_cfg.replace("D0 =", "DX ="), good_poly, -5),
        "poly_bad_count": (good_cfg, good_poly.replace("Number of total polymer:12800", "Number of total polymer:12"), -5),
        "poly_type_out_of_range": (good_cfg, good_poly.replace("Monomer type: 1 1", "Monomer type: 7 1"), -5),
        "truncated_matrix": (good_cfg, "\n".join(good_poly.splitlines()[:12]), -5),
    }
    for name, (cfg, poly, code) in cases.items():
        c, p = tmp_path / (name + ".cfg"), tmp_path / (name + ".poly")
        c.write_text(cfg)
        p.write_text(poly)
        with pytest.raises(nb.ScmfError) as e:
            SystemSpec.from_files(str(c), str(p), 1)
        assert e.value.code == code, name
    with pytest.raises(nb.ScmfError) as e:
        SystemSpec.from_files(str(tmp_path / "nope.dat"), str(tmp_path / "nope2.dat"), 1)
    assert e.value.code == -4


def test_spec_validation_errors():
    from new_arch_b200.spec import diblock_melt
    bad = diblock_melt(10, 8, 0.5, (4, 4, 4), 10.0, 50.0)
    bad.count_bits = 16
    bad.archs[0].n_chains = 10000  # 80,000 beads do not fit 16-bit counts
    h = bad.to_c()
    info = _lib.SpecInfo()
    _lib.check(_lib.lib().scmf_spec_get_info(h, C.byref(info)))
    assert info.n_beads == 80000
    out = C.c_void_p()
    rc = _lib.lib().scmf_system_create(h, None, C.byref(out))
    _lib.lib().scmf_spec_destroy(h)
    assert rc == -1 and b"16-bit" in _lib.lib().scmf_last_error()
    # an axis longer than the exact range of the FP32 fold allows
    long_axis = diblock_melt(10, 8, 0.5, ((1 << 20) + 1, 2, 1), 10.0, 50.0)
    h = long_axis.to_c()
    rc = _lib.lib().scmf_system_create(h, None, C.byref(out))
    _lib.lib().scmf_spec_destroy(h)
    assert rc == -1 and b"grid axis" in _lib.lib().scmf_last_error()
    # a negative chain count is refused where it is given
    neg = diblock_melt(10, 8, 0.5, (4, 4, 4), 10.0, 50.0)
    neg.archs[0].n_chains = -3
    with pytest.raises(nb.ScmfError) as e:
        h = neg.to_c()
        try:
            _lib.check(_lib.lib().scmf_system_create(h, None, C.byref(out)))
        finally:
            _lib.lib().scmf_spec_destroy(h)
    assert e.value.code == -1


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_no_device_is_an_error_not_a_fallback():
    from new_arch_b200.spec import diblock_melt
    with pytest.raises(nb.ScmfError) as e:
        nb.System(diblock_melt(10, 8, 0.5, (4, 4, 4), 10.0, 50.0))
    assert e.value.code == -2


def test_vtk_converter_known_answer(tmp_path):
    shutil.copy(os.path.join(GOLDEN, "density_240000_z3.dat"), tmp_path)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        nb.vtk_convert("density_240000_z3.dat", "mine.vtk")
    finally:
        os.chdir(cwd)
    assert filecmp.cmp(tmp_path / "mine.vtk", os.path.join(GOLDEN, "density_240000_z3.vtk"), shallow=False)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "out.vtk")), reason="reference checkout not mounted")
def test_vtk_converter_full_reference_file(tmp_path):
    shutil.copy(os.path.join(REF, "density_240000.dat"), tmp_path)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        nb.vtk_convert("density_240000.dat", "out.vtk")
    finally:
        os.chdir(cwd)
    assert filecmp.cmp(tmp_path / "out.vtk", os.path.join(REF, "out.vtk"), shallow=False)


def test_vtk_cli_matches_reference_argument_rules(tmp_path):
    exe = os.path.join(ROOT, "new_arch_b200", "_lib", "scmf_vtk")
    shutil.copy(os.path.join(GOLDEN, "density_240000_z3.dat"), tmp_path)
    r = subprocess.run([exe, "density_240000_z3.dat"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("2\n")
    assert filecmp.cmp(tmp_path / "out.vtk", os.path.join(GOLDEN, "density_240000_z3.vtk"), shallow=False)
    r = subprocess.run([exe, "missing.dat", "x.vtk"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode != 0 and "cannot open" in r.stderr


def test_vtk_auto_value_count(tmp_path):
    # a two-type density file: six values per point (vtk.c) misreads it, 'auto' does not
    p = tmp_path / "d.dat"
    lines = ["Nx=2, Ny=1, Nz=1\n", "dx=1, dy=1, dz=1\n", "0.5 0.25 1 2 \n", "0.75 0.125 3 4 \n"]
    p.write_text("".join(lines))
    nb.vtk_convert(str(p), str(tmp_path / "a.vtk"), 0)
    body = (tmp_path / "a.vtk").read_text().splitlines()
    assert body[-1].split() == ["0.2500", "0.6250"]


def test_coord_file_round_trip(tmp_path):
    xyz = (np.random.default_rng(0).normal(size=(50, 3)) * 7).astype(np.float32)
    p = tmp_path / "coord.dat"
    with open(p, "w") as f:
        for r in xyz:
            f.write("%g %g %g\n" % tuple(float(v) for v in r))
    got = nb.read_coords_file(str(p), 40, skip=10)
    assert np.allclose(got, xyz[10:], rtol=1e-5, atol=1e-5)
    with pytest.raises(nb.ScmfError) as e:
        nb.read_coords_file(str(p), 60)
    assert e.value.code == -5


def test_cli_refuses_multi_gpu(tmp_path):
    exe = os.path.join(ROOT, "new_arch_b200", "_lib", "scmf")
    r = subprocess.run([exe, "-GPU_N=2"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 2 and "one GPU" in r.stderr


def test_bench_reference_arm_contract():
    """bench.py --impl reference times the CPU port on this host and prints one
    JSON line with the keys the benchmark contract names; a rank other than 0
    prints nothing and exits 0."""
    import json
    import sys
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # the same workload config as the GPU arm prints (bench.workload_config of the large system)
    import bench
    from new_arch_b200.spec import large_system
    assert d["config"] == bench.workload_config(large_system(seed=7))
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=120, cwd=ROOT, env=env)
    assert r.returncode == 0 and not [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
