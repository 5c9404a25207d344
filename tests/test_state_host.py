"""CPU tests of the state around the hot path: the oracle's time-averaged
density and chain observables against independent numpy restatements, and the
checkpoint file format (header, sizes, checksum) read by the library's host
code without a GPU."""
import ctypes as C
import struct

import numpy as np
import pytest

import new_arch_b200 as nb
from new_arch_b200 import _lib
from new_arch_b200.spec import blend_system, diblock_melt
from oracle.oracle import OracleSystem


def _oracle(spec):
    o = OracleSystem(spec)
    o.init_coords()
    o.reset_density()
    o.update_omega()
    return o


# ------------------------------------------------------------ averaging
def test_oracle_average_sums_the_sampled_sweeps():
    spec = diblock_melt(120, 16, 0.4, (6, 5, 4), 20.0, 50.0, seed=8)
    a, b = _oracle(spec), _oracle(spec)
    a.average_start(3)
    a.step(10)
    want = np.zeros(spec.n_types * spec.n_cells, dtype=np.uint64)
    for s in range(1, 11):
        b.step(1)
        if s % 3 == 0:
            want += b.counts().astype(np.uint64)
    sums, n = a.average()
    assert n == 3
    assert np.array_equal(sums, want)
    a.average_sample()
    sums2, n2 = a.average()
    assert n2 == 4 and np.array_equal(sums2, want + a.counts().astype(np.uint64))
    a.average_start(0)
    assert a.average()[1] == 0


# ----------------------------------------------------------- observables
def _numpy_observables(xyz, ref, spec):
    out = []
    base = 0
    for a in spec.archs:
        L = a.length
        p = xyz[base:base + a.n_chains * L].astype(np.float64).reshape(a.n_chains, L, 3)
        r = ref[base:base + a.n_chains * L].astype(np.float64).reshape(a.n_chains, L, 3)
        base += a.n_chains * L
        cm = p.mean(axis=1)
        bonds = np.asarray(a.bonds).reshape(-1, 2)
        bv = p[:, bonds[:, 1], :] - p[:, bonds[:, 0], :]
        out.append({
            "re2": ((p[:, -1] - p[:, 0]) ** 2).mean(axis=0),
            "rg2": ((p - cm[:, None, :]) ** 2).mean(axis=1).mean(axis=0),
            "bond2": (bv ** 2).reshape(-1, 3).mean(axis=0),
            "msd": ((p - r) ** 2).reshape(-1, 3).mean(axis=0),
            "msd_com": ((cm - r.mean(axis=1)) ** 2).mean(axis=0),
        })
    return out


def test_oracle_observables_match_numpy():
    spec = blend_system(seed=3, n_chains=300, grid=(8, 8, 6))
    o = _oracle(spec)
    o.step(2)
    ref = o.coords().copy()
    o.analysis_reference()
    o.step(5)
    want = _numpy_observables(o.coords(), ref, spec)
    for ai in range(len(spec.archs)):
        got = o.analyze(ai)
        for k in ("re2", "rg2", "bond2", "msd", "msd_com"):
            np.testing.assert_allclose(got[k], want[ai][k], rtol=1e-9, err_msg=f"arch {ai} {k}")


def test_oracle_displacements_undefined_before_reference():
    spec = diblock_melt(20, 8, 0.5, (4, 4, 4), 10.0, 50.0, seed=1)
    o = _oracle(spec)
    got = o.analyze(0)
    assert np.all(np.isnan(got["msd"])) and np.all(np.isnan(got["msd_com"]))
    assert np.all(got["re2"] > 0)


# ------------------------------------------------------------ checkpoint
def _fnv1a64(data: bytes) -> int:
    h = 14695981039346656037
    for b in data:
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


HDR = "<I4i2iIqqQQQQQQdQQQ"


def _write_checkpoint(path, spec, step=7, avg_every=0, corrupt=None):
    h = spec.to_c()
    try:
        sh = C.c_uint64()
        _lib.check(_lib.lib().scmf_spec_hash(h, C.byref(sh)))
    finally:
        _lib.lib().scmf_spec_destroy(h)
    rng = np.random.default_rng(0)
    cells = spec.n_types * spec.n_cells
    payload = rng.standard_normal(3 * spec.n_beads).astype(np.float32).tobytes()
    payload += rng.standard_normal(cells).astype(np.float32).tobytes()
    if avg_every:
        payload += rng.integers(0, 1000, cells).astype(np.uint64).tobytes()
    hdr = struct.pack(HDR, 1, spec.n_types, spec.nx, spec.ny, spec.nz, spec.n_chains, len(spec.archs), avg_every,
                      spec.n_beads, spec.n_cells, spec.seed, sh.value, step, 5, 50, 700, -1.5,
                      3 if avg_every else 0, len(payload), _fnv1a64(payload))
    assert struct.calcsize(HDR) == 128 == C.sizeof(_lib.CheckpointHeader)
    blob = bytearray(b"SCMFCKPT" + hdr + payload)
    if corrupt == "payload":
        blob[-3] ^= 0x40
    elif corrupt == "magic":
        blob[0:8] = b"SCMFCKPX"
    elif corrupt == "truncate":
        blob = blob[:-5]
    elif corrupt == "version":
        blob[8] = 9
    with open(path, "wb") as f:
        f.write(blob)
    return sh.value


@pytest.mark.parametrize("avg_every", [0, 4])
def test_checkpoint_info_reads_the_documented_layout(tmp_path, avg_every):
    spec = diblock_melt(30, 8, 0.5, (4, 4, 4), 10.0, 50.0, seed=77)
    p = str(tmp_path / "ck.bin")
    sh = _write_checkpoint(p, spec, step=7, avg_every=avg_every)
    info = nb.checkpoint_info(p)
    assert info["version"] == 1 and info["step"] == 7 and info["seed"] == 77
    assert info["spec_hash"] == sh and info["n_beads"] == spec.n_beads and info["n_cells"] == spec.n_cells
    assert info["avg_every"] == avg_every and info["total_moves"] == 700 and info["e_field"] == -1.5


@pytest.mark.parametrize("corrupt,code", [("payload", -5), ("magic", -5), ("truncate", -5), ("version", -5)])
def test_checkpoint_info_rejects_damaged_files(tmp_path, corrupt, code):
    spec = diblock_melt(30, 8, 0.5, (4, 4, 4), 10.0, 50.0, seed=77)
    p = str(tmp_path / "ck.bin")
    _write_checkpoint(p, spec, corrupt=corrupt)
    with pytest.raises(nb.ScmfError) as e:
        nb.checkpoint_info(p)
    assert e.value.code == code


def test_spec_hash_tracks_trajectory_parameters():
    def hash_of(spec):
        h = spec.to_c()
        try:
            v = C.c_uint64()
            _lib.check(_lib.lib().scmf_spec_hash(h, C.byref(v)))
            return v.value
        finally:
            _lib.lib().scmf_spec_destroy(h)
    a = diblock_melt(30, 8, 0.5, (4, 4, 4), 10.0, 50.0, seed=1)
    assert hash_of(a) == hash_of(diblock_melt(30, 8, 0.5, (4, 4, 4), 10.0, 50.0, seed=2))  # seed is checked apart
    assert hash_of(a) != hash_of(diblock_melt(30, 8, 0.5, (4, 4, 4), 11.0, 50.0, seed=1))
    assert hash_of(a) != hash_of(diblock_melt(31, 8, 0.5, (4, 4, 4), 10.0, 50.0, seed=1))
    assert hash_of(a) != hash_of(diblock_melt(30, 8, 0.5, (4, 4, 5), 10.0, 50.0, seed=1))


# ------------------------------------------------ physics of the algorithm
def _ideal_chain_bond2(fault: bool) -> float:
    """<|b|^2> of field-free chains relaxed by the oracle from a third of the
    equilibrium bond length; the exact value is 3 / (2k)."""
    from oracle.oracle import set_threads
    import os
    spec = diblock_melt(1500, 8, 0.5, (8, 8, 8), 0.0, 0.0, seed=77, smc_a=0.1)
    spec.archs[0].init_sigma = 0.7 / np.sqrt(3.0) / 3.0
    set_threads(os.cpu_count() or 1)
    try:
        o = _oracle(spec)
        o.set_fault(fault)
        o.step(600)
        vals = []
        for _ in range(20):
            o.step(20)
            vals.append(o.analyze(0)["bond2"].sum())
    finally:
        set_threads(1)
    return float(np.mean(vals)) / (3.0 / (2.0 * spec.harmonic_normb))


def test_ideal_chain_statistics_detect_a_wrong_acceptance():
    """The statistics that the GPU physics test checks (tests/test_gpu_physics.py)
    hold for the oracle's algorithm and fail for a planted mistake: plain
    Metropolis on the bond energy with the drifted proposal, i.e. without the
    smart-MC correction."""
    assert abs(_ideal_chain_bond2(False) - 1.0) < 0.02
    assert abs(_ideal_chain_bond2(True) - 1.0) > 0.05
