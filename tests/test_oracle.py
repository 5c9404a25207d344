"""CPU tests of the oracle: known-answer vectors, the arithmetic building
blocks, the closed-form smart-MC energy, determinism of the OpenMP twin, and
the SCMF0 field against the reference's own density files."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as orc
from new_arch_b200.spec import Arch, SystemSpec, diblock_melt, interaction_matrix

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

# Philox4x32-10 known-answer vectors published with the algorithm
# (Salmon et al., SC'11; Random123 kat_vectors).
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    assert tuple(int(v) for v in orc.philox(ctr, key)) == want


def test_log_accuracy():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(2.0 ** -23, 1.0, 20000), rng.uniform(1.0, 1e6, 2000),
                         2.0 ** rng.uniform(-23, 0, 2000)]).astype(np.float32)
    worst = max(abs(orc.logf(float(x)) - math.log(float(x))) / max(abs(math.log(float(x))), 1e-30)
                for x in xs if abs(math.log(float(x))) > 1e-3)
    assert worst < 2.5e-7
    # absolute accuracy near 1, where log(x) -> 0
    near = np.float32(1.0) + np.arange(-2000, 2000, dtype=np.float32) * np.float32(2.0 ** -23)
    assert max(abs(orc.logf(float(x)) - math.log(float(x))) for x in near) < 2e-8


def _normal_words():
    """Random words, the two ends of the magnitude (f = 1 and f near 2^32), and
    words at and just below every segment boundary of the table, both signs."""
    rng = np.random.default_rng(4)
    words = [rng.integers(0, 2 ** 32, 60000, dtype=np.uint64),
             np.arange(0, 2048, dtype=np.uint64), np.uint64(0x7FFFFFFF) - np.arange(0, 2048, dtype=np.uint64)]
    for e in range(32):
        for j in range(16):
            f = (2 ** e) * (16 + j) // 16          # segment start (integer part), its odd neighbours
            for d in (-3, -1, 1, 3):
                v = f + d
                if 1 <= v < 2 ** 32 and v % 2 == 1:
                    words.append(np.array([(v - 1) // 2], dtype=np.uint64))
    w = np.concatenate(words)
    return np.concatenate([w, w | np.uint64(0x80000000)])


def test_normal_quantile_accuracy():
    """The normal of a word against an independent quantile (scipy's ndtri in
    FP64) of the same rounded variate: v = float32(2 (w mod 2^31) + 1) 2^-32,
    z = sign * -ndtri(v / 2).  Within 1.5e-7 relative above |z| = 0.5, within
    7.5e-8 absolute below; the tail reaches 6.3 sigma."""
    from scipy.special import ndtri
    words = _normal_words()
    f = ((words & np.uint64(0x7FFFFFFF)) * np.uint64(2) + np.uint64(1)).astype(np.float64).astype(np.float32)
    v = f.astype(np.float64) * 2.0 ** -32
    sign = np.where(words & np.uint64(0x80000000), -1.0, 1.0)
    want = sign * -ndtri(v / 2.0)
    got = np.array([orc.normal(int(w)) for w in words], dtype=np.float64)
    err = np.abs(got - want)
    big = np.abs(want) > 0.5
    assert (err[big] / np.abs(want[big])).max() < 1.5e-7
    assert err[~big].max() < 7.5e-8
    assert np.abs(want).max() > 6.3 and np.abs(got).max() > 6.3


def test_uniform_range():
    L = orc.lib()
    assert L.orc_u01(0) == pytest.approx(1.0)
    assert L.orc_u01(0xFFFFFFFF) == pytest.approx(2.0 ** -23)
    assert all(0.0 < L.orc_u01(int(w)) <= 1.0 for w in np.random.default_rng(3).integers(0, 2 ** 32, 1000))


def test_normals_statistics():
    rng = np.random.default_rng(4)
    n = np.array([orc.normals3(rng.integers(0, 2 ** 32, 4, dtype=np.uint64).astype(np.uint32)) for _ in range(40000)])
    assert abs(n.mean()) < 0.01
    assert abs(n.std() - 1.0) < 0.01
    # independence of the three components
    c = np.corrcoef(n.T)
    assert np.max(np.abs(c - np.eye(3))) < 0.02
    # fourth moment of a standard normal is 3
    assert abs((n ** 4).mean() - 3.0) < 0.1


def test_fold():
    L = orc.lib()
    for x, inv, n, want in [(0.0, 1.0, 16, 0), (15.99, 1.0, 16, 15), (16.0, 1.0, 16, 0), (-0.01, 1.0, 16, 15),
                            (-16.0, 1.0, 16, 0), (-16.5, 1.0, 16, 15), (100.2, 1.0, 16, 4), (-100.2, 1.0, 16, 11),
                            (0.5, 6.0, 24, 3), (-3.9, 6.0, 24, 0)]:
        assert L.orc_fold(x, inv, n) == want, (x, inv, n)


def test_closed_form_energy_matches_reference_expression():
    """The smart-MC energy the kernels evaluate, (A c/4)(c|d|^2 - 2 f.d), against
    the reference's literal bonded-energy + smc_deltaE expression in FP64."""
    import ctypes as C
    L = orc.lib()
    L.orc_dE_literal.restype = C.c_double
    L.orc_dE_literal.argtypes = [C.c_int] + [C.POINTER(C.c_float)] * 3 + [C.c_double, C.c_double]
    L.orc_dE_closed.restype = C.c_float
    L.orc_dE_closed.argtypes = [C.c_int] + [C.POINTER(C.c_float)] * 3 + [C.c_float, C.c_float]
    rng = np.random.default_rng(5)
    for _ in range(3000):
        deg = int(rng.integers(0, 5))
        k, A = float(rng.uniform(0.5, 50)), float(rng.uniform(0.001, 0.6))
        p = (rng.normal(size=3) * 4).astype(np.float32)
        q = (p + rng.normal(size=(max(deg, 1), 3)) * 0.6).astype(np.float32).reshape(-1)
        d = (rng.normal(size=3) * 0.5).astype(np.float32)
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        lit = L.orc_dE_literal(deg, ptr(q), ptr(p), ptr(d), k, A)
        cl = L.orc_dE_closed(deg, ptr(q), ptr(p), ptr(d), np.float32(2 * k), np.float32(A))
        # FP32 rounding of the two cancelling terms c|d|^2 and 2 f.d bounds the error
        f = 2 * k * (q.reshape(-1, 3)[:deg].astype(np.float64) - p).sum(axis=0)
        c = 2 * k * deg
        scale = A * c / 4 * (c * float(d @ d) + 2 * abs(float(f @ d))) + 1e-30
        assert abs(cl - lit) <= 1e-6 * scale + 1e-6, (deg, k, A, lit, cl, scale)


def _small_spec(**kw):
    return diblock_melt(300, 32, 0.4, (8, 9, 10), 20.0, 50.0, seed=11, **kw)


def test_openmp_twin_is_bit_identical():
    spec = _small_spec()
    runs = []
    for threads in (1, 4):
        orc.set_threads(threads)
        o = orc.OracleSystem(spec)
        o.init_coords()
        o.reset_density()
        o.update_omega()
        o.step(12)
        runs.append((o.coords(), o.counts(), o.omega(), o.stats()))
    orc.set_threads(1)
    (x1, c1, w1, s1), (x2, c2, w2, s2) = runs
    assert np.array_equal(x1.view(np.uint32), x2.view(np.uint32))
    assert np.array_equal(c1, c2)
    assert np.array_equal(w1.view(np.uint32), w2.view(np.uint32))
    assert s1["total_accepts"] == s2["total_accepts"]
    assert s1["e_field"] == pytest.approx(s2["e_field"], rel=1e-9)


def test_counts_conserved_and_match_positions():
    spec = _small_spec(field_rule=0)
    o = orc.OracleSystem(spec)
    o.init_coords()
    o.reset_density()
    o.update_omega()
    o.step(11)
    cnt = o.counts().reshape(spec.n_types, -1)
    assert int(cnt.sum()) == spec.n_beads
    # recount from the positions with numpy (floor mod n per axis)
    xyz = o.coords().astype(np.float64)
    ix = np.floor(xyz[:, 0]).astype(int) % spec.nx
    iy = np.floor(xyz[:, 1]).astype(int) % spec.ny
    iz = np.floor(xyz[:, 2]).astype(int) % spec.nz
    types = np.concatenate([np.tile(np.asarray(a.mono_type), a.n_chains) for a in spec.archs])
    want = np.zeros_like(cnt)
    np.add.at(want, (types, ix + spec.nx * (iy + spec.ny * iz)), 1)
    assert np.array_equal(cnt, want)


def test_field_rule_reference_skips_every_tenth():
    spec = _small_spec(field_rule=0)
    o = orc.OracleSystem(spec)
    o.init_coords()
    o.reset_density()
    o.update_omega()
    o.step(9)
    w9 = o.omega()
    o.step(1)            # step 10: omega not recomputed (test.cpp:42)
    assert np.array_equal(o.omega(), w9)
    o.step(1)            # step 11: recomputed
    assert not np.array_equal(o.omega(), w9)


def scmf0_reference(phi, xn, nref):
    """omega_field_update (device_function.cu:373-412) in FP64."""
    n = len(phi)
    w = np.zeros(n)
    for t in range(n):
        acc = sum(phi) - 1.0
        w[t] = xn[t + n * t] * acc / nref
        for s in range(n):
            if s != t:
                w[t] += -0.5 * xn[t + n * s] / nref * (phi[t] - phi[s])
    return w


def test_scmf0_mean_omega_matches_reference_density_files():
    """One cell holding 1/6/1 beads of three types has phi = 0.125/0.75/0.125,
    the per-type means of the reference's density_<step>.dat files; SCMF0 with
    kappaN=50, chiN=30, N_ref=32 must give their mean omega."""
    inv = json.load(open(os.path.join(GOLDEN, "density_invariants.json")))
    xn = interaction_matrix(3, 30.0, 50.0)
    mono = [0] + [1] * 6 + [2]
    spec = SystemSpec(3, 1, 1, 1, 1.0, 1.0, 1.0, xn, 32, 1.0, 0.0, archs=[Arch(8, 1, mono, [], 0.1)])
    o = orc.OracleSystem(spec)
    o.set_coords(np.full((8, 3), 0.5, np.float32))
    o.reset_density()
    o.update_omega()
    w = o.omega()
    for name, d in inv.items():
        assert d["counts_integral"] and d["bead_total_from_counts"] == 409600, name
        assert d["mean_phi"] == pytest.approx([0.125, 0.75, 0.125], abs=1e-6)
        if (d["nx"], d["ny"], d["nz"]) == (24, 24, 24):
            assert list(w) == pytest.approx(d["mean_omega"], abs=2e-6), name
        # SCMF0 structure for phi_A = phi_C: omega_A = omega_C = -omega_B / 2
        a, b, c = d["mean_omega"]
        assert a == pytest.approx(c, abs=1e-5) and a == pytest.approx(-b / 2, abs=2e-5)
    assert w == pytest.approx(scmf0_reference([0.125, 0.75, 0.125], xn, 32), abs=1e-6)


def test_log_lower_bounds_every_uniform():
    """The kernels reject a move without the logarithm (and without reading
    omega, with the omega span) when -dE <= log_lower(u), a bound linear in
    the bits of u.  That gives the oracle's outcome only if the bound lies at
    or below log_f(u) for every u the generator yields: checked over all 2^23
    of them with the constants of the device source."""
    import ctypes as C
    import re
    src = open(os.path.join(os.path.dirname(GOLDEN), "..", "new_arch_b200", "csrc", "scmf_math.cuh")).read()
    m = re.search(r"log_lower\(float u\).*?__fmaf_rn\(__uint2float_rn\(__float_as_uint\(u\)\), ([0-9a-fx.p+-]+)f, "
                  r"(-?[0-9a-fx.p+-]+)f\)", src, re.S)
    assert m, "log_lower not found"
    c1, c0 = float.fromhex(m.group(1)), float.fromhex(m.group(2))
    mm = C.c_float()
    bad = orc.lib().orc_log_lower_violations(c1, c0, C.byref(mm))
    assert bad == 0
    assert 0.0 < mm.value < 1e-3  # tight: a slack of 2^-12 and no more
    # the bound stays above -17, so dE >= 17 still rejects through it
    u_min = np.float32(2.0 ** -23)
    assert np.float32(u_min.view(np.uint32)) * np.float32(c1) + np.float32(c0) > -17.0


def test_multiply_high_fold_identity():
    """The device's branch-free fold for grid axes of 2 to 256 cells: with
    bias B = n * ceil(2^22 / n) and mag = ceil(2^32 / n), j = floor(t) + B and
    j - n * umulhi(j, mag) is floor(t) mod n.  Checked here in integers over
    every n, all small |floor(t)| and the ends of the valid range."""
    rng = np.random.default_rng(5)
    for n in range(2, 257):
        bias = n * (((1 << 22) + n - 1) // n)
        mag = np.uint64(((1 << 32) + n - 1) // n)
        fl = np.concatenate([np.arange(-3 * n, 3 * n), np.arange(-(1 << 22), -(1 << 22) + 2 * n),
                             np.arange((1 << 22) - 2 * n, 1 << 22), rng.integers(-(1 << 22), 1 << 22, 2000)])
        j = (fl + bias).astype(np.uint64)
        assert j.min() >= 0 and j.max() < (1 << 24)
        got = (j - ((j * mag) >> np.uint64(32)) * np.uint64(n)).astype(np.int64)
        assert np.array_equal(got, np.mod(fl, n)), n
