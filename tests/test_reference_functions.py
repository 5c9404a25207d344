"""The oracle against the reference's own functions, function by function.

oracle/Makefile's ref_harness target compiles the reference's
device_function.cu for the host (its CUDA and cuRAND names come from
oracle/ref_shim/) together with oracle/ref_harness.cpp, which calls:

* coord_to_index_unified_high (device_function.cu:313-360), the periodic
  cell fold, against the oracle's FP32 fold (orc_fold);
* omega_field_update (device_function.cu:373-412), the SCMF0 field in FP64,
  against the oracle's FP32 field of the same counts;
* trial_move_smc_arr + add_bond_forces_arr (device_function.cu:589-717) and
  calc_delta_energy_arr + calc_delta_bonded_energy_arr (:509-588), the
  smart-MC displacement and energy change for given Gaussian numbers, against
  the oracle's trial (closed-form bonded + smart-MC energy);
* mc_polymer_move_arr (device_function.cu:718-799), the whole sweep kernel,
  run on the host with a seeded generator in place of cuRAND, against the
  oracle's sweeps: equilibrium statistics (acceptance ratio, bond length,
  beads in favoured cells) agree within statistical error.

Tolerances state what FP32 against FP64 allows: folds identical except within
1e-5 cells of a cell face; omega within 1e-6 of its largest value; the
proposed position within 2e-6 (absolute, boxes of at most 32 cells plus a
relative 1e-6); the energy change within 1e-5 of the largest term of the
reference's sum (its bonded change and smart-MC term are of that size before
they cancel).  Skipped where the reference checkout is absent (the GPU boxes).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as orc_mod
from oracle.oracle import OracleSystem

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.join(os.path.dirname(HERE), "oracle")


@pytest.fixture(scope="module")
def ref():
    if orc_mod.reference_dir() is None:
        pytest.skip("reference checkout not present")
    subprocess.run(["make", "-s", "-C", ORACLE, "ref_harness"], check=True)
    L = C.CDLL(os.path.join(ORACLE, "_ref", "libref_harness.so"))
    d, f, i, i64 = C.c_double, C.POINTER(C.c_float), C.c_int, C.c_int64
    L.rh_fold.argtypes = [d, d, d, i, i, i, i, i64, f, C.POINTER(C.c_uint32)]
    L.rh_omega.argtypes = [i, i64, C.POINTER(C.c_int), C.POINTER(C.c_double), i, d, C.POINTER(C.c_double)]
    L.rh_trial.argtypes = [i, C.POINTER(C.c_int), f, i, d, d, f, d, d, d, i, i, i, i, C.POINTER(C.c_double), f,
                           C.POINTER(C.c_double)]
    L.rh_sweeps.restype = C.c_longlong
    L.rh_sweeps.argtypes = [i, i, C.POINTER(C.c_int), f, i, d, d, d, d, d, i, i, i, i, C.POINTER(C.c_double),
                            C.c_uint64]
    return L


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _spec(n_types, grid, box, archs, xn=None, nref=32, k=3.0 / (2 * 0.49), A=0.5):
    from new_arch_b200.spec import SystemSpec, interaction_matrix
    return SystemSpec(n_types, *grid, *box, xn or interaction_matrix(n_types, 25.0, 50.0), nref, k, A, seed=1,
                      archs=archs)


GRIDS = [((16, 16, 16), (16.0, 16.0, 16.0)),      # cell edge 1 (the synthetic workloads)
         ((24, 24, 24), (4.0, 4.0, 4.0)),         # the reference's configuration.dat (dx = 1/6)
         ((13, 7, 20), (6.5, 3.5, 20.0))]         # uneven axes, dx = 1/2


@pytest.mark.parametrize("grid,box", GRIDS)
def test_fold_matches_reference(ref, grid, box):
    rng = np.random.default_rng(5)
    n = 200_000
    lo, hi = -3.0 * np.array(box), 4.0 * np.array(box)
    xyz = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    # points on the cell faces of each axis (box edges included) and their FP32 neighbours
    extra = []
    for a, (g, b) in enumerate(zip(grid, box)):
        v = (np.arange(-2 * g, 3 * g + 1) * (b / g)).astype(np.float32)
        for w in (np.nextafter(v, np.float32(-np.inf)), v, np.nextafter(v, np.float32(np.inf))):
            pts = xyz[rng.integers(0, n, len(w))].copy()
            pts[:, a] = w
            extra.append(pts)
    xyz = np.concatenate([xyz] + extra).astype(np.float32)
    got = np.zeros(len(xyz), dtype=np.uint32)
    ref.rh_fold(*box, *grid, 1, len(xyz), _p(np.ascontiguousarray(xyz), C.c_float), _p(got, C.c_uint32))
    L = orc_mod.lib()
    inv = [np.float32(g / b) for g, b in zip(grid, box)]      # as the engine's constants (FP32 of n / L)
    ix = np.array([L.orc_fold(float(v), float(inv[0]), grid[0]) for v in xyz[:, 0]])
    iy = np.array([L.orc_fold(float(v), float(inv[1]), grid[1]) for v in xyz[:, 1]])
    iz = np.array([L.orc_fold(float(v), float(inv[2]), grid[2]) for v in xyz[:, 2]])
    n_cells = grid[0] * grid[1] * grid[2]
    want = n_cells + ix + grid[0] * (iy + grid[1] * iz)
    bad = np.nonzero(got != want)[0]
    if bad.size:
        # only FP32 / FP64 rounding at a cell face may differ
        t = xyz[bad].astype(np.float64) / (np.array(box) / np.array(grid))
        near = np.min(np.abs(t - np.round(t)), axis=1)
        assert np.all(near < 1e-5), f"{bad.size} folds differ away from cell faces: {xyz[bad[near >= 1e-5]][:3]}"
    if all(b == g for g, b in zip(grid, box)):
        # cell edge 1: x / dx is exact in both, so random points agree everywhere; the reference's
        # FP64 (k L + x) rounds only for tiny negative x just below a face
        assert np.all(bad >= n), "cell edge 1: random points must fold identically"
    assert np.sum(bad < n) <= 1e-4 * n, "too many random points on a cell face fold differently"


@pytest.mark.parametrize("n_types", [2, 3])
def test_field_matches_reference(ref, n_types):
    from new_arch_b200.spec import Arch, interaction_matrix
    rng = np.random.default_rng(7 + n_types)
    grid, box = (9, 8, 7), (9.0, 8.0, 7.0)
    n_cells = 9 * 8 * 7
    counts = rng.integers(0, 14, size=(n_types, n_cells))
    xn = interaction_matrix(n_types, 30.0, 50.0) if n_types == 3 else interaction_matrix(2, 25.0, 50.0)
    # one-bead chains of each type at the cell centres reproduce the counts
    archs = [Arch(1, int(counts[t].sum()), [t], [], 0.0) for t in range(n_types)]
    spec = _spec(n_types, grid, box, archs, xn=xn)
    cz, cy, cx = np.unravel_index(np.arange(n_cells), (7, 8, 9))
    centres = np.stack([cx, cy, cz], axis=1).astype(np.float32) + 0.5
    xyz = np.concatenate([np.repeat(centres, counts[t], axis=0) for t in range(n_types)])
    o = OracleSystem(spec)
    o.set_coords(xyz)
    o.reset_density()
    assert np.array_equal(o.counts(), counts.reshape(-1).astype(np.uint32))
    o.update_omega()
    scaling = n_cells / spec.n_beads
    w_ref = np.zeros(n_types * n_cells)
    c32 = np.ascontiguousarray(counts.reshape(-1), dtype=np.int32)
    ref.rh_omega(n_types, n_cells, _p(c32, C.c_int), _p(np.ascontiguousarray(xn, dtype=np.float64), C.c_double), 32,
                 scaling, _p(w_ref, C.c_double))
    w = o.omega().astype(np.float64)
    assert np.max(np.abs(w - w_ref)) <= 1e-6 * max(1.0, np.max(np.abs(w_ref)))


CASES = [
    # synthetic workload units: k = 3 / (2 b^2), b = 0.7, A = 0.5, cell edge 1
    dict(grid=(16, 16, 16), box=(16.0, 16.0, 16.0), k=3.0 / (2 * 0.49), A=0.5, sigma=0.7 / np.sqrt(3)),
    # the reference's configuration.dat: harmonic_normb = 1/(2 sigma^2) with sigma = 1/sqrt(3 (N-1)),
    # A = dt N/xi / N_ref = 0.17 / 32 (init_config.cu:480-484, 807), box 4 on 24^3 cells
    dict(grid=(24, 24, 24), box=(4.0, 4.0, 4.0), k=3.0 * 31 / 2, A=0.17 / 32, sigma=1 / np.sqrt(3 * 31)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_trial_matches_reference(ref, case):
    from new_arch_b200.spec import Arch, interaction_matrix
    cs = CASES[case]
    grid, box = cs["grid"], cs["box"]
    n_types, L = 2, 8
    n_cells = grid[0] * grid[1] * grid[2]
    types = [0] * 3 + [1] * 5
    spec = _spec(n_types, grid, box, [Arch(L, 1, types, [[i, i + 1] for i in range(L - 1)], cs["sigma"])],
                 k=cs["k"], A=cs["A"])
    o = OracleSystem(spec)
    rng = np.random.default_rng(11 + case)
    w32 = rng.normal(0.0, 0.8, n_types * n_cells).astype(np.float32)
    o.set_omega(w32)
    w64 = w32.astype(np.float64)
    t32 = np.ascontiguousarray(types, dtype=np.int32)
    inv = [np.float32(g / b) for g, b in zip(grid, box)]
    lib = orc_mod.lib()
    checked = 0
    for trial in range(3000):
        start = rng.random(3) * np.array(box)
        xyz = (start + np.cumsum(rng.normal(0.0, cs["sigma"], (L, 3)), axis=0)).astype(np.float32)
        if trial % 7 == 0:
            xyz -= np.float32(2.0) * np.array(box, dtype=np.float32)          # unwrapped, negative coordinates
        b = int(rng.integers(0, L))
        n = rng.normal(0.0, 1.0, 3).astype(np.float32)
        e_orc, p_orc = o.trial_energy(0, b, xyz, n)
        d_ref = np.zeros(3, dtype=np.float32)
        e_ref = np.zeros(2)
        pos = np.ascontiguousarray(xyz.reshape(-1))
        ref.rh_trial(L, _p(t32, C.c_int), _p(pos, C.c_float), b, cs["k"], cs["A"], _p(n, C.c_float), *box, *grid,
                     n_types, _p(w64, C.c_double), _p(d_ref, C.c_float), _p(e_ref, C.c_double))
        p_ref = (xyz[b] + d_ref).astype(np.float32)
        tol_p = 2e-6 + 1e-6 * np.abs(p_ref)
        assert np.all(np.abs(p_orc - p_ref) <= tol_p), (trial, p_orc, p_ref)
        # the same omega cells on both sides unless the proposal sits on a cell face
        new = xyz[b].astype(np.float64) + d_ref.astype(np.float64)
        cells_o = [lib.orc_fold(float(v), float(i), g) for v, i, g in zip(p_orc, inv, grid)]
        face = np.abs(new / (np.array(box) / np.array(grid)) - np.round(new / (np.array(box) / np.array(grid))))
        if np.min(face) < 1e-4:
            continue
        ref_cells = np.floor(new / (np.array(box) / np.array(grid))).astype(np.int64) % np.array(grid)
        assert list(ref_cells) == cells_o
        e_total = e_ref[0] + e_ref[1]
        # scale: the reference's bonded change and smart-MC term before they cancel
        scale = max(1.0, abs(e_ref[0]), abs(e_ref[1]))
        assert abs(e_orc - e_total) <= 1e-5 * scale, (trial, e_orc, e_total, e_ref)
        checked += 1
    assert checked > 2500


def _sweep_statistics(run, n_chains, L, blocks, per):
    """Per block of `per` sweeps: the acceptance ratio, and at its end the
    mean squared bond length and the fraction of A beads (the first half of
    each chain) in the cells of odd x, where the field favours them."""
    acc, b2, fav = [], [], []
    for blk in range(blocks):
        a, xyz = run(blk)
        c = xyz.reshape(n_chains, L, 3).astype(np.float64)
        acc.append(a / (per * n_chains * L))
        b2.append(np.mean(np.sum(np.diff(c, axis=1) ** 2, axis=2)))
        xa = np.floor(c[:, : L // 2, 0]).astype(np.int64) % 2
        fav.append(np.mean(xa == 1))
    return np.array(acc), np.array(b2), np.array(fav)


def test_sweeps_match_reference_statistics(ref):
    """The reference's whole sweep kernel, mc_polymer_move_arr
    (device_function.cu:718-799: per chain, L trials of beads picked at random
    with replacement, smart-MC proposals, Metropolis with exp), run on the host
    with a seeded generator in place of cuRAND, against the oracle's
    checkerboard sweeps of the same system: diblocks of 16 beads in a static
    field of +-0.5 alternating cell by cell along x, opposite for A and B
    beads.  The two update orders sample the same equilibrium, so after 400
    sweeps their acceptance ratios, mean squared bond lengths and fractions of
    A beads in favoured cells agree within statistical error (5 block standard
    errors).  The oracle with the smart-MC correction dropped (a mistake
    planted on purpose) does not."""
    from new_arch_b200.spec import Arch, interaction_matrix
    n_chains, L, G, A = 300, 16, 8, 0.2
    k = 3.0 / (2 * 0.49)
    types = [0] * 8 + [1] * 8
    spec = _spec(2, (G, G, G), (float(G),) * 3, [Arch(L, n_chains, types, [[j, j + 1] for j in range(L - 1)],
                                                     0.7 / np.sqrt(3.0))],
                 xn=interaction_matrix(2, 0.0, 0.0), nref=L, k=k, A=A)
    o = OracleSystem(spec)
    o.init_coords()
    x0 = o.coords().copy()
    prof = np.where(np.arange(G) % 2 == 0, 0.5, -0.5)                    # omega_A by x; exact in FP32
    w_a = np.broadcast_to(prof[None, None, :], (G, G, G)).reshape(-1)     # [z][y][x]
    w32 = np.concatenate([w_a, -w_a]).astype(np.float32)
    w64 = w32.astype(np.float64)
    t32 = np.ascontiguousarray(types, dtype=np.int32)
    pos = np.ascontiguousarray(x0.reshape(-1), dtype=np.float32)
    burn, blocks, per = 400, 30, 20

    def ref_run(n, seed):
        return ref.rh_sweeps(n_chains, L, _p(t32, C.c_int), _p(pos, C.c_float), n, k, A, float(G), float(G),
                             float(G), G, G, G, 2, _p(w64, C.c_double), seed)

    ref_run(burn, 1)
    r_acc, r_b2, r_fav = _sweep_statistics(lambda b: (ref_run(per, 100 + b), pos), n_chains, L, blocks, per)

    def oracle_stats(fault):
        orc = OracleSystem(spec)
        orc.set_coords(x0)
        orc.set_omega(w32)
        orc.set_fault(fault)
        orc.smc_move(burn)

        def run(_):
            a0 = orc.stats()["total_accepts"]
            orc.smc_move(per)
            return orc.stats()["total_accepts"] - a0, orc.coords()
        return _sweep_statistics(run, n_chains, L, blocks, per)

    def se(x):
        return x.std(axis=0) / np.sqrt(len(x))

    o_acc, o_b2, o_fav = oracle_stats(False)
    assert 0.05 < r_acc.mean() < 0.5   # moves are accepted often enough to equilibrate
    assert r_fav.mean() > 0.7          # the field does sort the beads
    for what, r, q in (("acceptance", r_acc, o_acc), ("bond length", r_b2, o_b2), ("favoured", r_fav, o_fav)):
        tol = 5 * np.hypot(se(r), se(q))
        assert abs(r.mean() - q.mean()) < tol, (what, r.mean(), q.mean(), tol)

    f_acc, f_b2, _ = oracle_stats(True)
    assert abs(r_b2.mean() - f_b2.mean()) > 10 * np.hypot(se(r_b2), se(f_b2))
