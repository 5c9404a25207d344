"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle.

Bead positions and density counts must be bit-identical; omega, energies
within 1e-6 relative.  Sizes are chosen so the single-threaded oracle finishes
in seconds."""
import numpy as np
import pytest

from tests._util import (assert_close, assert_coords_equal, assert_counts_equal, compare_state, oracle_for)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import new_arch_b200
    return new_arch_b200


def test_device_math_matches_oracle(nb):
    from new_arch_b200.system import debug_math
    from oracle import oracle as orc
    n = 1 << 16
    key = (0x12345678, 0x9abcdef0)
    words, logs, normals = debug_math(n, key)
    idx = np.random.default_rng(0).integers(0, n, 2000)
    for i in idx:
        w = orc.philox((int(i), 0, 0, 0), key)
        assert np.array_equal(words[i], w)
        assert np.float32(logs[i]).view(np.uint32) == np.float32(orc.logf(orc.lib().orc_u01(int(w[3])))).view(np.uint32)
        assert np.array_equal(np.asarray(normals[i], np.float32).view(np.uint32),
                              np.asarray(orc.normals3(w), np.float32).view(np.uint32))
    # statistical sanity of the device normals
    assert abs(float(normals.mean())) < 0.01
    assert abs(float(normals.std()) - 1.0) < 0.01


def test_init_grid_field(nb):
    spec = nb.spec.diblock_melt(300, 32, 0.5, (8, 8, 8), 20.0, 50.0, seed=42)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        compare_state(s, orc, "init")
        assert int(s.counts().sum()) == spec.n_beads


@pytest.mark.parametrize("rule", [0, 1])
def test_steps_bit_exact(nb, rule):
    spec = nb.spec.diblock_melt(250, 32, 0.3, (8, 10, 12), 25.0, 50.0, seed=7, field_rule=rule)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        for chunk in (1, 4, 7):      # crosses a step % 10 == 0 boundary
            s.step(chunk)
            orc.step(chunk)
            compare_state(s, orc, f"rule{rule} after {chunk}")


def test_reference_shaped_calls(nb):
    """smc_move -> reset_density_fields -> update_omega_fields_scmf0, as test.cpp:39-43."""
    spec = nb.spec.diblock_melt(120, 16, 0.5, (6, 6, 6), 15.0, 50.0, seed=3, field_rule=0)
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
            compare_state(s, orc, f"reference step {step}", energies=False)


def test_blend_mixed_lengths(nb):
    spec = nb.spec.blend_system(seed=11, n_chains=400, grid=(10, 10, 6))
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(6)
        orc.step(6)
        compare_state(s, orc, "blend")


@pytest.mark.parametrize("threads", [64, 128, 256])
def test_chains_across_warps(nb, threads):
    """Lengths whose ceil(L/2) does not divide 32 (48, 40, 24, 6, 5) run with
    chains laid across warp boundaries; in one batch beside lengths that fill
    warps exactly (32, 16), every system equals the oracle bit for bit."""
    from new_arch_b200.spec import diblock_melt
    lengths = (48, 40, 24, 6, 5, 32, 16)
    specs = [diblock_melt(max(3, int(7.8 * 6 * 6 * 5 / n)), n, 0.4, (6, 6, 5), 18.0, 50.0, seed=70 + n)
             for n in lengths]
    systems = [nb.System(sp) for sp in specs]
    for x in systems:
        x.init_coords()
    b = nb.Batch(systems, tune={"beads_per_tile": 1024, "threads_move": threads})
    b.step(4)
    for n, sp, x in zip(lengths, specs, systems):
        orc = oracle_for(sp)
        orc.step(4)
        compare_state(x, orc, f"L={n} threads={threads}")
    b.close()
    for x in systems:
        x.close()


@pytest.mark.parametrize("lengths", [(80,), (65, 100), (48, 96, 16)])
def test_long_linear_chains(nb, lengths):
    """Chains longer than 64 beads take the shared-memory kernel (each warp's
    chains staged with the even beads before the odd ones); every length in
    the system goes through it, against the oracle bit for bit."""
    from new_arch_b200.spec import SystemSpec, cell_units, diblock_arch, interaction_matrix
    k, sig = cell_units()
    archs = [diblock_arch(n, 0.5, max(2, int(7.8 * 8 * 8 * 6 / n / len(lengths))), sig) for n in lengths]
    spec = SystemSpec(2, 8, 8, 6, 8.0, 8.0, 6.0, interaction_matrix(2, 20.0, 50.0), 64, k, 0.5, 91,
                      nb.HAM_SCMF0, nb.FIELD_EVERY, 32, archs)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(5)
        orc.step(5)
        compare_state(s, orc, f"lengths {lengths}")


@pytest.mark.parametrize("threads", [64, 256])
@pytest.mark.parametrize("seeds", ["one", "same_high_word", "distinct_high_words"])
def test_chains_across_warps_key_modes(nb, threads, seeds):
    """Lengths laid across warps (48, 24, 12, 6) beside warp-filling ones
    (32, 16) in one batch, in every key mode and at two block sizes: each
    system equals the oracle bit for bit."""
    from new_arch_b200.spec import diblock_melt
    lengths = (48, 24, 12, 6, 32, 16)
    specs = [diblock_melt(max(3, int(7.8 * 8 * 6 * 5 / n)), n, 0.35, (8, 6, 5), 22.0, 50.0, seed=1)
             for n in lengths]
    for i, sp in enumerate(specs):
        sp.seed = {"one": 55, "same_high_word": 55 + i, "distinct_high_words": 55 + (i << 33)}[seeds]
    systems = [nb.System(sp) for sp in specs]
    for x in systems:
        x.init_coords()
    b = nb.Batch(systems, tune={"beads_per_tile": 1024, "threads_move": threads})
    b.step(4)
    for n, sp, x in zip(lengths, specs, systems):
        orc = oracle_for(sp)
        orc.step(4)
        compare_state(x, orc, f"L={n} threads={threads} seeds={seeds}")
    b.close()
    for x in systems:
        x.close()


def test_two_lengths_across_warps_one_system(nb):
    """One system of two architectures laid across warps (48 and 24 beads)."""
    from new_arch_b200.spec import SystemSpec, cell_units, diblock_arch, interaction_matrix
    k, sig = cell_units()
    spec = SystemSpec(2, 10, 8, 8, 10.0, 8.0, 8.0, interaction_matrix(2, 20.0, 50.0), 48, k, 0.5, 313,
                      nb.HAM_SCMF0, nb.FIELD_EVERY, 32, [diblock_arch(48, 0.3, 70, sig), diblock_arch(24, 0.5, 71, sig)])
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(5)
        orc.step(5)
        compare_state(s, orc, "L=48 and 24")


def test_chains_across_warps_alone(nb):
    from new_arch_b200.spec import diblock_melt
    spec = diblock_melt(700, 48, 0.3, (12, 10, 8), 25.0, 50.0, seed=48)
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        s.step(5)
        orc.step(5)
        compare_state(s, orc, "L=48 alone")


def test_branched_three_types_literal_field(nb):
    """A comb with side chains (greedy colouring), three monomer types, the
    literal field and 16-bit counts."""
    from new_arch_b200.spec import Arch, SystemSpec, interaction_matrix
    backbone = 12
    mono = [0] * backbone
    bonds = [[i, i + 1] for i in range(backbone - 1)]
    for j in range(0, backbone, 3):       # side chains of two beads at every third backbone bead
        a = len(mono)
        mono += [1, 2]
        bonds += [[j, a], [a, a + 1]]
    L = len(mono)
    spec = SystemSpec(3, 7, 6, 5, 7.0, 6.0, 5.0, interaction_matrix(3, 12.0, 40.0), 20, 3.0 / (2 * 0.49), 0.3,
                      seed=99, hamiltonian=1, field_rule=1, count_bits=16,
                      archs=[Arch(L, 60, mono, bonds, 0.7 / np.sqrt(3.0)),
                             Arch(8, 25, [2] * 8, [[i, i + 1] for i in range(7)], 0.5)])
    with nb.System(spec) as s:
        s.init_coords()
        orc = oracle_for(spec)
        compare_state(s, orc, "comb init")
        s.step(5)
        orc.step(5)
        compare_state(s, orc, "comb")


def test_set_coords_restart(nb):
    spec = nb.spec.diblock_melt(100, 24, 0.5, (6, 6, 6), 20.0, 50.0, seed=5)
    rng = np.random.default_rng(1)
    xyz = (rng.random((spec.n_beads, 3)) * 6.0 - 3.0).astype(np.float32)  # includes negative, unwrapped values
    from oracle.oracle import OracleSystem
    with nb.System(spec) as s:
        s.set_coords(xyz)
        s.set_step(40)
        orc = OracleSystem(spec)
        orc.set_coords(xyz)
        orc.set_step(40)
        orc.reset_density()
        orc.update_omega()
        assert_coords_equal(s.coords(), xyz, "round trip")
        s.step(3)
        orc.step(3)
        compare_state(s, orc, "restart")


def test_batch_bit_identical_to_alone(nb):
    specs = nb.spec.batched_mix(6, mix_seed=5, edge_scale=0.25)
    alone, batched = [], []
    for sp in specs:
        a = nb.System(sp)
        a.init_coords()
        a.step(5)
        alone.append((a.coords(), a.counts(), a.omega(), a.stats()))
        a.close()
    systems = [nb.System(sp) for sp in specs]
    for s in systems:
        s.init_coords()
    b = nb.Batch(systems, tune={"chains_per_tile": 7, "threads_move": 128, "persistent_ctas": 3})
    b.step(2)
    b.step(3)
    for s, (xyz, cnt, om, st) in zip(systems, alone):
        assert_coords_equal(s.coords(), xyz, "batched coords")
        assert_counts_equal(s.counts(), cnt, "batched counts")
        assert np.array_equal(s.omega(), om)
        g = s.stats()
        assert g["step"] == st["step"] == 5
        assert g["total_accepts"] == st["total_accepts"]
        assert_close([g["e_bond"]], [st["e_bond"]])
    b.close()
    for s in systems:
        s.close()


def _comb_spec(nb, seed):
    from new_arch_b200.spec import Arch, SystemSpec, interaction_matrix
    backbone = 9
    mono = [0] * backbone
    bonds = [[i, i + 1] for i in range(backbone - 1)]
    for j in range(0, backbone, 3):       # two-bead side chains at every third backbone bead
        a = len(mono)
        mono += [1, 1]
        bonds += [[j, a], [a, a + 1]]
    return SystemSpec(2, 6, 6, 5, 6.0, 6.0, 5.0, interaction_matrix(2, 15.0, 50.0), len(mono), 3.0 / (2 * 0.49), 0.5,
                      seed, nb.HAM_SCMF0, nb.FIELD_EVERY, 32, [Arch(len(mono), 60, mono, bonds, 0.7 / np.sqrt(3.0))])


@pytest.mark.parametrize("kernel", ["register", "long_chains", "any_graph"])
@pytest.mark.parametrize("seeds", ["one", "same_high_word", "distinct_high_words"])
def test_batch_key_modes_match_oracle(nb, seeds, kernel):
    """Systems batched into one launch take their Philox round keys from the
    kernel parameters when they share a seed, the second key word's only when
    they share the seed's upper 32 bits, and neither otherwise (each tile's
    key advanced in registers).  All three launch kinds equal the oracle, for
    each move kernel: a batch with a chain longer than 64 beads runs the
    long-chain kernel, one with a branched architecture the general one."""
    specs = nb.spec.batched_mix(3, mix_seed=11, edge_scale=0.25)
    if kernel == "long_chains":
        specs.append(nb.spec.diblock_melt(20, 80, 0.5, (6, 6, 6), 20.0, 50.0))
    elif kernel == "any_graph":
        specs.append(_comb_spec(nb, 0))
    for i, sp in enumerate(specs):
        sp.seed = {"one": 77, "same_high_word": 77 + i, "distinct_high_words": 77 + (i << 33)}[seeds]
    systems = [nb.System(sp) for sp in specs]
    for s in systems:
        s.init_coords()
    b = nb.Batch(systems, tune={"threads_move": 128})
    b.step(4)
    for i, (sp, s) in enumerate(zip(specs, systems)):
        orc = oracle_for(sp)
        orc.step(4)
        compare_state(s, orc, f"{kernel} {seeds} batch member {i}")
    b.close()
    for s in systems:
        s.close()


def test_autotune_keeps_state(nb):
    specs = nb.spec.batched_mix(3, mix_seed=9, edge_scale=0.25)
    systems = [nb.System(sp) for sp in specs]
    for s in systems:
        s.init_coords()
    before = [(s.coords(), s.counts(), s.stats()["step"]) for s in systems]
    b = nb.Batch(systems)
    t = b.autotune(1)
    assert t["threads_move"] in (128, 256, 512)
    for s, (xyz, cnt, st) in zip(systems, before):
        assert_coords_equal(s.coords(), xyz, "autotune restore")
        assert np.array_equal(s.counts(), cnt)
        assert s.stats()["step"] == st
    b.close()
    for s in systems:
        s.close()


def test_destroying_a_batched_system_is_deferred(nb):
    """A system destroyed while a batch still holds it stays alive until the
    batch is destroyed, so the batch keeps stepping correctly; it cannot join
    a new batch."""
    specs = nb.spec.batched_mix(3, mix_seed=13, edge_scale=0.25)
    systems = [nb.System(sp) for sp in specs]
    for s in systems:
        s.init_coords()
    b = nb.Batch(systems)
    held = systems[0].handle.value
    systems[0].close()                       # deferred: the batch still points at it
    b.step(3)
    orc = oracle_for(specs[1])
    orc.step(3)
    compare_state(systems[1], orc, "batch member after another member was destroyed")
    with pytest.raises(nb.ScmfError):
        import ctypes as C
        arr = (C.c_void_p * 1)(held)
        nb._lib.check(nb.lib().scmf_batch_create(arr, 1, None, None, C.byref(C.c_void_p())))
    b.close()                                # frees systems[0] now
    for s in systems[1:]:
        s.close()


def test_step_stats_equals_step_then_sweep_stats(nb):
    spec = nb.spec.diblock_melt(500, 16, 0.4, (8, 8, 8), 20.0, 50.0, seed=21)
    with nb.System(spec) as a, nb.System(spec) as b:
        a.init_coords()
        b.init_coords()
        for n in (1, 3):
            sa = a.step_stats(n)
            b.step(n)
            sb = b.sweep_stats()
            for k in ("step", "last_accepts", "total_accepts", "total_moves", "e_field", "error_word"):
                assert sa[k] == sb[k], k
        assert_counts_equal(a.counts(), b.counts(), "step_stats counts")


def test_edge_shapes(nb):
    """Single beads (no bonds), dimers, trimers, an architecture with no chains,
    and a system of a single chain: bit-exact against the oracle."""
    from new_arch_b200.spec import SystemSpec, cell_units, diblock_arch, homopolymer_arch, interaction_matrix
    k, sig = cell_units()
    cases = {
        "mixed short": [homopolymer_arch(1, 0, 300, sig), diblock_arch(2, 0.5, 200, sig),
                        diblock_arch(3, 0.34, 150, sig), homopolymer_arch(5, 1, 0, sig)],
        "one chain": [diblock_arch(32, 0.5, 1, sig)],
        # an odd-length architecture laid across warps with an odd chain count
        # shifts the next architecture to an odd bead: its pairs are not
        # float2-aligned, so the register kernel (which checks) moves them
        "odd offset": [diblock_arch(5, 0.4, 3, sig), diblock_arch(32, 0.5, 40, sig)],
        "one bead": [homopolymer_arch(1, 1, 1, sig)],
    }
    for name, archs in cases.items():
        spec = SystemSpec(2, 5, 4, 3, 5.0, 4.0, 3.0, interaction_matrix(2, 20.0, 50.0), 8, k, 0.5, 404,
                          nb.HAM_SCMF0, nb.FIELD_EVERY, 32, archs)
        with nb.System(spec) as s:
            s.init_coords()
            orc = oracle_for(spec)
            compare_state(s, orc, name + " init")
            s.step(6)
            orc.step(6)
            compare_state(s, orc, name)
            assert int(s.counts().sum()) == spec.n_beads
