"""Shared helpers of the parity tests: run the same spec on the GPU engine and
on the CPU oracle and compare.  Positions and counts must be bit-identical;
omega and energies within 1e-6 relative."""
from __future__ import annotations

import numpy as np

RTOL = 1e-6  # fields and energies


def bits(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_coords_equal(gpu_xyz, orc_xyz, what=""):
    g, o = bits(gpu_xyz).reshape(-1), bits(orc_xyz).reshape(-1)
    if not np.array_equal(g, o):
        bad = np.nonzero(g != o)[0]
        i = bad[0]
        raise AssertionError(f"{what}: {bad.size} coordinate words differ; first at {i}: "
                             f"gpu {np.asarray(gpu_xyz).reshape(-1)[i]!r} oracle {np.asarray(orc_xyz).reshape(-1)[i]!r}")


def assert_counts_equal(g, o, what=""):
    g, o = np.asarray(g), np.asarray(o)
    if not np.array_equal(g, o):
        bad = np.nonzero(g != o)[0]
        raise AssertionError(f"{what}: {bad.size} counts differ; first at {bad[0]}: gpu {g[bad[0]]} oracle {o[bad[0]]}")


def assert_close(g, o, rtol=RTOL, what=""):
    g = np.asarray(g, dtype=np.float64)
    o = np.asarray(o, dtype=np.float64)
    scale = max(1.0, float(np.max(np.abs(o))) if o.size else 1.0)
    err = float(np.max(np.abs(g - o))) / scale if o.size else 0.0
    assert err <= rtol, f"{what}: max relative error {err:.3e} > {rtol}"


def oracle_for(spec):
    from oracle.oracle import OracleSystem
    orc = OracleSystem(spec)
    orc.init_coords()
    orc.reset_density()
    orc.update_omega()
    return orc


def compare_state(sysm, orc, what="", energies=True):
    assert_coords_equal(sysm.coords(), orc.coords(), what + " coords")
    assert_counts_equal(sysm.counts(), orc.counts(), what + " counts")
    assert_close(sysm.omega(), orc.omega(), what=what + " omega")
    if energies:
        gs, os_ = sysm.stats(), orc.stats()
        assert gs["step"] == os_["step"], f"{what}: step {gs['step']} vs {os_['step']}"
        assert gs["total_accepts"] == os_["total_accepts"], f"{what}: accepts {gs['total_accepts']} vs {os_['total_accepts']}"
        assert_close([gs["e_bond"]], [os_["e_bond"]], what=what + " e_bond")
        assert_close([gs["e_field"]], [os_["e_field"]], what=what + " e_field")
