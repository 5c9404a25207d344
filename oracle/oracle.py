"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is the checker the CUDA engine is compared against; only tests,
the smoke check and the benchmark's CPU-baseline leg import this module.  It
restates the reference algorithm (ren5885a/New_arch device_function.cu:140-207,
313-360, 373-412, 444-454, 479-508, 509-799; test.cpp:37-43) in plain C.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def _cpu_has_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return " fma " in flags and " avx2 " in flags
    except OSError:
        return False


def reference_dir() -> str | None:
    """The reference checkout the recipes in this folder read (the Makefile's
    REF, which the environment variable REF overrides), or None when it is not
    present on this machine."""
    try:
        r = subprocess.run(["make", "-s", "-C", _HERE, "print-ref"], check=True, capture_output=True, text=True)
    except (OSError, subprocess.CalledProcessError):
        return None
    path = r.stdout.strip()
    return path if path and os.path.isdir(path) else None


def build(ref: bool = False) -> None:
    """Compile the oracle (and the reference's vtk.c into _ref/ when asked)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", _HERE] + targets, check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    name = "liboracle.so" if _cpu_has_fma() else "liboracle_generic.so"
    path = os.path.join(_HERE, "_build", name)
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    vp, i32, i64, u32p, f32p, f64p = C.c_void_p, C.c_int, C.c_int64, C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.POINTER(C.c_double)
    L.orc_create.restype = vp
    L.orc_create.argtypes = [i32, i32, i32, i32, C.c_double, C.c_double, C.c_double, f64p, i32,
                             C.c_double, C.c_double, C.c_uint64, i32, i32]
    L.orc_add_arch.restype = i32
    L.orc_add_arch.argtypes = [vp, i32, i32, C.POINTER(C.c_int), i32, C.POINTER(C.c_int), C.c_double]
    L.orc_finalize.argtypes = [vp]
    L.orc_destroy.argtypes = [vp]
    L.orc_set_threads.argtypes = [i32]
    L.orc_get_threads.restype = i32
    L.orc_n_beads.restype = i64
    L.orc_n_beads.argtypes = [vp]
    L.orc_n_cells.restype = i64
    L.orc_n_cells.argtypes = [vp]
    L.orc_n_chains.argtypes = [vp]
    for fn in ("orc_init_coords", "orc_reset_density", "orc_update_omega"):
        getattr(L, fn).argtypes = [vp]
    L.orc_smc_move.argtypes = [vp, i32]
    L.orc_step.argtypes = [vp, i32]
    L.orc_set_step.argtypes = [vp, C.c_uint64]
    L.orc_set_coords.argtypes = [vp, f32p]
    L.orc_get_coords.argtypes = [vp, f32p]
    L.orc_get_counts.argtypes = [vp, u32p]
    L.orc_get_omega.argtypes = [vp, f32p]
    L.orc_set_omega.argtypes = [vp, f32p]
    L.orc_get_stats.argtypes = [vp, C.POINTER(OrcStats)]
    L.orc_average_start.argtypes = [vp, C.c_uint32]
    L.orc_average_sample.argtypes = [vp]
    L.orc_average_get.restype = C.c_uint64
    L.orc_average_get.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.orc_analysis_reference.argtypes = [vp]
    L.orc_set_fault.argtypes = [vp, i32]
    L.orc_analyze.restype = i32
    L.orc_analyze.argtypes = [vp, i32, C.POINTER(C.c_double)]
    L.orc_philox4x32_10.argtypes = [u32p, u32p, u32p]
    L.orc_logf.restype = C.c_float
    L.orc_logf.argtypes = [C.c_float]
    L.orc_log_lower_violations.restype = C.c_long
    L.orc_log_lower_violations.argtypes = [C.c_float, C.c_float, C.POINTER(C.c_float)]
    L.orc_normal.restype = C.c_float
    L.orc_normal.argtypes = [C.c_uint32]
    L.orc_normals3.argtypes = [u32p, f32p, f32p, f32p]
    L.orc_u01.restype = C.c_float
    L.orc_u01.argtypes = [C.c_uint32]
    L.orc_set_shard.argtypes = [vp, C.POINTER(C.c_int), i64]
    L.orc_field_from.argtypes = [vp, u32p]
    L.orc_trial_energy.restype = C.c_float
    L.orc_trial_energy.argtypes = [vp, i32, i32, f32p, f32p, f32p, C.c_float, C.c_float, C.c_float, f32p]
    L.orc_fold.restype = i32
    L.orc_fold.argtypes = [C.c_float, C.c_float, i32]
    _lib = L
    return L


class OrcStats(C.Structure):
    _fields_ = [("step", C.c_uint64), ("last_accepts", C.c_uint64), ("total_accepts", C.c_uint64),
                ("total_moves", C.c_uint64), ("e_bond", C.c_double), ("e_field", C.c_double)]


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(_p(c, C.c_uint32), _p(k, C.c_uint32), _p(out, C.c_uint32))
    return out


def logf(x: float) -> float:
    return lib().orc_logf(C.c_float(x))


def normal(w: int) -> float:
    """The standard normal of one 32-bit word (tabulated inverse CDF)."""
    return lib().orc_normal(C.c_uint32(w))


def normals3(w):
    a = np.ascontiguousarray(w, dtype=np.uint32)
    n = [C.c_float() for _ in range(3)]
    lib().orc_normals3(_p(a, C.c_uint32), *[C.byref(v) for v in n])
    return tuple(v.value for v in n)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


class OracleSystem:
    """One SCMF system held by the oracle.  Built from a SystemSpec
    (new_arch_b200.spec.SystemSpec-like object with the same fields)."""

    def __init__(self, spec):
        L = lib()
        xn = np.ascontiguousarray(spec.xn, dtype=np.float64).ravel()
        self._h = L.orc_create(spec.n_types, spec.nx, spec.ny, spec.nz, spec.lx, spec.ly, spec.lz,
                               _p(xn, C.c_double), spec.nref, spec.harmonic_normb, spec.smc_a,
                               spec.seed, spec.hamiltonian, spec.field_rule)
        if not self._h:
            raise ValueError("oracle: invalid system parameters")
        for a in spec.archs:
            mt = np.ascontiguousarray(a.mono_type, dtype=np.int32)
            bd = np.ascontiguousarray(a.bonds, dtype=np.int32).reshape(-1)
            if bd.size == 0:
                bd = np.zeros(2, dtype=np.int32)
            rc = L.orc_add_arch(self._h, a.length, a.n_chains, _p(mt, C.c_int), len(a.bonds),
                                _p(bd, C.c_int), a.init_sigma)
            if rc != 0:
                raise ValueError("oracle: invalid architecture")
        L.orc_finalize(self._h)
        self.n_types = spec.n_types
        self.n_beads = L.orc_n_beads(self._h)
        self.n_cells = L.orc_n_cells(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    def init_coords(self):
        lib().orc_init_coords(self._h)

    def set_coords(self, xyz):
        a = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1)
        assert a.size == 3 * self.n_beads
        lib().orc_set_coords(self._h, _p(a, C.c_float))

    def coords(self):
        out = np.empty(3 * self.n_beads, dtype=np.float32)
        lib().orc_get_coords(self._h, _p(out, C.c_float))
        return out.reshape(-1, 3)

    def set_step(self, s):
        lib().orc_set_step(self._h, int(s))

    def smc_move(self, n=1):
        lib().orc_smc_move(self._h, int(n))

    def reset_density(self):
        lib().orc_reset_density(self._h)

    def update_omega(self):
        lib().orc_update_omega(self._h)

    def step(self, n=1):
        lib().orc_step(self._h, int(n))

    def counts(self):
        out = np.empty(self.n_types * self.n_cells, dtype=np.uint32)
        lib().orc_get_counts(self._h, _p(out, C.c_uint32))
        return out

    def omega(self):
        out = np.empty(self.n_types * self.n_cells, dtype=np.float32)
        lib().orc_get_omega(self._h, _p(out, C.c_float))
        return out

    def set_omega(self, w):
        a = np.ascontiguousarray(w, dtype=np.float32).reshape(-1)
        lib().orc_set_omega(self._h, _p(a, C.c_float))

    def stats(self):
        st = OrcStats()
        lib().orc_get_stats(self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in OrcStats._fields_}

    def average_start(self, every):
        lib().orc_average_start(self._h, int(every))

    def average_sample(self):
        lib().orc_average_sample(self._h)

    def average(self):
        """(sums uint64 [n_types * n_cells], number of samples)"""
        out = np.zeros(self.n_types * self.n_cells, dtype=np.uint64)
        n = lib().orc_average_get(self._h, _p(out, C.c_uint64))
        return out, int(n)

    def set_shard(self, rng_base, n_beads_total):
        """Make this system a chain shard: rng_base[a] is the whole-system id of its
        first chain of architecture a; the field scaling uses n_beads_total."""
        a = np.ascontiguousarray(rng_base, dtype=np.int32)
        lib().orc_set_shard(self._h, _p(a, C.c_int), int(n_beads_total))

    def field_from(self, counts):
        """omega and the field energy of the given counts (the sum over shards)."""
        a = np.ascontiguousarray(counts, dtype=np.uint32)
        lib().orc_field_from(self._h, _p(a, C.c_uint32))

    def trial_energy(self, arch, b, xyz, n):
        """(energy change, proposed position) of one trial of bead b of a chain of
        architecture `arch` at positions xyz[L, 3] with the normals n[3]."""
        a = np.ascontiguousarray(np.asarray(xyz, dtype=np.float32).T)
        p = np.zeros(3, dtype=np.float32)
        e = lib().orc_trial_energy(self._h, int(arch), int(b), _p(a[0], C.c_float), _p(a[1], C.c_float),
                                   _p(a[2], C.c_float), float(n[0]), float(n[1]), float(n[2]), _p(p, C.c_float))
        return e, p

    def set_fault(self, no_smc: bool):
        """Plant a known mistake (drop the smart-MC correction) to test the tests."""
        lib().orc_set_fault(self._h, int(bool(no_smc)))

    def analysis_reference(self):
        lib().orc_analysis_reference(self._h)

    def analyze(self, arch):
        """Means of re2, rg2, bond2, msd, msd_com per component (x, y, z)."""
        out = np.empty(15, dtype=np.float64)
        if lib().orc_analyze(self._h, int(arch), _p(out, C.c_double)) != 0:
            raise ValueError("oracle: no such architecture")
        v = out.reshape(5, 3)
        return {k: v[i] for i, k in enumerate(("re2", "rg2", "bond2", "msd", "msd_com"))}
