"""Python mirror of the engine's C ABI: one SCMF system on the GPU, batches of
systems, and the reference-shaped step pieces.

Method names follow the reference's host functions so a caller of the
reference finds the same pieces: smc_move (smc.cu:3-72),
reset_density_fields (mesh.cu:161-190), update_omega_fields_scmf0
(mesh.cu:217-248), io_out_density / io_out_coord (io.cpp:4-56, 95-118).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, List, Optional

import numpy as np

from . import _lib
from ._lib import check, lib
from .spec import SystemSpec


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(C.POINTER(t))


class System:
    """An SCMF system resident on the current CUDA device."""

    def __init__(self, spec: SystemSpec, stream: Optional[int] = None):
        L = lib()
        self.spec = spec
        h = spec.to_c()
        try:
            self._h = C.c_void_p()
            check(L.scmf_system_create(h, C.c_void_p(stream) if stream else None, C.byref(self._h)))
        finally:
            L.scmf_spec_destroy(h)
        info = _lib.SpecInfo()
        check(L.scmf_system_get_info(self._h, C.byref(info)))
        self.n_beads = info.n_beads
        self.n_cells = info.n_cells
        self.n_types = info.n_types
        self.n_chains = info.n_chains
        self.n_arch = info.n_arch

    # -------------------------------------------------------------- lifetime
    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().scmf_system_destroy(h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def stream(self) -> int:
        st = C.c_void_p()
        check(lib().scmf_system_stream(self._h, C.byref(st)))
        return st.value or 0

    # ----------------------------------------------------------------- state
    def init_coords(self) -> None:
        check(lib().scmf_init_coords(self._h))

    def set_coords(self, xyz) -> None:
        a = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1)
        check(lib().scmf_set_coords(self._h, _ptr(a, C.c_float), a.size))

    def coords(self) -> np.ndarray:
        out = np.empty(3 * self.n_beads, dtype=np.float32)
        check(lib().scmf_get_coords(self._h, _ptr(out, C.c_float), out.size))
        return out.reshape(-1, 3)

    def set_step(self, step: int) -> None:
        check(lib().scmf_set_step(self._h, int(step)))

    def counts(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Per-type cell counts [n_types * n_cells] (uint32), into `out` when
        given (e.g. a view of page-locked memory, which copies fastest)."""
        n = self.n_types * self.n_cells
        if out is None:
            out = np.empty(n, dtype=np.uint32)
        if out.dtype != np.uint32 or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"counts output must be a contiguous uint32 array of {n} elements")
        check(lib().scmf_get_counts(self._h, _ptr(out, C.c_uint32), out.size))
        return out

    def omega(self) -> np.ndarray:
        out = np.empty(self.n_types * self.n_cells, dtype=np.float32)
        check(lib().scmf_get_omega(self._h, _ptr(out, C.c_float), out.size))
        return out

    def set_omega(self, w) -> None:
        a = np.ascontiguousarray(w, dtype=np.float32).reshape(-1)
        check(lib().scmf_set_omega(self._h, _ptr(a, C.c_float), a.size))

    def stats(self) -> dict:
        st = _lib.Stats()
        check(lib().scmf_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.Stats._fields_ if k != "reserved"}

    def sweep_stats(self) -> dict:
        """Step, accepts and field energy of the last sweep (one small read; no
        bond-energy pass, e_bond is NaN unless current)."""
        st = _lib.Stats()
        check(lib().scmf_get_sweep_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.Stats._fields_ if k != "reserved"}

    # ----------------------------------------------------------------- steps
    def step(self, n_sweeps: int = 1) -> None:
        check(lib().scmf_step(self._h, int(n_sweeps)))

    def step_stats(self, n_sweeps: int = 1) -> dict:
        """n sweeps, then the statistics of the last one, in one round trip."""
        st = _lib.Stats()
        check(lib().scmf_step_stats(self._h, int(n_sweeps), C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.Stats._fields_ if k != "reserved"}

    def step_async(self, n_sweeps: int = 1) -> None:
        check(lib().scmf_step_async(self._h, int(n_sweeps)))

    def step_stats_async(self, n_sweeps: int, host_out_address: int) -> None:
        """n sweeps and a copy of their statistics into the scmf_stats at
        host_out_address (page-locked memory), enqueued without waiting; read
        it with stats_at() after synchronize()."""
        check(lib().scmf_step_stats_async(self._h, int(n_sweeps), C.c_void_p(host_out_address)))

    @staticmethod
    def stats_at(address: int) -> dict:
        st = _lib.Stats.from_address(address)
        return {k: getattr(st, k) for k, _ in _lib.Stats._fields_ if k != "reserved"}

    def step_profiled(self, n_sweeps: int = 1):
        """Runs n sweeps launch by launch with CUDA events; returns the summed
        device milliseconds of the move+grid kernel, of the field kernel, and
        the device time from the first launch to the end of the last."""
        a, b, t = C.c_float(), C.c_float(), C.c_float()
        check(lib().scmf_step_profiled(self._h, int(n_sweeps), C.byref(a), C.byref(b), C.byref(t)))
        return a.value, b.value, t.value

    def synchronize(self) -> None:
        check(lib().scmf_synchronize(self._h))

    def smc_move(self, n_sweeps: int = 1) -> None:
        check(lib().scmf_smc_move(self._h, int(n_sweeps)))

    def reset_density_fields(self) -> None:
        check(lib().scmf_reset_density_fields(self._h))

    def update_omega_fields_scmf0(self) -> None:
        check(lib().scmf_update_omega_fields_scmf0(self._h))

    # ---------------------------------------------------------------- output
    def io_out_density(self, step: int, path: Optional[str] = None) -> None:
        check(lib().scmf_write_density(self._h, path.encode() if path else None, int(step)))

    def io_out_coord(self, path: str = "coord.dat") -> None:
        check(lib().scmf_write_coords(self._h, path.encode()))

    # --------------------------------------------- time-averaged density
    def average_start(self, every: int = 1) -> None:
        """Sum the counts of every sweep s with s % every == 0 (0 stops)."""
        check(lib().scmf_average_start(self._h, int(every)))

    def average_sample(self) -> None:
        check(lib().scmf_average_sample(self._h))

    def average(self):
        """(sums uint64 [n_types * n_cells], number of samples)"""
        out = np.empty(self.n_types * self.n_cells, dtype=np.uint64)
        n = C.c_uint64()
        check(lib().scmf_average_get(self._h, _ptr(out, C.c_uint64), out.size, C.byref(n)))
        return out, n.value

    def io_out_aver_density(self, step: int, path: Optional[str] = None) -> None:
        check(lib().scmf_write_average_density(self._h, path.encode() if path else None, int(step)))

    # ------------------------------------------------------- checkpoints
    def checkpoint_write(self, path: str) -> None:
        check(lib().scmf_checkpoint_write(self._h, path.encode()))

    def checkpoint_read(self, path: str) -> None:
        check(lib().scmf_checkpoint_read(self._h, path.encode()))

    # -------------------------------------------------------- validation
    def validate(self, raise_on_error: bool = True) -> dict:
        """Device-side state checks (finite and in-range positions, counts equal
        to a fresh gridding and conserved per type, finite omega)."""
        v = _lib.Validation()
        rc = lib().scmf_validate(self._h, C.byref(v))
        if raise_on_error:
            check(rc)
        d = {k: getattr(v, k) for k, _ in _lib.Validation._fields_ if k != "reserved"}
        d["ok"] = rc == 0
        return d

    # ---------------------------------------------------------- analysis
    def analysis_reference(self) -> None:
        """Current positions become the origin of the displacements."""
        check(lib().scmf_analysis_reference(self._h))

    def analyze(self) -> list:
        """Per architecture: re2, rg2, bond2, msd, msd_com as (x, y, z, total)
        means, plus n_chains, n_beads, n_bonds and the acceptance ratio."""
        n = self.n_arch
        arr = (_lib.Observables * n)()
        check(lib().scmf_analyze(self._h, arr, n))
        out = []
        for o in arr:
            d = {k: np.array(list(getattr(o, k))) for k in ("re2", "rg2", "bond2", "msd", "msd_com")}
            d.update(arch=o.arch, n_chains=o.n_chains, n_beads=o.n_beads, n_bonds=o.n_bonds, acc_ratio=o.acc_ratio)
            out.append(d)
        return out


def checkpoint_info(path: str) -> dict:
    """Header of a checkpoint file, after checking its magic, sizes and checksum."""
    h = _lib.CheckpointHeader()
    check(lib().scmf_checkpoint_info(path.encode(), C.byref(h)))
    return {k: getattr(h, k) for k, _ in _lib.CheckpointHeader._fields_}


def read_coords_file(path: str, n_beads: int, skip: int = 0) -> np.ndarray:
    out = np.empty(3 * n_beads, dtype=np.float32)
    check(lib().scmf_read_coords_file(path.encode(), int(skip), _ptr(out, C.c_float), out.size))
    return out.reshape(-1, 3)


def vtk_convert(density_path: str, vtk_path: str, values_per_point: int = 6) -> None:
    check(lib().scmf_vtk_convert(density_path.encode(), vtk_path.encode(), int(values_per_point)))


class Batch:
    """Many systems advanced together by one persistent launch per phase."""

    def __init__(self, systems: Iterable[System], tune: Optional[dict] = None, stream: Optional[int] = None):
        self.systems: List[System] = list(systems)
        arr = (C.c_void_p * len(self.systems))(*[s.handle.value for s in self.systems])
        t = _tune(tune) if tune else None
        self._h = C.c_void_p()
        check(lib().scmf_batch_create(arr, len(self.systems), C.byref(t) if t else None,
                                      C.c_void_p(stream) if stream else None, C.byref(self._h)))

    def step(self, n_sweeps: int = 1) -> None:
        check(lib().scmf_batch_step(self._h, int(n_sweeps)))

    def step_async(self, n_sweeps: int = 1) -> None:
        check(lib().scmf_batch_step_async(self._h, int(n_sweeps)))

    def step_profiled(self, n_sweeps: int = 1):
        """Runs n sweeps launch by launch with CUDA events; returns the summed
        device milliseconds of the move launches, of the field launches, and
        the device time from the first launch to the end of the last."""
        a, b, t = C.c_float(), C.c_float(), C.c_float()
        check(lib().scmf_batch_step_profiled(self._h, int(n_sweeps), C.byref(a), C.byref(b), C.byref(t)))
        return a.value, b.value, t.value

    def tune_trials(self) -> list:
        """The tunings the last autotune timed, in order, each with its time (ms)."""
        n = C.c_int32()
        check(lib().scmf_batch_tune_trials(self._h, None, 0, C.byref(n)))
        arr = (_lib.TuneTrial * max(1, n.value))()
        check(lib().scmf_batch_tune_trials(self._h, arr, n.value, C.byref(n)))
        return [dict(_tune_dict(arr[i].tune), ms=arr[i].ms) for i in range(n.value)]

    def autotune(self, sweeps_per_trial: int = 2) -> dict:
        t = _lib.Tune()
        check(lib().scmf_batch_autotune(self._h, int(sweeps_per_trial), C.byref(t)))
        return _tune_dict(t)

    def tune(self) -> dict:
        t = _lib.Tune()
        check(lib().scmf_batch_get_tune(self._h, C.byref(t)))
        return _tune_dict(t)

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().scmf_batch_destroy(h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _tune(d: dict) -> _lib.Tune:
    t = _lib.Tune()
    t.use_graph = 1
    for k, v in d.items():
        setattr(t, k, int(v))
    return t


def _tune_dict(t: _lib.Tune) -> dict:
    return {k: getattr(t, k) for k, _ in _lib.Tune._fields_ if k != "reserved"}


def debug_math(n: int, key=(0, 0)):
    """Device Philox words, Metropolis log and normals for counters (i,0,0,0)."""
    words = np.zeros(4 * n, dtype=np.uint32)
    logs = np.zeros(n, dtype=np.float32)
    nr = np.zeros(3 * n, dtype=np.float32)
    check(lib().scmf_debug_math(key[0], key[1], n, _ptr(words, C.c_uint32), _ptr(logs, C.c_float),
                                _ptr(nr, C.c_float)))
    return words.reshape(-1, 4), logs, nr.reshape(-1, 3)
