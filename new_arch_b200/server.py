"""Python mirror of the served engine (scmf_server_* in include/scmf.h):
continuous batching of parameter-sweep solves under an HBM budget."""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional

import numpy as np

from . import _lib
from ._lib import check, lib
from .spec import SystemSpec


class Server:
    def __init__(self, hbm_budget_bytes: int, max_active: int = 0, sweeps_per_round: int = 0, use_graph: bool = False):
        opts = _lib.ServerOpts(int(hbm_budget_bytes), int(max_active), int(sweeps_per_round), int(bool(use_graph)), 0)
        self._h = C.c_void_p()
        check(lib().scmf_server_create(C.byref(opts), C.byref(self._h)))
        self._buffers: Dict[int, np.ndarray] = {}

    def submit(self, spec: SystemSpec, n_sweeps: int, want_counts: bool = True) -> int:
        h = spec.to_c()
        buf = np.empty(spec.n_types * spec.n_cells, dtype=np.uint32) if want_counts else None
        rid = C.c_uint64()
        try:
            check(lib().scmf_server_submit(self._h, h, int(n_sweeps),
                                           buf.ctypes.data_as(C.POINTER(C.c_uint32)) if buf is not None else None,
                                           C.byref(rid)))
        finally:
            lib().scmf_spec_destroy(h)
        if buf is not None:
            self._buffers[rid.value] = buf
        return rid.value

    def poll(self, max_results: int = 64, wait_ms: int = 0) -> List[dict]:
        arr = (_lib.Result * max_results)()
        n = C.c_int32()
        check(lib().scmf_server_poll(self._h, arr, max_results, C.byref(n), int(wait_ms)))
        out = []
        for i in range(n.value):
            r = arr[i]
            d = {k: getattr(r, k) for k, _ in _lib.Result._fields_ if k != "reserved"}
            d["counts"] = self._buffers.pop(r.id, None)
            out.append(d)
        return out

    def pending(self):
        q, a, b = C.c_int32(), C.c_int32(), C.c_uint64()
        check(lib().scmf_server_pending(self._h, C.byref(q), C.byref(a), C.byref(b)))
        return q.value, a.value, b.value

    def now(self) -> float:
        return lib().scmf_server_now(self._h)

    def cancel(self, rid: int) -> None:
        """Cancel a queued or running request; its result arrives with status -9."""
        check(lib().scmf_server_cancel(self._h, int(rid)))

    def drain(self, timeout_ms: int) -> None:
        """Wait until nothing is queued or running; ScmfError(-7) on timeout."""
        check(lib().scmf_server_drain(self._h, int(timeout_ms)))

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().scmf_server_destroy(h)
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
