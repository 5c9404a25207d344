"""The allocation-free field update, through the C ABI.

Callers that cannot allocate device memory (code running inside someone
else's stream capture or a loop that must never stall on an allocation, or an
application that owns all device memory and hands out pointers) pass their own
counts / omega / energy buffers to scmf_update_omega_noalloc, whose only
scratch is a fixed array inside the library.  This test allocates its buffers
itself (torch) and checks two calls in a row against the field update of the
regular entry point and against the oracle's field of the same positions,
within the tolerance of the other parity tests, for the SCMF0 and the literal
Hamiltonian and for a three-type system (runtime type count); this file is
collected last so that a stop-at-first-failure run has run everything else.
"""
import ctypes as C
import os

import numpy as np
import pytest

from tests._util import RTOL, assert_close

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _spec(case):
    from new_arch_b200 import HAM_LITERAL
    from new_arch_b200.spec import SystemSpec, diblock_melt
    if case == "three_types":
        # the reference's 3-type configuration (configuration.dat~) with its polymer.dat
        return SystemSpec.from_files(os.path.join(GOLDEN, "configuration_3types.dat"),
                                     os.path.join(GOLDEN, "polymer.dat"), 13)
    spec = diblock_melt(3000, 32, 0.3, (20, 18, 16), 25.0, 50.0, seed=13)
    if case == "literal":
        spec.hamiltonian = HAM_LITERAL
    return spec


@pytest.mark.parametrize("case", ["scmf0", "literal", "three_types"])
def test_noalloc_field_update_matches_regular_entry_point_and_oracle(case):
    import torch
    import new_arch_b200 as nb
    from new_arch_b200 import _lib
    from oracle.oracle import OracleSystem

    L = _lib.lib()
    spec = _spec(case)
    assert case != "three_types" or spec.n_types == 3
    xn = np.ascontiguousarray(spec.xn, dtype=np.float64)
    xn_p = xn.ctypes.data_as(C.POINTER(C.c_double))
    scaling = spec.n_cells / spec.n_beads
    d_omega = torch.empty(spec.n_types * spec.n_cells, dtype=torch.float32, device="cuda")
    d_energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    with nb.System(spec) as s:
        s.init_coords()
        for call in range(2):
            if call:
                s.step(3)                      # new counts for the second call
            counts = s.counts()
            s.update_omega_fields_scmf0()      # the regular entry point
            want_w, want_e = s.omega(), s.stats()["e_field"]
            orc = OracleSystem(spec)
            orc.set_coords(s.coords())
            orc.reset_density()
            orc.update_omega()
            d_counts = torch.from_numpy(counts.view(np.int32)).cuda()
            d_omega.fill_(float("nan"))
            d_energy.fill_(float("nan"))
            rc = L.scmf_update_omega_noalloc(d_counts.data_ptr(), d_omega.data_ptr(), spec.n_types, spec.n_cells,
                                             scaling, xn_p, spec.nref, spec.hamiltonian, d_energy.data_ptr(),
                                             stream.cuda_stream)
            _lib.check(rc)
            stream.synchronize()
            got_w, got_e = d_omega.cpu().numpy(), d_energy.item()
            assert_close(got_w, want_w, RTOL, f"{case}: omega vs entry point, call {call + 1}")
            assert_close([got_e], [want_e], RTOL, f"{case}: field energy vs entry point, call {call + 1}")
            assert np.array_equal(orc.counts(), counts), f"{case}: oracle recount differs, call {call + 1}"
            assert_close(got_w, orc.omega(), RTOL, f"{case}: omega vs oracle, call {call + 1}")
            assert_close([got_e], [orc.stats()["e_field"]], RTOL, f"{case}: field energy vs oracle, call {call + 1}")

    # sizes beyond the fixed scratch are refused, not truncated
    too_many = 2048 * 4096 + 1
    rc = L.scmf_update_omega_noalloc(d_omega.data_ptr(), d_omega.data_ptr(), 2, too_many, 1.0, xn_p, 32, 0,
                                     d_energy.data_ptr(), stream.cuda_stream)
    assert rc == -1
    assert b"exceeds" in L.scmf_last_error()
