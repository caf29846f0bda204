"""The no-allocation local-energy entry point against the allocating one.

dnq_ham_local_energy_noalloc exists for callers that may not allocate
device memory themselves (an XLA custom call inside XLA's memory plan, an
application with a fixed budget): its scratch is a file-scope device array.
Two calls in a row must each reproduce dnq_ham_local_energy, in FP64 and in
FP32; the file is named to run last so a failure here leaves the rest of a
``-x`` run intact.  It also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from detnqs_b200 import synthetic as S

pytestmark = pytest.mark.gpu

ENERGY_TOL = 1e-12


@pytest.fixture(scope="module")
def ham():
    import torch
    from detnqs_b200 import core, device, native
    sysm = S.make_system(16, 5, 5, 32, 2024)
    V = S.heat_bath_sample(sysm, 20000, 8)
    ctx = core.IntCtx.from_arrays(16, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    H = device.build(ctx, V, n_orb=16, policy=native.POLICY_STATIC, use_heatbath=True,
                     eps1=1e-6, want_vp=False)
    x = torch.from_numpy(S.normalized_psi(len(V), 6)).cuda()
    yield native, H, x
    H.close()
    ctx.close()


def _noalloc(native, H, x, eloc, precision):
    import torch
    out2 = np.zeros(2)
    native.check(native.lib.dnq_ham_local_energy_noalloc(
        H.handle, x.data_ptr(), eloc.data_ptr(), out2.ctypes.data, precision,
        torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out2


@pytest.mark.parametrize("prec_name", ["f64", "f32"])
def test_noalloc_matches_allocating_entry_point(ham, prec_name):
    import torch
    native, H, x = ham
    prec = native.F64 if prec_name == "f64" else native.F32
    ref_eloc = torch.empty_like(x)
    num, den = H.local_energy(x, eloc=ref_eloc, precision=prec)   # also prepares FP32 values
    torch.cuda.synchronize()
    ref = ref_eloc.cpu().numpy()
    for _ in range(2):                                              # two calls in a row
        eloc = torch.full_like(x, float("nan"))
        out2 = _noalloc(native, H, x, eloc, prec)
        got = eloc.cpu().numpy()
        assert abs(out2[0] - num) <= ENERGY_TOL * max(1.0, abs(num))
        assert abs(out2[1] - den) <= ENERGY_TOL * max(1.0, abs(den))
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)


def test_noalloc_rejects_host_buffers(ham):
    native, H, x = ham
    host = np.zeros(H.n_v)
    out2 = np.zeros(2)
    rc = native.lib.dnq_ham_local_energy_noalloc(H.handle, x.data_ptr(), host.ctypes.data,
                                                 out2.ctypes.data, native.F64, None)
    assert rc == native.ERR_INVALID
    assert b"device memory" in native.lib.dnq_last_error()
