"""The no-allocation local-energy entry point against the allocating one.

dnq_ham_local_energy_noalloc exists for callers that may not allocate
device memory themselves (an XLA custom call inside XLA's memory plan, an
application with a fixed budget): its scratch is a file-scope device array.
Two calls in a row must each reproduce dnq_ham_local_energy, in FP64 and in
FP32, with the energy pair returned to host or to device memory, and the
device's stream-ordered pool (which every allocating entry point of the
library draws from) must not grow its high-water mark during those calls.
The file is named to run last so a failure here leaves the rest of a ``-x``
run intact.  It also passes alone in a fresh process.
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


def _pool_used_high(native):
    """(used-now, high-water) bytes of the device's default stream-ordered
    pool, read through the CUDA runtime the library itself loaded."""
    cudart = C.CDLL("libcudart.so.12")
    pool = C.c_void_p()
    assert cudart.cudaDeviceGetDefaultMemPool(C.byref(pool), 0) == 0
    used, high = C.c_uint64(), C.c_uint64()
    assert cudart.cudaMemPoolGetAttribute(pool, 7, C.byref(used)) == 0    # UsedMemCurrent
    assert cudart.cudaMemPoolGetAttribute(pool, 8, C.byref(high)) == 0    # UsedMemHigh
    return cudart, pool, used.value, high.value


def _noalloc(native, H, x, eloc, precision, out2=None):
    import torch
    host = out2 is None
    if host:
        out2 = np.zeros(2)
    ptr = out2.ctypes.data if host else out2.data_ptr()
    native.check(native.lib.dnq_ham_local_energy_noalloc(
        H.handle, x.data_ptr(), eloc.data_ptr(), ptr, precision,
        torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out2 if host else out2.cpu().numpy()


@pytest.mark.parametrize("prec_name", ["f64", "f32"])
@pytest.mark.parametrize("out_on", ["host", "device"])
def test_noalloc_matches_allocating_entry_point(ham, prec_name, out_on):
    import torch
    native, H, x = ham
    prec = native.F64 if prec_name == "f64" else native.F32
    ref_eloc = torch.empty_like(x)
    num, den = H.local_energy(x, eloc=ref_eloc, precision=prec)   # also prepares FP32 values
    torch.cuda.synchronize()
    ref = ref_eloc.cpu().numpy()
    elocs = [torch.full_like(x, float("nan")) for _ in range(3)]
    outs = [None if out_on == "host" else torch.full((2,), float("nan"), dtype=torch.float64,
                                                     device=x.device) for _ in range(3)]
    # The first call of a process also makes the driver load the module that
    # holds the scratch array; the allocation check covers the calls after it.
    got = [_noalloc(native, H, x, elocs[0], prec, outs[0])]
    cudart, pool, used0, _ = _pool_used_high(native)
    zero = C.c_uint64(0)
    assert cudart.cudaMemPoolSetAttribute(pool, 8, C.byref(zero)) == 0     # reset high-water
    free0 = torch.cuda.mem_get_info()[0]
    got += [_noalloc(native, H, x, elocs[i], prec, outs[i]) for i in (1, 2)]   # two in a row
    _, _, used1, high1 = _pool_used_high(native)
    assert high1 <= used0 and used1 == used0, (used0, used1, high1)
    assert torch.cuda.mem_get_info()[0] == free0
    for i in range(3):
        out2 = got[i]
        assert abs(out2[0] - num) <= ENERGY_TOL * max(1.0, abs(num))
        assert abs(out2[1] - den) <= ENERGY_TOL * max(1.0, abs(den))
        np.testing.assert_allclose(elocs[i].cpu().numpy(), ref, rtol=1e-12, atol=0)


def test_noalloc_rejects_host_buffers(ham):
    native, H, x = ham
    host = np.zeros(H.n_v)
    out2 = np.zeros(2)
    rc = native.lib.dnq_ham_local_energy_noalloc(H.handle, x.data_ptr(), host.ctypes.data,
                                                 out2.ctypes.data, native.F64, None)
    assert rc == native.ERR_INVALID
    assert b"device memory" in native.lib.dnq_last_error()


def test_noalloc_rejects_overlapping_x_and_eloc(ham):
    import torch
    native, H, x = ham
    buf = torch.zeros(H.n_v + 8, dtype=torch.float64, device=x.device)
    buf[:H.n_v] = x
    out2 = np.zeros(2)
    for shift in (0, 8):                       # same buffer, and eloc 8 entries into x
        eloc_ptr = buf.data_ptr() + shift * 8
        rc = native.lib.dnq_ham_local_energy_noalloc(H.handle, buf.data_ptr(), eloc_ptr,
                                                     out2.ctypes.data, native.F64, None)
        assert rc == native.ERR_INVALID
        assert b"overlap" in native.lib.dnq_last_error()
