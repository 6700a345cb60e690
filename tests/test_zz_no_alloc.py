"""The allocation-free observables entry point, through the C ABI.

Callers that cannot allocate device memory (their device memory belongs to another allocator, or an
allocation's synchronisation is unaffordable, or their FFI cannot own a device buffer) use
`sck_observables_noalloc`, which keeps its partial sums in a fixed array inside the library. Its energies and
magnetizations must equal those of `sck_observables` with a caller workspace, on two calls in a row (the second
call reuses the array the first one left filled). This file is named to be collected last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import cases as C
from spin_colour_kernel_b200 import _lib as L
from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import system as sy

pytestmark = pytest.mark.gpu


def _both(A, S, storage, batch):
    """(E, M) from the workspace entry point and from the allocation-free one."""
    lib = L.lib()
    buf = A._buffers(S)
    s = A.sys
    stream = A._stream()
    E1 = torch.empty(batch, dtype=torch.float64, device=A.device)
    M1 = torch.empty((batch, s.b, s.n), dtype=torch.float64, device=A.device)
    ws = A._workspace(batch)
    L.check(lib.sck_observables(A._plan, ctypes.byref(buf), S.data_ptr(), storage, batch, E1.data_ptr(),
                                M1.data_ptr(), ws.data_ptr(), stream))
    E2 = torch.full((batch,), np.nan, dtype=torch.float64, device=A.device)
    M2 = torch.full((batch, s.b, s.n), np.nan, dtype=torch.float64, device=A.device)
    L.check(lib.sck_observables_noalloc(A._plan, ctypes.byref(buf), S.data_ptr(), storage, batch, E2.data_ptr(),
                                        M2.data_ptr(), stream))
    torch.cuda.synchronize()
    return E1.cpu().numpy(), M1.cpu().numpy(), E2.cpu().numpy(), M2.cpu().numpy()


@pytest.mark.parametrize("make, storage, batch", [
    (lambda: C.heisenberg_bcc_j1j2(sy, cr, 6), L.MODE_F32, 6),
    (lambda: sy.nanodot(Rd=2.5, L=3), L.MODE_F32, 3),
    (lambda: sy.ising("sc", 10), L.MODE_INT8, 40),
    (lambda: sy.ising("square", 12), L.MODE_PACKED, 70),
    # the tiled FP64 path (rows of 16 sites, 16 rows: 4 bands per replica), at the scratch limit exactly:
    # 4096 replicas x 4 blocks x 16 doubles = 2 MiB
    (lambda: C.heisenberg_bcc_j1j2(sy, cr, 16), L.MODE_F32, 4096),
    (lambda: C.heisenberg_bcc_j1j2(sy, cr, 8), L.MODE_QUAD, 10),
])
def test_no_alloc_observables_equal_workspace_observables(make, storage, batch):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200 import build
    from spin_colour_kernel_b200.sampler import Sampler
    build.build()
    s = make()
    kw = {"packed": storage == L.MODE_PACKED} if s.n == 1 else {}
    if storage == L.MODE_QUAD:
        kw["layout"] = "quad"
    A = Sampler(s, batch, device="cuda", seed=5, **kw)
    A.set_temperature(torch.linspace(0.5, 4.0, batch))
    S = A.init_spins(seed=1)
    for call in range(2):
        A.sweep(S, 1)
        E1, M1, E2, M2 = _both(A, S, storage, batch)
        np.testing.assert_allclose(E2, E1, rtol=1e-12, atol=1e-9, err_msg=f"call {call + 1}")
        np.testing.assert_allclose(M2, M1, rtol=1e-12, atol=1e-9, err_msg=f"call {call + 1}")


def test_no_alloc_observables_refuse_oversized_requests():
    """A request whose partial sums exceed the fixed array is refused (the plan's batch allows it, so only the
    size limit can reject it), and so is a batch beyond the plan's, before anything is launched."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200.sampler import Sampler
    s = C.heisenberg_bcc_j1j2(sy, cr, 16)
    A = Sampler(s, 4097, device="cuda", seed=1)
    S = A.init_spins(seed=1)
    buf = A._buffers(S)
    E = torch.empty(4097, dtype=torch.float64, device="cuda")
    rc = L.lib().sck_observables_noalloc(A._plan, ctypes.byref(buf), S.data_ptr(), L.MODE_F32, 4097, E.data_ptr(),
                                         None, A._stream())
    assert rc == L.ERR_INVALID and b"scratch" in L.lib().sck_last_error()
    rc = L.lib().sck_observables_noalloc(A._plan, ctypes.byref(buf), S.data_ptr(), L.MODE_F32, 4098, E.data_ptr(),
                                         None, A._stream())
    assert rc == L.ERR_INVALID and b"plan's batch" in L.lib().sck_last_error()
