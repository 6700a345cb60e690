"""Bounded device-side waits that give up are reported as SCK_ERR_TIMEOUT, through the C ABI.

Every spin-wait in the library's kernels has an iteration limit. A test-only knob shortens it to zero polls, so
that each wait which is not already satisfied gives up at once: the kernel still returns (nothing traps or hangs;
a block that gave up first waits, with the full limit, for its own copies or tensor-core products in flight),
its sites or output rows are left unwritten, and the host learns of it: the plan's next sweep refuses with
SCK_ERR_TIMEOUT until the status is read, and the status read (Sampler.check_waits, BlockProposal.check_waits)
raises and clears it. With the default limit restored the paths again equal their references.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import cases as C
from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import system as sy

pytestmark = pytest.mark.gpu


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200 import build
    build.build()


def _expect_timeout(fn):
    from spin_colour_kernel_b200 import _lib as L
    with pytest.raises(L.SckError) as e:
        fn()
    assert e.value.code == L.ERR_TIMEOUT, e.value


def test_tile_kernel_wait_that_gives_up_reports_timeout():
    """Tile kernels wait for their bricks' bulk copies; with zero polls every brick gives up, waits for its copies
    and leaves its sites unchanged: the whole sweep changes nothing, and the plan reports the timeout."""
    _need_gpu()
    from spin_colour_kernel_b200.sampler import Sampler
    s = sy.System("Heisenberg bcc J1-J2", 3, cr.make("bcc", (1, 2)), (64, 8, 8), (True,) * 3, {1: 1.0, 2: 0.3},
                  h=(0.0, 0.0, 0.1), cubic_k1=np.full((2, 8, 8, 64), 0.05, np.float32))
    B = 5
    A, R = Sampler(s, B, device="cuda", seed=3), Sampler(s, B, device="cuda", seed=3)
    assert A.tune(3, 0, 0)["specialised"] // 100 == 3
    assert R.tune(1, 0, 0)["specialised"] // 100 == 1
    for X in (A, R):
        X.set_temperature(torch.linspace(0.4, 3.0, B))
    S = A.init_spins(seed=7)
    S0 = S.clone()
    A.set_wait_limit(0)
    A.sweep(S, 1)
    torch.cuda.synchronize()
    assert torch.equal(S, S0)                          # every brick gave up
    _expect_timeout(lambda: A.sweep(S, 1))             # refused until the status is read
    _expect_timeout(A.check_waits)
    A.check_waits()                                    # cleared
    A.set_wait_limit(1 << 20)
    A.state.copy_(R.state)
    X = S.clone()
    A.sweep(S, 2)
    R.sweep(X, 2)
    A.check_waits()
    assert torch.equal(S, X)


def test_group_pipeline_wait_that_gives_up_reports_timeout():
    """The reference-layout group pipeline (L2 budget) orders its tasks by completion counters; with zero polls a
    task whose predecessor has not finished gives up, and the plan reports the timeout."""
    _need_gpu()
    from spin_colour_kernel_b200.sampler import Sampler
    s = C.heisenberg_bcc_j1j2(sy, cr, 16)
    B = 16
    A, R = Sampler(s, B, device="cuda", seed=21, packed=False), Sampler(s, B, device="cuda", seed=21, packed=False)
    per_rep = s.nsite * s.n * 4
    assert A.tune(True, len(A.classes) * per_rep * 2, 0)["group"] == 2   # eight groups of two replicas
    R.tune(True, 0, 0)
    for X in (A, R):
        X.set_temperature(torch.linspace(0.3, 3.0, B))
    S = A.init_spins(seed=6)
    A.set_wait_limit(0)
    A.sweep(S, 3)
    torch.cuda.synchronize()
    _expect_timeout(lambda: A.sweep(S, 1))
    _expect_timeout(A.check_waits)
    A.check_waits()
    A.set_wait_limit(1 << 20)
    A.state.copy_(R.state)
    X = S.clone()
    A.sweep(S, 3)
    R.sweep(X, 3)
    A.check_waits()
    assert torch.equal(S, X)


def test_tensor_core_gemm_wait_that_gives_up_reports_timeout():
    """The learned proposal's tcgen05 forward GEMM waits on its stages' mbarriers; with zero polls every block
    gives up after draining its products, and forward raises SCK_ERR_TIMEOUT; restored, the tcgen05 logits again
    equal the mma.sync kernel's."""
    _need_gpu()
    from spin_colour_kernel_b200.learned import BlockProposal, kaiming_params
    P = BlockProposal(16, 1, groups=16, params=kaiming_params(11))
    rng = np.random.default_rng(12)
    X = torch.from_numpy(rng.choice([-1.0, 1.0], size=(256, 160))).to(torch.bfloat16).cuda()
    P.check_waits()
    P.set_wait_limit(0)
    try:
        _expect_timeout(lambda: P.forward(X))          # 256 rows: the tcgen05 path
    finally:
        P.set_wait_limit(1 << 22)
    P.check_waits()                                    # cleared by the raising read
    l_umma, _ = P.forward(X)
    l_sync, _ = P.forward(X[:192])                     # 192 rows: the mma.sync path
    d = np.abs(l_umma[:192].cpu().numpy() - l_sync.cpu().numpy())
    assert np.median(d) < 1e-5 and d.max() < 0.05, (np.median(d), d.max())
