"""Host-side checks of the learned block proposal's C ABI (no device work): sizes, layout and refusals."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle import made as MD
from spin_colour_kernel_b200 import _lib as L
from spin_colour_kernel_b200 import learned as LP


def _sizes(groups, batch):
    p, a, t = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    rc = L.lib().sck_made_sizes(groups, batch, ctypes.byref(p), ctypes.byref(a), ctypes.byref(t))
    return rc, p.value, a.value, t.value


def test_sizes_and_refusals():
    rc, p, a, t = _sizes(16, 8192)
    assert rc == 0
    assert p >= LP.NPARAM * 4 + 2 * (264 * (160 + 512) + 72 * 256) and p % 256 == 0
    assert a == 2 * LP.NPARAM * 4
    assert t > 8192 * 256 * 2 * 6
    assert _sizes(17, 64)[0] == L.ERR_INVALID
    assert _sizes(64, 100)[0] == L.ERR_INVALID
    assert b"batch" in L.lib().sck_last_error()


def test_colour_step_refusals_before_any_launch():
    lib = L.lib()
    fake = ctypes.c_void_p(256)
    beta = ctypes.c_void_p(512)
    assert lib.sck_made_colour_step(None, 16, fake, 4, 16, beta, 0, 1, 0, None, None, None) == L.ERR_INVALID
    assert lib.sck_made_colour_step(fake, 16, fake, 4, 12, beta, 0, 1, 0, None, None, None) == L.ERR_INVALID
    assert lib.sck_made_colour_step(fake, 16, fake, 4, 16, beta, 8, 1, 0, None, None, None) == L.ERR_INVALID
    assert lib.sck_made_colour_step(fake, 32, fake, 4, 16, beta, 0, 1, 0, None, None, None) == L.ERR_INVALID
    # 17 x replicas x blocks must fit the int32 Philox counter
    assert lib.sck_made_colour_step(fake, 16, fake, 100000, 64, beta, 0, 1, 0, None, None, None) == L.ERR_COUNTER


def test_parameter_flattening_round_trips_and_matches_the_oracle_shapes():
    params = LP.kaiming_params(3)
    ref = MD.init_params(96, 64, 256, seed=3)
    for (W, b), (Wr, br) in zip(params, ref):
        assert W.shape == Wr.shape and b.shape == br.shape
        np.testing.assert_array_equal(W, Wr)
    flat = LP.flatten(params)
    assert flat.size == LP.NPARAM
    for (W, b), (W2, b2) in zip(params, LP.unflatten(flat)):
        np.testing.assert_array_equal(W, W2)
        np.testing.assert_array_equal(b, b2)


def test_block_colouring_is_searched_verified_and_names_parity_classes():
    """The block colouring comes from the site colouring's own search on the block graph (face, edge and corner
    neighbours): 8 colours, equal to the clique number, verified on the periodic box, and each colour is one
    parity class of the block coordinates, whose code the colour-step kernel takes."""
    from spin_colour_kernel_b200 import colouring as co
    from spin_colour_kernel_b200 import crystals as cr
    for nb in (2, 4, 16):
        col, codes = LP.block_colouring(nb)
        assert col.n_colours == 8 and sorted(codes) == list(range(8))
        assert co.verify_on_box(col, cr.make("sc", (1, 2, 3)), (nb,) * 3, (True,) * 3)
        grid = col.colour_grid(0, (nb,) * 3)
        z, y, x = np.meshgrid(np.arange(nb), np.arange(nb), np.arange(nb), indexing="ij")
        assert np.array_equal(np.asarray(codes)[grid], (x % 2) + 2 * (y % 2) + 4 * (z % 2))
    for bad in (1, 3):
        try:
            LP.block_colouring(bad)
        except ValueError:
            pass
        else:
            raise AssertionError(f"nb={bad} accepted")
