"""ctypes binding of libsckb200.so (include/sck.h).

The library is built in-tree by `python -m spin_colour_kernel_b200.build`. Loading fails loudly when it is
missing: there is no CPU path behind this package.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsckb200.so"

ABI_VERSION = 1
OK, ERR_INVALID, ERR_COUNTER, ERR_UNSUPPORTED, ERR_CUDA, ERR_TIMEOUT = 0, -1, -2, -3, -4, -5
MODE_INT8, MODE_F32, MODE_PACKED, MODE_BITWISE, MODE_BITWISE_INDEP, MODE_QUAD = 0, 1, 2, 3, 4, 5
METROPOLIS, BARKER = 0, 1
MAX_BASIS, MAX_BONDS, MAX_GROUPS, MAX_EXTRA, MAX_FACTORS, MAX_CLASSES = 4, 64, 8, 8, 4, 128

_i32, _i64, _f32, _f64, _vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p


class Bond(ctypes.Structure):
    _fields_ = [("alpha2", _i32), ("d", _i32 * 3), ("group", _i32), ("extra", _i32), ("J64", _f64)]


class Sublattice(ctypes.Structure):
    _fields_ = [("n_bonds", _i32), ("n_groups", _i32), ("group_end", _i32 * MAX_GROUPS),
                ("group_J", _f32 * MAX_GROUPS), ("group_apply", _i32 * MAX_GROUPS), ("n_extra", _i32),
                ("extra", (_f32 * 9) * MAX_EXTRA), ("extra64", (_f64 * 9) * MAX_EXTRA),
                ("bonds", Bond * MAX_BONDS)]


class SystemDesc(ctypes.Structure):
    _fields_ = [("abi_version", _i32), ("n", _i32), ("dim", _i32), ("b", _i32), ("L", _i32 * 3),
                ("periodic", _i32 * 3), ("acceptance", _i32), ("has_mask", _i32), ("has_cubic", _i32),
                ("h", _f32 * 3), ("h64", _f64 * 3), ("k2", _f32), ("k2_64", _f64), ("n_factors", _i32),
                ("m", _i32 * MAX_FACTORS), ("K", (_i32 * 3) * MAX_FACTORS), ("o", (_i32 * MAX_FACTORS) * MAX_BASIS),
                ("n_classes", _i32), ("classes", (_i32 * 2) * MAX_CLASSES), ("sub", Sublattice * MAX_BASIS)]


class Buffers(ctypes.Structure):
    _fields_ = [("spins", _vp), ("mask", _vp), ("k1", _vp), ("beta", _vp), ("table", _vp), ("state", _vp)]


_SIGNATURES = {
    "sck_abi_version": ([], _i32),
    "sck_last_error": ([], ctypes.c_char_p),
    "sck_struct_sizes": ([ctypes.POINTER(_i64)] * 4, _i32),
    "sck_plan_create": ([ctypes.POINTER(SystemDesc), _i32, _i32, ctypes.POINTER(_vp)], _i32),
    "sck_plan_destroy": ([_vp], _i32),
    "sck_plan_table_size": ([_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i32), ctypes.POINTER(_i32)], _i32),
    "sck_plan_shape": ([_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32)], _i32),
    "sck_plan_tune": ([_vp, _i32, _i64, _i64], _i32),
    "sck_plan_pipeline": ([_vp, _i32, _i32], _i32),
    "sck_plan_pipeline_chunks": ([_vp, _i32], _i32),
    "sck_plan_set_wait_limit": ([_vp, _i64], _i32),
    "sck_plan_wait_status": ([_vp, _vp], _i32),
    "sck_plan_path": ([_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i64), ctypes.POINTER(_i32),
                       ctypes.POINTER(_i32)], _i32),
    "sck_class_update": ([_vp, ctypes.POINTER(Buffers), _vp, _i32, _i32, _i32, _vp], _i32),
    "sck_sweep": ([_vp, ctypes.POINTER(Buffers), _i32, _vp], _i32),
    "sck_sync_sweep": ([_vp, ctypes.POINTER(Buffers), _vp, _i32, _vp], _i32),
    "sck_reference_sweep": ([_vp, ctypes.POINTER(Buffers), _i32, _vp], _i32),
    "sck_observables_workspace_size": ([_vp, _i32, ctypes.POINTER(_i64)], _i32),
    "sck_observables": ([_vp, ctypes.POINTER(Buffers), _vp, _i32, _i32, _vp, _vp, _vp, _vp], _i32),
    "sck_topological_charge": ([_vp, ctypes.POINTER(Buffers), _vp, _i32, _i32, _vp, _vp], _i32),
    "sck_observables_accumulate": ([_vp, ctypes.POINTER(Buffers), _vp, _i32, _i32, ctypes.c_double, _vp, _vp, _vp,
                                    _vp, _vp, _vp, _vp], _i32),
    "sck_sweep_measure_workspace_size": ([_vp, ctypes.POINTER(_i64)], _i32),
    "sck_sweep_measure": ([_vp, ctypes.POINTER(Buffers), _i32, _vp, _vp, _vp, _vp], _i32),
    "sck_observables_noalloc": ([_vp, ctypes.POINTER(Buffers), _vp, _i32, _i32, _vp, _vp, _vp], _i32),
    "sck_wait_timeouts": ([ctypes.POINTER(_i64)], _i32),
    "sck_pack": ([_vp, _vp, _vp, _vp], _i32),
    "sck_quad_pack": ([_vp, _vp, _vp, _vp], _i32),
    "sck_quad_unpack": ([_vp, _vp, _vp, _vp], _i32),
    "sck_unpack": ([_vp, _vp, _vp, _vp, _vp], _i32),
    "sck_advance": ([_vp, _i32, _vp], _i32),
    "sck_batch_create": ([ctypes.POINTER(_vp), _i32, _i64, ctypes.POINTER(_vp)], _i32),
    "sck_batch_destroy": ([_vp], _i32),
    "sck_batch_workspace_size": ([_vp, ctypes.POINTER(_i64)], _i32),
    "sck_batch_bind": ([_vp, ctypes.POINTER(Buffers), _vp, _vp], _i32),
    "sck_batch_sweep": ([_vp, _vp, _i32, _vp], _i32),
    "sck_batch_info": ([_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32), ctypes.POINTER(_i64)], _i32),
    "sck_batch_set_wait_limit": ([_vp, _i64], _i32),
    "sck_batch_wait_status": ([_vp, _vp], _i32),
    # learned block proposal (include/sck_made.h)
    "sck_made_sizes": ([_i32, _i32, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)], _i32),
    "sck_made_prepare": ([_vp, _i32, _vp], _i32),
    "sck_made_gather": ([_vp, _i32, _i32, _vp, _vp], _i32),
    "sck_made_forward": ([_vp, _i32, _vp, _i32, _vp, _vp, _vp, _vp], _i32),
    "sck_made_grads": ([_vp, _i32, _vp, _i32, _vp, _vp, _vp, _vp], _i32),
    "sck_made_train_step": ([_vp, _vp, _i32, _vp, _i32, _f32, _f32, _f32, _f32, _i32, _vp, _vp, _vp], _i32),
    "sck_made_colour_step": ([_vp, _i32, _vp, _i32, _i32, _vp, _i32, _i64, _i32, _vp, _vp, _vp], _i32),
    "sck_made_set_wait_limit": ([_i64], _i32),
    "sck_made_wait_status": ([_vp], _i32),
}

EXPORTS = tuple(_SIGNATURES)
_lib = None


class SckError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libsckb200 error {code}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """The loaded library (built in-tree); raises when it is absent or does not match this binding."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH.name} is not built: run `python -m spin_colour_kernel_b200.build` "
                               "(this package has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        if L.sck_abi_version() != ABI_VERSION:
            raise RuntimeError("libsckb200 ABI version does not match this binding")
        sizes = [_i64() for _ in range(4)]
        L.sck_struct_sizes(*[ctypes.byref(s) for s in sizes])
        want = [ctypes.sizeof(SystemDesc), ctypes.sizeof(Sublattice), ctypes.sizeof(Bond), ctypes.sizeof(Buffers)]
        if [s.value for s in sizes] != want:
            raise RuntimeError(f"libsckb200 struct layout mismatch: {[s.value for s in sizes]} != {want}")
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != OK:
        msg = lib().sck_last_error().decode(errors="replace")
        if rc in (ERR_INVALID, ERR_COUNTER, ERR_UNSUPPORTED):
            raise ValueError(msg)
        raise SckError(rc, msg)
