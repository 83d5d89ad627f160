"""ctypes mirror of include/lbflow.h and the loader for liblbflow_b200.so.

The structures here are the binary layout of the C ABI; `lbf_sizeof` in the
library is checked against them when the library is loaded, so a header change
that is not mirrored here fails loudly instead of corrupting memory.
"""
from __future__ import annotations

import ctypes as C
import os

# --- enums (include/lbflow.h) ----------------------------------------------
LBF_OK, LBF_EINVAL, LBF_ENOMEM, LBF_EDEVICE, LBF_ETIMEOUT, LBF_ENAN, LBF_EUNSUPPORTED, LBF_ESTATE = range(8)
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "EDEVICE", 4: "ETIMEOUT", 5: "ENAN",
                6: "EUNSUPPORTED", 7: "ESTATE"}

LBF_D2Q5, LBF_D2Q9, LBF_D3Q15, LBF_D3Q19, LBF_D3Q27 = range(5)
LBF_WEST, LBF_EAST, LBF_SOUTH, LBF_NORTH, LBF_BOTTOM, LBF_TOP = range(6)
LBF_BGK, LBF_TRT, LBF_MRT, LBF_CENTRAL = range(4)
LBF_BC_NO_SLIP, LBF_BC_BOUNCE_BACK, LBF_BC_ANTI_BOUNCE_BACK, LBF_BC_ZOU_HE, LBF_BC_PERIODIC = range(5)
(LBF_SBC_ANTI_BOUNCE_BACK, LBF_SBC_ANTI_BB_NO_FLUX, LBF_SBC_BB_NO_FLUX,
 LBF_SBC_ZEROTH_ORDER_NO_FLUX, LBF_SBC_SECOND_ORDER_NO_FLUX, LBF_SBC_PERIODIC) = range(6)
LBF_INNER_ANTI_BOUNCE_BACK, LBF_INNER_BOUNCE_BACK = range(2)
LBF_STORE_F64, LBF_STORE_F32, LBF_STORE_F16DEV, LBF_STORE_BF16DEV = range(4)
LBF_COMPAT_REFERENCE, LBF_COMPAT_PHYSICS = range(2)

(LBF_OPT_BLOCK_X, LBF_OPT_STAGE, LBF_OPT_PIPE, LBF_OPT_PIPE_STAGES, LBF_OPT_COMPACT, LBF_OPT_Z_BEGIN, LBF_OPT_Z_END,
 LBF_OPT_SPARSE, LBF_OPT_STREAMING, LBF_OPT_SROUND, LBF_OPT_WAIT_LIMIT, LBF_OPT_SEED_OFFSET) = range(12)
LBF_STREAM_PULL, LBF_STREAM_PUSH, LBF_STREAM_INPLACE = range(3)
LBF_MAX_SCALARS = 4
LBF_BATCH_OPT_CHUNK_LAUNCH = 0

LBF_CLASS_SOLID = 0x1
LBF_CLASS_BOUNCE_BACK = 0x2
LBF_CLASS_FACE_SHIFT = 2

STORAGE_NAMES = {LBF_STORE_F64: "f64", LBF_STORE_F32: "f32", LBF_STORE_F16DEV: "f16dev",
                 LBF_STORE_BF16DEV: "bf16dev"}
STORAGE_BYTES = {LBF_STORE_F64: 8, LBF_STORE_F32: 4, LBF_STORE_F16DEV: 2, LBF_STORE_BF16DEV: 2}


class CollisionDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("_pad", C.c_int32), ("tau", C.c_double),
                ("omega_plus", C.c_double), ("omega_minus", C.c_double),
                ("relaxation", C.c_double * 27)]


class BcDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("has_density", C.c_int32), ("density", C.c_double),
                ("has_velocity", C.c_int32 * 3), ("_pad", C.c_int32),
                ("velocity", C.c_double * 3)]


class DomainDesc(C.Structure):
    _fields_ = [("velocity_set", C.c_int32), ("storage", C.c_int32), ("n", C.c_int64 * 3),
                ("collision", CollisionDesc), ("has_force", C.c_int32), ("compat", C.c_int32),
                ("force", C.c_double * 3), ("bc", BcDesc * 6), ("face_order", C.c_int32 * 6),
                ("node_type", C.c_void_p), ("initial_density", C.c_double),
                ("initial_velocity", C.c_double * 3), ("initial_density_field", C.c_void_p),
                ("initial_velocity_field", C.c_void_p)]


class ScalarBcDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("unknown_populations_only", C.c_int32),
                ("scalar_value", C.c_double)]


class ScalarDesc(C.Structure):
    _fields_ = [("velocity_set", C.c_int32), ("inner_boundary_condition", C.c_int32),
                ("collision", CollisionDesc), ("has_source", C.c_int32),
                ("has_adsorption", C.c_int32), ("source_value", C.c_double),
                ("initial_scalar_value", C.c_double), ("initial_scalar_field", C.c_void_p),
                ("bc", ScalarBcDesc * 6), ("adsorption_rate", C.c_double),
                ("desorption_rate", C.c_double), ("q_max", C.c_double),
                ("initial_q_ads", C.c_double)]


class LbfError(RuntimeError):
    """A non-zero lbf_status from the library, with lbf_last_error()'s message."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"lbflow_b200: {STATUS_NAMES.get(status, status)}: {message}")


# --- exported symbols and their signatures -----------------------------------
_P = C.c_void_p
_I32, _I64, _D = C.c_int32, C.c_int64, C.c_double
_PD, _PI32, _PI64, _PU32 = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_uint32)

SIGNATURES = {
    "lbf_abi_version": (_I32, []),
    "lbf_last_error": (C.c_char_p, []),
    "lbf_sizeof": (C.c_size_t, [_I32]),
    "lbf_velocity_set_tables": (_I32, [_I32, _PI32, _PI32, _PI32, _PD, _PI32, _PI32, _PI32, _PD, _PD]),
    "lbf_domain_create": (_I32, [C.POINTER(DomainDesc), C.POINTER(_P)]),
    "lbf_scalar_attach": (_I32, [_P, C.POINTER(ScalarDesc)]),
    "lbf_domain_init": (_I32, [_P, _P]),
    "lbf_domain_step": (_I32, [_P, _I64, _I64, _P]),
    "lbf_domain_run": (_I32, [_P, _I64, _I64, _D, _D, _D, _PI64, _P]),
    "lbf_domain_residuals": (_I32, [_P, _PD, _PI64]),
    "lbf_domain_get_moments": (_I32, [_P, _PD, _PD, _PD, _P]),
    "lbf_domain_get_q_ads": (_I32, [_P, _PD]),
    "lbf_domain_get_scalar": (_I32, [_P, _I32, _PD, _P]),
    "lbf_domain_get_q_ads_at": (_I32, [_P, _I32, _PD]),
    "lbf_domain_inventory": (_I32, [_P, _PD, _P]),
    "lbf_domain_get_node_class": (_I32, [_P, _PU32, _PU32]),
    "lbf_domain_time_step": (_I32, [_P, _PI64]),
    "lbf_domain_set_option": (_I32, [_P, _I32, _I64]),
    "lbf_domain_get_option": (_I32, [_P, _I32, _PI64]),
    "lbf_domain_device_bytes": (_I32, [_P, _PI64]),
    "lbf_domain_destroy": (_I32, [_P]),
    "lbf_solve": (_I32, [C.POINTER(DomainDesc), C.POINTER(ScalarDesc), _I64, _PD, _PD, _PD, _P]),
    "lbf_inventory_noalloc": (_I32, [_P, _P, _P, _P, _P, _I64, _I32, _P, _P]),
    "lbf_domain_checkpoint_bytes": (_I32, [_P, _PI64]),
    "lbf_domain_save": (_I32, [_P, _P, _I64, _P]),
    "lbf_domain_load": (_I32, [_P, _P, _I64, _P]),
    "lbf_domain_halo_info": (_I32, [_P, _PI32, _PI64, _PI64]),
    "lbf_domain_halo_pack": (_I32, [_P, _I32, _P, _P]),
    "lbf_domain_halo_unpack": (_I32, [_P, _I32, _P, _P]),
    "lbf_domain_step_part": (_I32, [_P, _I32, _I64, _P]),
    "lbf_domain_estimate_bytes": (_I32, [C.POINTER(DomainDesc), C.POINTER(ScalarDesc), _PI64]),
    "lbf_batch_create": (_I32, [_I64, _I64, C.POINTER(_P)]),
    "lbf_batch_admit": (_I32, [_P, _P, _I64, _D, _D, _D]),
    "lbf_batch_step": (_I32, [_P, _I64, _P]),
    "lbf_batch_poll": (_I32, [_P, C.POINTER(_P), _PI32, _I32, _PI32, _I32]),
    "lbf_batch_evict": (_I32, [_P, _P]),
    "lbf_batch_info": (_I32, [_P, _PI64, _PI64, _PI64, _PI64]),
    "lbf_batch_set_option": (_I32, [_P, _I32, _I64]),
    "lbf_batch_destroy": (_I32, [_P]),
    "lbf_format_csv": (_I32, [_P, _I64, _I32, _P, _I64, _PI64, _I32]),
    "lbf_format_coordinates": (_I32, [_PI64, _I32, _D, _P, _P, _I64, _PI64, _I32]),
}

_LIB_NAME = "liblbflow_b200.so"
_lib = None


def library_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), _LIB_NAME)


def load() -> C.CDLL:
    """Load the in-tree liblbflow_b200.so; raise if it has not been built.

    There is no fallback: the CUDA library is the only implementation of the
    engine.
    """
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("LBF_LIBRARY") or library_path()   # an alternative build, if given
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C lbflow_b200/csrc`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for which, st in enumerate((DomainDesc, ScalarDesc, BcDesc, CollisionDesc)):
        if lib.lbf_sizeof(which) != C.sizeof(st):
            raise ImportError(f"ABI mismatch for {st.__name__}: library {lib.lbf_sizeof(which)} "
                              f"bytes, binding {C.sizeof(st)} bytes")
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != LBF_OK:
        msg = _lib.lbf_last_error().decode() if _lib is not None else ""
        raise LbfError(status, msg)
