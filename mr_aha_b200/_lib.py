"""ctypes binding of ``libmr_aha_c.so``: library loading, struct mirrors,
enums and prototypes.

Mirrors the reference binding's ``python/mr_aha/_lib.py`` (struct layouts
``_lib.py:172-250`` and the operator structs, prototypes ``:581-698``,
library search ``:487-531``): the same field order and C types, the same
``MR_AHA_LIBRARY`` override. The library is searched for in
``$MR_AHA_LIBRARY`` and in this package's ``lib/`` directory (where
``python -m mr_aha_b200.build`` puts it). There is no fallback: importing this
module fails when the CUDA library is missing.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

DEFAULT_MASK_RADIUS = 2
OP_MAX_DEVICES = 16
OP_ALL_DEVICES = -1
OP_SHARE_PRIMARY = 1
OP_TOEP_SOURCES = {0: "supplied", 1: "broadcast", 2: "split", 3: "replicate", 4: "none"}

KF_COMPLEX64 = 0
KF_BF16 = 1
KF_INT16 = 2
KERNEL_FORMATS = {"complex64": KF_COMPLEX64, "bf16": KF_BF16, "int16": KF_INT16}


class MRError(RuntimeError):
    """A library call returned a negative ``mr_status``."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class _Enum:
    _FROM_STR: dict = {}
    _TO_STR: dict = {}

    @classmethod
    def parse(cls, value):
        if isinstance(value, int):
            return int(value)
        try:
            return cls._FROM_STR[str(value).lower()]
        except KeyError:
            raise ValueError(
                f"{cls.__name__}: expected one of {sorted(cls._FROM_STR)}; got {value!r}"
            ) from None


class TrajType(_Enum):
    TWO_D = 0
    THREE_D = 1
    STACK = 2
    _FROM_STR = {"2d": 0, "3d": 1, "stack": 2}
    _TO_STR = {0: "2D", 1: "3D", 2: "stack"}


class Triangulation(_Enum):
    LOWER = 0
    UPPER = 1
    _FROM_STR = {"lower": 0, "upper": 1}
    _TO_STR = {0: "lower", 1: "upper"}


class OpMethod(_Enum):
    TOEPLITZ = 0
    NUFFT = 1
    _FROM_STR = {"toeplitz": 0, "nufft": 1}
    _TO_STR = {0: "toeplitz", 1: "nufft"}


class ToepDist(_Enum):
    AUTO = 0
    SPLIT = 1
    REPLICATE = 2
    BROADCAST = 3
    _FROM_STR = {"auto": 0, "split": 1, "replicate": 2, "broadcast": 3, "off": 3}
    _TO_STR = {0: "auto", 1: "split", 2: "replicate", 3: "broadcast"}


class MRConfig(ctypes.Structure):
    """Mirror of ``struct mr_config`` (field order and C types are the ABI)."""

    _fields_ = [
        ("traj_type", ctypes.c_int),
        ("n_spatial", ctypes.c_int),
        ("n_dim", ctypes.c_int * 3),
        ("phi2_dim", ctypes.c_int * 3),
        ("L", ctypes.c_int),
        ("triangulation", ctypes.c_int),
        ("is_masked", ctypes.c_int),
        ("num_masked", ctypes.c_int64),
        ("n_coils", ctypes.c_int),
        ("eps", ctypes.c_double),
        ("gpu_device_id", ctypes.c_int),
        ("stream", ctypes.c_void_p),
        ("mem_fraction", ctypes.c_double),
        ("verbose", ctypes.c_int),
        ("mask_radius", ctypes.c_int),
    ]


class MROpInputs(ctypes.Structure):
    _fields_ = [
        ("d_SEs", ctypes.c_void_p),
        ("d_phi2", ctypes.c_void_p),
        ("d_traj", ctypes.c_void_p),
        ("Ntrajs", ctypes.c_int64),
        ("Nkx", ctypes.c_int64),
        ("d_mask", ctypes.c_void_p),
        ("d_phi2_toep", ctypes.c_void_p),
    ]


class MROpOptions(ctypes.Structure):
    _fields_ = [
        ("method", ctypes.c_int),
        ("devices", ctypes.POINTER(ctypes.c_int)),
        ("n_devices", ctypes.c_int),
        ("toep_dist", ctypes.c_int),
        ("flags", ctypes.c_int),
        ("nufft_upsampfac", ctypes.c_double),
        ("nufft_gpu_method", ctypes.c_int),
    ]


class MROpInfo(ctypes.Structure):
    _fields_ = [
        ("method", ctypes.c_int),
        ("n_devices", ctypes.c_int),
        ("devices", ctypes.c_int * OP_MAX_DEVICES),
        ("coil_begin", ctypes.c_int * OP_MAX_DEVICES),
        ("coil_count", ctypes.c_int * OP_MAX_DEVICES),
        ("group", ctypes.c_int * OP_MAX_DEVICES),
        ("n_split_coils", ctypes.c_int),
        ("peer_access", ctypes.c_int),
        ("peer_bandwidth_gbs", ctypes.c_double),
        ("toep_source", ctypes.c_int),
        ("toep_devices", ctypes.c_int),
        ("toep_ms", ctypes.c_double),
        ("toep_component_ms", ctypes.c_double),
        ("toep_gather_gbs", ctypes.c_double),
        ("create_ms", ctypes.c_double),
    ]


#: Every symbol of ``include/mr_aha/mr_aha.h`` and ``mr_aha_b200.h``:
#: name -> (restype, argtypes).
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
PROTOTYPES = {
    "mr_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "mr_last_error": (ctypes.c_char_p, []),
    "mr_backend": (ctypes.c_char_p, []),
    "mr_version": (ctypes.c_int, []),
    "mr_config_defaults": (ctypes.c_int, [ctypes.POINTER(MRConfig), ctypes.c_int]),
    "mr_config_validate": (ctypes.c_int, [ctypes.POINTER(MRConfig)]),
    "mr_num_tri": (_I64, [ctypes.c_int]),
    "mr_image_size": (_I64, [ctypes.POINTER(MRConfig)]),
    "mr_pad_size": (_I64, [ctypes.POINTER(MRConfig)]),
    "mr_phi2_toep_size": (_I64, [ctypes.POINTER(MRConfig)]),
    "mr_x_size": (_I64, [ctypes.POINTER(MRConfig)]),
    "mr_se_size": (_I64, [ctypes.POINTER(MRConfig)]),
    "mr_aha_plan_create": (ctypes.c_int, [ctypes.POINTER(MRConfig), ctypes.POINTER(_P)]),
    "mr_aha_plan_execute": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "mr_aha_plan_destroy": (ctypes.c_int, [_P]),
    "mr_aha_toeplitz": (ctypes.c_int, [ctypes.POINTER(MRConfig), _P, _P, _P, _P, _P]),
    "mr_op_options_defaults": (ctypes.c_int, [ctypes.POINTER(MROpOptions)]),
    "mr_op_create": (ctypes.c_int, [ctypes.POINTER(MRConfig), ctypes.POINTER(MROpInputs),
                                    ctypes.POINTER(MROpOptions), ctypes.POINTER(_P)]),
    "mr_op_execute": (ctypes.c_int, [_P, _P, _P]),
    "mr_op_info": (ctypes.c_int, [_P, ctypes.POINTER(MROpInfo)]),
    "mr_op_kernel": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P)]),
    "mr_op_destroy": (ctypes.c_int, [_P]),
    "mr_op_abandon": (ctypes.c_int, [_P]),
    "mr_calc_toep": (ctypes.c_int, [ctypes.POINTER(MRConfig), _P, _P, _I64, _I64, _P, _P]),
    "mr_calc_toep_from_psf": (ctypes.c_int, [ctypes.POINTER(MRConfig), _P, _I64, _I64, _P, _P]),
    "mr_calc_mask": (ctypes.c_int, [ctypes.POINTER(MRConfig), _P, _I64, _I64, _P,
                                    ctypes.POINTER(_I64)]),
    "mr_b200_op_set_kernel_format": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "mr_b200_op_kernel_format": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_op_launches": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_op_device_status": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_op_execute_host": (ctypes.c_int, [_P, _P, _P]),
    "mr_b200_op_save_kernel16": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), _P, _P]),
    "mr_b200_op_load_kernel16": (ctypes.c_int, [_P, ctypes.c_int, _P, _P]),
    "mr_b200_op_host_sync": (ctypes.c_int, [_P]),
    "mr_b200_op_host_release": (ctypes.c_int, [_P]),
    "mr_b200_trace_launches": (ctypes.c_int, [ctypes.c_int]),
    "mr_b200_trace_read": (_I64, [ctypes.c_char_p, ctypes.c_size_t]),
    "mr_b200_aha_toeplitz_noalloc": (ctypes.c_int, [ctypes.POINTER(MRConfig), _P, _P, _P, _P,
                                                    _P]),
    "mr_b200_op_profile": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_float),
                                          ctypes.c_char_p, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_op_autotune": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    "mr_b200_batch_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.POINTER(_P)]),
    "mr_b200_batch_execute": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _P]),
    "mr_b200_batch_destroy": (ctypes.c_int, [_P]),
    "mr_b200_op_blocked_copy": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_op_device_bytes": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "mr_b200_cg_busy": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_cg_iterations": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_cg_create": (ctypes.c_int, [_P, _P, _P, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(_P)]),
    "mr_b200_cg_step": (ctypes.c_int, [_P, ctypes.c_int]),
    "mr_b200_cg_residuals": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int)]),
    "mr_b200_cg_destroy": (ctypes.c_int, [_P]),
    "mr_b200_cg_solve": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
}

LIB_DIR = Path(__file__).resolve().parent / "lib"
LIB_NAME = "libmr_aha_c.so"


def library_path() -> Path:
    override = os.environ.get("MR_AHA_LIBRARY")
    if override:
        return Path(override)
    return LIB_DIR / LIB_NAME


def _load() -> ctypes.CDLL:
    path = library_path()
    if not path.exists():
        raise OSError(
            f"{path} not found: build the CUDA library first "
            f"(python -m mr_aha_b200.build); there is no CPU fallback"
        )
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _LazyLib:
    """Loads the library on first use, so that the package (and its build
    script) import without it; any call then fails loudly if it is missing."""

    _cdll = None

    def __getattr__(self, name):
        if _LazyLib._cdll is None:
            _LazyLib._cdll = _load()
        return getattr(_LazyLib._cdll, name)


lib = _LazyLib()


def backend() -> str:
    return lib.mr_backend().decode()


def check(status: int, what: str) -> None:
    """Raise :class:`MRError` with the library's message for a failed call."""
    if status != 0:
        msg = lib.mr_last_error().decode(errors="replace")
        name = lib.mr_status_string(int(status)).decode()
        raise MRError(int(status), f"{what} failed: {name}: {msg}")
