"""ctypes binding of the C ABI in ``include/acfdtd_b200.h`` (``libacfdtd_b200.so``).

The library is built in-tree by ``build.py`` (nvcc, sm_100a). There is no fallback: if the
shared object is missing or fails to load, every solver constructor raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

__all__ = ["AcfConfig", "library", "check", "NativeError", "LIBRARY_PATH", "EXPORTED_SYMBOLS"]

LIBRARY_PATH = Path(__file__).resolve().parent / "libacfdtd_b200.so"
MAX_RELAXATION = 4

FIELD_P, FIELD_VX, FIELD_VY, FIELD_VZ, FIELD_PSI0 = 0, 1, 2, 3, 4

_STATUS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "out of memory", 4: "bad state",
           5: "non-finite state"}

#: Bits of a handle's device status word (acf_device_status).
STATUS_WAIT_TIMEOUT, STATUS_NON_FINITE = 1, 2
ERR_STATE, ERR_NUMERIC = 4, 5

#: Every entry point declared in include/acfdtd_b200.h.
EXPORTED_SYMBOLS = (
    "acf_abi_version", "acf_struct_size", "acf_last_error", "acf_device_count",
    "acf_create", "acf_destroy", "acf_is_double", "acf_set_sources", "acf_set_receivers",
    "acf_read_recording", "acf_upload", "acf_download", "acf_run", "acf_set_graph",
    "acf_energy_terms", "acf_field_pointer", "acf_profile_enable", "acf_profile_read",
    "acf_launch_count", "acf_synchronize", "acf_host_alloc", "acf_host_free",
    "acf_energy_terms_noalloc", "acf_set_launch",
    "acf_batch_create", "acf_batch_destroy", "acf_batch_room_count", "acf_batch_set_sources",
    "acf_batch_set_receivers", "acf_batch_read_recording", "acf_batch_upload",
    "acf_batch_download", "acf_batch_run", "acf_batch_set_graph", "acf_batch_set_launch",
    "acf_batch_energy_terms", "acf_batch_profile_enable", "acf_batch_profile_read",
    "acf_batch_launch_count", "acf_set_coefficients", "acf_adjoint_prepare",
    "acf_adjoint_shell_size", "acf_forward_record", "acf_adjoint_run", "acf_adjoint_download",
    "acf_reset_state", "acf_set_scheme", "acf_get_scheme", "acf_set_staging", "acf_device_status",
    "acf_batch_set_scheme", "acf_adjoint_checkpoint_interval", "acf_set_device",
    "acf_batch_adjoint_prepare", "acf_batch_adjoint_shell_size", "acf_batch_forward_record",
    "acf_batch_adjoint_run", "acf_batch_reset_state", "acf_batch_set_coefficients",
    "acf_set_prefetch", "acf_get_prefetch", "acf_batch_set_prefetch", "acf_copy_plane",
    "acf_solver_device", "acf_energy_terms_planes", "acf_run_slabs", "acf_batch_device_status",
    "acf_set_wait_test", "acf_schroeder_decay", "acf_decay_fit", "acf_clarity",
    "acf_spectral_divide", "acf_pressure_only_energy_terms", "acf_set_time_blocking",
    "acf_get_time_blocking",
)

SCHEME_TWO_SWEEPS, SCHEME_FUSED, SCHEME_FUSED_STAGED, SCHEME_PRESSURE_ONLY = 0, 1, 2, 3

GRAD_WALLS, GRAD_AIR = 1, 2


class NativeError(RuntimeError):
    """A C ABI call returned a non-zero status."""

    def __init__(self, status: int, call: str, message: str):
        super().__init__(f"{call}: {_STATUS.get(status, status)}: {message}")
        self.status = status


class AcfConfig(ctypes.Structure):
    """Field-for-field mirror of ``acf_config``; its size is checked against the library."""

    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("n_relax", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("vel_coef", ctypes.c_double), ("pres_coef", ctypes.c_double),
        ("src_coef", ctypes.c_double), ("relax_scale", ctypes.c_double),
        ("relax_decay", ctypes.c_double * MAX_RELAXATION),
        ("relax_mean", ctypes.c_double * MAX_RELAXATION),
        ("relax_gain", ctypes.c_double * MAX_RELAXATION),
        ("wall_shell", ctypes.POINTER(ctypes.c_double) * 6),
        ("cell", ctypes.POINTER(ctypes.c_double) * 3),
        ("face", ctypes.POINTER(ctypes.c_double) * 3),
    ]


_lib: ctypes.CDLL | None = None

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I64P = ctypes.POINTER(ctypes.c_int64)
_DP = ctypes.POINTER(ctypes.c_double)

_SIGNATURES = {
    "acf_abi_version": (ctypes.c_int, []),
    "acf_struct_size": (ctypes.c_size_t, []),
    "acf_last_error": (ctypes.c_char_p, []),
    "acf_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "acf_create": (ctypes.c_int, [ctypes.POINTER(AcfConfig), ctypes.POINTER(_P)]),
    "acf_destroy": (ctypes.c_int, [_P]),
    "acf_is_double": (ctypes.c_int, [_P]),
    "acf_set_sources": (ctypes.c_int, [_P, _I64, _I64P, _I64P, _DP, _I64]),
    "acf_set_receivers": (ctypes.c_int, [_P, _I64, _I64P, _I64P]),
    "acf_read_recording": (ctypes.c_int, [_P, _I64, _I64, _I64, _P, _P]),
    "acf_upload": (ctypes.c_int, [_P, ctypes.c_int, _P, _P]),
    "acf_download": (ctypes.c_int, [_P, ctypes.c_int, _P, _P]),
    "acf_run": (ctypes.c_int, [_P, _I64, _I64, _P]),
    "acf_set_graph": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_set_launch": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "acf_energy_terms": (ctypes.c_int, [_P, ctypes.c_double, _DP, _P]),
    "acf_field_pointer": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P), _I64P]),
    "acf_profile_enable": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_profile_read": (ctypes.c_int, [_P, _DP, _DP, _I64P]),
    "acf_launch_count": (ctypes.c_int64, [_P]),
    "acf_synchronize": (ctypes.c_int, [_P]),
    "acf_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(_P)]),
    "acf_host_free": (ctypes.c_int, [_P]),
    "acf_energy_terms_noalloc": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                                _P, _P]),
    "acf_batch_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(AcfConfig),
                                        ctypes.POINTER(_P)]),
    "acf_batch_destroy": (ctypes.c_int, [_P]),
    "acf_batch_room_count": (ctypes.c_int, [_P]),
    "acf_batch_set_sources": (ctypes.c_int, [_P, ctypes.c_int32, _I64, _I64P, _I64P, _DP, _I64]),
    "acf_batch_set_receivers": (ctypes.c_int, [_P, ctypes.c_int32, _I64, _I64P, _I64P]),
    "acf_batch_read_recording": (ctypes.c_int, [_P, ctypes.c_int32, _I64, _I64, _I64, _P, _P]),
    "acf_batch_upload": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int, _P, _P]),
    "acf_batch_download": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int, _P, _P]),
    "acf_batch_run": (ctypes.c_int, [_P, _I64, _I64, _P]),
    "acf_batch_set_graph": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_batch_set_launch": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "acf_batch_energy_terms": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, _DP, _P]),
    "acf_batch_profile_enable": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_batch_profile_read": (ctypes.c_int, [_P, _DP, _DP, _I64P]),
    "acf_batch_launch_count": (ctypes.c_int64, [_P]),
    "acf_set_coefficients": (ctypes.c_int, [_P, ctypes.POINTER(AcfConfig)]),
    "acf_adjoint_prepare": (ctypes.c_int, [_P, ctypes.c_int32, _I64, ctypes.c_int32]),
    "acf_adjoint_shell_size": (ctypes.c_int64, [_P]),
    "acf_forward_record": (ctypes.c_int, [_P, _I64, _I64, _P]),
    "acf_adjoint_run": (ctypes.c_int, [_P, _DP, _DP, _DP, _DP, _P]),
    "acf_adjoint_download": (ctypes.c_int, [_P, ctypes.c_int, _P, _P]),
    "acf_reset_state": (ctypes.c_int, [_P, _P]),
    "acf_set_scheme": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_get_scheme": (ctypes.c_int, [_P]),
    "acf_set_staging": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "acf_batch_set_scheme": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_adjoint_checkpoint_interval": (ctypes.c_int32, [_P]),
    "acf_set_device": (ctypes.c_int, [ctypes.c_int32]),
    "acf_device_status": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "acf_batch_device_status": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "acf_set_wait_test": (ctypes.c_int, [_P, _I64, ctypes.c_int32]),
    "acf_pressure_only_energy_terms": (ctypes.c_int, [_P, _DP, _P]),
    "acf_schroeder_decay": (ctypes.c_int, [_P, _I64, _I64, ctypes.c_double, _P, _P]),
    "acf_decay_fit": (ctypes.c_int, [_P, _I64, _I64, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, _P, _P, _P]),
    "acf_clarity": (ctypes.c_int, [_P, _I64, _I64, _I64, _P, _P]),
    "acf_spectral_divide": (ctypes.c_int, [_P, _P, _I64, _I64, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, _P, _P, _P]),
    "acf_batch_adjoint_prepare": (ctypes.c_int, [_P, _I64]),
    "acf_batch_adjoint_shell_size": (ctypes.c_int64, [_P, ctypes.c_int32]),
    "acf_batch_forward_record": (ctypes.c_int, [_P, _I64, _I64, _P]),
    "acf_batch_adjoint_run": (ctypes.c_int, [_P, _DP, _DP, _DP, _P]),
    "acf_batch_reset_state": (ctypes.c_int, [_P, _P]),
    "acf_batch_set_coefficients": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(AcfConfig)]),
    "acf_set_prefetch": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_get_prefetch": (ctypes.c_int, [_P]),
    "acf_set_time_blocking": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_get_time_blocking": (ctypes.c_int, [_P]),
    "acf_batch_set_prefetch": (ctypes.c_int, [_P, ctypes.c_int32]),
    "acf_copy_plane": (ctypes.c_int, [_P, _I64, _P, _I64, ctypes.c_int, _P]),
    "acf_solver_device": (ctypes.c_int, [_P]),
    "acf_energy_terms_planes": (ctypes.c_int, [_P, ctypes.c_double, _I64, _I64, ctypes.c_int32, _DP, _P]),
    "acf_run_slabs": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                     ctypes.POINTER(ctypes.c_int32), _I64, _I64, _P]),
}


def library() -> ctypes.CDLL:
    """Load the CUDA library once; raise if it is absent or does not match this binding."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise RuntimeError(
            f"{LIBRARY_PATH.name} is not built; run `python -c 'import __graft_entry__ as g; "
            "g.build()'` or `python -m ac_fdtd_b200.build` (needs nvcc)"
        )
    lib = ctypes.CDLL(str(LIBRARY_PATH))
    for name, (restype, argtypes) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if lib.acf_struct_size() != ctypes.sizeof(AcfConfig):
        raise RuntimeError(
            "the ctypes mirror of acf_config no longer matches the C definition: "
            f"{ctypes.sizeof(AcfConfig)} bytes here, {lib.acf_struct_size()} bytes there"
        )
    _lib = lib
    return lib


def check(status: int, call: str) -> None:
    if status != 0:
        message = library().acf_last_error()
        raise NativeError(status, call, message.decode() if message else "")
