"""ctypes binding of the C ABI in ``include/hit3d.h``.

The shared library ``_lib/libhit3d_b200.so`` is built in-tree by ``build.py``
(``__graft_entry__.build()`` runs it).  There is no fallback: if the library
is missing every compute call raises, naming the build command.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# The in-tree build; HIT3D_LIB names another build of the same library (e.g.
# one made with different compile options) to load instead.
LIB_PATH = os.environ.get("HIT3D_LIB") or os.path.join(_HERE, "_lib", "libhit3d_b200.so")

HIT_OK = 0
HIT_E_INVALID = -1
HIT_E_CUDA = -2
HIT_E_ALLOC = -3
HIT_E_NONFINITE = -4
HIT_E_UNSUPPORTED = -5

HIT_DTYPE_F32 = 0
HIT_DTYPE_F64 = 1

HIT_FORCING_NONE = 0
HIT_FORCING_LINEAR = 1
HIT_FORCING_BAND = 2
HIT_FORCING_HOLD_ENERGY = 3

HIT_FLAG_ASSUME_DEALIASED = 1
HIT_FLAG_INTEGRATING_FACTOR = 2
HIT_NUM_KERNEL_CLASSES = 6
KERNEL_CLASSES = ("x-inverse", "y-inverse", "z-pass", "y-forward", "x-forward+epilogue", "forcing-coef")

# Every entry point of include/hit3d.h: name -> (restype, argtypes)
_vp, _i, _d, _i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64


class HitParams(ctypes.Structure):
    """``hit_params`` of include/hit3d.h."""

    _fields_ = [
        ("nu", ctypes.c_double),
        ("forcing_kind", ctypes.c_int),
        ("flags", ctypes.c_uint),
        ("A", ctypes.c_double),
        ("eps", ctypes.c_double),
        ("kmin", ctypes.c_double),
        ("kmax", ctypes.c_double),
        ("E_target", ctypes.c_double),
        ("tau", ctypes.c_double),
    ]


_PP = ctypes.POINTER(HitParams)

SIGNATURES = {
    "hit_plan_create": (_i, [_i, _i, _i, _d, _d, _d, _i, ctypes.POINTER(_vp)]),
    "hit_plan_destroy": (_i, [_vp]),
    "hit_plan_num_shells": (_i, [_vp]),
    "hit_to_physical": (_i, [_vp, _vp, _i, _vp, _vp]),
    "hit_to_spectral": (_i, [_vp, _vp, _i, _vp, _vp]),
    "hit_dealias_project": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "hit_shell_scale": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "hit_check_dealiased": (_i, [_vp, _vp, _vp, _vp]),
    "hit_rhs": (_i, [_vp, _vp, _PP, _d, _vp, _vp]),
    "hit_rk4_step": (_i, [_vp, _vp, _PP, _d, _d, _vp, _vp]),
    "hit_rollout": (_i, [_vp, _vp, _PP, _d, _i64, _d, _vp, _vp]),
    "hit_rhs_forced": (_i, [_vp, _vp, _PP, _vp, _d, _vp, _vp]),
    "hit_device_status": (_i, [ctypes.POINTER(ctypes.c_int)]),
    "hit_set_wait_limit": (_i, [_i]),
    "hit_rk4_step_forced_vjp": (_i, [_vp, _vp, _PP, _vp, _d, _d, _vp, _vp, _vp, _vp, _vp]),
    "hit_sgs_force_vjp": (_i, [_vp, _vp, _vp, _vp]),
    "hit_axis_fft": (_i, [_vp, _vp, _vp, _i, _i, _i, _vp]),
    "hit_velocity_gradients_vjp": (_i, [_vp, _vp, _vp, _vp]),
    "hit_mlp_vjp": (_i, [_vp, _vp, _vp, _i64, _i64, _vp, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hit_rollout_forced": (_i, [_vp, _vp, _PP, _vp, _d, _i64, _d, _vp, _vp]),
    "hit_les_rollout": (_i, [_vp, _vp, _PP, _vp, _d, _i64, _vp, _vp, _vp]),
    "hit_profile_rollout": (_i, [_vp, _vp, _PP, _d, _i64, _vp, _vp, _vp, _vp]),
    "hit_rhs_vjp": (_i, [_vp, _vp, _PP, _d, _vp, _vp, _vp, _vp]),
    "hit_rk4_step_vjp": (_i, [_vp, _vp, _PP, _d, _d, _vp, _vp, _vp, _vp]),
    "hit_rollout_vjp": (_i, [_vp, _vp, _PP, _d, _i64, _d, _i, _vp, _vp, _vp, _vp]),
    "hit_energy_spectrum": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "hit_energy_budget": (_i, [_vp, _vp, _PP, _vp, _vp]),
    "hit_tc_gemm_bf16": (_i, [_vp, _i, _vp, _i, _vp, _i, _i, _i, _i, _vp, _vp]),
    "hit_mlp_forward": (_i, [_vp, _vp, _i64, _vp, _vp, _vp]),
    "hit_mlp_forward_strided": (_i, [_vp, _vp, _i64, _i64, _i64, _vp, _i64, _i64, _i, _vp, _vp]),
    "hit_velocity_gradients": (_i, [_vp, _vp, _vp, _vp]),
    "hit_add_sgs_force": (_i, [_vp, _vp, _vp, _vp]),
    "hit_sgs_force": (_i, [_vp, _vp, _vp, _vp]),
    "hit_mlp_workspace_bytes": (_i64, [_i64]),
    "hit_mlp_train_grads": (_i, [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hit_energy_spectrum_noalloc": (_i, [_i, _i, _i, _d, _d, _d, _i, _vp, _vp, _vp, _vp]),
    "hit_last_error_string": (ctypes.c_char_p, []),
}


class MlpWeights(ctypes.Structure):
    """hit_mlp_weights (include/hit3d.h): device pointers of the closure MLP."""
    _fields_ = [(n, ctypes.c_void_p) for n in ("w1t", "w2t", "w3t", "w4t", "w2", "w3", "w4", "b2", "b3", "b4")]


class HitError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, func, code, message):
        super().__init__(f"{func} failed with status {code}: {message}")
        self.code = code


_lib = None
_lock = threading.Lock()


def load(path=LIB_PATH):
    """dlopen the library and bind every signature (no GPU needed)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(
                f"{path} is missing: build it with `python 3dhit_b200/build.py` "
                "(or __graft_entry__.build()); there is no non-CUDA fallback")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def call(name, *args):
    """Call an entry point and raise HitError on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != HIT_OK:
        msg = lib.hit_last_error_string().decode(errors="replace")
        if rc == HIT_E_INVALID:
            raise ValueError(f"{name}: {msg}")
        raise HitError(name, rc, msg)
    return rc


class DeviceWaitError(RuntimeError):
    """A bounded wait inside a transform kernel gave up: the results of the
    calls since the last check are not valid."""


def check_device(where=""):
    """Raise `DeviceWaitError` if a bounded TMA wait of a transform pass gave
    up since the last check (``hit_device_status``, which reads and clears
    the flag; it synchronises with the current device)."""
    st = ctypes.c_int(0)
    call("hit_device_status", ctypes.byref(st))
    if st.value:
        raise DeviceWaitError(f"a TMA tile wait of a transform kernel gave up{' in ' + where if where else ''}; "
                              "the results since the last check are not valid")


def stream_ptr(device):
    """The current torch stream of `device` as a void* (cudaStream_t)."""
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Plan:
    """Owns one ``hit_plan`` (one grid, one dtype, one device)."""

    def __init__(self, Nx, Ny, Nz, Lx, Ly, Lz, f64, device):
        self.device = torch.device(device)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            call("hit_plan_create", Nx, Ny, Nz, float(Lx), float(Ly), float(Lz),
                 HIT_DTYPE_F64 if f64 else HIT_DTYPE_F32, ctypes.byref(h))
        self.handle = h
        self.num_shells = load().hit_plan_num_shells(h)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            try:
                _lib.hit_plan_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None
