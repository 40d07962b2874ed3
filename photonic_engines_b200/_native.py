"""ctypes binding of the CUDA library `libpe_b200.so` (C ABI declared in include/pe_b200.h).

The library is the only compute path: when it is missing, or no CUDA device is visible, every
sampling call raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PE_LIB", os.path.join(_HERE, "libpe_b200.so"))

PE_OK = 0
PE_ERR_ARG = -1
PE_ERR_SIZE = -2
PE_ERR_CUDA = -3
PE_ERR_DEVICE = -4
PE_PRECISION_F64 = 0
PE_PRECISION_MIXED = 1
PE_PRECISION_COMPENSATED = 2
PE_MAX_PHOTONS = 64
PE_MIXED_MAX_PHOTONS = 32          # the FP32 forms are compiled up to 32 columns: FP64 beyond


def check_photons(n: int, precision: str, what: str = "photons per stream") -> None:
    """ValueError unless the library runs chains of n photons in this precision."""
    if n > PE_MAX_PHOTONS:
        raise ValueError(f"at most {PE_MAX_PHOTONS} {what} (got {n})")
    if precision in ("mixed", "compensated") and n > PE_MIXED_MAX_PHOTONS:
        raise ValueError(f"precision={precision!r} runs at most {PE_MIXED_MAX_PHOTONS} {what} (got {n}); "
                         f"use precision='f64'")
PRECISIONS = {"f64": PE_PRECISION_F64, "mixed": PE_PRECISION_MIXED, "compensated": PE_PRECISION_COMPENSATED}

_lib = None
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int


class NativeError(RuntimeError):
    """A status < 0 returned by the CUDA library, or the library missing."""


def load() -> ctypes.CDLL:
    """Load libpe_b200.so (raises NativeError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeError(f"{LIB_PATH} is missing: build it with `python -m photonic_engines_b200.build` "
                          "(there is no non-CUDA path)")
    L = ctypes.CDLL(LIB_PATH)
    L.pe_version.restype = _i32
    L.pe_version.argtypes = []
    L.pe_max_modes.restype = _i32
    L.pe_max_modes.argtypes = [_i32]
    L.pe_chain_workspace_bytes.restype = ctypes.c_size_t
    L.pe_chain_workspace_bytes.argtypes = [_i64]
    L.pe_fock_chain.restype = _i32
    L.pe_fock_chain.argtypes = [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp,
                                _vp, _vp, _vp, _i32, _vp, _i32, _vp, ctypes.c_size_t, _i32, _i32, _i32, _vp]
    L.pe_fock_chain_split.restype = _i32
    L.pe_fock_chain_split.argtypes = [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                                      _vp, _vp, _vp, _vp, _i32, _vp, _i32, _i32, _i32, _vp, ctypes.c_size_t, _i32, _i32,
                                      _vp]
    L.pe_fock_chain_warp.restype = _i32
    L.pe_fock_chain_warp.argtypes = [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                                     _vp, _vp, _vp, _vp, _i32, _vp, _i32, _vp, ctypes.c_size_t, _i32, _i32, _vp]
    L.pe_fock_chain_range.restype = _i32
    L.pe_fock_chain_range.argtypes = [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                                      _vp, _vp, _vp, _vp, _i32, _vp, _i32, _vp, ctypes.c_size_t, _i32, _i32, _i32,
                                      _vp, _i32, _i32, _vp]
    L.pe_fock_chain_range_split.restype = _i32
    L.pe_fock_chain_range_split.argtypes = [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _vp, _vp, _vp, _i32, _vp, _vp,
                                            _vp, _vp, _vp, _vp, _vp, _i32, _vp, _i32, _vp, ctypes.c_size_t, _i32,
                                            _i32, _vp, _i32, _i32, _i32, _i64, _vp]
    L.pe_range_split_workspace_bytes.restype = ctypes.c_size_t
    L.pe_range_split_workspace_bytes.argtypes = [_i64, _i32]
    L.pe_chain_split_workspace_bytes.restype = ctypes.c_size_t
    L.pe_chain_split_workspace_bytes.argtypes = [_i64, _i32]
    L.pe_fock_chain_adaptive.restype = _i32
    L.pe_fock_chain_adaptive.argtypes = [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _vp, _vp, _i32, _vp, _vp, _vp,
                                         _vp, _vp, _i32, _vp, _vp, _vp, _i32, _i32, _i32, _vp, ctypes.c_size_t, _i32,
                                         _i32, _i32, _vp]
    L.pe_adaptive_workspace_bytes.restype = ctypes.c_size_t
    L.pe_adaptive_workspace_bytes.argtypes = [_i64, _i32]
    L.pe_emitter_weights.restype = _i32
    L.pe_emitter_weights.argtypes = [_vp, _i32, _i32, _vp, _i32, _vp, _i64, _i32, _i32, _i32, _vp, _vp, _vp, _i64, _vp,
                                     _vp, _vp, _vp, _i64, _vp, _vp, _vp, ctypes.c_size_t, _vp]
    L.pe_emitter_workspace_bytes.restype = ctypes.c_size_t
    L.pe_emitter_workspace_bytes.argtypes = []
    L.pe_emitter_count.restype = _i32
    L.pe_emitter_count.argtypes = [_vp, _vp, _i64, _i32, _vp, _vp, _vp, _i32, _i32, _vp, _vp, ctypes.c_size_t, _vp]
    L.pe_emitter_step.restype = _i32
    L.pe_emitter_step.argtypes = [_vp, _i32, _i32, _vp, _i32, _vp, _vp, _vp, _i64, _i32, _i32, _i32, _vp, _vp, _vp,
                                  _vp, _vp, _vp, _vp, _i32, _i32, _vp, _vp, _i64, _vp, _vp, _vp, ctypes.c_size_t,
                                  _vp]
    L.pe_fock_chain_noalloc.restype = _i32
    L.pe_fock_chain_noalloc.argtypes = [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                                        _vp, _vp, _vp, _vp, _i32, _vp, _i32, _vp, _i32, _i32, _i32, _vp]
    L.pe_cofactors_rows.restype = _i32
    L.pe_cofactors_rows.argtypes = [_i32, _vp, _vp, _i64, _i32, _i32, _vp, _vp, ctypes.c_size_t, _i32, _i32, _vp]
    L.pe_partition_shots.restype = _i32
    L.pe_partition_shots.argtypes = [_vp, _vp, _vp, _vp, _i64, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.pe_scatter_occupations.restype = _i32
    L.pe_scatter_occupations.argtypes = [_vp, _vp, _vp, _i64, _i32, _vp, _i32, _i64, _vp, _vp]
    L.pe_pipe_probe.restype = _i32
    L.pe_pipe_probe.argtypes = [_i32, _i32, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double), _vp]
    L.pe_read_status.restype = _i32
    L.pe_read_status.argtypes = [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i64), _vp]
    L.pe_status_string.restype = ctypes.c_char_p
    L.pe_status_string.argtypes = [_i32]
    L.pe_last_cuda_error.restype = ctypes.c_char_p
    L.pe_last_cuda_error.argtypes = []
    L.pe_split_slots.restype = _i32
    L.pe_split_slots.argtypes = [_i32, _i32, _i32, _i32]
    _lib = L
    return L


# every symbol the C header declares (checked by the CPU test that loads the library)
EXPORTED = ("pe_version", "pe_max_modes", "pe_chain_workspace_bytes", "pe_fock_chain", "pe_fock_chain_noalloc",
            "pe_fock_chain_split", "pe_chain_split_workspace_bytes", "pe_split_slots", "pe_fock_chain_warp",
            "pe_fock_chain_range", "pe_fock_chain_range_split", "pe_range_split_workspace_bytes",
            "pe_fock_chain_adaptive", "pe_adaptive_workspace_bytes", "pe_emitter_weights",
            "pe_emitter_workspace_bytes", "pe_emitter_count", "pe_emitter_step",
            "pe_cofactors_rows", "pe_partition_shots", "pe_scatter_occupations", "pe_pipe_probe", "pe_read_status",
            "pe_status_string", "pe_last_cuda_error")


def check(rc: int, what: str) -> None:
    if rc != PE_OK:
        msg = load().pe_status_string(rc).decode()
        if rc == PE_ERR_CUDA:
            msg += ": " + load().pe_last_cuda_error().decode()
        raise NativeError(f"{what}: status {rc} ({msg})")


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not torch.cuda.is_available():
        raise NativeError("no CUDA device is visible: the B200 sampler has no CPU path")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must be a CUDA tensor (got {t.device})")


def workspace(device: torch.device) -> torch.Tensor:
    """A fresh device workspace for one call (queue counter + status word)."""
    n = int(load().pe_chain_workspace_bytes(0))
    return torch.empty(n, dtype=torch.uint8, device=device)


def read_status(ws: torch.Tensor) -> tuple[int, int]:
    st = _i32(0)
    det = _i64(0)
    check(load().pe_read_status(ptr(ws), ctypes.byref(st), ctypes.byref(det), stream_handle(ws.device)),
          "pe_read_status")
    return int(st.value), int(det.value)


def pipe_peak_tflops(precision: str, device, iters: int = 4096, reps: int = 5) -> float:
    """Measured FP64 ("f64") or FP32 ("mixed") FMA-pipe peak of the device, TFLOP/s (best of `reps`)."""
    L = load()
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    out = torch.empty(sms * 8 * 256, dtype=torch.float64, device=device)
    fl = ctypes.c_double(0.0)
    best = 0.0
    s = stream_handle(out.device)
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        check(L.pe_pipe_probe(PRECISIONS[precision], iters, ptr(out), out.numel() * 8, ctypes.byref(fl), s),
              "pe_pipe_probe")
        e1.record()
        e1.synchronize()
        best = max(best, fl.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best
