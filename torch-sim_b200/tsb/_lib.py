"""ctypes binding of the C ABI in ``include/tsb.h`` (library ``libtsb.so``).

This is the only way Python reaches the kernels: every op passes raw device
pointers, sizes and the current CUDA stream.  There is no CPU fallback -- if
the library is missing or a CUDA device is absent the ops raise.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import torch

from .build import LIB_PATH

TSB_OK = 0
TSB_ERR_INVALID_ARG = 1
TSB_ERR_CAPACITY = 2
TSB_ERR_NONFINITE = 3
TSB_ERR_TIMEOUT = 4
TSB_ERR_CUDA = 5
TSB_ERR_UNSUPPORTED = 6
TSB_ERR_WORKSPACE = 7

F32, F64 = 0, 1
POT_LJ, POT_MORSE, POT_SOFT, POT_PLIFE = 0, 1, 2, 3
NL_SELF_INTERACTION, NL_HALF = 1, 2
OUT_FORCES, OUT_STRESS, OUT_ENERGIES, OUT_STRESSES, MATH_FP64 = 1, 2, 4, 8, 16
INT_NVE, INT_LANGEVIN, INT_NOSE_HOOVER, INT_VRESCALE = 0, 1, 2, 3

_vp, _i64, _u64, _i32, _dbl, _sz, _int = (C.c_void_p, C.c_int64, C.c_uint64, C.c_int32,
                                         C.c_double, C.c_size_t, C.c_int)

_FIRE_ARGS = [_int, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
              _vp, _vp, _vp, _vp, _dbl, _int, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _int, _vp,
              _sz, _vp]

# name -> (restype, argtypes); mirrors include/tsb.h exactly
PROTOTYPES = {
    "tsb_version": (C.c_char_p, []),
    "tsb_status_string": (C.c_char_p, [_int]),
    "tsb_nl_workspace_size": (_sz, [_i64, _i64]),
    "tsb_nl_build": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _int, _dbl, _int, _vp, _i64,
                            _vp, _vp, _i64, _vp, _vp, _sz, _vp]),
    "tsb_pair_workspace_size": (_sz, [_i64, _i64]),
    "tsb_pair_forward": (_int, [_int, _vp, _int, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _int,
                                _dbl, _int, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _sz,
                                _vp]),
    "tsb_md_kick": (_int, [_vp, _vp, _vp, _vp, _dbl, _i64, _int, _vp]),
    "tsb_md_drift": (_int, [_vp, _vp, _vp, _vp, _vp, _dbl, _i64, _int, _vp]),
    "tsb_md_baoab_boa": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u64, _u64,
                                _vp, _i64, _int, _vp]),
    "tsb_adjoint_workspace_size": (_sz, [_i64, _i64, _i64]),
    "tsb_vv_kick_drift": (_int, [_vp, _vp, _vp, _vp, _dbl, _dbl, _vp, _vp, _i64, _vp]),
    "tsb_vv_kick": (_int, [_vp, _vp, _dbl, _vp, _i64, _vp]),
    "tsb_adj_kick": (_int, [_vp, _vp, _vp, _dbl, _i64, _vp]),
    "tsb_lj_hvp": (_int, [_vp, _int, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _dbl, _vp, _dbl, _vp,
                          _vp, _i64, _vp, _sz, _vp]),
    "tsb_rdf_hist": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _dbl, _int, _dbl, _vp, _i64, _vp,
                            _sz, _vp]),
    "tsb_rdf_hist_grad": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _dbl, _int, _dbl, _vp, _vp,
                                 _i64, _vp, _sz, _vp]),
    "tsb_verlet_workspace_size": (_sz, [_i64]),
    "tsb_verlet_build": (_int, [_vp, _vp, _i64, _int, _dbl, _dbl, _vp, _vp, _int, _vp, _vp,
                                _vp, _vp, _sz, _vp]),
    "tsb_verlet_check": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _int, _dbl, _vp, _vp, _sz,
                                _vp]),
    "tsb_verlet_forces": (_int, [_int, _vp, _int, _vp, _vp, _i64, _vp, _int, _dbl, _int, _vp,
                                 _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "tsb_npt_crescale_iso": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp, _vp,
                                    _vp, _vp, _vp, _vp, _u64, _u64, _vp, _sz, _vp]),
    "tsb_npt_crescale_aniso": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp,
                                      _vp, _vp, _vp, _vp, _vp, _u64, _u64, _vp, _sz, _vp]),
    "tsb_npt_crescale_tri": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp, _vp,
                                    _vp, _vp, _vp, _vp, _vp, _vp, _int, _vp, _u64, _u64, _vp,
                                    _sz, _vp]),
    "tsb_npt_langevin_aniso_pre": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp,
                                          _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                          _vp, _vp, _vp, _u64, _u64, _vp, _sz, _vp]),
    "tsb_npt_langevin_aniso_post": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp,
                                           _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                           _u64, _u64, _vp, _sz, _vp]),
    "tsb_npt_nh_iso_pre": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp,
                                  _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "tsb_npt_nh_iso_post": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp, _vp,
                                   _vp, _vp, _vp, _vp, _sz, _vp]),
    "tsb_vlist_workspace_size": (_sz, [_i64, _i64]),
    "tsb_vlist_reset": (_int, [_i64, _i64, _vp, _sz, _vp]),
    "tsb_vlist_check": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _int, _dbl, _dbl, _dbl, _vp, _vp,
                               _sz, _vp]),
    "tsb_vlist_build": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _int, _dbl, _dbl, _vp, _vp,
                               _int, _i64, _vp, _vp, _sz, _vp]),
    "tsb_vlist_hvp_scratch_size": (_sz, [_i64, _int]),
    "tsb_vlist_lj_hvp": (_int, [_vp, _int, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _dbl, _vp,
                                _dbl, _vp, _vp, _vp, _sz, _vp, _sz, _vp]),
    "tsb_vlist_forces": (_int, [_int, _vp, _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64,
                                _int, _dbl, _dbl, _int, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "tsb_fire_workspace_size": (_sz, [_i64]),
    "tsb_fire_ase_pre": (_int, _FIRE_ARGS),
    "tsb_fire_vv_pre": (_int, _FIRE_ARGS),
    "tsb_fire_vv_post": (_int, _FIRE_ARGS),
    "tsb_frechet_cell_forces": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _int, _vp, _int,
                                       _vp]),
    "tsb_fire_converged": (_int, [_vp, _vp, _i64, _i64, _vp, _dbl, _vp, _vp, _int, _vp, _sz,
                                  _vp]),
    "tsb_fused_max_atoms": (_int, []),
    "tsb_fused_workspace_size": (_sz, [_i64, _i64]),
    "tsb_fused_md": (_int, [_int, _int, _vp, _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64,
                            _i64, _vp, _dbl, _dbl, _i64, _vp, _vp, _vp, _u64, _u64, _vp, _vp,
                            _vp, _vp, _vp, _vp, _sz, _vp]),
    "tsb_fused_md_static": (_int, [_int, _int, _vp, _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                   _i64, _i64, _vp, _dbl, _dbl, _i64, _vp, _vp, _vp, _u64,
                                   _u64, _vp, _vp, _vp, _vp]),
    "tsb_fused_md_nvt": (_int, [_int, _int, _vp, _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                _i64, _i64, _vp, _dbl, _dbl, _i64, _vp, _vp, _vp, _vp, _vp,
                                _vp, _vp, _vp, _int, _int, _int, _u64, _u64, _vp, _vp, _vp,
                                _vp, _vp, _vp, _sz, _vp]),
    "tsb_fused_md_ex": (_int, [_int, _int, _vp, _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64,
                               _i64, _vp, _dbl, _dbl, _i64, _vp, _vp, _vp, _vp, _vp, _vp,
                               _vp, _vp, _vp, _int, _int, _int, _u64, _u64, _vp, _vp, _vp,
                               _i64, _i64, _int, _i64, _dbl, _vp, _vp, _vp, _vp, _vp, _sz,
                               _vp]),
    "tsb_npt_workspace_size": (_sz, [_i64]),
    "tsb_npt_langevin_iso_pre": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp,
                                        _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                        _vp, _vp, _vp, _u64, _u64, _vp, _sz, _vp]),
    "tsb_npt_langevin_iso_post": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp,
                                         _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                         _vp, _u64, _u64, _vp, _sz, _vp]),
    "tsb_thermostat_workspace_size": (_sz, [_i64]),
    "tsb_kinetic_energy": (_int, [_vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _sz, _vp]),
    "tsb_nhc_half_step": (_int, [_vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp, _vp, _vp,
                                 _vp, _vp, _vp, _int, _int, _int, _int, _vp, _sz, _vp]),
    "tsb_vrescale": (_int, [_vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp, _vp, _vp, _u64,
                            _u64, _vp, _vp, _sz, _vp]),
}

_lib = None
_lock = threading.Lock()


class TsbError(RuntimeError):
    """A tsb C-ABI call returned a non-zero status."""

    def __init__(self, name, status, msg=""):
        self.status = status
        super().__init__(f"{name} failed: status {status} ({status_string(status)}) {msg}")


def lib_path() -> str:
    return os.environ.get("TSB_LIB", LIB_PATH)


def load(path: str | None = None):
    """Load libtsb.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or lib_path()
        if not os.path.exists(p):
            raise RuntimeError(
                f"tsb CUDA library not found at {p}; build it with "
                "`python -m tsb.build` (nvcc, sm_100a). There is no CPU fallback.")
        lib = C.CDLL(p)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def status_string(status: int) -> str:
    try:
        return load().tsb_status_string(int(status)).decode()
    except Exception:  # noqa: BLE001
        return "?"


def call(name: str, *args):
    st = getattr(load(), name)(*args)
    if st != TSB_OK:
        raise TsbError(name, st)
    return st


_MAX_SYS_CACHE: dict = {}


def max_system_atoms(system_idx: torch.Tensor, n_systems: int) -> int:
    """Largest system's atom count (the binning hint of the C ABI), cached per
    system_idx tensor version (one device read when it changes)."""
    key = (system_idx.data_ptr(), system_idx._version, system_idx.shape[0], n_systems)
    hit = _MAX_SYS_CACHE.get(key)
    if hit is None:
        if system_idx.numel() == 0:
            hit = 0
        else:
            hit = int(torch.bincount(system_idx, minlength=n_systems).max())
        if len(_MAX_SYS_CACHE) > 64:
            _MAX_SYS_CACHE.clear()
        _MAX_SYS_CACHE[key] = hit
    return hit


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float64:
        return F64
    if dtype == torch.float32:
        return F32
    raise TypeError(f"tsb kernels support float32/float64, got {dtype}")


_PBC_CACHE: dict = {}


def pbc_rows(pbc, n_systems: int, device) -> torch.Tensor:
    """Periodic flags as a contiguous uint8 [S, 3] tensor from a bool, a 0-d or
    [3] tensor (every system alike), an [S, 3] tensor or a flat [3 S] one.

    Flags given on the host (a bool, a list or a CPU tensor) are converted once
    and cached per (flags, S, device), so later calls -- inside a CUDA-graph
    capture too -- copy nothing from the host."""
    if not (torch.is_tensor(pbc) and pbc.device.type == "cuda"):
        flags = torch.as_tensor(pbc).reshape(-1).tolist()
        key = (tuple(bool(f) for f in flags), int(n_systems), str(torch.device(device)))
        hit = _PBC_CACHE.get(key)
        if hit is None:
            if len(_PBC_CACHE) > 64:
                _PBC_CACHE.clear()
            hit = _pbc_rows(torch.as_tensor(pbc, device=device), n_systems)
            _PBC_CACHE[key] = hit
        return hit
    return _pbc_rows(pbc, n_systems)


def _pbc_rows(p: torch.Tensor, n_systems: int) -> torch.Tensor:
    if p.ndim == 0:
        p = p.reshape(1).expand(3)
    if p.ndim == 1 and p.shape[0] == 3:
        p = p.unsqueeze(0).expand(n_systems, 3)
    elif p.ndim == 1 and p.shape[0] == 3 * n_systems:
        p = p.reshape(n_systems, 3)
    if tuple(p.shape) != (n_systems, 3):
        raise ValueError(f"pbc of shape {tuple(p.shape)} does not fit {n_systems} systems")
    return p.to(torch.uint8).contiguous()


def require_cuda(t: torch.Tensor, what: str = "tensor") -> None:
    if not t.is_cuda:
        raise RuntimeError(f"tsb ops run on CUDA only ({what} is on {t.device}); "
                           "there is no CPU fallback")


class Workspace:
    """Per-device grow-only scratch buffer handed to the C ABI."""

    _bufs: dict = {}

    @classmethod
    def get(cls, device: torch.device, nbytes: int) -> torch.Tensor:
        # one buffer per (device, stream): calls are stream-ordered, so reuse on
        # the same stream is safe and concurrent streams never share scratch
        key = (device.type, device.index, stream_ptr(device))
        buf = cls._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes * 1.25), 1 << 20), dtype=torch.uint8,
                              device=device)
            cls._bufs[key] = buf
        return buf

    @classmethod
    def clear(cls) -> None:
        cls._bufs.clear()
