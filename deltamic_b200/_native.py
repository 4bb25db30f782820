"""ctypes binding of ``lib/libdeltamic_b200.so`` (the C ABI in include/deltamic_b200.h).

The library is required: there is no CPU or PyTorch fallback.  ``lib()`` raises
``RuntimeError`` when the shared object is missing or fails to load.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libdeltamic_b200.so")

DM_OK = 0
DM_BAND_HERMITIAN = 1
DM_ERR_INVALID_ARG = 1
DM_ERR_BAD_INDEX = 2
DM_ERR_SIZE = 4
DM_ERR_WORKSPACE = 8
DM_ERR_CUDA = 16
DM_ERR_TIMEOUT = 32
DM_ERR_UNSUPPORTED = 64
DM_ERR_NONFINITE = 128

ABI_VERSION = 2

# Entry points and their (restype, argtypes); every symbol of the public header.
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_SZ = ctypes.c_size_t
_F = ctypes.c_float
_INT = ctypes.c_int
_I32 = ctypes.c_int32


class DmBox(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3),
                ("shape", ctypes.c_int32 * 3), ("band_flags", ctypes.c_int32)]


_BOXP = ctypes.POINTER(DmBox)


class DmCell(ctypes.Structure):
    _fields_ = [("nv", ctypes.c_int64), ("nt", ctypes.c_int64), ("n_band", ctypes.c_int64),
                ("grid_offset", ctypes.c_int64), ("box", DmBox)]


class DmBatch(ctypes.Structure):
    _fields_ = [("ncells", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("nv", ctypes.c_int64), ("nt", ctypes.c_int64), ("n_band", ctypes.c_int64),
                ("grid_elems", ctypes.c_int64), ("fwd_workspace", ctypes.c_int64),
                ("bwd_workspace", ctypes.c_int64), ("topology_bytes", ctypes.c_int64),
                ("image_workspace", ctypes.c_int64), ("plan", ctypes.c_int64 * 12),
                ("cells", ctypes.c_void_p)]


_BATCHP = ctypes.POINTER(DmBatch)


class DmBandboxBatch(ctypes.Structure):
    _fields_ = [("ncells", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("workspace_bytes", ctypes.c_int64), ("plan", ctypes.c_int64 * 128),
                ("cells", ctypes.c_void_p), ("workspace", ctypes.c_void_p)]


_BBBP = ctypes.POINTER(DmBandboxBatch)

SIGNATURES = {
    "dm_abi_version": (_INT, []),
    "dm_status_string": (ctypes.c_char_p, [_INT]),
    "dm_device_error": (_INT, [_P, ctypes.POINTER(_INT), _P]),
    "dm_narrowband_workspace_size": (_SZ, [_I64]),
    "dm_narrowband_compact": (_INT, [_P, _I64, _F, _P, _P, _P, _SZ, _P]),
    "dm_narrowband_compact64": (_INT, [_P, _I64, ctypes.c_double, _P, _P, _P, _SZ, _P]),
    "dm_narrowband_hermitian": (_INT, [_P, _I64, _I64, _P, _P]),
    "dm_topology_size": (_SZ, [_I64, _I64]),
    "dm_topology_build": (_INT, [_P, _I64, _I64, _P, _SZ, _P]),
    "dm_meshft_forward_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft_forward": (_INT, [_P, _I64, _P, _I64, _P, _BOXP, _P, _I64, _P, _P, _P, _P, _SZ,
                                 _P]),
    "dm_meshft_forward_noalloc": (_INT, [_P, _I64, _P, _I64, _P, _BOXP, _P, _I64, _P, _P, _P,
                                         _P]),
    "dm_meshft_forward_noalloc_device_error": (_INT, [ctypes.POINTER(_INT), _P]),
    "dm_meshft_forward_xi_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft_forward_xi": (_INT, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P, _SZ, _P]),
    "dm_meshft_backward_xi_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft_backward_xi": (_INT, [_P, _I64, _P, _I64, _P, _P, _P, _P, _I64, _P, _P, _P, _P,
                                     _SZ, _P]),
    "dm_meshft64_forward_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft64_forward": (_INT, [_P, _I64, _P, _I64, _P, _BOXP, _P, _P, _I64, _P, _P, _P, _P,
                                   _SZ, _P]),
    "dm_meshft64_backward_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft64_backward": (_INT, [_P, _I64, _P, _I64, _P, _BOXP, _P, _P, _I64, _P, _P, _P,
                                    ctypes.c_double, _P, _P, _P, _P, _P, _SZ, _P]),
    "dm_meshft_volume_forward_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft_volume_forward": (_INT, [_P, _I64, _P, _I64, _P, _BOXP, _P, _I64, _P, _P, _P,
                                        _P, _P, _SZ, _P]),
    "dm_meshft_volume_backward_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft_volume_backward": (_INT, [_P, _I64, _P, _I64, _P, _BOXP, _P, _I64, _P, _P, _P,
                                         _F, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "dm_meshft_backward_workspace_size": (_SZ, [_I64, _I64, _I64]),
    "dm_meshft_backward": (_INT, [_P, _I64, _P, _I64, _P, _BOXP, _P, _I64, _P, _P, _P, _F, _P,
                                  _P, _P, _P, _P, _P, _SZ, _P]),
    "dm_aniso_gaussian_psf": (_INT, [_P, _P, _I32, _P, _I32, _P, _I32, _P, _P]),
    "dm_aniso_gaussian_psf_grad_workspace_size": (_SZ, [_I64]),
    "dm_aniso_gaussian_psf_grad": (_INT, [_P, _P, _P, _P, _I32, _P, _I32, _P, _I32, _P, _P,
                                          _SZ, _P]),
    "dm_radial_basis": (_INT, [_P, _I32, _P, _P, _I64, _P, _P, _P, _P]),
    "dm_radial_basis_grad_workspace_size": (_SZ, [_I64, _I32]),
    "dm_radial_basis_grad": (_INT, [_P, _P, _I32, _P, _P, _I64, _P, _P, _I32, _P, _P, _P, _P,
                                    _SZ, _P]),
    "dm_radial_intensity_workspace_size": (_SZ, [_I64, _I32]),
    "dm_radial_intensity": (_INT, [_P, _I64, _I32, _P, _I64, _P, _P, _P, _P, _SZ, _P]),
    "dm_radial_intensity_backward": (_INT, [_P, _P, _P, _P, _I64, _I32, _P, _P, _P, _P, _SZ,
                                            _P]),
    "dm_pupil_defocus": (_INT, [_P, _P, _P, _I32, _I32, _I32, _P, _P]),
    "dm_pupil_defocus_grad_workspace_size": (_SZ, [_I32, _I32, _I32]),
    "dm_pupil_defocus_backward": (_INT, [_P, _P, _P, _P, _I32, _I32, _I32, _P, _P, _P, _P, _SZ,
                                         _P]),
    "dm_shifted_intensity": (_INT, [_P, _I32, _I32, _I32, _P, _P]),
    "dm_shifted_intensity_backward": (_INT, [_P, _P, _I32, _I32, _I32, _P, _P]),
    "dm_zernike": (_INT, [_P, _P, _I64, _P, _I32, _P, _P]),
    "dm_mask_workspace_size": (_SZ, [_I64, _I32, _BOXP]),
    "dm_membrane_mask": (_INT, [_P, _I64, _P, _I64, _I32, _BOXP, ctypes.c_double, _I32, _P, _P,
                                _SZ, _P]),
    "dm_instance_mask": (_INT, [_P, _I64, _P, _I64, _BOXP, _I32, _P, _P, _SZ, _P]),
    "dm_batch_desc_size": (_SZ, [_INT]),
    "dm_batch_plan": (_INT, [ctypes.POINTER(DmCell), _INT, _P, _SZ, _BATCHP, _P]),
    "dm_bandbox_batch_desc_size": (_SZ, [_INT]),
    "dm_bandbox_batch_workspace_size": (_INT, [ctypes.POINTER(DmCell), _P, _INT,
                                               ctypes.POINTER(ctypes.c_size_t)]),
    "dm_bandbox_batch_plan": (_INT, [ctypes.POINTER(DmCell), _P, _INT, _P, _SZ, _P, _SZ, _BBBP,
                                     _P]),
    "dm_bandbox_batch_render_loss": (_INT, [_BBBP, _P, _P, _P, _INT, _P, _F, _P, _P, _P, _P]),
    "dm_bandbox_batch_device_error": (_INT, [_BBBP, ctypes.POINTER(_INT), _P]),
    "dm_batched_topology_build": (_INT, [_BATCHP, _P, _P, _SZ, _P]),
    "dm_batched_meshft_forward": (_INT, [_BATCHP, _P, _P, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "dm_batched_meshft_backward": (_INT, [_BATCHP, _P, _P, _P, _P, _P, _P, _P, _F, _P, _P, _P,
                                          _P, _P, _P, _SZ, _P]),
    "dm_batched_image_loss": (_INT, [_BATCHP, _P, _INT, _P, _F, _P, _P, _P, _P, _SZ, _P]),
    "dm_gaussian_otf": (_INT, [_P, _P, ctypes.c_int32, _P, ctypes.c_int32, _P, ctypes.c_int32,
                               _P, _P]),
    "dm_gaussian_otf64": (_INT, [_P, _P, ctypes.c_int32, _P, ctypes.c_int32, _P, ctypes.c_int32,
                                 _P, _P]),
    "dm_gaussian_otf64_sigma_grad": (_INT, [_P, _P, _I64, _P, _P, ctypes.c_int32, _P,
                                            ctypes.c_int32, _P, ctypes.c_int32, _P, _P, _SZ, _P]),
    "dm_gaussian_otf_grad_workspace_size": (_SZ, [_I64]),
    "dm_gaussian_otf_sigma_grad": (_INT, [_P, _P, _I64, _P, _P, ctypes.c_int32, _P,
                                          ctypes.c_int32, _P, ctypes.c_int32, _P, _P, _SZ, _P]),
    "dm_image_loss_workspace_size": (_SZ, [_I64]),
    "dm_image_loss": (_INT, [_P, _I64, _INT, _P, _F, _P, _P, _P, _P, _SZ, _P]),
    "dm_normalize_workspace_size": (_SZ, [_I64]),
    "dm_normalize": (_INT, [_P, _I64, ctypes.c_double, _P, _P, _P, _SZ, _P]),
    "dm_normalize_backward": (_INT, [_P, _P, _I64, ctypes.c_double, _P, _P, _P, _SZ, _P]),
    "dm_normalize64": (_INT, [_P, _I64, ctypes.c_double, _P, _P, _P, _SZ, _P]),
    "dm_normalize64_backward": (_INT, [_P, _P, _I64, ctypes.c_double, _P, _P, _P, _SZ, _P]),
    "dm_band_bounds": (_INT, [_P, _I64, _BOXP, _P, _P]),
    "dm_render_loss_bandbox_supported": (_INT, [_BOXP, ctypes.POINTER(ctypes.c_int32)]),
    "dm_render_loss_bandbox_workspace_size": (_SZ, [_BOXP, ctypes.POINTER(ctypes.c_int32)]),
    "dm_render_loss_bandbox": (_INT, [_P, _P, _I64, _BOXP, ctypes.POINTER(ctypes.c_int32), _P,
                                      _INT, _P, _F, _P, _P, _P, _P, _SZ, _P]),
    "dm_conv3d_s2_workspace_size": (_SZ, [_INT] * 6),
    "dm_conv3d_s2_forward": (_INT, [_P, _INT, _INT, _INT, _INT, _INT, _P, _P, _INT, _P, _P, _P]),
    "dm_conv3d_s2_device_error": (_INT, [ctypes.POINTER(_INT), _P]),
    "dm_conv3d_s2_forward_workspace_size": (_SZ, [_INT] * 6),
    "dm_conv3d_s2_forward_ws": (_INT, [_P, _INT, _INT, _INT, _INT, _INT, _P, _P, _INT, _P, _P,
                                       _P, _SZ, _P]),
    "dm_conv3d_s2_backward": (_INT, [_P, _INT, _INT, _INT, _INT, _INT, _P, _INT, _P, _P, _P, _P,
                                     _P, _P, _SZ, _P]),
    "dm_conv3d_s2_backward_bf16": (_INT, [_P, _INT, _INT, _INT, _INT, _INT, _P, _INT, _P, _P,
                                          _P, _P, _P, _P, _SZ, _P]),
    "dm_voxelize": (_INT, [_P, _I64, _P, _I64, _BOXP, _P, _P, _P]),
    "dm_adam_step": (_INT, [_P, _P, _P, _P, _I64, _F, _F, _F, _F, _P, _P]),
    "dm_precond_apply": (_INT, [_P, _I64, _I64, _P, _P, _P]),
    "dm_precond_chebyshev": (_INT, [_P, _P, _I64, _F, ctypes.c_double, ctypes.c_double, _INT,
                                    _P, _P, _P, _P]),
    "dm_otf_from_spectrum": (_INT, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P]),
    "dm_otf_from_spectrum_backward": (_INT, [_P, _P, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, _P, _P]),
    "dm_vector_adam_step": (_INT, [_P, _P, _P, _P, _I64, _F, _F, _F, _F, _P, _P]),
    "dm_launch_count": (ctypes.c_longlong, []),
    "dm_set_variants": (_INT, [_INT, _INT]),
    "dm_get_variants": (_INT, [ctypes.POINTER(_INT)] * 4),
    "dm_peak_probe": (_INT, [_INT, _INT, ctypes.POINTER(ctypes.c_double), _P]),
    "dm_selftest_bounded_wait": (_INT, [_INT, ctypes.c_uint32, _P, _P]),
    "dm_profile_enable": (_INT, [_INT]),
    "dm_profile_read": (_INT, [_INT, ctypes.POINTER(_INT), ctypes.POINTER(_F)]),
}

_lib = None
_lock = threading.Lock()


def lib():
    """The loaded library (loads it on first use; raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"deltamic_b200 native library not found at {LIB_PATH}; build it with "
                "`python -m deltamic_b200.build` (nvcc, sm_100a). There is no CPU fallback.")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        if handle.dm_abi_version() != ABI_VERSION:
            raise RuntimeError("libdeltamic_b200.so ABI version mismatch; rebuild it")
        _lib = handle
    return _lib


class DeltaMicError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().dm_status_string(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


def check(status: int, where: str) -> None:
    if status != DM_OK:
        raise DeltaMicError(status, where)


def ptr(t) -> int | None:
    """Device address of a tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def make_box(box_size, box_shape) -> DmBox:
    b = DmBox()
    for d in range(3):
        b.lo[d] = float(box_size[d][0])
        b.hi[d] = float(box_size[d][1])
        b.shape[d] = int(box_shape[d])
    b.band_flags = 0
    return b


def require_cuda(t: torch.Tensor, name: str, dtype=None) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor (deltamic_b200 has no CPU path)")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


class Workspace:
    """Grow-only device scratch buffer per (device, purpose)."""

    def __init__(self):
        self._bufs: dict = {}

    def get(self, key, nbytes: int, device) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        k = (key, str(device))
        buf = self._bufs.get(k)
        if buf is None or buf.numel() < nbytes:
            buf = torch.zeros(nbytes, dtype=torch.uint8, device=device)
            self._bufs[k] = buf
        return buf


WORKSPACES = Workspace()
