"""Host mirror of the reference's TiledDeviceOutput (src/calculator/tiled_device_output.jl) over the
library's epb_tiled object, plus ind_range_for_k_range (src/band_states.jl:416-428) and
residency_use_block. Shapes are Julia's (column-major); `i_axis` is 1-based as in the reference; k
indices and state ranges are 1-based."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

_KIND = {4: "f32", 8: "f64", 16: "c128"}
_NP = {4: np.float32, 8: np.float64, 16: np.complex128}


def ind_range_for_k_range(iks, nk, kstart, kend):
    """range(first, last + 1) of the 1-based states whose k lies in kstart:kend (empty when none);
    EpbError when they are not contiguous."""
    iks = np.ascontiguousarray(np.asarray(iks, dtype=np.int64))
    a, b = C.c_int64(), C.c_int64()
    check(_lib.lib().epb_ind_range_for_k_range(iks.ctypes.data if iks.size else None, iks.size, int(nk), int(kstart),
                                               int(kend), C.byref(a), C.byref(b)))
    return range(a.value, b.value + 1)


def tile_capacity(iks, nk, n_batch_max):
    iks = np.ascontiguousarray(np.asarray(iks, dtype=np.int64))
    c = C.c_int64()
    check(_lib.lib().epb_tiled_plan(iks.ctypes.data if iks.size else None, iks.size, int(nk), int(n_batch_max),
                                    C.byref(c)))
    return c.value


def residency_use_block(full_bytes, headroom=1.2, ctx=None):
    ctx = ctx or _lib.default_context()
    b = C.c_int()
    check(_lib.lib().epb_residency_use_block(ctx.h, int(full_bytes), float(headroom), C.byref(b)))
    return bool(b.value)


class TiledDeviceOutput:
    def __init__(self, dims, i_axis, iks, nk, *, narr=1, elem_bytes=8, force_block=None, headroom=1.2,
                 n_batch_max=1, ctx=None):
        self.ctx = ctx or _lib.default_context()
        self.dims = tuple(int(d) for d in dims)
        self.i_axis = int(i_axis)
        if not 1 <= self.i_axis <= len(self.dims):
            raise ValueError(f"i_axis {i_axis} out of range for dims {self.dims}")
        self.elem = int(elem_bytes)
        self.narr = int(narr)
        iks = np.ascontiguousarray(np.asarray(iks, dtype=np.int64))
        d = np.asarray(self.dims, dtype=np.int64)
        fb = -1 if force_block is None else (1 if force_block else 0)
        h = C.c_void_p()
        check(_lib.lib().epb_tiled_create(self.ctx.h, d.ctypes.data, len(self.dims), self.i_axis - 1, self.narr,
                                          self.elem, fb, float(headroom), iks.ctypes.data if iks.size else None,
                                          iks.size, int(nk), int(n_batch_max), C.byref(h)))
        self.h = h

    def _info(self):
        info = _lib.TiledInfo()
        check(_lib.lib().epb_tiled_get_info(self.h, C.byref(info)))
        return info

    def tile_begin(self, kstart, kend):
        check(_lib.lib().epb_tiled_begin(self.ctx.h, self.h, int(kstart), int(kend)))
        return self

    def is_allocated(self):
        return bool(self._info().allocated)

    def is_block(self):
        return bool(self._info().block)

    def tile_offset(self):
        return self._info().tile_offset

    def tile_length(self):
        return self._info().tile_length

    def tile_stride(self):
        return self._info().tile_stride

    def device_array(self, k=1):
        """The k-th (1-based) device buffer as a torch view in Julia byte layout, extent tile_stride along
        the tiled axis."""
        from .outer_q import _view

        p = C.c_void_p()
        check(_lib.lib().epb_tiled_device_array(self.h, int(k) - 1, C.byref(p)))
        shape = list(self.dims)
        shape[self.i_axis - 1] = self.tile_stride()
        return _view(p.value, tuple(shape), _KIND[self.elem], None)

    def tile_download(self, k=1):
        """Array k on the host (Fortran order): the current tile in block mode, all of it in full mode."""
        shape = list(self.dims)
        if self.is_block():
            shape[self.i_axis - 1] = self.tile_length()
        out = np.zeros(shape, dtype=_NP[self.elem], order="F")
        check(_lib.lib().epb_tiled_download(self.ctx.h, self.h, int(k) - 1, out.ctypes.data))
        return out

    def tile_free(self):
        check(_lib.lib().epb_tiled_free(self.h))
        return self

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().epb_tiled_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
