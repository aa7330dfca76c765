"""Host image buffers with the layout the AGO CPU kernels expect: byte strides, padding
rows/columns around the image (HAF stencils read one or two pixels outside the area they
process), and a controllable address alignment (HAF kernels pick their scalar/SIMD split
from the destination address)."""
from __future__ import annotations

import numpy as np


class Img:
    def __init__(self, h, w, dtype=np.uint8, channels=1, pad=4, stride=None, align_off=0, fill=None, rng=None):
        self.h, self.w, self.dtype, self.channels = h, w, np.dtype(dtype), channels
        bpp = self.dtype.itemsize * channels
        self.stride = stride if stride is not None else ((w * bpp + 15) // 16) * 16 + 64
        self.pad = pad
        total = (h + 2 * pad) * self.stride + 256
        self.raw = np.zeros(total, dtype=np.uint8)
        if rng is not None:
            self.raw[:] = rng.integers(0, 256, total, dtype=np.uint8)
        base = self.raw.ctypes.data
        start = pad * self.stride + 64
        start += (-(base + start) % 64) + align_off
        self.off = start
        self.bpp = bpp
        if fill is not None:
            self.set(fill)

    @property
    def ptr(self) -> int:
        """Address of pixel (0, 0)."""
        return self.raw.ctypes.data + self.off

    def row_ptr(self, y: int) -> int:
        return self.ptr + y * self.stride

    def view(self) -> np.ndarray:
        """(h, w[, c]) view of the image pixels."""
        a = np.lib.stride_tricks.as_strided(
            self.raw[self.off:], shape=(self.h, self.w * self.bpp), strides=(self.stride, 1))
        a = a.view(self.dtype) if self.dtype.itemsize > 1 else a
        if self.channels > 1:
            a = a.reshape(self.h, self.w, self.channels)
        return a

    def set(self, arr: np.ndarray) -> None:
        v = self.view()
        v[...] = np.asarray(arr, dtype=self.dtype).reshape(v.shape)

    def get(self) -> np.ndarray:
        return np.array(self.view())
