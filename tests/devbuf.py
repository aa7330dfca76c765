"""Device image buffers for calling the C ABI directly (torch only provides the memory)."""
from __future__ import annotations

import numpy as np
import torch


class DevImg:
    def __init__(self, h, w, dtype=np.uint8, channels=1, stride=None, align_off=0, device="cuda:0"):
        self.h, self.w, self.dtype, self.channels = h, w, np.dtype(dtype), channels
        self.bpp = self.dtype.itemsize * channels
        self.stride = stride if stride is not None else ((w * self.bpp + 255) // 256) * 256
        nbytes = h * self.stride + 512
        self.t = torch.zeros(nbytes, dtype=torch.uint8, device=device)
        base = self.t.data_ptr()
        self.off = (-base % 256) + align_off

    @property
    def ptr(self) -> int:
        return self.t.data_ptr() + self.off

    def row_ptr(self, y):
        return self.ptr + y * self.stride

    def upload(self, arr: np.ndarray) -> "DevImg":
        a = np.ascontiguousarray(np.asarray(arr, dtype=self.dtype)).view(np.uint8).reshape(self.h, self.w * self.bpp)
        host = np.zeros((self.h, self.stride), np.uint8)
        host[:, : self.w * self.bpp] = a
        flat = torch.from_numpy(host.reshape(-1))
        self.t[self.off: self.off + self.h * self.stride].copy_(flat)
        return self

    def download(self) -> np.ndarray:
        torch.cuda.synchronize()
        raw = self.t[self.off: self.off + self.h * self.stride].cpu().numpy().reshape(self.h, self.stride)
        a = np.ascontiguousarray(raw[:, : self.w * self.bpp]).view(self.dtype)
        if self.channels > 1:
            a = a.reshape(self.h, self.w, self.channels)
        return a


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream
