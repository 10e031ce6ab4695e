"""Helpers for the GPU parity tests: device buffers and C-ABI calls."""
import ctypes as C

import numpy as np
import torch

from firewebapp_b200 import _lib
from firewebapp_b200._lib import FsGrid, check, ptr

DEV = torch.device("cuda")


def dev(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


class Grid:
    """FsGrid on device plus the tensors it points into."""

    def __init__(self, nz, ny, nx, dx, dy, dz, da=None, db=None):
        self.nz, self.ny, self.nx = int(nz), int(ny), int(nx)
        self.shape = (self.nz, self.ny, self.nx)
        self.n = self.nz * self.ny * self.nx
        self.dz = dev(dz)
        self.da = dev(da if da is not None else dz)
        self.db = dev(db if db is not None else dz)
        self.g = FsGrid(self.nx, self.ny, self.nz, float(dx), float(dy), ptr(self.dz),
                        ptr(self.da), ptr(self.db))

    @property
    def ref(self):
        return C.byref(self.g)


def stream():
    return torch.cuda.current_stream().cuda_stream


def lib():
    return _lib.lib()


def call(name, *args):
    st = getattr(lib(), name)(*args)
    check(st, name)
    return st
