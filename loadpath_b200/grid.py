"""Device layout of one grid level and the host <-> device conversions.

A level with (nx, ny, nz) cells keeps
  node fields  (3, nx+1, ny+1, pz)   pz = nz+1 rounded up to a multiple of 4
  cell fields  (nx, ny, pz)          the same pitch (cells nz..pz-1 are zero padding)
  node mask    (nx+1, ny+1, pz) uint8
so that 16-byte vector loads along z stay aligned. Padding entries are zero and every kernel
keeps them zero.
"""
from __future__ import annotations

import numpy as np
import torch

__all__ = ["DevGrid", "torch_dtype", "stream_handle"]


def torch_dtype(dt) -> torch.dtype:
    dt = np.dtype(dt)
    if dt == np.float32:
        return torch.float32
    if dt == np.float64:
        return torch.float64
    raise ValueError(f"unsupported precision {dt}")


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


class DevGrid:
    def __init__(self, cells, device="cuda"):
        self.nx, self.ny, self.nz = (int(c) for c in cells)
        self.NX, self.NY, self.NZ = self.nx + 1, self.ny + 1, self.nz + 1
        self.pz = (self.NZ + 3) // 4 * 4
        self.cpz = self.pz
        self.device = torch.device(device)

    @property
    def cells(self):
        return (self.nx, self.ny, self.nz)

    @property
    def node_shape(self):
        return (3, self.NX, self.NY, self.NZ)

    @property
    def args(self):
        """The five ints the C ABI takes for a level."""
        return (self.nx, self.ny, self.nz, self.pz, self.cpz)

    @property
    def n_node_field(self) -> int:
        return 3 * self.NX * self.NY * self.pz

    @property
    def n_cell_field(self) -> int:
        return self.nx * self.ny * self.cpz

    def node_field(self, dtype) -> torch.Tensor:
        return torch.zeros((3, self.NX, self.NY, self.pz), dtype=dtype, device=self.device)

    def cell_field(self, dtype) -> torch.Tensor:
        return torch.zeros((self.nx, self.ny, self.cpz), dtype=dtype, device=self.device)

    def mask_field(self) -> torch.Tensor:
        return torch.zeros((self.NX, self.NY, self.pz), dtype=torch.uint8, device=self.device)

    # host <-> device -------------------------------------------------------------------
    def nodes_to_dev(self, a: np.ndarray, dtype, out: torch.Tensor | None = None) -> torch.Tensor:
        """(3, NX, NY, NZ) host array -> padded device node field."""
        a = np.asarray(a)
        assert a.shape == self.node_shape, (a.shape, self.node_shape)
        t = out if out is not None else self.node_field(dtype)
        host = torch.from_numpy(np.ascontiguousarray(a)).to(dtype)
        t[:, :, :, :self.NZ].copy_(host, non_blocking=False)
        return t

    def nodes_to_host(self, t: torch.Tensor) -> np.ndarray:
        return t[:, :, :, :self.NZ].cpu().numpy().copy()

    def cells_to_dev(self, a: np.ndarray, dtype, out: torch.Tensor | None = None) -> torch.Tensor:
        a = np.asarray(a)
        assert a.shape == self.cells, (a.shape, self.cells)
        t = out if out is not None else self.cell_field(dtype)
        t[:, :, :self.nz].copy_(torch.from_numpy(np.ascontiguousarray(a)).to(dtype))
        return t

    def cells_to_host(self, t: torch.Tensor) -> np.ndarray:
        return t[:, :, :self.nz].cpu().numpy().copy()

    def mask_to_host(self, t: torch.Tensor) -> np.ndarray:
        """uint8 mask -> float (3, NX, NY, NZ) 0/1 solved-dof mask (the reference's level.mask)."""
        m = t[:, :, :self.NZ].cpu().numpy()
        return np.stack([(m >> c) & 1 for c in range(3)]).astype(np.float64)

    def bits_to_dev(self, boolgrid: np.ndarray) -> torch.Tensor:
        """bool (3, NX, NY, NZ) -> uint8 bits per node (bit c = component c)."""
        b = np.asarray(boolgrid, bool)
        bits = (b[0].astype(np.uint8) | (b[1].astype(np.uint8) << 1) | (b[2].astype(np.uint8) << 2))
        t = self.mask_field()
        t[:, :, :self.NZ].copy_(torch.from_numpy(np.ascontiguousarray(bits)))
        return t
