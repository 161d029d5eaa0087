"""Device layout of one grid level and the host <-> device conversions.

A level with (nx, ny, nz) cells cuts z into chunks of four planes, the chunk index slowest:
  node fields  (3, pz/4, ny+1, nx+1, 4)   pz = nz+1 rounded up to a multiple of 4
  cell fields  (pz/4, ny, nx, 4)          the same pitch (cells nz..pz-1 are zero padding)
  node mask    (pz/4, ny+1, nx+1, 4) uint8
so a chunk's four planes of a row of x are one contiguous run (16 bytes per column in float32):
tile loads and stores move whole rows. Padding entries are zero and every kernel keeps them
zero. Host arrays are in grid order, (3, NX, NY, NZ) for nodes and (nx, ny, nz) for cells.
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
        return torch.zeros((3, self.pz // 4, self.NY, self.NX, 4), dtype=dtype, device=self.device)

    def cell_field(self, dtype) -> torch.Tensor:
        return torch.zeros((self.cpz // 4, self.ny, self.nx, 4), dtype=dtype, device=self.device)

    def mask_field(self) -> torch.Tensor:
        return torch.zeros((self.pz // 4, self.NY, self.NX, 4), dtype=torch.uint8, device=self.device)

    # layout <-> grid order (torch, on either side) ---------------------------------------
    def node_grid(self, t: torch.Tensor) -> torch.Tensor:
        """device node field (or mask, without the component axis) -> grid order
        (3, NX, NY, NZ) / (NX, NY, NZ), a new contiguous tensor on t's device."""
        if t.dim() == 5:
            g = t.permute(0, 3, 2, 1, 4).reshape(3, self.NX, self.NY, self.pz)
            return g[..., :self.NZ].contiguous()
        g = t.permute(2, 1, 0, 3).reshape(self.NX, self.NY, self.pz)
        return g[..., :self.NZ].contiguous()

    def cell_grid(self, t: torch.Tensor) -> torch.Tensor:
        """device cell field -> grid order (nx, ny, nz), a new contiguous tensor."""
        return t.permute(2, 1, 0, 3).reshape(self.nx, self.ny, self.cpz)[..., :self.nz].contiguous()

    def set_nodes(self, t: torch.Tensor, a: torch.Tensor) -> torch.Tensor:
        """t (node field or mask) <- a in grid order ((3, NX, NY, NZ) or (NX, NY, NZ), any device);
        the z padding is zeroed."""
        lead = (3,) if t.dim() == 5 else ()
        full = torch.zeros(lead + (self.NX, self.NY, self.pz), dtype=t.dtype, device=t.device)
        full[..., :self.NZ] = a.to(device=t.device, dtype=t.dtype)
        v = full.view(lead + (self.NX, self.NY, self.pz // 4, 4))
        t.copy_(v.permute(0, 3, 2, 1, 4) if lead else v.permute(2, 1, 0, 3))
        return t

    def set_cells(self, t: torch.Tensor, a) -> torch.Tensor:
        """t (cell field) <- a in grid order ((nx, ny, nz) tensor, or a scalar for every cell);
        the z padding is zeroed."""
        full = torch.zeros((self.nx, self.ny, self.cpz), dtype=t.dtype, device=t.device)
        if isinstance(a, torch.Tensor):
            full[..., :self.nz] = a.to(device=t.device, dtype=t.dtype)
        else:
            full[..., :self.nz] = a
        t.copy_(full.view(self.nx, self.ny, self.cpz // 4, 4).permute(2, 1, 0, 3))
        return t

    # host <-> device -------------------------------------------------------------------
    def nodes_to_dev(self, a: np.ndarray, dtype, out: torch.Tensor | None = None) -> torch.Tensor:
        """(3, NX, NY, NZ) host array -> padded device node field."""
        a = np.asarray(a)
        assert a.shape == self.node_shape, (a.shape, self.node_shape)
        t = out if out is not None else self.node_field(dtype)
        return self.set_nodes(t, torch.from_numpy(np.ascontiguousarray(a)))

    def nodes_to_host(self, t: torch.Tensor) -> np.ndarray:
        return self.node_grid(t).cpu().numpy()

    def cells_to_dev(self, a: np.ndarray, dtype, out: torch.Tensor | None = None) -> torch.Tensor:
        a = np.asarray(a)
        assert a.shape == self.cells, (a.shape, self.cells)
        t = out if out is not None else self.cell_field(dtype)
        return self.set_cells(t, torch.from_numpy(np.ascontiguousarray(a)))

    def cells_to_host(self, t: torch.Tensor) -> np.ndarray:
        return self.cell_grid(t).cpu().numpy()

    def mask_to_host(self, t: torch.Tensor) -> np.ndarray:
        """uint8 mask -> float (3, NX, NY, NZ) 0/1 solved-dof mask (the reference's level.mask)."""
        m = self.node_grid(t).cpu().numpy()
        return np.stack([(m >> c) & 1 for c in range(3)]).astype(np.float64)

    def bits_to_dev(self, boolgrid: np.ndarray) -> torch.Tensor:
        """bool (3, NX, NY, NZ) -> uint8 bits per node (bit c = component c)."""
        b = np.asarray(boolgrid, bool)
        bits = (b[0].astype(np.uint8) | (b[1].astype(np.uint8) << 1) | (b[2].astype(np.uint8) << 2))
        return self.set_nodes(self.mask_field(), torch.from_numpy(np.ascontiguousarray(bits)))
