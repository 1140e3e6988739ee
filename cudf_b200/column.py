"""Device columns and tables (the roles of pylibcudf's Column and Table,
python/cudf/cudf/_lib/pylibcudf/column.pyx and table.pyx), backed by torch
CUDA tensors.  Null masks are libcudf's LSB-first 32-bit validity words."""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .types import CAI_TYPESTR, FROM_TORCH, NUMPY_DTYPE, TORCH_DTYPE, TypeId


def pack_mask(valid: torch.Tensor) -> torch.Tensor:
    """bool[n] (device) -> int32[(n+31)//32] validity words, bit i = row i valid."""
    n = valid.numel()
    words = (n + 31) // 32
    padded = torch.zeros(words * 32, dtype=torch.int64, device=valid.device)
    padded[:n] = valid.to(torch.int64)
    w = (padded.view(words, 32) << torch.arange(32, device=valid.device, dtype=torch.int64)).sum(1)
    return w.to(torch.int64).bitwise_and(0xFFFFFFFF).to(torch.int32) if words else torch.zeros(0, dtype=torch.int32, device=valid.device)


def unpack_mask(words: torch.Tensor, n: int) -> torch.Tensor:
    """int32 validity words -> bool[n] on the same device."""
    if n == 0:
        return torch.zeros(0, dtype=torch.bool, device=words.device)
    w = words.to(torch.int64).bitwise_and(0xFFFFFFFF)
    bits = (w.unsqueeze(1) >> torch.arange(32, device=words.device, dtype=torch.int64)) & 1
    return bits.reshape(-1)[:n].to(torch.bool)


class Column:
    """A fixed-width device column: data tensor, optional validity words, offset."""

    def __init__(self, type_id: int, data: torch.Tensor, mask: Optional[torch.Tensor] = None,
                 size: Optional[int] = None, offset: int = 0, null_count: Optional[int] = None,
                 _owner=None):
        self.type_id = TypeId(type_id)
        self._data = data
        self._mask = mask
        self._raw = None  # (data ptr, mask ptr) of an engine-owned result not yet wrapped
        self.offset = int(offset)
        self.size = int(data.numel() - self.offset if size is None else size)
        self._null_count = null_count
        self._owner = _owner

    @staticmethod
    def from_device_buffers(type_id: int, data_ptr: int, mask_ptr: int, size: int, null_count: int,
                            owner) -> "Column":
        """A zero-copy column over engine-owned device buffers.  The torch
        views are made on first access, so results nobody reads cost no
        wrapping; `owner` keeps the buffers alive."""
        c = Column.__new__(Column)
        c.type_id = TypeId(type_id)
        c._data = None
        c._mask = None
        c._raw = (int(data_ptr or 0), int(mask_ptr or 0))
        c.offset = 0
        c.size = int(size)
        c._null_count = int(null_count)
        c._owner = owner
        return c

    def _materialize(self):
        if self._raw is not None:
            dp, mp = self._raw
            self._raw = None
            self._data = tensor_from_device(dp, self.size, self.type_id, self._owner)
            self._mask = mask_from_device(mp, self.size, self._owner)

    @property
    def data(self) -> torch.Tensor:
        self._materialize()
        return self._data

    @data.setter
    def data(self, t: torch.Tensor):
        self._raw = None
        self._data = t

    @property
    def mask(self) -> Optional[torch.Tensor]:
        self._materialize()
        return self._mask

    @mask.setter
    def mask(self, m: Optional[torch.Tensor]):
        self._materialize()
        self._mask = m

    # -- construction ---------------------------------------------------
    @staticmethod
    def from_tensor(t: torch.Tensor, valid: Optional[torch.Tensor] = None,
                    type_id: Optional[int] = None) -> "Column":
        if type_id is None:
            type_id = FROM_TORCH[t.dtype]
        t = t.contiguous()
        if valid is None:
            mask = None
        elif valid.dtype in (torch.int32, torch.uint32) and valid.numel() == (t.shape[0] + 31) // 32:
            mask = valid.to(t.device).contiguous()  # packed validity words, LSB first
        else:
            mask = pack_mask(valid.to(device=t.device, dtype=torch.bool))
        return Column(type_id, t, mask)

    @staticmethod
    def from_numpy(arr, valid=None, type_id: Optional[int] = None, device="cuda") -> "Column":
        arr = np.array(arr, copy=True, order="C") if not np.asarray(arr).flags.writeable else np.ascontiguousarray(arr)
        if type_id is None:
            type_id = {np.dtype(v): k for k, v in NUMPY_DTYPE.items()
                       if k not in (TypeId.BOOL8,) and k < 12}[arr.dtype]
        type_id = TypeId(type_id)
        if type_id == TypeId.BOOL8:
            t = torch.from_numpy(arr.astype(np.uint8) != 0)
        else:
            t = torch.from_numpy(arr.astype(NUMPY_DTYPE[type_id], copy=False).view(NUMPY_DTYPE[type_id]))
        t = t.to(device)
        v = None if valid is None else torch.from_numpy(np.asarray(valid, dtype=bool)).to(device)
        return Column.from_tensor(t, v, type_id)

    # -- views ----------------------------------------------------------
    def gb_view(self) -> _lib.GbColumn:
        if self._raw is not None:
            dp, mp = self._raw
            return _lib.GbColumn(int(self.type_id), self.size, dp if self.size else 0, mp, 0)
        return _lib.GbColumn(int(self.type_id), self.size, self.data.data_ptr() if self.data.numel() else 0,
                             0 if self.mask is None else self.mask.data_ptr(), self.offset)

    @property
    def null_count(self) -> int:
        if self._null_count is None:
            if self.mask is None:
                self._null_count = 0
            else:
                v = unpack_mask(self.mask, self.offset + self.size)[self.offset:]
                self._null_count = int((~v).sum().item())
        return self._null_count

    def valid(self) -> Optional[torch.Tensor]:
        if self.mask is None:
            return None
        return unpack_mask(self.mask, self.offset + self.size)[self.offset:]

    def values(self) -> torch.Tensor:
        return self.data[self.offset:self.offset + self.size]

    def to_numpy(self):
        """(values ndarray, valid bool ndarray | None) on the host."""
        d = self.values()
        if self.type_id == TypeId.BOOL8:
            vals = d.to(torch.uint8).cpu().numpy()
        elif d.dtype in (torch.uint16, torch.uint32, torch.uint64):
            vals = d.cpu().numpy()
        else:
            vals = d.cpu().numpy()
        v = self.valid()
        return vals, (None if v is None else v.cpu().numpy())

    def __len__(self):
        return self.size

    def __repr__(self):
        return f"Column({self.type_id.name}, size={self.size}, nullable={self.mask is not None})"


class Table:
    def __init__(self, columns: Sequence[Column]):
        self.columns = list(columns)

    def num_columns(self) -> int:
        return len(self.columns)

    def num_rows(self) -> int:
        return self.columns[0].size if self.columns else 0

    def __getitem__(self, i):
        return self.columns[i]

    def __len__(self):
        return len(self.columns)


class HostStaging:
    """Pinned host buffers reused across device->host copies of results.

    A copy into pageable host memory (``tensor.cpu()``) runs at a few GB/s,
    one into pinned memory at the PCIe rate (~55 GB/s on B200 hosts), so
    callers that read results back every call keep one of these.  The arrays
    ``to_host`` returns are views into the staging buffers: they stay valid
    until the next ``to_host`` call on the same staging object."""

    def __init__(self):
        self._bufs: list = []

    def to_host(self, tensors: Sequence[torch.Tensor], stream=None) -> list:
        out = []
        for i, t in enumerate(tensors):
            nbytes = t.numel() * t.element_size()
            if i >= len(self._bufs) or self._bufs[i].numel() < nbytes:
                buf = torch.empty(max(nbytes, 1), dtype=torch.uint8).pin_memory()
                if i >= len(self._bufs):
                    self._bufs.append(buf)
                else:
                    self._bufs[i] = buf
            view = self._bufs[i][:nbytes].view(t.dtype) if nbytes else torch.empty(0, dtype=t.dtype)
            if nbytes:
                view.copy_(t.reshape(-1), non_blocking=True)
            out.append(view)
        if stream is not None:
            stream.synchronize()
        else:
            torch.cuda.current_stream().synchronize()
        return [v.numpy() for v in out]


class _CAI:
    """__cuda_array_interface__ view of an engine-owned buffer; keeps the owner alive."""

    def __init__(self, ptr: int, n: int, type_id: int, owner, stream: int):
        self.__cuda_array_interface__ = {
            "shape": (n,), "typestr": CAI_TYPESTR[type_id], "data": (ptr, False), "version": 3,
            "strides": None, "stream": None,
        }
        self._owner = owner


def tensor_from_device(ptr: int, n: int, type_id: int, owner, stream: int = 0) -> torch.Tensor:
    if n == 0 or not ptr:
        return torch.empty(0, dtype=TORCH_DTYPE[TypeId(type_id)], device="cuda")
    return torch.as_tensor(_CAI(ptr, n, type_id, owner, stream), device="cuda")


def mask_from_device(ptr: int, n: int, owner) -> Optional[torch.Tensor]:
    if not ptr:
        return None
    words = max(1, (n + 31) // 32)
    return torch.as_tensor(_CAI(ptr, words, TypeId.INT32, owner, 0), device="cuda")
