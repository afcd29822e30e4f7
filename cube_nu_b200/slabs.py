"""Runs split into z-slabs over ranks (``Params.nslab > 1``): the host side.

The reference decomposes its box into nn^3 images that exchange ghost layers of particles
(buffer_particle.f90:29-375), transpose the PM1 pencils (pencil_fft.f90:81-325) and reduce
the dt criteria (kick.f90:316-346) through coarrays.  This library splits the box along z
into slabs of whole tile layers, one rank each, and does that work itself; it needs two
collectives from the host, passed as the callbacks of ``cube_comm`` (include/cube_gpu.h).
``TorchComm`` implements them with torch.distributed: NCCL on device memory (the message
buffers are wrapped in place), or gloo through host copies.  The other helpers cut a
whole-box particle state into the slabs' parts and join them again.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import ALLREDUCE_FN, SENDRECV_FN, CComm, load
from .params import Params

DT_F32, DT_I64, DT_F64, DT_I32 = 0, 1, 2, 3
OP_SUM, OP_MAX = 0, 1
_NP_DTYPE = {DT_F32: np.float32, DT_I64: np.int64, DT_F64: np.float64, DT_I32: np.int32}


class _DeviceArray:
    """A raw device pointer as a CUDA array (the __cuda_array_interface__ protocol), so
    torch can wrap the library's buffer without a copy."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


class TorchComm:
    """cube_comm over a torch.distributed process group: rank r of the group steps slab r.

    allreduce and sendrecv are called by the library from inside a step, on the calling
    thread; a Python exception is kept in ``errors`` and reported to the library as a
    failure (CUBE_E_COMM)."""

    def __init__(self, group=None, device: int | None = None):
        import torch
        import torch.distributed as dist

        self.torch, self.dist, self.group = torch, dist, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.nccl = dist.get_backend(group) == "nccl"
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device) \
            if torch.cuda.is_available() else None
        self.errors: list[BaseException] = []
        self._ar = ALLREDUCE_FN(self._allreduce)
        self._sr = SENDRECV_FN(self._sendrecv)

    # ---- buffers ----
    def _view(self, ptr: int, n: int, dtype, device: int):
        torch = self.torch
        if n == 0:
            return None
        if device:
            return torch.as_tensor(_DeviceArray(ptr, n, dtype), device=self.device)
        arr = np.ctypeslib.as_array((ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr))
        return torch.from_numpy(arr.view(dtype))

    def _staged(self, t, device: int):
        """The tensor the backend works on: NCCL wants device memory, gloo host memory."""
        if t is None:
            return None
        if self.nccl and not device:
            return t.to(self.device)
        if not self.nccl and device:
            return t.cpu()
        return t

    # ---- the callbacks ----
    def _allreduce(self, user, buf, count, dtype, op, device):
        try:
            t = self._view(buf, count, _NP_DTYPE[dtype], device)
            if t is None:
                return 0
            w = self._staged(t, device)
            self.dist.all_reduce(w, op=self.dist.ReduceOp.SUM if op == OP_SUM else self.dist.ReduceOp.MAX,
                                 group=self.group)
            if w is not t:
                t.copy_(w)
            if device:
                self.torch.cuda.current_stream(self.device).synchronize()
            return 0
        except BaseException as e:  # reported to the library as a failed collective
            self.errors.append(e)
            return 1

    def _sendrecv(self, user, up, sn_up, down, sn_down, below, rn_below, above, rn_above, device):
        try:
            dist = self.dist
            lo, hi = (self.rank - 1) % self.size, (self.rank + 1) % self.size
            views = [self._view(p, n, np.uint8, device) for p, n in
                     ((up, sn_up), (down, sn_down), (below, rn_below), (above, rn_above))]
            work = [self._staged(v, device) for v in views]
            # sends up, then down; receives from below (sent up there), then from above: with
            # two slabs both neighbours are one rank and the messages pair up in this order
            # (tags keep them apart where the backend uses tags)
            ops = []
            if work[0] is not None:
                ops.append(dist.P2POp(dist.isend, work[0], hi, self.group, 1))
            if work[1] is not None:
                ops.append(dist.P2POp(dist.isend, work[1], lo, self.group, 2))
            if work[2] is not None:
                ops.append(dist.P2POp(dist.irecv, work[2], lo, self.group, 1))
            if work[3] is not None:
                ops.append(dist.P2POp(dist.irecv, work[3], hi, self.group, 2))
            if ops:
                for r in dist.batch_isend_irecv(ops):
                    r.wait()
            for v, w in zip(views[2:], work[2:]):
                if v is not None and w is not v:
                    v.copy_(w)
            if device:
                self.torch.cuda.current_stream(self.device).synchronize()
            return 0
        except BaseException as e:
            self.errors.append(e)
            return 1

    def as_c(self) -> CComm:
        return CComm(None, self._ar, self._sr)


# ---------------------------------------------------------------------------------
# Whole-box states and slabs
# ---------------------------------------------------------------------------------
def slab_params(p: Params, nslab: int, slab: int) -> Params:
    import dataclasses

    q = dataclasses.replace(p, nslab=nslab, slab=slab)
    q.validate()
    return q


def slab_cells(p: Params, which: int) -> np.ndarray:
    """Global storage indices of a slab's cell set (cube_slab_cells): 0 own cells, 1 the
    layer sent down, 2 the layer sent up, 3 ghosts from below, 4 ghosts from above."""
    L = load()
    cp = p.to_c()
    n = L.cube_slab_cells(ctypes.byref(cp), which, None, 0)
    if n < 0:
        raise ValueError("cube_slab_cells: bad geometry")
    out = np.empty(n, dtype=np.int64)
    L.cube_slab_cells(ctypes.byref(cp), which, out.ctypes.data_as(ctypes.c_void_p), n)
    return out


def cell_range(p: Params, nslab: int, slab: int) -> tuple[int, int]:
    """[c0, c1): the slab's cells in storage order (whole tile layers are contiguous)."""
    per = p.nt ** 3 * p.nnt ** 2 * (p.nnt // nslab)
    return slab * per, (slab + 1) * per


def split_state(p: Params, xp, vp, pid, rhoc, nslab: int):
    """The slabs' parts of a whole-box state in storage order: per slab (xp, vp, pid, rhoc)
    with rhoc the global array, zero outside the slab."""
    start = np.concatenate([[0], np.cumsum(rhoc, dtype=np.int64)])
    parts = []
    for s in range(nslab):
        c0, c1 = cell_range(p, nslab, s)
        a, b = int(start[c0]), int(start[c1])
        r = np.zeros_like(rhoc)
        r[c0:c1] = rhoc[c0:c1]
        parts.append((xp[a:b].copy(), vp[a:b].copy(), pid[a:b].copy(), r))
    return parts


def join_states(parts):
    """Inverse of split_state: the slabs' own particles, in slab order, are the whole box
    in storage order."""
    xp = np.concatenate([q[0] for q in parts])
    vp = np.concatenate([q[1] for q in parts])
    pid = np.concatenate([q[2] for q in parts])
    rhoc = np.sum([q[3] for q in parts], axis=0).astype(np.int32)
    return xp, vp, pid, rhoc
