"""x-slab decomposition of one periodic lattice over ranks (one process per GPU).

The reference runs one lattice in one process and marks where an MPI halo
exchange would go (GFTEvolver ``Core/Source/Lattice.cpp:779``).  Here rank r of
W owns planes [x0, x1) of the global x axis (the slowest index, so a plane of
every field array is contiguous) and holds them as a lattice of x1 - x0 + 2
planes: its own planes at local 1 .. nloc and one ghost plane on each side.
The step kernels run unchanged on that lattice; after every step the level just
written has its ghost planes refreshed from the neighbours (local plane 1 goes
to the left neighbour's ghost nloc+1, plane nloc to the right neighbour's ghost
0), before the Gauss-law kernel or the next step reads them.  The exchange runs
through ``torch.distributed`` (NCCL send/recv of the plane of each of the 7 or
8 field arrays, ordered on the library's stream); observables rows are combined
over ranks in FP64 (sums, site-weighted means and maxima).

The host logic here -- ``partition``, ``HaloExchange`` with its transports and
``combine_rows`` -- is independent of the device: the CPU tests drive it with
``gloo`` ranks over the oracle.
"""
from __future__ import annotations

import ctypes
import dataclasses

from . import _lib
from .evolver import Evolver, LatticeParams

ROW_SUMS = ("energy", "potential", "gradient", "kinetic", "magnetic", "electric")
ROW_MEANS = ("plaq_su2", "plaq_u1", "phi_sq")


def partition(nx: int, world: int, rank: int) -> tuple[int, int]:
    """Planes [x0, x1) of rank `rank`: an even split, the first nx % world ranks one plane more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    if nx < world:
        raise ValueError(f"{nx} planes cannot be split over {world} ranks")
    base, extra = divmod(nx, world)
    x0 = rank * base + min(rank, extra)
    return x0, x0 + base + (1 if rank < extra else 0)


def slab_params(params: LatticeParams, x0: int, x1: int) -> LatticeParams:
    """The local lattice of planes [x0, x1) plus one ghost plane on each side."""
    return dataclasses.replace(params, nx=x1 - x0 + 2)


class SelfTransport:
    """One rank: the lattice is periodic onto itself."""

    def exchange(self, send_lo, send_hi, recv_lo, recv_hi) -> None:
        for d, s in zip(recv_lo, send_hi):
            d.copy_(s)
        for d, s in zip(recv_hi, send_lo):
            d.copy_(s)


class DistTransport:
    """Neighbour exchange over torch.distributed point-to-point operations.

    Every rank posts, per field array and in the same order: send of its first
    own plane to the left, receive of the right neighbour's first plane into its
    right ghost, send of its last own plane to the right, receive of the left
    neighbour's last plane into its left ghost.  Point-to-point messages between
    two ranks match in posting order, so the pairs line up also when left and
    right are the same rank (two ranks).
    """

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self._ops = {}  # the operation list per set of plane tensors (they are fixed views)

    def _global(self, r: int) -> int:
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def exchange(self, send_lo, send_hi, recv_lo, recv_hi) -> None:
        dist = self.dist
        key = tuple(t.data_ptr() for t in (*send_lo, *recv_lo))
        ops = self._ops.get(key)
        if ops is None:
            left = self._global((self.rank - 1) % self.world)
            right = self._global((self.rank + 1) % self.world)
            ops = []
            for k in range(len(send_lo)):
                ops.append(dist.P2POp(dist.isend, send_lo[k], left, self.group))
                ops.append(dist.P2POp(dist.irecv, recv_hi[k], right, self.group))
                ops.append(dist.P2POp(dist.isend, send_hi[k], right, self.group))
                ops.append(dist.P2POp(dist.irecv, recv_lo[k], left, self.group))
            self._ops[key] = ops
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class HaloExchange:
    """Refreshes the ghost planes (local 0 and nloc + 1) of one level.

    `planes(level, x)` returns the tensors of plane x of every field array of a
    level (views of the field storage, same order on every rank).
    """

    def __init__(self, planes, nloc: int, transport):
        self.planes = planes
        self.nloc = nloc
        self.transport = transport

    def __call__(self, level: int) -> None:
        n = self.nloc
        self.transport.exchange(self.planes(level, 1), self.planes(level, n), self.planes(level, 0),
                                self.planes(level, n + 1))


def combine_rows(rows: list[dict], own_sites: int, group=None, device=None) -> list[dict]:
    """Whole-lattice observables rows from every rank's rows over its own sites.

    Energies and integrated Gauss residuals add, maximum residuals take the
    maximum, means (plaquettes, <phi^dag phi>) are weighted by the ranks' site
    counts.  All ranks must pass rows of the same steps.
    """
    import torch
    import torch.distributed as dist
    if not rows or not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return rows
    n = len(rows)
    neq = len(rows[0]["gauss_int"])  # Gauss constraints per row (gaugeNum)
    sums = torch.zeros((n, len(ROW_SUMS) + len(ROW_MEANS) + neq + 1), dtype=torch.float64)
    maxs = torch.zeros((n, neq), dtype=torch.float64)
    for i, r in enumerate(rows):
        vals = [r[k] for k in ROW_SUMS] + [r[k] * own_sites for k in ROW_MEANS] + list(r["gauss_int"]) + [own_sites]
        sums[i] = torch.tensor(vals, dtype=torch.float64)
        maxs[i] = torch.tensor(r["gauss_max"], dtype=torch.float64)
    if device is not None:
        sums, maxs = sums.to(device), maxs.to(device)
    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(maxs, op=dist.ReduceOp.MAX, group=group)
    sums, maxs = sums.cpu(), maxs.cpu()
    out = []
    for i, r in enumerate(rows):
        o = dict(r)
        s = sums[i].tolist()
        total = s[-1]
        for j, k in enumerate(ROW_SUMS):
            o[k] = s[j]
        for j, k in enumerate(ROW_MEANS):
            o[k] = s[len(ROW_SUMS) + j] / total
        o["gauss_int"] = s[len(ROW_SUMS) + len(ROW_MEANS):len(ROW_SUMS) + len(ROW_MEANS) + neq]
        o["gauss_max"] = maxs[i].tolist()
        out.append(o)
    return out


def share_id(make_id, rank: int, world: int, group=None) -> bytes:
    """Bytes made by rank 0 of the group (make_id()), the same on every rank: the id a
    group of ranks uses to join one NCCL communicator (any torch.distributed backend)."""
    import torch.distributed as dist
    data = make_id() if rank == 0 else None
    if world > 1:
        if not (dist.is_available() and dist.is_initialized()):
            raise RuntimeError("sharing an id over several ranks needs an initialised process group")
        obj = [data]
        src = 0 if group is None else dist.get_global_rank(group, 0)
        dist.broadcast_object_list(obj, src=src, group=group)
        data = obj[0]
    return data


class _DeviceBuffer:
    """A device range as a CUDA-array-interface object (zero-copy torch view)."""

    def __init__(self, ptr: int, nbytes: int, typestr: str, itemsize: int):
        self.__cuda_array_interface__ = {"shape": (nbytes // itemsize,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class SlabEvolver:
    """This rank's x-slab of a periodic lattice on its GPU (libgft_b200), ghost
    planes exchanged after every step.

    Without an initialised process group (or with one rank) the slab is the
    whole lattice and the exchange is a local copy: the result equals
    ``Evolver`` on the whole lattice.
    """

    def __init__(self, params: LatticeParams, form: str = "mixed", device: int = 0, group=None, transport=None,
                 rank: int | None = None, world: int | None = None, auto_exchange: bool = True,
                 exchange: str = "python", timeout_s: float = 300.0):
        """rank / world override the process group's (several slabs driven by one process, e.g. in
        tests); auto_exchange=False leaves the ghost refresh to the caller (``halo``).

        exchange="python": the ghost refresh runs after every step from a callback, through
        ``transport`` (torch.distributed point-to-point operations, or a local copy on one rank).
        exchange="library": gft_evolve posts it itself over NCCL (gft_set_slab_nccl): the boundary
        planes go out on a second stream while the interior planes are computed, with no host
        callback per step; its final wait gives up after ``timeout_s`` seconds."""
        import torch
        import torch.distributed as dist
        self.global_params = params
        dist_on = dist.is_available() and dist.is_initialized()
        self.world = world if world is not None else (dist.get_world_size(group) if dist_on else 1)
        self.rank = rank if rank is not None else (dist.get_rank(group) if dist_on else 0)
        self.group = group
        self.x0, self.x1 = partition(params.nx, self.world, self.rank)
        self.nloc = self.x1 - self.x0
        self.own_sites = self.nloc * params.ny * params.nz
        self.device = device
        self.local = Evolver(slab_params(params, self.x0, self.x1), form=form, device=device)
        lib, h = self.local.lib, self.local.h
        _lib.check(lib.gft_set_slab(h, self.x0 - 1, params.nx, 1, self.nloc + 1), h)
        import numpy as np
        itemsize = np.dtype(self.local.dtype).itemsize
        self._typestr = "<f8" if itemsize == 8 else "<f4"
        self._itemsize = itemsize
        self._views = {}
        self._transport = transport
        self._halo = None
        self._stream = torch.cuda.ExternalStream(self.local.stream, device=f"cuda:{device}")
        self._error = None
        self._cb = _lib.EXCHANGE_FN(self._on_exchange)
        self.exchange = exchange
        if exchange == "library":
            self._join_nccl(timeout_s)
        elif exchange != "python":
            raise ValueError(f"exchange must be 'python' or 'library', not {exchange!r}")
        elif auto_exchange:
            _lib.check(lib.gft_set_exchange(h, ctypes.cast(self._cb, ctypes.c_void_p), None), h)

    def _join_nccl(self, timeout_s: float) -> None:
        """One NCCL communicator over the ranks of the group: rank 0 makes its id, the group shares it."""
        lib, h = self.local.lib, self.local.h

        def make_id() -> bytes:
            buf = ctypes.create_string_buffer(128)
            _lib.check(lib.gft_nccl_unique_id(buf))
            return buf.raw

        id_buf = ctypes.create_string_buffer(share_id(make_id, self.rank, self.world, self.group), 128)
        _lib.check(lib.gft_set_slab_nccl(h, id_buf, self.world, self.rank, float(timeout_s)), h)

    # plane views of the library's field storage
    def _planes(self, level: int, x: int):
        key = (level, x)
        if key not in self._views:
            import torch
            ptrs = (ctypes.c_void_p * 11)()  # at most 11 arrays (2HDM with a Higgs-family field)
            sizes = (ctypes.c_size_t * 11)()
            n = _lib.check(self.local.lib.gft_level_planes(self.local.h, level, x, ptrs, sizes, 11), self.local.h)
            self._views[key] = [
                torch.as_tensor(_DeviceBuffer(ptrs[k], sizes[k], self._typestr, self._itemsize),
                                device=f"cuda:{self.device}")
                for k in range(n)]
        return self._views[key]

    @property
    def halo(self) -> HaloExchange:
        """The ghost refresh of this slab (created on first use: a process group is needed only then)."""
        if self._halo is None:
            t = self._transport
            if t is None:
                t = DistTransport(self.group) if self.world > 1 else SelfTransport()
            self._halo = HaloExchange(self._planes, self.nloc, t)
        return self._halo

    def _on_exchange(self, h, level, user):
        import torch
        try:
            with torch.cuda.stream(self._stream):
                self.halo(level)
            return 0
        except Exception as ex:  # reported by evolve()
            self._error = ex
            return 1

    def init_fields(self, ic) -> None:
        """Device initial data: each rank generates the global lattice's data of its planes (and ghosts)."""
        self.local.init_fields(ic)

    def upload_global(self, scalars, vectors, time_iter: int = 0) -> None:
        """Upload this rank's planes (and ghosts) from whole-lattice arrays in the reference layout."""
        import numpy as np
        idx = [(x % self.global_params.nx) for x in range(self.x0 - 1, self.x1 + 1)]
        self.local.upload(np.ascontiguousarray(scalars[:, idx]), np.ascontiguousarray(vectors[:, idx]), time_iter)

    def download_own(self, dtype=None):
        """This rank's own planes (reference layout, both levels)."""
        sc, ve = self.local.download(dtype)
        return sc[:, 1:self.nloc + 1], ve[:, 1:self.nloc + 1]

    def planes(self, level: int, x: int):
        """Device tensors viewing plane x (local index, 0 and nloc + 1 are ghosts) of every field array."""
        return self._planes(level, x)

    def evolve(self, n_steps: int) -> list[dict]:
        self._error = None
        try:
            rows = self.local.evolve(n_steps)
        except _lib.GftError:
            if self._error is not None:
                raise RuntimeError(f"halo exchange failed: {self._error}") from self._error
            raise
        return combine_rows(rows, self.own_sites, self.group,
                            device=f"cuda:{self.device}" if self.world > 1 else None)

    @property
    def time_iter(self) -> int:
        return self.local.time_iter

    def close(self) -> None:
        if getattr(self, "local", None) is not None:
            if self.exchange == "python":
                self.local.lib.gft_set_exchange(self.local.h, None, None)
            self.local.close()
            self.local = None
