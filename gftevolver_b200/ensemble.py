"""Ensembles of independent lattices on one GPU (over the gft_batch_* C ABI).

The reference evolves one lattice per process (``Lattice::evolve``,
GFTEvolver ``Core/Source/Lattice.cpp:755-876``); an ensemble of realisations
with different seeds and sizes is a loop of such runs.  ``Ensemble`` evolves
all members together: one persistent kernel launch per time step walks a work
list of tiles of every member, whole logging periods replay from a CUDA graph,
and ``autotune()`` picks the tile shape and march depth by timing them on the
ensemble itself.  Every member evolves exactly as ``Evolver`` with
``set_kernel(2, tile, march)`` would (mixed form).

On several GPUs the members are replicas, not a decomposition: with one process
per GPU, ``ShardedEnsemble`` deals them round-robin (``member_shard``) and each
rank evolves its share as an ``Ensemble``; the ranks exchange no fields, and the
analyser rows meet only when ``gather_rows`` is called.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .evolver import InitialData, LatticeParams, _row_dict, make_config


class Ensemble:
    """Members share the model, the device, the analysers' cadence and the step counter."""

    def __init__(self, params: list[LatticeParams], device: int = 0):
        if not params:
            raise ValueError("an ensemble needs at least one member")
        self.lib = _lib.load()
        self.params = list(params)
        cfgs = (_lib.GftConfig * len(params))(*[make_config(p, "mixed", device) for p in params])
        b = ctypes.c_void_p()
        _lib.check(self.lib.gft_batch_create(cfgs, len(params), ctypes.byref(b)))
        self.b = b
        self.last_warnings = 0

    def close(self) -> None:
        if getattr(self, "b", None):
            self.lib.gft_batch_destroy(self.b)
            self.b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.params)

    def init_fields(self, ics: list[InitialData]) -> None:
        if len(ics) != len(self):
            raise ValueError("one InitialData per member")
        arr = (_lib.GftIC * len(ics))()
        for c, ic in zip(arr, ics):
            c.seed = int(ic.seed)
            for k in range(8):
                c.mean[k] = ic.mean[k]
                c.sigma[k] = ic.sigma[k]
            c.theta_sigma, c.eps_sigma = ic.theta_sigma, ic.eps_sigma
            c.wall_width, c.wall_value = ic.wall_width, ic.wall_value
        _lib.check_batch(self.lib.gft_batch_init_fields(self.b, arr), self.b)

    def _shapes(self, m: int):
        p = self.params[m]
        return (2, p.nx, p.ny, p.nz, p.nsc), (2, p.nx, p.ny, p.nz, p.nve)

    def upload(self, m: int, scalars: np.ndarray, vectors: np.ndarray, time_iter: int = 0) -> None:
        ss, vs = self._shapes(m)
        if scalars.shape != ss or vectors.shape != vs:
            raise ValueError(f"expected shapes {ss} and {vs}")
        sc = np.ascontiguousarray(scalars, dtype=np.float32)
        ve = np.ascontiguousarray(vectors, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check_batch(self.lib.gft_batch_upload_f32(self.b, m, sc.ctypes.data_as(fp), ve.ctypes.data_as(fp),
                                                       int(time_iter)), self.b)

    def download(self, m: int):
        ss, vs = self._shapes(m)
        sc = np.empty(ss, np.float32)
        ve = np.empty(vs, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check_batch(self.lib.gft_batch_download_f32(self.b, m, sc.ctypes.data_as(fp), ve.ctypes.data_as(fp)),
                         self.b)
        return sc, ve

    def evolve(self, n_steps: int) -> list[list[dict]]:
        """Advance every member n_steps; returns, per member, the analyser rows logged on the way."""
        max_rows = n_steps + 1
        rows = (_lib.GftObservables * (max_rows * len(self)))()
        n = ctypes.c_int(0)
        self.last_warnings = _lib.check_batch(
            self.lib.gft_batch_evolve(self.b, int(n_steps), rows, max_rows, ctypes.byref(n)), self.b)
        neq = self.params[0].neq  # Gauss constraints per row: gaugeNum, shared by the members
        return [[_row_dict(rows[m * max_rows + r], neq) for r in range(n.value)] for m in range(len(self))]

    def set_kernel(self, tile: int, march: int, use_graphs: bool = True) -> None:
        _lib.check_batch(self.lib.gft_batch_set_kernel(self.b, int(tile), int(march), int(bool(use_graphs))), self.b)

    def autotune(self, trial_steps: int = 4):
        """Time every admissible (tile, march) on the ensemble; keep and return the fastest."""
        t, m = ctypes.c_int(0), ctypes.c_int(0)
        _lib.check_batch(self.lib.gft_batch_autotune(self.b, int(trial_steps), ctypes.byref(t), ctypes.byref(m)),
                         self.b)
        return t.value, m.value

    @property
    def last_ms(self) -> float:
        return float(self.lib.gft_batch_last_ms(self.b))

    @property
    def launch_count(self) -> int:
        return int(self.lib.gft_batch_launch_count(self.b))

    @property
    def time_iter(self) -> int:
        return int(self.lib.gft_batch_time_iter(self.b))

    @property
    def stream(self) -> int:
        return int(self.lib.gft_batch_stream(self.b) or 0)

    @property
    def device_bytes(self) -> int:
        return int(self.lib.gft_batch_device_bytes(self.b))

    @property
    def nsite(self) -> int:
        return sum(p.nsite for p in self.params)


def member_shard(n_members: int, rank: int, world: int) -> list[int]:
    """The members that rank `rank` of `world` evolves when `n_members` realisations
    are dealt round-robin over one process per GPU (member m goes to rank m % world)."""
    if world < 1 or not 0 <= rank < world or n_members < 0:
        raise ValueError(f"bad shard request: {n_members} members, rank {rank} of {world}")
    return list(range(rank, n_members, world))


def gather_member_rows(local_rows: list, n_members: int, rank: int, world: int, group=None) -> list:
    """Every member's analyser rows, in member order, on every rank, from each rank's
    rows of its own members (`local_rows[k]` belongs to member_shard(...)[k]).  One
    all_gather of Python objects through torch.distributed; it is the only exchange
    of a sharded ensemble and runs outside the step loop."""
    import torch.distributed as dist

    mine = member_shard(n_members, rank, world)
    if len(local_rows) != len(mine):
        raise ValueError(f"rank {rank} holds {len(mine)} members but passed rows for {len(local_rows)}")
    got = [None] * world
    dist.all_gather_object(got, list(local_rows), group=group)
    out = [None] * n_members
    for r in range(world):
        for k, m in enumerate(member_shard(n_members, r, world)):
            out[m] = got[r][k]
    return out


class ShardedEnsemble:
    """This rank's round-robin share of an ensemble (one process per GPU).

    rank / world default to torch.distributed's when a process group is
    initialised, else to a single rank.  A rank with no members (fewer members
    than ranks) holds no device state and evolves nothing."""

    def __init__(self, params: list[LatticeParams], device: int = 0, rank: int | None = None,
                 world: int | None = None):
        if rank is None or world is None:
            import torch.distributed as dist
            on = dist.is_available() and dist.is_initialized()
            if rank is None:
                rank = dist.get_rank() if on else 0
            if world is None:
                world = dist.get_world_size() if on else 1
        self.n_members, self.rank, self.world = len(params), rank, world
        self.members = member_shard(len(params), rank, world)
        self.local = Ensemble([params[m] for m in self.members], device=device) if self.members else None

    def init_fields(self, ics: list[InitialData]) -> None:
        if len(ics) != self.n_members:
            raise ValueError("one InitialData per member of the whole ensemble")
        if self.local is not None:
            self.local.init_fields([ics[m] for m in self.members])

    def evolve(self, n_steps: int) -> list[list[dict]]:
        """Advance this rank's members; their rows, in member_shard order."""
        return self.local.evolve(n_steps) if self.local is not None else []

    def gather_rows(self, local_rows: list, group=None) -> list:
        return gather_member_rows(local_rows, self.n_members, self.rank, self.world, group)

    def close(self) -> None:
        if self.local is not None:
            self.local.close()
            self.local = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
