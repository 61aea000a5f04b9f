"""Ensembles of independent lattices on one GPU (over the gft_batch_* C ABI).

The reference evolves one lattice per process (``Lattice::evolve``,
GFTEvolver ``Core/Source/Lattice.cpp:755-876``); an ensemble of realisations
with different seeds and sizes is a loop of such runs.  ``Ensemble`` evolves
all members together: one persistent kernel launch per time step walks a work
list of tiles of every member, whole logging periods replay from a CUDA graph,
and ``autotune()`` picks the tile shape and march depth by timing them on the
ensemble itself.  Every member evolves exactly as ``Evolver`` with
``set_kernel(2, tile, march)`` would (mixed form).
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
        return (2, p.nx, p.ny, p.nz, p.nsc), (2, p.nx, p.ny, p.nz, 15)

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
        return [[_row_dict(rows[m * max_rows + r]) for r in range(n.value)] for m in range(len(self))]

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
