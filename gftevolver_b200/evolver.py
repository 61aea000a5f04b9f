"""Python front end of the B200 evolver (over the C ABI in include/gft.h).

``Evolver`` owns one device handle: both time levels of the fields, the model
parameters, the step counter and the analysers' logging cadence -- the state
the reference keeps in ``Lattice`` and ``Model`` (Core/Header/Lattice.hpp:22-212,
Core/Header/Model.hpp:23-266).  Host arrays use the reference layout
``scalars[2, nx, ny, nz, nsc]``, ``vectors[2, nx, ny, nz, 3 * dw]`` (dw = 5 link
words per direction, 6 or 9 with a 2HDM Higgs-family U(1) phase or SU(2)
quaternion, ``WilsonLoops/Source/TwoHDM.cpp:210-242``; 4, 5 or 7 in the generator
representation).
"""
from __future__ import annotations

import ctypes
from dataclasses import asdict, dataclass, field

import numpy as np

from . import _lib

FORMS = {
    "ref32": (_lib.GFT_FORM_REF, 4),
    "ref64": (_lib.GFT_FORM_REF, 8),
    "fp64": (_lib.GFT_FORM_FP64, 8),
    "mixed": (_lib.GFT_FORM_MIXED, 4),
}
STORAGE_DTYPE = {"ref32": np.float32, "ref64": np.float64, "fp64": np.float64, "mixed": np.float32}


@dataclass
class LatticeParams:
    """Model and lattice parameters (the values of the reference's .cfg files)."""

    model: int = _lib.GFT_MODEL_SM
    nx: int = 32
    ny: int = 32
    nz: int = 32
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0
    dt: float = 0.05
    g: float = 0.65
    gp: float = 0.35
    gpp: float = 0.5           # Higgs-family coupling g'' (TwoHDM gaugeNum 5/7)
    div_tol: float = 1e-9
    damping: float = 0.0
    nt_damped: int = 0
    lam: float = 0.13
    eta_sqr: float = 1.0
    m1: float = 0.5
    m2: float = 0.5
    l1: float = 0.065
    l2: float = 0.065
    l3: float = 0.2
    m12r: float = 0.2
    l4p5: float = -0.1
    l6r: float = 0.0
    l7r: float = 0.0
    m12i: float = 0.0
    l4m5: float = 0.0
    l5i: float = 0.0
    l6i: float = 0.0
    l7i: float = 0.0
    break_son: int = 1
    break_uhalfn: int = 1
    apply_norm: int = 0
    energy_offset: float = 0.0
    energy_every: int = 0
    gauss_every: int = 0
    fixed_axes: int = 0        # bit a: both faces of axis a Fixed (frozen shell), else periodic
    higgs_family: int = 0      # 2HDM Higgs-family gauge field: 0 none, 1 U(1) (gaugeNum 5), 2 SU(2) (gaugeNum 7)
    generator_rep: int = 0     # host links as 3 generators w (U = exp(i w.sigma)) instead of quaternions
    energy_local_every: int = 0  # Energy local densities kept every n steps (gft_local_fields); 0 = none
    gauss_local_every: int = 0   # GaugeCondition local violations kept every n steps; 0 = none

    @property
    def nsc(self) -> int:
        return 4 if self.model == _lib.GFT_MODEL_SM else 8

    @property
    def nve(self) -> int:
        """Link words per site in the reference layout (3 directions x 5, 6 or 9; generators 4, 5 or 7)."""
        lw = 3 if self.generator_rep else 4
        return 3 * (1 + lw + {0: 0, 1: 1, 2: lw}[self.higgs_family])

    @property
    def neq(self) -> int:
        """Gauge equations per direction = Gauss constraints per row (gaugeNum)."""
        return {0: 4, 1: 5, 2: 7}[self.higgs_family]

    @property
    def nsite(self) -> int:
        return self.nx * self.ny * self.nz

    def as_dict(self) -> dict:
        return asdict(self)


@dataclass
class InitialData:
    """Device-generated initial data (both levels equal: E = 0, pi = 0)."""

    seed: int = 1
    mean: list = field(default_factory=lambda: [0.0] * 8)
    sigma: list = field(default_factory=lambda: [0.1] * 8)
    theta_sigma: float = 0.0
    eps_sigma: float = 0.0
    wall_width: float = 0.0
    wall_value: float = 1.0


ROW_KEYS = ("energy", "potential", "gradient", "kinetic", "magnetic", "electric")


def _row_dict(r: _lib.GftObservables, neq: int = 4) -> dict:
    d = {"time_iter": r.time_iter, "has_energy": bool(r.has_energy), "has_gauss": bool(r.has_gauss)}
    for k in ROW_KEYS:
        d[k] = r.__getattribute__(k)
    d["gauss_int"] = list(r.gauss_int)[:neq]
    d["gauss_max"] = list(r.gauss_max)[:neq]
    d["plaq_su2"], d["plaq_u1"], d["phi_sq"] = r.plaq_su2, r.plaq_u1, r.phi_sq
    return d


def make_config(params: LatticeParams, form: str = "mixed", device: int = 0) -> _lib.GftConfig:
    """The C ABI's gft_config for these parameters."""
    if form not in FORMS:
        raise ValueError(f"unknown form {form!r}; choose one of {sorted(FORMS)}")
    cfg = _lib.GftConfig()
    for name, _ in _lib.GftConfig._fields_:
        if name in ("form", "storage_bytes", "device"):
            continue
        setattr(cfg, name, getattr(params, name))
    cfg.form, cfg.storage_bytes = FORMS[form]
    cfg.device = device
    return cfg


class Evolver:
    """One lattice on one GPU, evolved by the CUDA kernels of libgft_b200.so."""

    def __init__(self, params: LatticeParams, form: str = "mixed", device: int = 0):
        if form not in FORMS:
            raise ValueError(f"unknown form {form!r}; choose one of {sorted(FORMS)}")
        self.lib = _lib.load()
        self.params = params
        self.form = form
        self.dtype = STORAGE_DTYPE[form]
        cfg = _lib.GftConfig()
        for name, _ in _lib.GftConfig._fields_:
            if name in ("form", "storage_bytes", "device"):
                continue
            setattr(cfg, name, getattr(params, name))
        cfg.form, cfg.storage_bytes = FORMS[form]
        cfg.device = device
        h = ctypes.c_void_p()
        _lib.check(self.lib.gft_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.last_warnings = 0

    # -- checkpoint / restart --------------------------------------------------
    def save(self, path: str) -> None:
        """Checkpoint: both time levels (reference layout, storage precision), the
        step counter, the form and the parameters, in one .npz file.  Restarting
        from it continues bit for bit (the step depends only on the two levels and
        time_iter)."""
        sc, ve = self.download()
        np.savez(path, scalars=sc, vectors=ve, time_iter=self.time_iter, form=self.form,
                 params=np.array(repr(asdict(self.params))))

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Evolver":
        """Restart from a checkpoint written by save()."""
        import ast
        z = np.load(path, allow_pickle=False)
        params = LatticeParams(**ast.literal_eval(str(z["params"])))
        ev = cls(params, form=str(z["form"]), device=device)
        ev.upload(z["scalars"], z["vectors"], int(z["time_iter"]))
        return ev

    # -- lifetime ------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gft_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- fields --------------------------------------------------------------
    def _shapes(self):
        p = self.params
        return (2, p.nx, p.ny, p.nz, p.nsc), (2, p.nx, p.ny, p.nz, p.nve)

    def upload(self, scalars: np.ndarray, vectors: np.ndarray, time_iter: int = 0) -> None:
        ss, vs = self._shapes()
        if scalars.shape != ss or vectors.shape != vs:
            raise ValueError(f"expected shapes {ss} and {vs}, got {scalars.shape} and {vectors.shape}")
        if scalars.dtype == np.float64:
            sc = np.ascontiguousarray(scalars)
            ve = np.ascontiguousarray(vectors, dtype=np.float64)
            fn, ptr = self.lib.gft_upload_f64, ctypes.POINTER(ctypes.c_double)
        else:
            sc = np.ascontiguousarray(scalars, dtype=np.float32)
            ve = np.ascontiguousarray(vectors, dtype=np.float32)
            fn, ptr = self.lib.gft_upload_f32, ctypes.POINTER(ctypes.c_float)
        _lib.check(fn(self.h, sc.ctypes.data_as(ptr), ve.ctypes.data_as(ptr), int(time_iter)), self.h)

    def upload_ptr(self, scalars_ptr: int, vectors_ptr: int, f64: bool, time_iter: int = 0) -> None:
        """Upload from raw host pointers (e.g. pinned torch tensors)."""
        if f64:
            P = ctypes.POINTER(ctypes.c_double)
            fn = self.lib.gft_upload_f64
        else:
            P = ctypes.POINTER(ctypes.c_float)
            fn = self.lib.gft_upload_f32
        _lib.check(fn(self.h, ctypes.cast(scalars_ptr, P), ctypes.cast(vectors_ptr, P), int(time_iter)), self.h)

    def download(self, dtype=None):
        dtype = np.dtype(dtype or self.dtype)
        ss, vs = self._shapes()
        sc = np.empty(ss, dtype=dtype)
        ve = np.empty(vs, dtype=dtype)
        self.download_into(sc, ve)
        return sc, ve

    def download_into(self, sc: np.ndarray, ve: np.ndarray) -> None:
        if sc.dtype == np.float64:
            fn, ptr = self.lib.gft_download_f64, ctypes.POINTER(ctypes.c_double)
        else:
            fn, ptr = self.lib.gft_download_f32, ctypes.POINTER(ctypes.c_float)
        _lib.check(fn(self.h, sc.ctypes.data_as(ptr), ve.ctypes.data_as(ptr)), self.h)

    def download_ptr(self, scalars_ptr: int, vectors_ptr: int, f64: bool) -> None:
        if f64:
            P, fn = ctypes.POINTER(ctypes.c_double), self.lib.gft_download_f64
        else:
            P, fn = ctypes.POINTER(ctypes.c_float), self.lib.gft_download_f32
        _lib.check(fn(self.h, ctypes.cast(scalars_ptr, P), ctypes.cast(vectors_ptr, P)), self.h)

    def upload_device(self, scalars_ptr: int, vectors_ptr: int, f64: bool, time_iter: int = 0) -> None:
        """Upload from reference-layout buffers already in device memory (e.g. CUDA torch tensors)."""
        fn = self.lib.gft_upload_device_f64 if f64 else self.lib.gft_upload_device_f32
        _lib.check(fn(self.h, ctypes.c_void_p(scalars_ptr), ctypes.c_void_p(vectors_ptr), int(time_iter)), self.h)

    def download_device(self, scalars_ptr: int, vectors_ptr: int, f64: bool) -> None:
        """Write both levels, reference layout, into device buffers (e.g. CUDA torch tensors)."""
        fn = self.lib.gft_download_device_f64 if f64 else self.lib.gft_download_device_f32
        _lib.check(fn(self.h, ctypes.c_void_p(scalars_ptr), ctypes.c_void_p(vectors_ptr)), self.h)

    def init_fields(self, ic: InitialData) -> None:
        c = _lib.GftIC()
        c.seed = int(ic.seed)
        for k in range(8):
            c.mean[k] = float((list(ic.mean) + [0.0] * 8)[k])
            c.sigma[k] = float((list(ic.sigma) + [0.0] * 8)[k])
        c.theta_sigma, c.eps_sigma = float(ic.theta_sigma), float(ic.eps_sigma)
        c.wall_width, c.wall_value = float(ic.wall_width), float(ic.wall_value)
        _lib.check(self.lib.gft_init_fields(self.h, ctypes.byref(c)), self.h)

    # -- time stepping -------------------------------------------------------
    def evolve(self, n_steps: int, max_rows: int | None = None) -> list:
        """Advance n_steps; returns the analyser rows logged on the way."""
        if max_rows is None:
            max_rows = n_steps + 1
        rows = (_lib.GftObservables * max(max_rows, 1))()
        n = ctypes.c_int(0)
        self.last_warnings = _lib.check(
            self.lib.gft_evolve(self.h, int(n_steps), rows, int(max_rows), ctypes.byref(n)), self.h)
        return [_row_dict(rows[i], self.params.neq) for i in range(n.value)]

    def set_graphs(self, on: bool = True) -> None:
        """Replay whole logging periods of small lattices from a CUDA graph (default) or launch directly."""
        _lib.check(self.lib.gft_set_graphs(self.h, int(bool(on))), self.h)

    def set_wait_limit(self, ns: int = 0) -> None:
        """Time limit of the tiled kernel's plane waits in ns (0: the 2 s default); see gft_set_wait_limit."""
        _lib.check(self.lib.gft_set_wait_limit(self.h, int(ns)), self.h)

    def set_kernel(self, kind: int = 0, tile: int = 0, march: int = 32) -> None:
        """Step kernel of the throughput forms: 0 auto, 1 one thread per site, 2 TMA-staged tiles."""
        _lib.check(self.lib.gft_set_kernel(self.h, int(kind), int(tile), int(march)), self.h)

    def observe(self) -> dict:
        r = _lib.GftObservables()
        _lib.check(self.lib.gft_observe(self.h, ctypes.byref(r)), self.h)
        return _row_dict(r, self.params.neq)

    @property
    def time_iter(self) -> int:
        return int(self.lib.gft_time_iter(self.h))

    def step_kernel_ms(self):
        n = ctypes.c_int(0)
        ms = self.lib.gft_step_kernel_ms(self.h, ctypes.byref(n))
        return ms, n.value

    @property
    def launch_count(self) -> int:
        """Kernels launched by evolve() on this handle so far."""
        return int(self.lib.gft_launch_count(self.h))

    def local_fields(self):
        """Per-site analyser outputs of the latest local-output step: (energy[nsite, 6] or None,
        step, gauss[nsite, gaugeNum] or None, step); see gft_local_fields."""
        p = self.params
        fp = ctypes.POINTER(ctypes.c_float)
        e = np.zeros((p.nsite, 6), np.float32) if p.energy_local_every > 0 else None
        g = np.zeros((p.nsite, p.neq), np.float32) if p.gauss_local_every > 0 else None
        es, gs = ctypes.c_int(-1), ctypes.c_int(-1)
        _lib.check(self.lib.gft_local_fields(self.h, e.ctypes.data_as(fp) if e is not None else None,
                                             g.ctypes.data_as(fp) if g is not None else None, ctypes.byref(es),
                                             ctypes.byref(gs)), self.h)
        return e, es.value, g, gs.value

    @property
    def step_kernel_name(self) -> str:
        """The step kernel gft_evolve launches for this handle (ref / fast / tiled)."""
        return self.lib.gft_step_kernel_name(self.h).decode()

    @property
    def stream(self) -> int:
        return int(self.lib.gft_stream(self.h) or 0)

    @property
    def device_bytes(self) -> int:
        return int(self.lib.gft_device_bytes(self.h))
