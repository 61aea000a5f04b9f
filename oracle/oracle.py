"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for the GFTEvolver leapfrog step.

Python front end (ctypes) of ``gft_oracle.c``, the plain-C restatement of the
reference's per-site update (``Core/Source/Lattice.cpp:755-876``,
``Core/Source/Model.cpp:339-375``, ``Gradients/Source/StandardModel.cpp``,
``Gradients/Source/TwoHDM.cpp``, ``WilsonLoops/Source/StandardModel.cpp``,
``Potentials/Source/SO_N.cpp``, ``Potentials/Source/Double_SO_N.cpp``) and of
its Energy and GaugeCondition analysers.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, as the
checker; the product never imports it.

Arrays use the reference layout: ``scalars[2, nx, ny, nz, nsc]`` and
``vectors[2, nx, ny, nz, 3 * dw]`` (per direction ``[theta_Y, c0, c1, c2, c3]``,
plus the 2HDM Higgs-family phase ``theta_H`` (dw = 6) or quaternion ``d0..d3``
(dw = 9), ``WilsonLoops/Source/TwoHDM.cpp:210-242``); in the generator
representation ``[theta_Y, w1, w2, w3]`` (+ ``theta_H`` or ``w'1..w'3``: dw = 4, 5, 7).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "liborc.so")

MODEL_SM = 1
MODEL_2HDM = 2
HF_NONE, HF_U1, HF_SU2 = 0, 1, 2   # 2HDM Higgs-family gauge group (gaugeNum 4, 5, 7)
MAX_EQ = 7


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("dt", ctypes.c_double),
        ("g", ctypes.c_double), ("gp", ctypes.c_double),
        ("div_tol", ctypes.c_double),
        ("damping", ctypes.c_double), ("nt_damped", ctypes.c_int),
        ("lam", ctypes.c_double), ("eta_sqr", ctypes.c_double),
        ("m1", ctypes.c_double), ("m2", ctypes.c_double), ("l1", ctypes.c_double), ("l2", ctypes.c_double),
        ("l3", ctypes.c_double),
        ("m12r", ctypes.c_double), ("l4p5", ctypes.c_double), ("l6r", ctypes.c_double), ("l7r", ctypes.c_double),
        ("m12i", ctypes.c_double), ("l4m5", ctypes.c_double), ("l5i", ctypes.c_double), ("l6i", ctypes.c_double),
        ("l7i", ctypes.c_double),
        ("break_son", ctypes.c_int), ("break_uhalfn", ctypes.c_int), ("apply_norm", ctypes.c_int),
        ("energy_offset", ctypes.c_double),
        ("energy_every", ctypes.c_int), ("gauss_every", ctypes.c_int),
        ("fixed_axes", ctypes.c_int),
        ("higgs_family", ctypes.c_int), ("gpp", ctypes.c_double),
        ("generator_rep", ctypes.c_int),
        ("energy_local_every", ctypes.c_int), ("gauss_local_every", ctypes.c_int),
    ]


class OrcRow(ctypes.Structure):
    _fields_ = [
        ("time_iter", ctypes.c_int),
        ("has_energy", ctypes.c_int), ("has_gauss", ctypes.c_int),
        ("energy", ctypes.c_double), ("potential", ctypes.c_double), ("gradient", ctypes.c_double),
        ("kinetic", ctypes.c_double), ("magnetic", ctypes.c_double), ("electric", ctypes.c_double),
        ("gauss_int", ctypes.c_double * MAX_EQ), ("gauss_max", ctypes.c_double * MAX_EQ),
        ("plaq_su2", ctypes.c_double), ("plaq_u1", ctypes.c_double), ("phi_sq", ctypes.c_double),
        ("ref_energy", ctypes.c_double * 6),
        ("ref_gauss_int", ctypes.c_double * MAX_EQ),
    ]


@dataclass
class Params:
    """Physics parameters of one run (the reference's .cfg values)."""

    model: int = MODEL_SM
    nx: int = 8
    ny: int = 8
    nz: int = 8
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0
    dt: float = 0.05
    g: float = 0.65
    gp: float = 0.35
    gpp: float = 0.5
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
    fixed_axes: int = 0        # bit a: both faces of axis a Fixed (else periodic)
    higgs_family: int = HF_NONE  # 2HDM Higgs-family gauge field (HF_*)
    generator_rep: int = 0     # links stored as 3 generators w (U = exp(i w.sigma)) instead of quaternions
    energy_local_every: int = 0  # Energy local densities every n steps (0 = none)
    gauss_local_every: int = 0   # GaugeCondition local violations every n steps (0 = none)

    @property
    def nsc(self) -> int:
        return 4 if self.model == MODEL_SM else 8

    @property
    def dw(self) -> int:
        """Link words per direction."""
        if self.generator_rep:
            return {HF_NONE: 4, HF_U1: 5, HF_SU2: 7}[self.higgs_family]
        return {HF_NONE: 5, HF_U1: 6, HF_SU2: 9}[self.higgs_family]

    @property
    def nve(self) -> int:
        return 3 * self.dw

    @property
    def neq(self) -> int:
        """Gauge equations per direction = Gauss constraints (gaugeNum)."""
        return {HF_NONE: 4, HF_U1: 5, HF_SU2: 7}[self.higgs_family]

    @property
    def nsite(self) -> int:
        return self.nx * self.ny * self.nz

    def to_c(self) -> OrcConfig:
        c = OrcConfig()
        for name, _ in OrcConfig._fields_:
            setattr(c, name, getattr(self, name))
        return c


_lock = threading.Lock()
_lib = None


def build_oracle(force: bool = False) -> str:
    """Compile gft_oracle.c (float and double storage) into oracle/_build/liborc.so."""
    src = os.path.join(HERE, "gft_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= max(
        os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "gft_oracle.h"))
    ):
        return LIB_PATH
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    for s, prefix in (("float", "orc32_"), ("double", "orc64_")):
        obj = os.path.join(BUILD_DIR, f"gft_oracle_{prefix[:-1]}.o")
        subprocess.check_call([
            "gcc", "-O2", "-std=c11", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
            f"-DORC_S={s}", f"-DORC_PREFIX={prefix}", "-c", src, "-o", obj,
        ])
        objs.append(obj)
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call(["gcc", "-shared", "-o", tmp] + objs + ["-lm"])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def _load():
    global _lib
    with _lock:
        if _lib is None:
            build_oracle()
            lib = ctypes.CDLL(LIB_PATH)
            for p, fp in (("orc32_", ctypes.POINTER(ctypes.c_float)), ("orc64_", ctypes.POINTER(ctypes.c_double))):
                f = getattr(lib, p + "evolve")
                f.restype = ctypes.c_int
                f.argtypes = [ctypes.POINTER(OrcConfig), fp, fp, ctypes.c_int, ctypes.c_int,
                              ctypes.POINTER(OrcRow), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
                f = getattr(lib, p + "gauss")
                f.restype = ctypes.c_int
                f.argtypes = [ctypes.POINTER(OrcConfig), fp, fp, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
                f = getattr(lib, p + "init_fields")
                f.restype = None
                f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              fp, fp, ctypes.c_ulonglong,
                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                              ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]
            _lib = lib
    return _lib


def _ptr(a: np.ndarray):
    if a.dtype == np.float32:
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _prefix(dtype) -> str:
    if np.dtype(dtype) == np.float32:
        return "orc32_"
    if np.dtype(dtype) == np.float64:
        return "orc64_"
    raise TypeError(f"oracle storage must be float32 or float64, got {dtype}")


@dataclass
class ICSpec:
    """Initial data: Gaussian scalars (+ optional tanh wall on component 0), random links."""

    seed: int = 1
    mean: list = field(default_factory=lambda: [0.0] * 8)
    sigma: list = field(default_factory=lambda: [0.1] * 8)
    theta_sigma: float = 0.0
    eps_sigma: float = 0.0
    wall_width: float = 0.0
    wall_value: float = 1.0


def init_fields(p: Params, ic: ICSpec, dtype=np.float32):
    """Both time levels of the initial data (E = 0, pi = 0) in the reference layout."""
    lib = _load()
    sc = np.zeros((2, p.nx, p.ny, p.nz, p.nsc), dtype=dtype)
    ve = np.zeros((2, p.nx, p.ny, p.nz, p.nve), dtype=dtype)
    mean = (ctypes.c_double * 8)(*[float(v) for v in (list(ic.mean) + [0.0] * 8)[:8]])
    sig = (ctypes.c_double * 8)(*[float(v) for v in (list(ic.sigma) + [0.0] * 8)[:8]])
    getattr(lib, _prefix(dtype) + "init_fields")(
        p.nx, p.ny, p.nz, p.nsc, p.higgs_family, p.generator_rep, _ptr(sc), _ptr(ve), ctypes.c_ulonglong(ic.seed), mean, sig,
        float(ic.theta_sigma), float(ic.eps_sigma), float(ic.wall_width), float(ic.wall_value))
    return sc, ve


ROW_KEYS = ("energy", "potential", "gradient", "kinetic", "magnetic", "electric")


def evolve(p: Params, scalars: np.ndarray, vectors: np.ndarray, nsteps: int, time_iter0: int = 0,
           local: bool = False):
    """Evolve in place; returns (rows, warn) with rows a list of dicts, and with local=True
    also the per-site outputs of the last local-output step: (rows, warn, energy[nsite, 6],
    gauss[nsite, gaugeNum]) (zeros where no step computed them)."""
    lib = _load()
    assert scalars.flags.c_contiguous and vectors.flags.c_contiguous
    assert scalars.dtype == vectors.dtype
    assert scalars.shape == (2, p.nx, p.ny, p.nz, p.nsc), scalars.shape
    assert vectors.shape == (2, p.nx, p.ny, p.nz, p.nve), vectors.shape
    max_rows = nsteps + 1
    rows = (OrcRow * max_rows)()
    warn = ctypes.c_int(0)
    cfg = p.to_c()
    loc_e = np.zeros((p.nsite, 6), np.float64)
    loc_g = np.zeros((p.nsite, p.neq), np.float64)
    dp = ctypes.POINTER(ctypes.c_double)
    n = getattr(lib, _prefix(scalars.dtype) + "evolve")(
        ctypes.byref(cfg), _ptr(scalars), _ptr(vectors), time_iter0, nsteps, rows, max_rows, ctypes.byref(warn),
        loc_e.ctypes.data_as(dp), loc_g.ctypes.data_as(dp))
    if n < 0:
        raise ValueError(f"oracle rejected the configuration (code {n})")
    out = []
    for r in rows[: min(n, max_rows)]:
        d = {"time_iter": r.time_iter, "has_energy": bool(r.has_energy), "has_gauss": bool(r.has_gauss)}
        for k in ROW_KEYS:
            d[k] = getattr(r, k)
        d["gauss_int"] = list(r.gauss_int)[: p.neq]
        d["gauss_max"] = list(r.gauss_max)[: p.neq]
        d["plaq_su2"], d["plaq_u1"], d["phi_sq"] = r.plaq_su2, r.plaq_u1, r.phi_sq
        d["ref_energy"] = list(r.ref_energy)
        d["ref_gauss_int"] = list(r.ref_gauss_int)[: p.neq]
        out.append(d)
    if local:
        return out, warn.value, loc_e, loc_g
    return out, warn.value


def gauss(p: Params, scalars: np.ndarray, vectors: np.ndarray, time_iter: int):
    """The Gauss row of two levels as they stand after step time_iter (the post-evolve
    analyser of evolve, without stepping): (gauss_int[neq], gauss_max[neq], loc_g[nsite, neq])
    with loc_g the signed violations rounded to float."""
    lib = _load()
    assert scalars.flags.c_contiguous and vectors.flags.c_contiguous
    assert scalars.dtype == vectors.dtype
    assert scalars.shape == (2, p.nx, p.ny, p.nz, p.nsc), scalars.shape
    assert vectors.shape == (2, p.nx, p.ny, p.nz, p.nve), vectors.shape
    gi = np.zeros(MAX_EQ, np.float64)
    gm = np.zeros(MAX_EQ, np.float64)
    loc_g = np.zeros((p.nsite, p.neq), np.float64)
    dp = ctypes.POINTER(ctypes.c_double)
    cfg = p.to_c()
    n = getattr(lib, _prefix(scalars.dtype) + "gauss")(
        ctypes.byref(cfg), _ptr(scalars), _ptr(vectors), int(time_iter), gi.ctypes.data_as(dp), gm.ctypes.data_as(dp),
        loc_g.ctypes.data_as(dp))
    if n < 0:
        raise ValueError(f"oracle rejected the configuration (code {n})")
    return gi[: p.neq].copy(), gm[: p.neq].copy(), loc_g
