"""Generate the golden fixtures in tests/golden/ by running the reference itself.

Each fixture holds the initial data, the reference's fields after ``nt``
steps and the Energy / GaugeCondition analysers' raw sums per logged step,
produced by the unmodified GFTEvolver sources compiled by
``oracle/build_ref.sh`` (``oracle/_ref/ref32`` = float storage as shipped,
``oracle/_ref/ref64`` = the same sources with float -> double).

Run from the repository root in the container where the reference is
mounted:  ``sh oracle/build_ref.sh && python tests/golden/make_golden.py``
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from oracle import refrun  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

RANDOM_LINKS = dict(theta_sigma=0.1, eps_sigma=0.1)

# name -> (params overrides, IC overrides, steps, storage list)
CASES = {
    "sm_4x5x6": (dict(model=orc.MODEL_SM, nx=4, ny=5, nz=6, energy_every=2, gauss_every=3),
                 dict(seed=11, mean=[1.0] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 10, ("f32", "f64")),
    "2hdm_5x4x3": (dict(model=orc.MODEL_2HDM, nx=5, ny=4, nz=3, energy_every=2, gauss_every=3),
                   dict(seed=12, mean=[0.7] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 10, ("f32", "f64")),
    "sm_1x1x1": (dict(model=orc.MODEL_SM, nx=1, ny=1, nz=1, energy_every=1, gauss_every=1),
                 dict(seed=13, mean=[1.0] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 5, ("f32",)),
    "sm_2x2x2": (dict(model=orc.MODEL_SM, nx=2, ny=2, nz=2, energy_every=1, gauss_every=2),
                 dict(seed=14, mean=[1.0] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 5, ("f32", "f64")),
    "sm_3x1x7": (dict(model=orc.MODEL_SM, nx=3, ny=1, nz=7, energy_every=1, gauss_every=1),
                 dict(seed=15, mean=[1.0] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 5, ("f32",)),
    "sm_damped_aniso_6x5x4": (dict(model=orc.MODEL_SM, nx=6, ny=5, nz=4, dx=0.5, dy=0.7, dz=1.3, damping=1.0,
                                   nt_damped=4, energy_every=3, gauss_every=2),
                              dict(seed=16, mean=[0.5] * 8, sigma=[0.2] * 8, **RANDOM_LINKS), 8, ("f32",)),
    "sm_identity_8x8x8": (dict(model=orc.MODEL_SM, nx=8, ny=8, nz=8, energy_every=5, gauss_every=5),
                          dict(seed=17, mean=[0.0] * 8, sigma=[0.1] * 8), 10, ("f32", "f64")),
    "2hdm_wall_4x4x12": (dict(model=orc.MODEL_2HDM, nx=4, ny=4, nz=12, energy_every=4, gauss_every=4),
                         dict(seed=18, mean=[0.0] * 8, sigma=[0.05] * 8, wall_width=2.0, wall_value=1.0), 8, ("f64",)),
    # Fixed faces on x and z (Lattice.cfg face types 1 1 3 3 1 1): a frozen shell, analysers over the rest
    "sm_fixed_xz_6x5x7": (dict(model=orc.MODEL_SM, nx=6, ny=5, nz=7, energy_every=2, gauss_every=3, fixed_axes=5),
                          dict(seed=19, mean=[1.0] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 8, ("f32", "f64")),
    "2hdm_fixed_y_5x6x4": (dict(model=orc.MODEL_2HDM, nx=5, ny=6, nz=4, energy_every=2, gauss_every=2, fixed_axes=2),
                           dict(seed=20, mean=[0.7] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 6, ("f32",)),
    # 2HDM with a Higgs-family gauge field: U(1) (gaugeNum 5) and SU(2) (gaugeNum 7), coupling g''
    "2hdm_hf_u1_4x5x3": (dict(model=orc.MODEL_2HDM, nx=4, ny=5, nz=3, energy_every=2, gauss_every=3, higgs_family=orc.HF_U1,
                              gpp=0.47),
                         dict(seed=21, mean=[0.7] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 8, ("f32", "f64")),
    "2hdm_hf_su2_5x3x4": (dict(model=orc.MODEL_2HDM, nx=5, ny=3, nz=4, energy_every=3, gauss_every=2, higgs_family=orc.HF_SU2,
                               gpp=0.52),
                          dict(seed=22, mean=[0.7] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 8, ("f32", "f64")),
    # generator link representation (links stored as w, U = exp(i w.sigma)): SM, and 2HDM with a family SU(2)
    "sm_gen_4x5x6": (dict(model=orc.MODEL_SM, nx=4, ny=5, nz=6, energy_every=2, gauss_every=3, generator_rep=1),
                     dict(seed=23, mean=[1.0] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 8, ("f32", "f64")),
    "2hdm_gen_hf_su2_4x3x5": (dict(model=orc.MODEL_2HDM, nx=4, ny=3, nz=5, energy_every=3, gauss_every=2,
                                   higgs_family=orc.HF_SU2, gpp=0.52, generator_rep=1),
                              dict(seed=24, mean=[0.7] * 8, sigma=[0.1] * 8, **RANDOM_LINKS), 8, ("f32", "f64")),
}


# Benchmark configuration 1 at its own size (SM 32^3, identity links, Higgs N(0, 0.1^2), analysers
# every 10 steps): too large for a field fixture, so the reference's final fields are kept as a
# SHA-256 digest of their bytes (both levels, reference layout) next to the analysers' raw sums.
DIGESTS = {
    "config1_sm_32": (dict(model=orc.MODEL_SM, nx=32, ny=32, nz=32, energy_every=10, gauss_every=10),
                      dict(seed=7, mean=[0.0] * 8, sigma=[0.1] * 8), 10, ("f32", "f64")),
}


def field_digest(sc: np.ndarray, ve: np.ndarray) -> str:
    """SHA-256 of the scalar then the vector array bytes (C order)."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(sc).tobytes())
    h.update(np.ascontiguousarray(ve).tobytes())
    return h.hexdigest()


def make_digest(name: str) -> None:
    pover, icover, nt, storages = DIGESTS[name]
    p = orc.Params(**pover)
    ic = orc.ICSpec(**icover)
    out = {"params": p.__dict__, "ic": ic.__dict__, "nt": nt, "runs": {}}
    for st in storages:
        fp64 = st == "f64"
        dtype = np.float64 if fp64 else np.float32
        sc, ve = orc.init_fields(p, ic, dtype)
        ic_digest = field_digest(sc, ve)
        rs, rv, rows, _ = refrun.run(p, sc, ve, nt, fp64=fp64)
        out["runs"][st] = {
            "generator": "oracle/_ref/" + ("ref64" if fp64 else "ref32"),
            "ic_sha256": ic_digest, "fields_sha256": field_digest(rs, rv),
            "rows": [{"time_iter": r["time_iter"], "has_energy": r["has_energy"], "has_gauss": r["has_gauss"],
                      "ref_energy": r["ref_energy"], "ref_gauss_int": r["ref_gauss_int"],
                      "gauss_max": r["gauss_max"]} for r in rows],
        }
    path = os.path.join(HERE, f"{name}_digest.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print("wrote", os.path.relpath(path, ROOT), os.path.getsize(path), "bytes")


def make(name: str) -> None:
    pover, icover, nt, storages = CASES[name]
    p = orc.Params(**pover)
    ic = orc.ICSpec(**icover)
    for st in storages:
        fp64 = st == "f64"
        dtype = np.float64 if fp64 else np.float32
        sc, ve = orc.init_fields(p, ic, dtype)
        rs, rv, rows, _ = refrun.run(p, sc, ve, nt, fp64=fp64)
        meta = {"params": p.__dict__, "ic": ic.__dict__, "nt": nt, "storage": st,
                "generator": "oracle/_ref/" + ("ref64" if fp64 else "ref32")}
        out = os.path.join(HERE, f"{name}_{st}.npz")
        np.savez_compressed(
            out, ic_scalars=sc, ic_vectors=ve, scalars=rs, vectors=rv,
            row_time_iter=np.array([r["time_iter"] for r in rows], dtype=np.int64),
            row_has_energy=np.array([r["has_energy"] for r in rows], dtype=bool),
            row_has_gauss=np.array([r["has_gauss"] for r in rows], dtype=bool),
            row_ref_energy=np.array([r["ref_energy"] for r in rows], dtype=np.float64).reshape(-1, 6),
            row_ref_gauss_int=np.array([r["ref_gauss_int"] for r in rows], dtype=np.float64).reshape(-1, p.neq),
            row_gauss_max=np.array([r["gauss_max"] for r in rows], dtype=np.float64).reshape(-1, p.neq),
            meta=np.array(json.dumps(meta)))
        print("wrote", os.path.relpath(out, ROOT), os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if not (refrun.available(False) and refrun.available(True)):
        sys.exit("reference binaries missing: run sh oracle/build_ref.sh first")
    for n in (sys.argv[1:] or list(CASES) + list(DIGESTS)):
        if n in DIGESTS:
            make_digest(n)
        else:
            make(n)
