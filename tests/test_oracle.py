"""The CPU oracle against the reference itself (CPU only).

The golden fixtures were produced by the unmodified reference sources
(tests/golden/make_golden.py); the oracle must reproduce them bit for bit:
fields after every step and the analysers' float running sums (which also
pins the reference's site order, boundary regions first).
"""
import os

import numpy as np
import pytest

from conftest import golden_files, load_golden

GOLDEN = golden_files()


def _params(oracle_mod, meta):
    return oracle_mod.Params(**meta["params"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_reproduces_reference_golden(oracle_mod, path):
    z, meta = load_golden(path)
    p = _params(oracle_mod, meta)
    sc = z["ic_scalars"].copy()
    ve = z["ic_vectors"].copy()
    rows, warn = oracle_mod.evolve(p, sc, ve, meta["nt"])
    assert warn == 0
    # bit-exact fields (both time levels)
    np.testing.assert_array_equal(sc, z["scalars"])
    np.testing.assert_array_equal(ve, z["vectors"])
    # analyser rows: same steps, bit-exact sums in the reference's precision and order
    assert [r["time_iter"] for r in rows] == list(z["row_time_iter"])
    assert [r["has_energy"] for r in rows] == list(z["row_has_energy"])
    assert [r["has_gauss"] for r in rows] == list(z["row_has_gauss"])
    for r, e, gi, gm in zip(rows, z["row_ref_energy"], z["row_ref_gauss_int"], z["row_gauss_max"]):
        if r["has_energy"]:
            assert r["ref_energy"] == list(e)
        if r["has_gauss"]:
            assert r["ref_gauss_int"] == list(gi)
            assert r["gauss_max"] == list(gm)


def test_golden_ic_is_reproducible(oracle_mod):
    """The oracle's initial-data generator regenerates the stored initial data."""
    for path in GOLDEN:
        z, meta = load_golden(path)
        p = _params(oracle_mod, meta)
        ic = oracle_mod.ICSpec(**meta["ic"])
        dtype = np.float64 if meta["storage"] == "f64" else np.float32
        sc, ve = oracle_mod.init_fields(p, ic, dtype)
        np.testing.assert_allclose(sc, z["ic_scalars"], rtol=0, atol=4 * np.finfo(dtype).eps)
        np.testing.assert_allclose(ve, z["ic_vectors"], rtol=0, atol=4 * np.finfo(dtype).eps)


def test_oracle_free_field_limit(oracle_mod):
    """g = g' = 0, lambda = 0 and identity links: the scalar update is the lattice wave equation."""
    p = oracle_mod.Params(nx=5, ny=4, nz=6, g=0.0, gp=0.0, lam=0.0)
    ic = oracle_mod.ICSpec(seed=5, mean=[0.3] * 8, sigma=[0.2] * 8)
    sc, ve = oracle_mod.init_fields(p, ic, np.float64)
    phi = sc[1].copy()
    past = sc[0].copy()
    oracle_mod.evolve(p, sc, ve, 1)
    lap = -6.0 * phi
    for ax in range(3):
        lap += np.roll(phi, 1, axis=ax) + np.roll(phi, -1, axis=ax)
    expect = 2 * phi - past + p.dt ** 2 * lap
    np.testing.assert_allclose(sc[0], expect, rtol=0, atol=1e-15)


@pytest.mark.parametrize("model,hf,fixed,dtype,time_iter", [
    (1, 0, 0, np.float64, 0), (1, 0, 0, np.float32, 3), (1, 0, 5, np.float64, 2), (2, 0, 0, np.float64, 1),
    (2, 0, 0, np.float32, 0), (2, 1, 0, np.float64, 1), (2, 2, 0, np.float32, 2), (2, 2, 3, np.float64, 0)])
def test_oracle_gauss_matches_its_post_evolve_row(oracle_mod, model, hf, fixed, dtype, time_iter):
    """gauss() on the levels after a step reproduces that step's own Gauss row and local
    violations exactly (the same pass over the same fields, no step), with the Higgs-family
    constraints of gaugeNum 5 and 7 and Fixed faces."""
    p = oracle_mod.Params(model=model, nx=5, ny=4, nz=6, gauss_every=1, gauss_local_every=1, higgs_family=hf,
                          fixed_axes=fixed)
    ic = oracle_mod.ICSpec(seed=9, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(p, ic, dtype)
    rows, _, _, loc_g = oracle_mod.evolve(p, sc, ve, 1, time_iter0=time_iter, local=True)
    gi, gm, lg = oracle_mod.gauss(p, sc, ve, time_iter)
    assert list(gi) == rows[0]["gauss_int"] and list(gm) == rows[0]["gauss_max"]
    assert np.array_equal(lg, loc_g)
    assert max(gm) > 0.0


def test_oracle_rejects_bad_config(oracle_mod):
    p = oracle_mod.Params(model=7, nx=2, ny=2, nz=2)
    sc = np.zeros((2, 2, 2, 2, p.nsc), np.float32)
    ve = np.zeros((2, 2, 2, 2, 15), np.float32)
    with pytest.raises(ValueError):
        oracle_mod.evolve(p, sc, ve, 1)
    # a Higgs-family field exists only in the 2HDM (WilsonLoops::TwoHDM)
    p = oracle_mod.Params(model=oracle_mod.MODEL_SM, nx=2, ny=2, nz=2, higgs_family=oracle_mod.HF_U1)
    sc = np.zeros((2, 2, 2, 2, p.nsc), np.float32)
    ve = np.zeros((2, 2, 2, 2, p.nve), np.float32)
    with pytest.raises(ValueError):
        oracle_mod.evolve(p, sc, ve, 1)


def test_local_outputs_match_the_reference(oracle_mod, tmp_path):
    """Energy's local densities and GaugeCondition's local violations (Analysers/Source/Energy.cpp:117-163,
    191-207; GaugeCondition.cpp:117-140, 194-212) against the reference's own files, and the fields bit
    for bit: the energy pass (storeEnergy) runs on the union of the global and local Energy cadences."""
    from oracle import refrun
    if not refrun.available(False):
        pytest.skip("reference binaries not built in this environment")
    for model, hf, el, gl, ee, ge, fixed in ((1, 0, 3, 2, 2, 0, 2), (2, 2, 2, 3, 0, 4, 0)):
        p = oracle_mod.Params(model=model, nx=4, ny=5, nz=3, energy_every=ee, gauss_every=ge, higgs_family=hf,
                              gpp=0.5, energy_local_every=el, gauss_local_every=gl, fixed_axes=fixed)
        ic = oracle_mod.ICSpec(seed=5, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
        sc, ve = oracle_mod.init_fields(p, ic, np.float32)
        work = tmp_path / f"m{model}"
        work.mkdir()
        rsc, rve, _, _ = refrun.run(p, sc, ve, 7, workdir=str(work))
        o_sc, o_ve = sc.copy(), ve.copy()
        _, _, le, lg = oracle_mod.evolve(p, o_sc, o_ve, 7, local=True)
        np.testing.assert_array_equal(o_sc, rsc)
        np.testing.assert_array_equal(o_ve, rve)
        last_e = max(t for t in range(7) if t % el == 0)
        last_g = max(t for t in range(7) if t % gl == 0)
        fe = np.loadtxt(work / "Data" / "Continual" / f"local_quantities_{last_e}.dat").reshape(6, -1).T
        fg = np.loadtxt(work / "Data" / "Continual" / f"local_quantities_gauge_{last_g}.dat").reshape(-1, p.neq)
        # the files print 6 significant digits
        np.testing.assert_allclose(fe, le, rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(fg, lg, rtol=1e-5, atol=1e-9)


def test_live_reference_matches_oracle_when_built(oracle_mod):
    """If oracle/_ref was built here (the reference is mounted), compare live on a fresh random case."""
    from oracle import refrun
    if not (refrun.available(False) and refrun.available(True)):
        pytest.skip("reference binaries not built in this environment")
    cases = [(oracle_mod.MODEL_SM, 0, 0), (oracle_mod.MODEL_2HDM, 0, 0), (oracle_mod.MODEL_2HDM, oracle_mod.HF_U1, 0),
             (oracle_mod.MODEL_2HDM, oracle_mod.HF_SU2, 0), (oracle_mod.MODEL_SM, 0, 1),
             (oracle_mod.MODEL_2HDM, oracle_mod.HF_U1, 1)]
    for model, hf, gen in cases:
        for dtype in (np.float32, np.float64):
            p = oracle_mod.Params(model=model, nx=3, ny=4, nz=5, energy_every=2, gauss_every=2, higgs_family=hf, gpp=0.44,
                                  generator_rep=gen)
            ic = oracle_mod.ICSpec(seed=99, mean=[0.8] * 8, sigma=[0.15] * 8, theta_sigma=0.2, eps_sigma=0.2)
            sc, ve = oracle_mod.init_fields(p, ic, dtype)
            sc0, ve0 = sc.copy(), ve.copy()
            oracle_mod.evolve(p, sc, ve, 4)
            rs, rv, _, _ = refrun.run(p, sc0, ve0, 4, fp64=dtype == np.float64)
            np.testing.assert_array_equal(sc, rs)
            np.testing.assert_array_equal(ve, rv)


def test_oracle_reproduces_reference_at_config1_size(oracle_mod):
    """Benchmark configuration 1 at its own size (SM 32^3, identity links, Higgs
    N(0, 0.1^2), 10 steps, analysers every 10): the oracle's fields hash to the
    reference's (tests/golden/config1_sm_32_digest.json, made by the reference
    binaries) and its analyser sums equal the reference's, in both storages."""
    import hashlib
    import json

    from conftest import GOLDEN_DIR
    with open(os.path.join(GOLDEN_DIR, "config1_sm_32_digest.json")) as f:
        d = json.load(f)
    p = oracle_mod.Params(**d["params"])
    ic = oracle_mod.ICSpec(**d["ic"])

    def digest(sc, ve):
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(sc).tobytes())
        h.update(np.ascontiguousarray(ve).tobytes())
        return h.hexdigest()

    for st, run in d["runs"].items():
        dtype = np.float64 if st == "f64" else np.float32
        sc, ve = oracle_mod.init_fields(p, ic, dtype)
        assert digest(sc, ve) == run["ic_sha256"], st
        rows, warn = oracle_mod.evolve(p, sc, ve, d["nt"])
        assert warn == 0
        assert digest(sc, ve) == run["fields_sha256"], st
        assert len(rows) == len(run["rows"])
        for r, g in zip(rows, run["rows"]):
            assert r["time_iter"] == g["time_iter"]
            if g["has_energy"]:
                assert r["ref_energy"] == g["ref_energy"]
            if g["has_gauss"]:
                assert r["ref_gauss_int"] == g["ref_gauss_int"]
                assert r["gauss_max"] == g["gauss_max"]
