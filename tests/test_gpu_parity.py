"""CUDA path vs the oracle and the reference's golden fixtures (GPU).

Tolerances (stated per form):
  ref32  float storage, reference arithmetic (FP64 per site, no FMA): equal to
         the reference except where CUDA's sin/cos/asin differ from glibc in
         the last bit; fields within 8 float ulps of |value| and at most 1% of
         words differ at all; energies within 1e-6 relative.
  ref64  double storage, reference arithmetic: fields within 1e-13 relative.
  fp64   plain FP64 form (reassociated): fields within 1e-12 relative
         (max |a - b| / max |b| per field array) after 10 steps, observables
         within 1e-12 relative.
  mixed  FP32 storage / mixed arithmetic vs the FP64 oracle: fields within
         6e-6 absolute after 10 steps (|fields| ~ 1), energies 1e-6 relative.
         With two FP32 time levels the rounding of each new level (<= 6e-8)
         is a velocity error that the leapfrog integrates twice, so the
         deviation grows like 6e-8 * n^1.5 per word (rms ~6e-7 at n = 10; the
         bound covers the maximum over ~1e5 words).  The reference's own
         float build carries the same storage error.
"""
import os

import numpy as np
import pytest

from conftest import golden_files, load_golden

pytestmark = pytest.mark.gpu

GOLDEN = golden_files()


def _lp(meta_params):
    from gftevolver_b200 import LatticeParams
    return LatticeParams(**meta_params)


def run_gpu(params, form, sc, ve, nt, time_iter=0):
    from gftevolver_b200 import Evolver
    with Evolver(params, form=form) as ev:
        ev.upload(sc, ve, time_iter)
        rows = ev.evolve(nt)
        warn = ev.last_warnings
        osc, ove = ev.download(sc.dtype)
    return osc, ove, rows, warn


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def ulp_close(a, b, nulp):
    a = np.asarray(a)
    b = np.asarray(b)
    tol = nulp * np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(a.dtype))
    return np.abs(a.astype(np.float64) - b.astype(np.float64)) <= tol.astype(np.float64) + 1e-30


@pytest.mark.parametrize("path", [p for p in GOLDEN if p.endswith("_f32.npz")],
                         ids=[os.path.basename(p) for p in GOLDEN if p.endswith("_f32.npz")])
def test_ref32_matches_reference_golden(path):
    z, meta = load_golden(path)
    p = _lp(meta["params"])
    sc, ve, rows, warn = run_gpu(p, "ref32", z["ic_scalars"], z["ic_vectors"], meta["nt"])
    assert warn == 0
    for got, want in ((sc, z["scalars"]), (ve, z["vectors"])):
        ok = ulp_close(got, want, 8)
        assert ok.all(), f"max diff {np.max(np.abs(got - want))}"
        assert np.mean(got != want) <= 0.01
    assert [r["time_iter"] for r in rows] == list(z["row_time_iter"])
    dv = p.dx * p.dy * p.dz
    for r, e, gm in zip(rows, z["row_ref_energy"], z["row_gauss_max"]):
        if r["has_energy"]:
            np.testing.assert_allclose(r["energy"], e[0] * dv, rtol=2e-5)
        if r["has_gauss"]:
            np.testing.assert_allclose(r["gauss_max"], gm, rtol=1e-5, atol=1e-12)


@pytest.mark.parametrize("path", [p for p in GOLDEN if p.endswith("_f64.npz")],
                         ids=[os.path.basename(p) for p in GOLDEN if p.endswith("_f64.npz")])
@pytest.mark.parametrize("form,tol", [("ref64", 1e-13), ("fp64", 1e-12)])
def test_fp64_forms_match_reference_golden(path, form, tol):
    z, meta = load_golden(path)
    p = _lp(meta["params"])
    sc, ve, rows, warn = run_gpu(p, form, z["ic_scalars"], z["ic_vectors"], meta["nt"])
    assert warn == 0
    assert rel_err(sc, z["scalars"]) <= tol
    assert rel_err(ve, z["vectors"]) <= tol
    dv = p.dx * p.dy * p.dz
    for r, e, gm in zip(rows, z["row_ref_energy"], z["row_gauss_max"]):
        if r["has_energy"]:
            np.testing.assert_allclose(r["energy"], e[0] * dv, rtol=1e-11)
        if r["has_gauss"]:
            # Gauss residuals are rounding-level numbers; compare on the scale of the charge terms
            assert np.all(np.abs(np.array(r["gauss_max"]) - gm) <= 1e-12)


@pytest.mark.parametrize("model", [1, 2], ids=["sm", "2hdm"])
@pytest.mark.parametrize("shape,fixed", [((8, 8, 8), 0), ((5, 6, 7), 0), ((16, 12, 33), 0), ((8, 8, 32), 5),
                                         ((7, 8, 32), 7)])
def test_forms_vs_oracle_random(oracle_mod, model, shape, fixed):
    """Random links and Gaussian scalars, 10 steps, all forms against the oracle
    (periodic, and with Fixed faces on x and z or on every axis: a frozen shell)."""
    nx, ny, nz = shape
    op = oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, energy_every=5, gauss_every=5, fixed_axes=fixed)
    ic = oracle_mod.ICSpec(seed=1234 + nx, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8,
                           theta_sigma=0.1, eps_sigma=0.1)
    p = _lp(op.__dict__)
    sc64, ve64 = oracle_mod.init_fields(op, ic, np.float64)
    o_sc, o_ve = sc64.copy(), ve64.copy()
    o_rows, _ = oracle_mod.evolve(op, o_sc, o_ve, 10)
    # plain FP64 form
    sc, ve, rows, _ = run_gpu(p, "fp64", sc64, ve64, 10)
    assert rel_err(sc, o_sc) <= 1e-12
    assert rel_err(ve, o_ve) <= 1e-12
    for a, b in zip(rows, o_rows):
        assert a["time_iter"] == b["time_iter"]
        if b["has_energy"]:
            for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric"):
                assert abs(a[k] - b[k]) <= 1e-12 * max(abs(b["energy"]), 1.0), k
            assert abs(a["plaq_su2"] - b["plaq_su2"]) <= 1e-13
            assert abs(a["plaq_u1"] - b["plaq_u1"]) <= 1e-13
            assert abs(a["phi_sq"] - b["phi_sq"]) <= 1e-12
    # mixed form against the FP64 oracle
    sc32, ve32 = oracle_mod.init_fields(op, ic, np.float32)
    sc, ve, rows, _ = run_gpu(p, "mixed", sc32, ve32, 10)
    assert np.max(np.abs(sc.astype(np.float64) - o_sc)) <= 6e-6
    assert np.max(np.abs(ve.astype(np.float64) - o_ve)) <= 6e-6
    for a, b in zip(rows, o_rows):
        if b["has_energy"]:
            assert abs(a["energy"] - b["energy"]) <= 1e-6 * abs(b["energy"])
    # reference arithmetic, float storage, against the float oracle
    o32_sc, o32_ve = sc32.copy(), ve32.copy()
    oracle_mod.evolve(op, o32_sc, o32_ve, 10)
    sc, ve, rows, _ = run_gpu(p, "ref32", sc32, ve32, 10)
    assert ulp_close(sc, o32_sc, 8).all()
    assert ulp_close(ve, o32_ve, 8).all()


@pytest.mark.parametrize("hf", [1, 2], ids=["hf_u1", "hf_su2"])
@pytest.mark.parametrize("shape,fixed", [((8, 8, 8), 0), ((5, 6, 7), 0), ((6, 8, 12), 2)])
def test_higgs_family_forms_vs_oracle(oracle_mod, hf, shape, fixed):
    """2HDM with a Higgs-family U(1) (gaugeNum 5) or SU(2) (gaugeNum 7) gauge field,
    random links of both groups, 10 steps: every form against the oracle, the
    Gauss rows with all gaugeNum constraints."""
    nx, ny, nz = shape
    op = oracle_mod.Params(model=2, nx=nx, ny=ny, nz=nz, energy_every=5, gauss_every=5, fixed_axes=fixed,
                           higgs_family=hf, gpp=0.47)
    ic = oracle_mod.ICSpec(seed=4321 + nx + hf, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    p = _lp(op.__dict__)
    sc64, ve64 = oracle_mod.init_fields(op, ic, np.float64)
    assert ve64.shape[-1] == (18 if hf == 1 else 27)
    o_sc, o_ve = sc64.copy(), ve64.copy()
    o_rows, _ = oracle_mod.evolve(op, o_sc, o_ve, 10)
    sc, ve, rows, warn = run_gpu(p, "fp64", sc64, ve64, 10)
    assert warn == 0
    assert rel_err(sc, o_sc) <= 1e-12
    assert rel_err(ve, o_ve) <= 1e-12
    assert [r["time_iter"] for r in rows] == [r["time_iter"] for r in o_rows]
    for a, b in zip(rows, o_rows):
        if b["has_energy"]:
            for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric"):
                assert abs(a[k] - b[k]) <= 1e-12 * max(abs(b["energy"]), 1.0), k
        if b["has_gauss"]:
            assert len(a["gauss_max"]) == op.neq
            np.testing.assert_allclose(a["gauss_int"], b["gauss_int"], rtol=1e-9, atol=1e-13)
            np.testing.assert_allclose(a["gauss_max"], b["gauss_max"], rtol=1e-9, atol=1e-13)
    # mixed form against the FP64 oracle
    sc32, ve32 = oracle_mod.init_fields(op, ic, np.float32)
    sc, ve, rows, _ = run_gpu(p, "mixed", sc32, ve32, 10)
    assert np.max(np.abs(sc.astype(np.float64) - o_sc)) <= 6e-6
    assert np.max(np.abs(ve.astype(np.float64) - o_ve)) <= 6e-6
    for a, b in zip(rows, o_rows):
        if b["has_energy"]:
            assert abs(a["energy"] - b["energy"]) <= 1e-6 * abs(b["energy"])
    # reference arithmetic, float storage, against the float oracle (rows in the reference's order)
    o32_sc, o32_ve = sc32.copy(), ve32.copy()
    o32_rows, _ = oracle_mod.evolve(op, o32_sc, o32_ve, 10)
    sc, ve, rows, _ = run_gpu(p, "ref32", sc32, ve32, 10)
    assert ulp_close(sc, o32_sc, 8).all()
    assert ulp_close(ve, o32_ve, 8).all()
    for a, b in zip(rows, o32_rows):
        if b["has_gauss"]:
            np.testing.assert_allclose(a["gauss_max"], b["gauss_max"], rtol=1e-5, atol=1e-12)


@pytest.mark.parametrize("hf", [1, 2], ids=["hf_u1", "hf_su2"])
def test_higgs_family_device_initial_data(oracle_mod, hf):
    from gftevolver_b200 import Evolver, InitialData
    op = oracle_mod.Params(model=2, nx=5, ny=6, nz=7, higgs_family=hf)
    spec = dict(seed=91, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    with Evolver(_lp(op.__dict__), form="fp64") as ev:
        ev.init_fields(InitialData(**spec))
        g_sc, g_ve = ev.download()
    o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**spec), np.float64)
    assert np.max(np.abs(g_sc - o_sc)) <= 4e-14
    assert np.max(np.abs(g_ve - o_ve)) <= 1e-14


def test_higgs_family_is_refused_where_not_built(oracle_mod):
    """The tiled kernel and the ensemble evolve gaugeNum 4 only."""
    from gftevolver_b200 import Evolver, _lib
    op = oracle_mod.Params(model=2, nx=8, ny=8, nz=32, higgs_family=1)
    with Evolver(_lp(op.__dict__), form="mixed") as ev:
        assert ev.lib.gft_set_kernel(ev.h, 2, 0, 8) == _lib.GFT_E_UNSUPPORTED
        assert ev.step_kernel_name == "fast_step_kernel"


@pytest.mark.parametrize("model,hf", [(1, 0), (2, 0), (2, 1), (2, 2)], ids=["sm", "2hdm", "2hdm_hf_u1", "2hdm_hf_su2"])
@pytest.mark.parametrize("shape", [(8, 8, 32), (5, 6, 7)])
def test_generator_representation_forms_vs_oracle(oracle_mod, model, hf, shape):
    """Links stored as generators (WilsonLoops/Source/StandardModel.cpp:76-160): the
    reference-arithmetic form converts on every access as the reference does; the
    throughput forms convert at the transfer and evolve quaternions (8 x 8 x 32 SM
    mixed runs the tiled kernel)."""
    nx, ny, nz = shape
    op = oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, energy_every=5, gauss_every=5, higgs_family=hf,
                           gpp=0.47, generator_rep=1)
    ic = oracle_mod.ICSpec(seed=777 + nz + hf, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8,
                           theta_sigma=0.1, eps_sigma=0.1)
    p = _lp(op.__dict__)
    sc64, ve64 = oracle_mod.init_fields(op, ic, np.float64)
    assert ve64.shape[-1] == op.nve
    o_sc, o_ve = sc64.copy(), ve64.copy()
    o_rows, _ = oracle_mod.evolve(op, o_sc, o_ve, 10)
    for form in ("fp64", "ref64"):
        sc, ve, rows, warn = run_gpu(p, form, sc64, ve64, 10)
        assert warn == 0
        assert rel_err(sc, o_sc) <= 1e-12, form
        assert rel_err(ve, o_ve) <= 1e-12, form
        for a, b in zip(rows, o_rows):
            if b["has_energy"]:
                assert abs(a["energy"] - b["energy"]) <= 1e-12 * abs(b["energy"]), form
            if b["has_gauss"]:
                np.testing.assert_allclose(a["gauss_max"], b["gauss_max"], rtol=1e-8, atol=1e-13)
    sc32, ve32 = oracle_mod.init_fields(op, ic, np.float32)
    from gftevolver_b200 import Evolver
    with Evolver(p, form="mixed") as ev:
        if model == 1 and shape == (8, 8, 32):
            ev.set_kernel(2, 0, 32)  # the staged step (too few tiles for the automatic choice)
        ev.upload(sc32, ve32, 0)
        rows = ev.evolve(10)
        sc, ve = ev.download()
        if model == 1 and shape == (8, 8, 32):
            assert ev.step_kernel_name == "tiled_step_kernel"
    assert np.max(np.abs(sc.astype(np.float64) - o_sc)) <= 6e-6
    assert np.max(np.abs(ve.astype(np.float64) - o_ve)) <= 6e-6
    for a, b in zip(rows, o_rows):
        if b["has_energy"]:
            assert abs(a["energy"] - b["energy"]) <= 1e-6 * abs(b["energy"])
    o32_sc, o32_ve = sc32.copy(), ve32.copy()
    oracle_mod.evolve(op, o32_sc, o32_ve, 10)
    sc, ve, rows, _ = run_gpu(p, "ref32", sc32, ve32, 10)
    assert ulp_close(sc, o32_sc, 8).all()
    assert ulp_close(ve, o32_ve, 8).all()


@pytest.mark.parametrize("form,dtype,tol", [("ref32", np.float32, 0.0), ("fp64", np.float64, 1e-15)])
def test_generator_representation_device_initial_data(oracle_mod, form, dtype, tol):
    """Device initial data in the generator representation: w = eps n."""
    from gftevolver_b200 import Evolver, InitialData
    op = oracle_mod.Params(model=2, nx=5, ny=6, nz=7, higgs_family=2, generator_rep=1)
    spec = dict(seed=93, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    with Evolver(_lp(op.__dict__), form=form) as ev:
        ev.init_fields(InitialData(**spec))
        g_sc, g_ve = ev.download()
    o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**spec), dtype)
    assert np.max(np.abs(g_sc.astype(np.float64) - o_sc)) <= max(tol, 1e-7 if dtype == np.float32 else 0) * 4
    assert np.max(np.abs(g_ve.astype(np.float64) - o_ve)) <= max(tol, 1e-7 if dtype == np.float32 else 0)


@pytest.mark.parametrize("form", ["ref32", "fp64", "mixed"])
@pytest.mark.parametrize("model,hf,fixed", [(1, 0, 0), (2, 1, 0), (1, 0, 4)])
def test_local_outputs_vs_oracle(oracle_mod, form, model, hf, fixed):
    """Per-site Energy densities and signed Gauss violations of the last local-output step
    (gft_local_fields) against the oracle; local cadences differ from the global ones, so the
    fields also check that the energy pass runs on their union."""
    nx, ny, nz = 6, 8, 32
    op = oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, energy_every=4, gauss_every=0, higgs_family=hf,
                           gpp=0.47, fixed_axes=fixed, energy_local_every=3, gauss_local_every=2)
    ic = oracle_mod.ICSpec(seed=55, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                           eps_sigma=0.1)
    dtype = np.float32 if form in ("ref32", "mixed") else np.float64
    sc0, ve0 = oracle_mod.init_fields(op, ic, dtype)
    o_sc, o_ve = sc0.copy(), ve0.copy()
    o_dtype = np.float32 if form == "ref32" else np.float64
    if o_dtype != dtype:
        o_sc, o_ve = o_sc.astype(o_dtype), o_ve.astype(o_dtype)
    _, _, o_le, o_lg = oracle_mod.evolve(op, o_sc, o_ve, 8, local=True)
    from gftevolver_b200 import Evolver
    with Evolver(_lp(op.__dict__), form=form) as ev:
        ev.upload(sc0, ve0, 0)
        ev.evolve(8)
        le, es, lg, gs = ev.local_fields()
        sc, ve = ev.download()
    assert (es, gs) == (6, 6)
    tol = {"ref32": (2e-6, 1e-9), "fp64": (1e-6, 1e-9), "mixed": (1e-4, 1e-6)}[form]
    np.testing.assert_allclose(le, o_le, rtol=tol[0], atol=tol[1] * np.abs(o_le).max())
    # the SM violations are rounding-level numbers: ref32 / fp64 reproduce the oracle's; in the mixed
    # form they are the FP32 storage noise of the two levels (~1e-8 .. 1e-7 here), so the mixed form is
    # held to an absolute bound (the Higgs-family violation of the reference's equations is O(1e-4))
    scale = np.abs(o_lg).max()
    if form == "mixed":
        assert np.max(np.abs(lg - o_lg)) <= 1e-6
    else:
        gtol = {"ref32": 1e-6, "fp64": 1e-7}[form]
        assert np.max(np.abs(lg - o_lg)) <= gtol * max(scale, 1e-3)
    if fixed:
        frozen = np.zeros((nx, ny, nz), bool)
        frozen[:, :, 0] = frozen[:, :, -1] = True
        assert np.all(le.reshape(nx, ny, nz, 6)[frozen] == 0) and np.all(lg.reshape(nx, ny, nz, -1)[frozen] == 0)
    if form == "ref32":
        assert ulp_close(sc, o_sc, 8).all() and ulp_close(ve, o_ve, 8).all()
    elif form == "fp64":
        assert rel_err(sc, o_sc) <= 1e-12 and rel_err(ve, o_ve) <= 1e-12


def test_time_iter_parity_and_chunking(oracle_mod):
    """Evolving 3 + 4 steps equals 7 steps; the now/past slot follows time_iter (Lattice.cpp:773)."""
    op = oracle_mod.Params(nx=6, ny=5, nz=4, energy_every=2, gauss_every=3)
    ic = oracle_mod.ICSpec(seed=3, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float64)
    o_sc, o_ve = sc.copy(), ve.copy()
    o_rows, _ = oracle_mod.evolve(op, o_sc, o_ve, 7)
    from gftevolver_b200 import Evolver
    with Evolver(_lp(op.__dict__), form="fp64") as ev:
        ev.upload(sc, ve, 0)
        rows = ev.evolve(3) + ev.evolve(4)
        assert ev.time_iter == 7
        g_sc, g_ve = ev.download()
    assert rel_err(g_sc, o_sc) <= 1e-12 and rel_err(g_ve, o_ve) <= 1e-12
    assert [r["time_iter"] for r in rows] == [r["time_iter"] for r in o_rows]


def test_device_initial_data_matches_oracle(oracle_mod):
    from gftevolver_b200 import Evolver, InitialData
    op = oracle_mod.Params(model=2, nx=6, ny=7, nz=20)
    spec = dict(seed=77, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1, wall_width=5.0,
                wall_value=1.0)
    for form, dtype, tol in (("fp64", np.float64, 1e-14), ("mixed", np.float32, 2.5e-7)):
        with Evolver(_lp(op.__dict__), form=form) as ev:
            ev.init_fields(InitialData(**spec))
            g_sc, g_ve = ev.download()
        o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**spec), dtype)
        assert np.max(np.abs(g_sc.astype(np.float64) - o_sc)) <= tol * 4
        assert np.max(np.abs(g_ve.astype(np.float64) - o_ve)) <= tol


def test_domain_warning_is_reported(oracle_mod):
    """A link RHS outside asin's / sqrt's domain sets GFT_W_* bits (the reference prints "Panic", StandardModel.cpp:474-491)."""
    op = oracle_mod.Params(nx=4, ny=4, nz=4)
    ic = oracle_mod.ICSpec(seed=9, mean=[1.0] * 8, sigma=[0.5] * 8, theta_sigma=1.0, eps_sigma=1.0)
    sc, ve = oracle_mod.init_fields(op, ic, np.float64)
    sc *= 300.0  # currents g^2 J dt^2 of order 10: |RHS| > 1 at many sites
    _, _, _, warn = run_gpu(_lp(op.__dict__), "fp64", sc, ve, 1)
    o_sc, o_ve = sc.copy(), ve.copy()
    _, owarn = oracle_mod.evolve(op, o_sc, o_ve, 1)
    assert owarn & 3 != 0
    assert warn & 3 == owarn & 3


def test_observe_does_not_advance(oracle_mod):
    from gftevolver_b200 import Evolver
    op = oracle_mod.Params(nx=8, ny=8, nz=8, energy_every=1)
    ic = oracle_mod.ICSpec(seed=4, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float64)
    with Evolver(_lp(op.__dict__), form="fp64") as ev:
        ev.upload(sc, ve, 0)
        o = ev.observe()
        assert ev.time_iter == 0
        r = ev.evolve(1)[0]
        a_sc, a_ve = ev.download()
    assert abs(o["energy"] - r["energy"]) <= 1e-12 * abs(r["energy"])
    o_sc, o_ve = sc.copy(), ve.copy()
    oracle_mod.evolve(op, o_sc, o_ve, 1)
    assert rel_err(a_sc, o_sc) <= 1e-12


@pytest.mark.parametrize("form", ["mixed", "fp64"])
def test_device_buffer_transfers_match_host_transfers(oracle_mod, form):
    """gft_upload_device_* / gft_download_device_* move the same reference-layout words as the host calls."""
    import torch
    from gftevolver_b200 import Evolver
    op = oracle_mod.Params(nx=8, ny=6, nz=32, energy_every=2, gauss_every=2)
    ic = oracle_mod.ICSpec(seed=12, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    dtype = np.float64 if form == "fp64" else np.float32
    sc, ve = oracle_mod.init_fields(op, ic, dtype)
    f64 = form == "fp64"
    d_sc = torch.from_numpy(sc).cuda()
    d_ve = torch.from_numpy(ve).cuda()
    with Evolver(_lp(op.__dict__), form=form) as a, Evolver(_lp(op.__dict__), form=form) as b:
        a.upload(sc, ve, 0)
        b.upload_device(d_sc.data_ptr(), d_ve.data_ptr(), f64, 0)
        ra, rb = a.evolve(3), b.evolve(3)
        h_sc, h_ve = a.download()
        o_sc, o_ve = torch.empty_like(d_sc), torch.empty_like(d_ve)
        b.download_device(o_sc.data_ptr(), o_ve.data_ptr(), f64)
    assert np.array_equal(h_sc, o_sc.cpu().numpy()) and np.array_equal(h_ve, o_ve.cpu().numpy())
    assert [r["energy"] for r in ra] == [r["energy"] for r in rb]


def test_step_kernel_name_follows_form_and_shape(oracle_mod):
    """The automatic choice takes the staged step for the SM model when its tiles fill
    0.8 of a wave of resident CTAs (mixed form) or 5 waves (FP64), else one thread per site."""
    from gftevolver_b200 import Evolver
    op = oracle_mod.Params(nx=8, ny=8, nz=32)  # one tile
    with Evolver(_lp(op.__dict__), form="mixed") as ev:
        assert ev.step_kernel_name == "fast_step_kernel"
        ev.set_kernel(2, 0, 32)
        assert ev.step_kernel_name == "tiled_step_kernel"
        ev.set_kernel(1, 0, 32)
        assert ev.step_kernel_name == "fast_step_kernel"
    with Evolver(_lp(op.__dict__), form="fp64") as ev:
        assert ev.step_kernel_name == "fast_step_kernel"
        ev.set_kernel(2, 0, 32)
        assert ev.step_kernel_name == "tiled_step_kernel"
    big = oracle_mod.Params(nx=64, ny=256, nz=256)  # 8 x 32 tiles, march 32: 512 tiles = 1.7 waves of 296
    with Evolver(_lp(big.__dict__), form="mixed") as ev:
        assert ev.step_kernel_name == "tiled_step_kernel"
    with Evolver(_lp(big.__dict__), form="fp64") as ev:  # FP64: 3.5 waves of 148, under 5
        assert ev.step_kernel_name == "fast_step_kernel"
        ev.set_kernel(0, 3, 16)  # automatic with 16 x 16 tiles, march 16: 1024 tiles = 6.9 waves
        assert ev.step_kernel_name == "tiled_step_kernel"
    with Evolver(_lp(op.__dict__), form="ref32") as ev:
        assert ev.step_kernel_name == "ref_step_kernel"
    odd = oracle_mod.Params(nx=5, ny=3, nz=7)
    with Evolver(_lp(odd.__dict__), form="mixed") as ev:
        assert ev.step_kernel_name == "fast_step_kernel"
        ev.set_kernel(0, 0, 32)  # automatic, with a tile the lattice does not divide into
        assert ev.step_kernel_name == "fast_step_kernel"
    two = oracle_mod.Params(model=2, nx=8, ny=8, nz=32)  # 2HDM: one thread per site unless asked
    with Evolver(_lp(two.__dict__), form="mixed") as ev:
        assert ev.step_kernel_name == "fast_step_kernel"
        ev.set_kernel(2, 0, 32)
        assert ev.step_kernel_name == "tiled_step_kernel"


@pytest.mark.parametrize("form", ["mixed", "fp64", "ref32"])
def test_checkpoint_restart_continues_bit_for_bit(tmp_path, oracle_mod, form):
    from gftevolver_b200 import Evolver, InitialData
    op = oracle_mod.Params(nx=8, ny=8, nz=32, energy_every=3, gauss_every=4)
    with Evolver(_lp(op.__dict__), form=form) as ev:
        ev.init_fields(InitialData(seed=8, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1))
        ev.evolve(5)
        ev.save(str(tmp_path / "ck.npz"))
        rows_a = ev.evolve(6)
        a = ev.download()
    with Evolver.load(str(tmp_path / "ck.npz")) as ev:
        assert ev.time_iter == 5 and ev.form == form
        rows_b = ev.evolve(6)
        b = ev.download()
    assert rows_a == rows_b
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
