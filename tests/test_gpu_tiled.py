"""The TMA-staged tiled step kernel (mixed form) against the one-thread-per-site
kernel and the oracle (GPU).

Both kernels evaluate the same per-site arithmetic (gft_step_body.cuh); only
where the neighbours come from differs (shared-memory planes vs L1/L2).  The
compiler may contract multiply-adds differently in the two instantiations, so
after one step the fields agree to 2 float ulps of the field scale (|phi|, |U|
~ 1: 2.4e-7 absolute); after 7 steps, where such differences are integrated
like storage rounding, to 2e-6 absolute, and both stay within the mixed-form
bound of the FP64 oracle.  Cases cover every tile shape, march
lengths that do not divide nx, lattices where every tile touches the periodic
boundary, and the 2HDM model.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(oracle_mod, model, shape, seed=31, fixed_axes=0):
    from gftevolver_b200 import LatticeParams
    nx, ny, nz = shape
    op = oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, energy_every=3, gauss_every=3, fixed_axes=fixed_axes)
    ic = oracle_mod.ICSpec(seed=seed, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                           eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float32)
    return op, LatticeParams(**op.__dict__), sc, ve


def _run(p, sc, ve, nt, kind, tile=0, march=32):
    from gftevolver_b200 import Evolver
    with Evolver(p, form="mixed") as ev:
        ev.set_kernel(kind, tile, march)
        ev.upload(sc, ve, 0)
        rows = ev.evolve(nt)
        out = ev.download()
    return out[0], out[1], rows


def _maxdiff(a, b):
    return float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64))))


@pytest.mark.parametrize("model", [1, 2], ids=["sm", "2hdm"])
@pytest.mark.parametrize("shape,tile,march", [
    ((8, 8, 32), 0, 32),      # one tile per plane: every halo wraps
    ((12, 16, 64), 0, 5),     # march does not divide nx
    ((7, 8, 32), 1, 3),
    ((9, 12, 48), 2, 4),      # 4 x 16 tiles
    ((3, 4, 16), 2, 1),       # march 1
    ((20, 16, 32), 1, 64),    # march > nx
    ((10, 32, 48), 3, 6),     # 16 x 16 tiles
    ((4, 16, 16), 3, 32),     # 16 x 16, one tile per plane
])
@pytest.mark.parametrize("fixed_axes", [0, 3], ids=["periodic", "fixed_xy"])
def test_tiled_matches_global_kernel(oracle_mod, model, shape, tile, march, fixed_axes):
    op, p, sc, ve = _setup(oracle_mod, model, shape, fixed_axes=fixed_axes)
    g1 = _run(p, sc, ve, 1, kind=1)
    t1 = _run(p, sc, ve, 1, kind=2, tile=tile, march=march)
    assert _maxdiff(t1[0], g1[0]) <= 2.4e-7 and _maxdiff(t1[1], g1[1]) <= 2.4e-7
    g_sc, g_ve, g_rows = _run(p, sc, ve, 7, kind=1)
    t_sc, t_ve, t_rows = _run(p, sc, ve, 7, kind=2, tile=tile, march=march)
    assert _maxdiff(t_sc, g_sc) <= 2e-6 and _maxdiff(t_ve, g_ve) <= 2e-6
    assert len(t_rows) == len(g_rows)
    for a, b in zip(t_rows, g_rows):
        assert a["time_iter"] == b["time_iter"]
        for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric", "plaq_su2", "plaq_u1"):
            assert abs(a[k] - b[k]) <= 1e-6 * max(1.0, abs(b[k])), k
    # and against the FP64 oracle within the mixed-form bound
    o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(seed=31, mean=[1.0 if model == 1 else 0.7] * 8,
                                                              sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1),
                                        np.float64)
    oracle_mod.evolve(op, o_sc, o_ve, 7)
    assert np.max(np.abs(t_sc.astype(np.float64) - o_sc)) <= 6e-6
    assert np.max(np.abs(t_ve.astype(np.float64) - o_ve)) <= 6e-6


def test_tiled_rejects_indivisible_lattice(oracle_mod):
    from gftevolver_b200 import Evolver, GftError
    _, p, sc, ve = _setup(oracle_mod, 1, (4, 6, 20))
    with Evolver(p, form="mixed") as ev:
        with pytest.raises(GftError):
            ev.set_kernel(2, 0, 8)
        ev.upload(sc, ve, 0)
        ev.evolve(2)  # automatic choice falls back to the one-thread-per-site kernel


@pytest.mark.parametrize("shape,tile,march,fixed", [
    ((8, 8, 32), 0, 32, 0),      # every halo wraps
    ((10, 24, 96), 0, 4, 0),     # an interior 8 x 32 tile; march does not divide nx
    ((9, 48, 128), 0, 4, 0),     # 8 of 24 tiles per chunk interior: the march without per-plane barriers
    ((6, 48, 48), 3, 32, 0),     # an interior 16 x 16 tile
    ((10, 24, 96), 0, 4, 5),     # Fixed faces on x and z (frozen sites inside x-marches)
    ((8, 8, 32), 0, 32, 7),      # Fixed faces on every axis
])
def test_fp64_tiled_matches_oracle(oracle_mod, shape, tile, march, fixed):
    """The FP64 form through the staged tiled step (gft_set_kernel kind 2; the automatic FP64
    SM kernel on large lattices): the FP64 bar, 1e-12 relative to the FP64 oracle after 10
    steps; energy terms within 1e-12 of the total."""
    from gftevolver_b200 import Evolver, LatticeParams
    nx, ny, nz = shape
    op = oracle_mod.Params(model=1, nx=nx, ny=ny, nz=nz, energy_every=3, gauss_every=4, fixed_axes=fixed)
    ic = oracle_mod.ICSpec(seed=33, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float64)
    with Evolver(LatticeParams(**op.__dict__), form="fp64") as ev:
        ev.set_kernel(2, tile, march)
        assert ev.step_kernel_name == "tiled_step_kernel"
        ev.upload(sc, ve, 0)
        rows = ev.evolve(10)
        g_sc, g_ve = ev.download()
    o_rows, _ = oracle_mod.evolve(op, sc, ve, 10)
    for a, b in ((g_sc, sc), (g_ve, ve)):
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) <= 1e-12
    assert [r["time_iter"] for r in rows] == [r["time_iter"] for r in o_rows]
    for a, b in zip(rows, o_rows):
        if b["has_energy"]:  # components relative to the total energy, as for the one-site FP64 step
            for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric"):
                assert abs(a[k] - b[k]) <= 1e-12 * max(abs(b["energy"]), 1.0), k
            assert abs(a["plaq_su2"] - b["plaq_su2"]) <= 1e-13
            assert abs(a["phi_sq"] - b["phi_sq"]) <= 1e-12
        if b["has_gauss"]:
            # rounding level on periodic lattices; next to frozen sites the residual is the
            # oracle's (the Fixed faces break the constraint there, as in the reference)
            np.testing.assert_allclose(a["gauss_max"], b["gauss_max"], rtol=1e-8, atol=1e-12)


@pytest.mark.parametrize("kind,shape,tile,march,fixed", [
    (1, (10, 24, 96), 0, 4, 0),   # after the one-thread-per-site step
    (2, (10, 24, 96), 0, 4, 0),   # after the tiled step: an interior 8 x 32 tile; march does not divide nx
    (2, (8, 8, 32), 0, 32, 0),    # every halo wraps
    (2, (6, 48, 48), 3, 32, 0),   # 16 x 16 tiles with interior tiles
    (2, (9, 12, 48), 2, 1, 0),    # 4 x 16 tiles, march 1
    (2, (7, 8, 32), 1, 3, 0),     # 4 x 32 tiles
    (2, (10, 24, 96), 0, 4, 5),   # Fixed faces on x and z
    (2, (8, 8, 32), 0, 32, 7),    # Fixed faces on every axis
])
def test_gauss_pass_matches_oracle_on_the_same_fields(oracle_mod, kind, shape, tile, march, fixed):
    """The mixed form's Gauss pass (fast_gauss_kernel, FP64 from the stored floats) against
    the oracle's FP64 Gauss pass over the very fields the GPU's last step left, downloaded and
    widened exactly to double: both evaluate the residual in FP64 from the same inputs, so
    the maximum and the integral agree to 1e-12 relative, and every local violation (rounded
    to float) to one float ulp plus 1e-16: the kernel may contract multiply-adds where the
    oracle rounds twice, a difference of order 1e-17 on terms of order 0.1, which the float
    rounding of the smallest violations (down to 1e-13) can show."""
    nx, ny, nz = shape
    op = oracle_mod.Params(model=1, nx=nx, ny=ny, nz=nz, gauss_every=1, gauss_local_every=1, fixed_axes=fixed)
    _check_gauss_on_same_fields(oracle_mod, op, kind, tile, march, mean=1.0)


@pytest.mark.parametrize("hf", [0, 1, 2], ids=["2hdm", "2hdm_hf_u1", "2hdm_hf_su2"])
def test_gauss_pass_2hdm_matches_oracle_on_the_same_fields(oracle_mod, hf):
    """As above for the 2HDM model: both doublets, and the Higgs-family constraints of gaugeNum
    5 and 7 (one thread per site; the kernel the automatic choice takes for 2HDM)."""
    op = oracle_mod.Params(model=2, nx=6, ny=8, nz=32, gauss_every=1, gauss_local_every=1, higgs_family=hf)
    _check_gauss_on_same_fields(oracle_mod, op, 1, 0, 32, mean=0.7)


def _check_gauss_on_same_fields(oracle_mod, op, kind, tile, march, mean):
    from gftevolver_b200 import Evolver, LatticeParams
    ic = oracle_mod.ICSpec(seed=41, mean=[mean] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float32)
    with Evolver(LatticeParams(**op.__dict__), form="mixed") as ev:
        ev.set_kernel(kind, tile, march)
        assert ev.step_kernel_name == ("tiled_step_kernel" if kind == 2 else "fast_step_kernel")
        ev.upload(sc, ve, 0)
        rows = ev.evolve(3)
        g_sc, g_ve = ev.download()
        _, _, lg, gstep = ev.local_fields()
    assert rows[-1]["time_iter"] == 2 and rows[-1]["has_gauss"] and gstep == 2
    gi, gm, o_lg = oracle_mod.gauss(op, g_sc.astype(np.float64), g_ve.astype(np.float64), 2)
    np.testing.assert_allclose(rows[-1]["gauss_max"], gm, rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(rows[-1]["gauss_int"], gi, rtol=1e-12, atol=1e-18)
    assert max(gm) > 0.0
    tol = np.spacing(np.abs(o_lg).astype(np.float32)).astype(np.float64) + 1e-16
    excess = np.abs(lg.astype(np.float64) - o_lg) - tol
    assert excess.max() <= 0.0, (excess.max(), o_lg.flat[np.argmax(excess)])
