"""Parity at the benchmark configurations and on the staged tiles that carry them (GPU).

* Configuration 1 at its own size: SM 32^3, identity links, Higgs N(0, 0.1^2),
  g = 0.65, g' = 0.35, lambda = 0.13, v = 1, dt = 0.05, analysers every 10
  steps.  The oracle is pinned to the reference binaries at this size by a
  digest of their fields (tests/test_oracle.py); here every GPU form runs 10
  steps against it: fp64 <= 1e-12 relative, ref64 <= 1e-13, ref32 within 8
  float ulps on at least 99 % of the words, mixed <= 6e-6 absolute; the rows'
  energies, Gauss residuals and average plaquettes likewise.
* The staged (TMA ring + halo staging) tiled kernel on lattices with interior
  tiles -- tiles whose halo touches no lattice face, the case that makes up
  most of a 256^3 step -- for every tile shape and both models, single
  handles and an ensemble, against the FP64 oracle (mixed bound 6e-6) and
  against the one-thread-per-site kernel (2 float ulps after one step).
* The benchmark sizes themselves (SM 256^3, 2HDM 192^3): the mixed form
  against the FP64 form (itself pinned to the oracle at small sizes) on the
  same device-generated initial data, with asserted bounds: after 10 steps
  every stored word within 1e-5 absolute; over 1000 steps at 256^3 the energy
  of the mixed form within 1e-6 relative of the FP64 energy at every logging
  step, the FP64 Gauss residual at rounding level (<= 1e-12), the mixed
  form's Gauss residual below its FP32 storage floor bound (<= 1e-5), and
  every stored word within 1e-3 absolute.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# ---------------------------------------------------------------------------
# configuration 1 (SM 32^3 FP64, identity links) against the oracle
# ---------------------------------------------------------------------------
CONFIG1 = dict(nx=32, ny=32, nz=32, dt=0.05, g=0.65, gp=0.35, lam=0.13, eta_sqr=1.0, energy_every=10,
               gauss_every=10)


def _ulp_close(a, b, nulp):
    tol = nulp * np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(a.dtype))
    return np.abs(a.astype(np.float64) - b.astype(np.float64)) <= tol.astype(np.float64) + 1e-30


@pytest.mark.parametrize("form", ["fp64", "ref64", "ref32", "mixed"])
def test_config1_sm32_identity_links_vs_oracle(oracle_mod, form):
    from gftevolver_b200 import Evolver, InitialData, LatticeParams
    op = oracle_mod.Params(model=oracle_mod.MODEL_SM, **CONFIG1)
    ic = dict(seed=7, mean=[0.0] * 8, sigma=[0.1] * 8)
    host_dtype = np.float32 if form in ("ref32", "mixed") else np.float64
    orc_dtype = np.float32 if form == "ref32" else np.float64
    nt = 10
    with Evolver(LatticeParams(**op.__dict__), form=form) as ev:
        ev.init_fields(InitialData(**ic))
        rows = ev.evolve(nt)
        assert ev.last_warnings == 0
        g_sc, g_ve = ev.download(host_dtype)
    o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**ic), orc_dtype)
    o_rows, warn = oracle_mod.evolve(op, o_sc, o_ve, nt)
    assert warn == 0
    if form == "ref32":
        for a, b in ((g_sc, o_sc), (g_ve, o_ve)):
            close = _ulp_close(a, b, 8)
            assert close.all()
            assert np.mean(a != b) <= 0.01
    else:
        for a, b in ((g_sc, o_sc), (g_ve, o_ve)):
            a64, b64 = a.astype(np.float64), b.astype(np.float64)
            if form == "mixed":
                assert np.max(np.abs(a64 - b64)) <= 6e-6
            else:
                tol = 1e-12 if form == "fp64" else 1e-13
                assert np.max(np.abs(a64 - b64)) / np.max(np.abs(b64)) <= tol
    obs_tol = {"fp64": 1e-12, "ref64": 1e-12, "ref32": 1e-6, "mixed": 1e-6}[form]
    assert [r["time_iter"] for r in rows] == [r["time_iter"] for r in o_rows]
    for a, b in zip(rows, o_rows):
        if b["has_energy"]:
            for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric", "plaq_su2", "plaq_u1",
                      "phi_sq"):
                assert abs(a[k] - b[k]) <= obs_tol * max(1.0, abs(b[k])), (k, a[k], b[k])
        if b["has_gauss"]:
            # FP64 forms: residuals at rounding level in both; the float forms carry FP32 storage noise
            gtol = 1e-12 if form in ("fp64", "ref64") else 1e-5
            assert max(a["gauss_max"]) <= gtol and max(b["gauss_max"]) <= gtol


# ---------------------------------------------------------------------------
# staged tiled kernel with interior tiles
# ---------------------------------------------------------------------------
TILES = {0: (8, 32), 1: (4, 32), 2: (4, 16), 3: (16, 16)}


def _interior_tiles(shape, tile):
    """Number of (y, z) tiles whose one-site halo stays inside the lattice (no wrap)."""
    _, ny, nz = shape
    ty, tz = TILES[tile]
    return sum(1 for y0 in range(0, ny, ty) for z0 in range(0, nz, tz)
               if y0 != 0 and y0 + ty != ny and z0 != 0 and z0 + tz != nz)


INTERIOR_CASES = [
    ((10, 24, 96), 0, 4),   # 8 x 32: y tiles 0/8/16, z tiles 0/32/64 -> tile (8, 32) interior
    ((6, 12, 96), 1, 4),    # 4 x 32: tile (4, 32) interior
    ((6, 48, 48), 3, 32),   # 16 x 16: tile (16, 16) interior; march longer than nx
    ((5, 12, 48), 2, 2),    # 4 x 16: tile (4, 16) interior
]


def _ic(model, seed):
    return dict(seed=seed, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)


@pytest.mark.parametrize("model", [1, 2], ids=["sm", "2hdm"])
@pytest.mark.parametrize("shape,tile,march", INTERIOR_CASES, ids=["8x32", "4x32", "16x16", "4x16"])
def test_staged_interior_tiles_vs_oracle(oracle_mod, model, shape, tile, march):
    from gftevolver_b200 import Evolver, InitialData, LatticeParams
    assert _interior_tiles(shape, tile) >= 1
    nx, ny, nz = shape
    op = oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, energy_every=3, gauss_every=4)
    p = LatticeParams(**op.__dict__)
    ic = _ic(model, 41)

    def run(kind, nt):
        with Evolver(p, form="mixed") as ev:
            ev.set_kernel(kind, tile, march)
            ev.init_fields(InitialData(**ic))
            rows = ev.evolve(nt)
            name = ev.step_kernel_name
            sc, ve = ev.download()
        return sc, ve, rows, name

    # one step against the one-thread-per-site kernel: contraction-level agreement
    t_sc, t_ve, _, name = run(2, 1)
    assert "tiled" in name
    g_sc, g_ve, _, _ = run(1, 1)
    assert np.max(np.abs(t_sc - g_sc)) <= 2.4e-7 and np.max(np.abs(t_ve - g_ve)) <= 2.4e-7
    # ten steps (plain staged steps and logging steps) against the FP64 oracle
    t_sc, t_ve, rows, _ = run(2, 10)
    o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**ic), np.float64)
    o_rows, _ = oracle_mod.evolve(op, o_sc, o_ve, 10)
    assert np.max(np.abs(t_sc.astype(np.float64) - o_sc)) <= 6e-6
    assert np.max(np.abs(t_ve.astype(np.float64) - o_ve)) <= 6e-6
    assert [r["time_iter"] for r in rows] == [r["time_iter"] for r in o_rows]
    for a, b in zip(rows, o_rows):
        if b["has_energy"]:
            for k in ("energy", "plaq_su2", "plaq_u1", "phi_sq"):
                assert abs(a[k] - b[k]) <= 1e-5 * max(1.0, abs(b[k])), k


@pytest.mark.parametrize("model", [1, 2], ids=["sm", "2hdm"])
@pytest.mark.parametrize("tile,shapes", [
    (0, [(10, 24, 96), (6, 16, 64)]),
    (3, [(6, 48, 48), (4, 32, 64)]),
], ids=["8x32", "16x16"])
def test_ensemble_interior_tiles_vs_single_and_oracle(oracle_mod, model, tile, shapes):
    from gftevolver_b200 import Ensemble, Evolver, InitialData, LatticeParams
    assert _interior_tiles(shapes[0], tile) >= 1
    ops = [oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, energy_every=3, gauss_every=3)
           for nx, ny, nz in shapes]
    ps = [LatticeParams(**op.__dict__) for op in ops]
    ics = [_ic(model, 60 + k) for k in range(len(shapes))]
    nt = 7
    with Ensemble(ps) as ens:
        ens.set_kernel(tile, 4)
        ens.init_fields([InitialData(**ic) for ic in ics])
        ens.evolve(nt)
        out = [ens.download(m) for m in range(len(ps))]
    for m, (op, p, ic) in enumerate(zip(ops, ps, ics)):
        with Evolver(p, form="mixed") as ev:
            ev.set_kernel(2, tile, 4)
            ev.init_fields(InitialData(**ic))
            ev.evolve(nt)
            sc, ve = ev.download()
        assert np.max(np.abs(out[m][0] - sc)) <= 2e-6
        assert np.max(np.abs(out[m][1] - ve)) <= 2e-6
        o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**ic), np.float64)
        oracle_mod.evolve(op, o_sc, o_ve, nt)
        assert np.max(np.abs(out[m][0].astype(np.float64) - o_sc)) <= 6e-6
        assert np.max(np.abs(out[m][1].astype(np.float64) - o_ve)) <= 6e-6


# ---------------------------------------------------------------------------
# benchmark sizes: mixed form against the FP64 form on the device
# ---------------------------------------------------------------------------
def _bench_workload(model, n, every=10):
    from gftevolver_b200 import GFT_MODEL_2HDM, GFT_MODEL_SM, InitialData, LatticeParams
    if model == "sm":
        p = LatticeParams(model=GFT_MODEL_SM, nx=n, ny=n, nz=n, dt=0.05, g=0.65, gp=0.35, lam=0.13, eta_sqr=1.0,
                          energy_every=every, gauss_every=every)
        ic = InitialData(seed=20240101, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    else:
        p = LatticeParams(model=GFT_MODEL_2HDM, nx=n, ny=n, nz=n, dt=0.05, g=0.65, gp=0.35, m1=0.5, m2=0.5,
                          l1=0.065, l2=0.065, l3=0.2, m12r=0.2, l4p5=-0.1, energy_every=every, gauss_every=every)
        ic = InitialData(seed=20240102, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    return p, ic


def _mixed_and_fp64(p, ic, steps):
    """Evolve both forms from the same device initial data; returns the rows of
    each and the largest |word difference| of the scalars and of the links."""
    import torch

    from gftevolver_b200 import Evolver
    rows, fields = {}, {}
    for form in ("mixed", "fp64"):
        with Evolver(p, form=form) as ev:
            ev.init_fields(ic)
            rows[form] = ev.evolve(steps)
            assert ev.last_warnings == 0, form
            dt = torch.float64 if form == "fp64" else torch.float32
            sc = torch.empty((2, p.nx, p.ny, p.nz, p.nsc), dtype=dt, device="cuda:0")
            ve = torch.empty((2, p.nx, p.ny, p.nz, p.nve), dtype=dt, device="cuda:0")
            ev.download_device(sc.data_ptr(), ve.data_ptr(), form == "fp64")
            torch.cuda.synchronize()
            fields[form] = (sc, ve)
    d_sc = (fields["mixed"][0].double() - fields["fp64"][0]).abs().max().item()
    d_ve = (fields["mixed"][1].double() - fields["fp64"][1]).abs().max().item()
    del fields
    torch.cuda.empty_cache()
    return rows, d_sc, d_ve


@pytest.mark.parametrize("model,n", [("sm", 256), ("2hdm", 192)])
def test_benchmark_size_mixed_vs_fp64_ten_steps(model, n):
    p, ic = _bench_workload(model, n)
    rows, d_sc, d_ve = _mixed_and_fp64(p, ic, 10)
    assert d_sc <= 1e-5 and d_ve <= 1e-5, (d_sc, d_ve)
    for a, b in zip(rows["mixed"], rows["fp64"]):
        assert a["time_iter"] == b["time_iter"]
        if b["has_energy"]:
            assert abs(a["energy"] - b["energy"]) <= 1e-6 * abs(b["energy"])
            assert abs(a["plaq_su2"] - b["plaq_su2"]) <= 1e-6


def test_thousand_step_precision_at_256():
    """The mixed form's error budget over 1000 steps at SM 256^3 (analysers every 10)."""
    p, ic = _bench_workload("sm", 256)
    rows, d_sc, d_ve = _mixed_and_fp64(p, ic, 1000)
    e32 = [r["energy"] for r in rows["mixed"] if r["has_energy"]]
    e64 = [r["energy"] for r in rows["fp64"] if r["has_energy"]]
    assert len(e32) == len(e64) == 100
    rel = max(abs(a - b) / abs(b) for a, b in zip(e32, e64))
    assert rel <= 1e-6, rel
    g32 = max(max(r["gauss_max"]) for r in rows["mixed"] if r["has_gauss"])
    g64 = max(max(r["gauss_max"]) for r in rows["fp64"] if r["has_gauss"])
    assert g64 <= 1e-12, g64
    assert g32 <= 1e-5, g32
    assert d_sc <= 1e-3 and d_ve <= 1e-3, (d_sc, d_ve)


# ---------------------------------------------------------------------------
# small lattices: whole logging periods replayed from a CUDA graph
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("form,shape,every,steps,kind", [
    ("fp64", (32, 32, 32), (10, 10), 47, 0),    # configuration 1; a tail shorter than a period
    ("mixed", (8, 8, 32), (3, 2), 20, 2),       # tiled kernel, period lcm(2, 3, 2) = 6
    ("mixed", (8, 8, 32), (3, 2), 20, 0),       # the automatic choice: one thread per site here
    ("ref32", (6, 5, 4), (2, 3), 13, 0),        # reference arithmetic, odd shape
])
def test_graph_replay_equals_direct_launches(form, shape, every, steps, kind):
    from gftevolver_b200 import Evolver, InitialData, LatticeParams
    nx, ny, nz = shape
    p = LatticeParams(nx=nx, ny=ny, nz=nz, energy_every=every[0], gauss_every=every[1])
    ic = InitialData(seed=5, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    out = []
    for graphs in (True, False):
        with Evolver(p, form=form) as ev:
            ev.set_graphs(graphs)
            if kind:
                ev.set_kernel(kind, 0, 32)
            ev.init_fields(ic)
            l0 = ev.launch_count
            rows = ev.evolve(5)          # starts off a period boundary, then whole periods and a tail
            rows += ev.evolve(steps)
            launches = ev.launch_count - l0
            assert ev.time_iter == 5 + steps
            out.append((ev.download(), rows, launches))
    (a, ra, la), (b, rb, lb) = out
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert la == lb
    assert [r["time_iter"] for r in ra] == [r["time_iter"] for r in rb]
    for x, y in zip(ra, rb):
        for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric", "plaq_su2", "plaq_u1",
                  "phi_sq"):
            assert x[k] == y[k], k
        assert x["gauss_max"] == y["gauss_max"] and x["gauss_int"] == y["gauss_int"]


def test_graph_replay_across_damping_and_a_kernel_switch():
    """Damped steps launch one by one and the graph takes over after them; switching the
    kernel mid-run drops the captured period and the next one is captured afresh."""
    from gftevolver_b200 import Evolver, InitialData, LatticeParams
    p = LatticeParams(nx=8, ny=8, nz=32, energy_every=4, gauss_every=2, damping=1.0, nt_damped=7)
    ic = InitialData(seed=6, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    out = []
    for graphs in (True, False):
        with Evolver(p, form="mixed") as ev:
            ev.set_graphs(graphs)
            ev.set_kernel(2, 0, 32)         # the staged step first
            ev.init_fields(ic)
            rows = ev.evolve(13)           # damped 0..6, then whole periods of 4
            ev.set_kernel(1, 0, 32)         # one thread per site from here on
            rows += ev.evolve(9)
            out.append((ev.download(), rows))
    (a, ra), (b, rb) = out
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert [r["time_iter"] for r in ra] == [r["time_iter"] for r in rb]
    assert [r["energy"] for r in ra] == [r["energy"] for r in rb]
    assert [r["gauss_max"] for r in ra] == [r["gauss_max"] for r in rb]
