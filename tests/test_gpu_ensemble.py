"""Ensembles (gft_batch_*): one persistent launch per step over the tiles of
every member, logging periods replayed from a CUDA graph, autotuned tiles (GPU).

Every member must evolve as a single handle does with the same tile shape and
march depth (gft_set_kernel(kind=2, tile, march)): the per-site arithmetic is
the same code (run_tile of gft_tiled_tile.cuh).  The two kernels are separate
instantiations, so the compiler may contract multiply-adds differently (the
2HDM logging variant also spills differently): after one step the fields agree
to 2 float ulps of the field scale, and such differences are integrated like
storage rounding, so after 7 steps the bound is the tiled-kernel test's 2e-6
absolute; energies agree to 1e-7 relative and the Gauss residuals (FP32
storage noise themselves) to 1e-10 per site on average.  Graph replay versus direct
launches runs the same kernels with the same parameters: bit-identical.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _members(oracle_mod, model, shapes, every=(2, 3)):
    from gftevolver_b200 import LatticeParams
    ps, ics = [], []
    for k, (nx, ny, nz) in enumerate(shapes):
        op = oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, energy_every=every[0], gauss_every=every[1])
        ps.append(LatticeParams(**op.__dict__))
        ics.append(dict(seed=100 + k, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                        eps_sigma=0.1))
    return ps, ics


def _single(p, ic, nt, tile, march):
    from gftevolver_b200 import Evolver, InitialData
    with Evolver(p, form="mixed") as ev:
        ev.set_kernel(2, tile, march)
        ev.init_fields(InitialData(**ic))
        rows = ev.evolve(nt)
        sc, ve = ev.download()
    return sc, ve, rows


def _compare_rows(ra, rb, nsite, tol=1e-7):
    assert [r["time_iter"] for r in ra] == [r["time_iter"] for r in rb]
    for a, b in zip(ra, rb):
        for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric", "plaq_su2", "plaq_u1",
                  "phi_sq"):
            assert abs(a[k] - b[k]) <= tol * max(abs(b[k]), 1e-30), (k, a[k], b[k])
        # the mixed form's Gauss residual is itself FP32 storage noise, so two evolutions that
        # differ at the contraction level differ in it by that noise: bound the difference per
        # site (1e-10 averaged, 1e-8 at the worst site; dV = 1) rather than relative to it
        for k in range(4):
            assert abs(a["gauss_max"][k] - b["gauss_max"][k]) <= 1e-8
            assert abs(a["gauss_int"][k] - b["gauss_int"][k]) <= 1e-10 * nsite


@pytest.mark.parametrize("model,shapes", [
    (1, [(16, 8, 16), (8, 12, 32), (24, 4, 16)]),
    (2, [(8, 8, 16), (12, 4, 32)]),
    (1, [(32, 16, 48), (8, 32, 16)]),   # 16 x 16 tiles
])
def test_members_evolve_like_single_handles(oracle_mod, model, shapes):
    from gftevolver_b200 import Ensemble, InitialData
    ps, ics = _members(oracle_mod, model, shapes)
    nt = 7
    tile = 3 if all(p.ny % 16 == 0 and p.nz % 16 == 0 for p in ps) else 2
    with Ensemble(ps) as ens:
        ens.set_kernel(tile, 8)
        ens.init_fields([InitialData(**ic) for ic in ics])
        rows = ens.evolve(nt)
        assert ens.time_iter == nt
        out = [ens.download(m) for m in range(len(ps))]
    for m, (p, ic) in enumerate(zip(ps, ics)):
        sc, ve, r1 = _single(p, ic, nt, tile, 8)
        assert np.max(np.abs(out[m][0] - sc)) <= 2e-6
        assert np.max(np.abs(out[m][1] - ve)) <= 2e-6
        _compare_rows(rows[m], r1, p.nsite)


def test_two_launch_groups_and_uneven_chunks_evolve_like_single_handles(oracle_mod):
    """70 members: two launch groups (64 members' parameters per launch), each with its own
    per-CTA tile lists; x-lengths 8, 12 and 20 at march 8 give chunks of 8 and 4 planes, so
    the lists deal tiles of unequal cost.  Members on both sides of the group boundary evolve
    as single handles do."""
    from gftevolver_b200 import Ensemble, InitialData
    shapes = [((8, 12, 20)[k % 3], 8, 16) for k in range(70)]
    ps, ics = _members(oracle_mod, 1, shapes, every=(3, 3))
    nt = 5
    with Ensemble(ps) as ens:
        ens.set_kernel(2, 8)
        ens.init_fields([InitialData(**ic) for ic in ics])
        rows = ens.evolve(nt)
        out = {m: ens.download(m) for m in (0, 1, 62, 63, 64, 65, 69)}
    assert all(np.isfinite(r["energy"]) for mr in rows for r in mr if r["has_energy"])
    for m, (sc_e, ve_e) in out.items():
        sc, ve, r1 = _single(ps[m], ics[m], nt, 2, 8)
        assert np.max(np.abs(sc_e - sc)) <= 2e-6, m
        assert np.max(np.abs(ve_e - ve)) <= 2e-6, m
        _compare_rows(rows[m], r1, ps[m].nsite)


def test_march_longer_than_every_member(oracle_mod):
    """A march of 64 planes over members 8 and 12 planes long: every tile is one whole
    member chunk, and the Gauss pass keeps one partial row per plane of the longest member."""
    from gftevolver_b200 import Ensemble, InitialData
    ps, ics = _members(oracle_mod, 1, [(8, 8, 16), (12, 8, 32)], every=(2, 2))
    nt = 5
    with Ensemble(ps) as ens:
        ens.set_kernel(2, 64)
        ens.init_fields([InitialData(**ic) for ic in ics])
        rows = ens.evolve(nt)
        out = [ens.download(m) for m in range(len(ps))]
    for m, (p, ic) in enumerate(zip(ps, ics)):
        sc, ve, r1 = _single(p, ic, nt, 2, 64)
        assert np.max(np.abs(out[m][0] - sc)) <= 2e-6
        assert np.max(np.abs(out[m][1] - ve)) <= 2e-6
        _compare_rows(rows[m], r1, p.nsite)


def test_graph_replay_equals_direct_launches(oracle_mod):
    from gftevolver_b200 import Ensemble, InitialData
    ps, ics = _members(oracle_mod, 1, [(16, 8, 16), (32, 16, 32), (8, 4, 16)], every=(2, 2))
    res = []
    for graphs in (True, False):
        with Ensemble(ps) as ens:
            ens.set_kernel(2, 16, use_graphs=graphs)
            ens.init_fields([InitialData(**ic) for ic in ics])
            r1, r2 = ens.evolve(4), ens.evolve(9)  # periods of 2 steps, then a ragged tail
            rows = [a + b for a, b in zip(r1, r2)]
            res.append((rows, [ens.download(m) for m in range(len(ps))]))
    (ra, fa), (rb, fb) = res
    assert ra == rb
    for (a_sc, a_ve), (b_sc, b_ve) in zip(fa, fb):
        assert np.array_equal(a_sc, b_sc) and np.array_equal(a_ve, b_ve)


def test_member_within_mixed_bound_of_oracle(oracle_mod):
    from gftevolver_b200 import Ensemble
    op = oracle_mod.Params(nx=12, ny=8, nz=16, energy_every=5, gauss_every=5)
    ic = oracle_mod.ICSpec(seed=5, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float64)
    from gftevolver_b200 import LatticeParams
    other = LatticeParams(nx=16, ny=4, nz=32, energy_every=5, gauss_every=5)
    with Ensemble([LatticeParams(**op.__dict__), other]) as ens:
        ens.upload(0, sc, ve, 0)
        ens.upload(1, *_random_fields(other), 0)
        ens.evolve(10)
        g_sc, g_ve = ens.download(0)
    o_sc, o_ve = sc.copy(), ve.copy()
    oracle_mod.evolve(op, o_sc, o_ve, 10)
    assert np.max(np.abs(g_sc - o_sc)) <= 6e-6
    assert np.max(np.abs(g_ve - o_ve)) <= 6e-6


def _random_fields(p):
    rng = np.random.default_rng(1)
    sc = (1.0 + 0.1 * rng.standard_normal((2, p.nx, p.ny, p.nz, p.nsc))).astype(np.float32)
    ve = np.zeros((2, p.nx, p.ny, p.nz, 15), np.float32)
    ve[..., 1::5] = 1.0  # identity links, theta = 0
    return sc, ve


def test_autotune_restores_fields_and_counter(oracle_mod):
    from gftevolver_b200 import Ensemble, InitialData
    ps, ics = _members(oracle_mod, 1, [(32, 8, 32), (16, 16, 32)])
    with Ensemble(ps) as ens:
        ens.init_fields([InitialData(**ic) for ic in ics])
        ens.evolve(3)
        before = [ens.download(m) for m in range(len(ps))]
        tile, march = ens.autotune(2)
        assert tile in (0, 1, 2, 3) and march in (8, 16, 32, 64)
        assert ens.time_iter == 3
        after = [ens.download(m) for m in range(len(ps))]
        for (a, b), (c, d) in zip(before, after):
            assert np.array_equal(a, c) and np.array_equal(b, d)
        rows = ens.evolve(4)
        assert [r["time_iter"] for r in rows[0]] == [3, 4, 6]  # gauss every 3, energy every 2


def test_device_initial_data_per_member_matches_evolver(oracle_mod):
    from gftevolver_b200 import Ensemble, Evolver, InitialData
    ps, ics = _members(oracle_mod, 2, [(8, 4, 16), (4, 8, 32)])
    with Ensemble(ps) as ens:
        ens.init_fields([InitialData(**ic) for ic in ics])
        got = [ens.download(m) for m in range(len(ps))]
    for m, (p, ic) in enumerate(zip(ps, ics)):
        with Evolver(p, form="mixed") as ev:
            ev.init_fields(InitialData(**ic))
            sc, ve = ev.download()
        assert np.array_equal(got[m][0], sc) and np.array_equal(got[m][1], ve)


def test_member_with_fixed_faces_evolves_like_a_single_handle(oracle_mod):
    """A member with Fixed y faces (frozen shell) next to a periodic one."""
    import dataclasses

    from gftevolver_b200 import Ensemble, InitialData
    ps, ics = _members(oracle_mod, 1, [(16, 16, 32), (8, 16, 16)])
    ps[1] = dataclasses.replace(ps[1], fixed_axes=2)
    with Ensemble(ps) as ens:
        ens.set_kernel(3, 8)
        ens.init_fields([InitialData(**ic) for ic in ics])
        rows = ens.evolve(7)
        out = [ens.download(m) for m in range(len(ps))]
    for m, (p, ic) in enumerate(zip(ps, ics)):
        sc, ve, r1 = _single(p, ic, 7, 3, 8)
        assert np.max(np.abs(out[m][0] - sc)) <= 2e-6 and np.max(np.abs(out[m][1] - ve)) <= 2e-6
        _compare_rows(rows[m], r1, p.nsite)
    # the frozen shell kept its initial values
    with Ensemble(ps[1:]) as one:
        one.init_fields([InitialData(**ics[1])])
        init = one.download(0)
    assert np.array_equal(out[1][0][:, :, 0], init[0][:, :, 0]) and np.array_equal(out[1][1][:, :, -1], init[1][:, :, -1])


def test_sharded_ensemble_halves_match_the_whole(oracle_mod):
    """Two round-robin shards (ranks 0 and 1 of 2, run one after the other on one GPU)
    evolve their members exactly as the whole ensemble does: same kernel instance,
    same tile and march, each member's tiles and reductions independent of the others."""
    from gftevolver_b200 import Ensemble, InitialData, ShardedEnsemble
    ps, ics = _members(oracle_mod, 1, [(16, 8, 16), (8, 12, 32), (24, 4, 16), (8, 8, 32), (16, 16, 16)])
    ics = [InitialData(**ic) for ic in ics]
    with Ensemble(ps) as whole:
        whole.set_kernel(2, 8)
        whole.init_fields(ics)
        w_rows = whole.evolve(6)
        w_fields = [whole.download(m) for m in range(len(ps))]
    got_rows = [None] * len(ps)
    for rank in range(2):
        with ShardedEnsemble(ps, rank=rank, world=2) as se:
            assert se.members == list(range(rank, len(ps), 2))
            se.local.set_kernel(2, 8)
            se.init_fields(ics)
            rows = se.evolve(6)
            for k, m in enumerate(se.members):
                got_rows[m] = rows[k]
                sc, ve = se.local.download(k)
                assert np.array_equal(sc, w_fields[m][0]) and np.array_equal(ve, w_fields[m][1])
    assert got_rows == w_rows


@pytest.mark.parametrize("hf", [1, 2], ids=["family_u1", "family_su2"])
def test_higgs_family_members_evolve_like_single_handles(oracle_mod, hf):
    """2HDM members with a Higgs-family field (gaugeNum 5 / 7): the ensemble takes the
    single handle's one-thread-per-site launches member after member, so every member
    equals a single handle bit for bit, analyser rows included (gaugeNum Gauss
    constraints), in lattices of any shape; replaying logging periods from a graph
    changes nothing; there is no tile shape to tune."""
    from gftevolver_b200 import Ensemble, Evolver, InitialData, LatticeParams
    shapes = [(8, 6, 10), (5, 8, 16), (12, 4, 7)]
    ps, ics = [], []
    for k, (nx, ny, nz) in enumerate(shapes):
        op = oracle_mod.Params(model=2, nx=nx, ny=ny, nz=nz, energy_every=2, gauss_every=3, higgs_family=hf,
                               gpp=0.47)
        ps.append(LatticeParams(**op.__dict__))
        ics.append(dict(seed=700 + k, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1))
    nt = 7
    res = []
    for graphs in (True, False):
        with Ensemble(ps) as ens:
            ens.set_kernel(0, 8, use_graphs=graphs)
            ens.init_fields([InitialData(**ic) for ic in ics])
            rows = ens.evolve(nt)
            res.append((rows, [ens.download(m) for m in range(len(ps))]))
            if graphs:
                with pytest.raises(Exception):
                    ens.autotune(2)
    (ra, fa), (rb, fb) = res
    assert ra == rb
    for (a_sc, a_ve), (b_sc, b_ve) in zip(fa, fb):
        assert np.array_equal(a_sc, b_sc) and np.array_equal(a_ve, b_ve)
    neq = 5 if hf == 1 else 7
    for m, (p, ic) in enumerate(zip(ps, ics)):
        with Evolver(p, form="mixed") as ev:
            ev.init_fields(InitialData(**ic))
            r1 = ev.evolve(nt)
            sc, ve = ev.download()
        assert fa[m][1].shape[-1] == (18 if hf == 1 else 27)
        assert np.array_equal(fa[m][0], sc) and np.array_equal(fa[m][1], ve), m
        assert ra[m] == r1, m
        assert all(len(r["gauss_max"]) == neq for r in r1 if r["has_gauss"])
