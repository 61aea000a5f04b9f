"""The split-site tiled step (kernel kind 4): each site's update divided between a
links thread and a scalars thread (GPU).

On plain steps the links thread computes the SU(2) staple sums and the SU(2) link
update, the scalars thread everything else and hands it the link momentum and the
currents through shared memory; logging steps run the one-site tiled kernel.  The
arithmetic is the one-site step's expression by expression, so the two agree to
contraction-level rounding: 2 float ulps of the field scale (2.4e-7) after one
step, 2e-6 after 7 steps, and both within the mixed form's 6e-6 of the FP64 oracle
after 10 steps.  Cases: tiles that all wrap, interior tiles, march lengths that
do not divide nx, a march of one plane, and an x-slab exchanging over NCCL.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ic(seed):
    return dict(seed=seed, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)


def _run(p, ic, nt, kind, march, tile=0):
    from gftevolver_b200 import Evolver, InitialData
    with Evolver(p, form="mixed") as ev:
        ev.set_kernel(kind, tile, march)
        ev.init_fields(InitialData(**ic))
        rows = ev.evolve(nt)
        assert ev.last_warnings == 0
        name = ev.step_kernel_name
        sc, ve = ev.download()
    return sc, ve, rows, name


@pytest.mark.parametrize("shape,march", [
    ((8, 8, 32), 32),       # every halo wraps
    ((10, 24, 96), 4),      # interior 8 x 16 tiles
    ((12, 16, 64), 5),      # march does not divide nx
    ((3, 8, 16), 1),        # march 1, one tile per plane
    ((6, 16, 48), 32),      # march longer than nx
])
def test_split_step_matches_one_site_step_and_oracle(oracle_mod, shape, march):
    from gftevolver_b200 import LatticeParams
    nx, ny, nz = shape
    op = oracle_mod.Params(model=oracle_mod.MODEL_SM, nx=nx, ny=ny, nz=nz, energy_every=4, gauss_every=4)
    p = LatticeParams(**op.__dict__)
    ic = _ic(93)
    tile = 0 if nz % 32 == 0 else 2  # the logging steps' one-site tile
    a1 = _run(p, ic, 1, 2, march, tile)
    b1 = _run(p, ic, 1, 4, march, tile)
    assert b1[3] == "tiled_split_kernel"
    assert np.max(np.abs(a1[0] - b1[0])) <= 2.4e-7 and np.max(np.abs(a1[1] - b1[1])) <= 2.4e-7
    a7 = _run(p, ic, 7, 2, march, tile)
    b7 = _run(p, ic, 7, 4, march, tile)
    assert np.max(np.abs(a7[0] - b7[0])) <= 2e-6 and np.max(np.abs(a7[1] - b7[1])) <= 2e-6
    for ra, rb in zip(a7[2], b7[2]):
        assert ra["time_iter"] == rb["time_iter"]
        for k in ("energy", "magnetic", "electric", "kinetic", "plaq_su2", "plaq_u1", "phi_sq"):
            assert abs(ra[k] - rb[k]) <= 1e-6 * max(1.0, abs(ra[k])), k
    b10 = _run(p, ic, 10, 4, march, tile)
    o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**ic), np.float64)
    oracle_mod.evolve(op, o_sc, o_ve, 10)
    assert np.max(np.abs(b10[0].astype(np.float64) - o_sc)) <= 6e-6
    assert np.max(np.abs(b10[1].astype(np.float64) - o_ve)) <= 6e-6


def test_split_step_is_refused_where_not_built():
    from gftevolver_b200 import Evolver, GftError, LatticeParams
    for c in (dict(model=2, nx=4, ny=8, nz=32), dict(model=1, nx=4, ny=8, nz=32, fixed_axes=2),
              dict(model=1, nx=4, ny=12, nz=32)):
        with Evolver(LatticeParams(**c), form="mixed") as ev:
            with pytest.raises(GftError):
                ev.set_kernel(4, 0 if c["ny"] % 8 == 0 else 1, 8)
