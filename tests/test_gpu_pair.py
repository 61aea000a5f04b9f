"""The two-sites-per-thread tiled step (kernel kind 3, paired FP32 arithmetic) (GPU).

On plain steps each thread evolves two sites of the tile (rows ty and
ty + TY/2) with Blackwell's paired FP32 instructions; logging steps run the
one-site tiled kernel.  Each half of a paired instruction rounds as the scalar
instruction does and the sums are formed in the same order, so the paired step
agrees with the one-site tiled step to contraction-level rounding: 2 float ulps
of the field scale (2.4e-7 absolute) after one step, 2e-6 after 7 steps (such
differences integrate like storage rounding), and both stay within the mixed
form's 6e-6 of the FP64 oracle after 10 steps.  Cases cover tiles that all
wrap, interior tiles, both tile shapes the kernel is built for, and march
lengths that do not divide nx.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ic(seed):
    return dict(seed=seed, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)


def _run(p, ic, nt, kind, tile, march):
    from gftevolver_b200 import Evolver, InitialData
    with Evolver(p, form="mixed") as ev:
        ev.set_kernel(kind, tile, march)
        ev.init_fields(InitialData(**ic))
        rows = ev.evolve(nt)
        assert ev.last_warnings == 0
        name = ev.step_kernel_name
        sc, ve = ev.download()
    return sc, ve, rows, name


@pytest.mark.parametrize("shape,tile,march", [
    ((8, 8, 32), 0, 32),      # one tile per plane: every halo wraps
    ((10, 24, 96), 0, 4),     # interior 8 x 32 tile
    ((12, 16, 64), 0, 5),     # march does not divide nx
    ((3, 8, 32), 0, 1),       # march 1
    ((6, 48, 48), 3, 4),      # interior 16 x 16 tile
    ((5, 16, 32), 3, 32),     # 16 x 16, march longer than nx
])
def test_pair_step_matches_one_site_step_and_oracle(oracle_mod, shape, tile, march):
    from gftevolver_b200 import LatticeParams
    nx, ny, nz = shape
    op = oracle_mod.Params(model=oracle_mod.MODEL_SM, nx=nx, ny=ny, nz=nz, energy_every=4, gauss_every=4)
    p = LatticeParams(**op.__dict__)
    ic = _ic(91)
    a1 = _run(p, ic, 1, 2, tile, march)
    b1 = _run(p, ic, 1, 3, tile, march)
    assert b1[3] == "tiled_pair_kernel"
    assert np.max(np.abs(a1[0] - b1[0])) <= 2.4e-7 and np.max(np.abs(a1[1] - b1[1])) <= 2.4e-7
    # step 0 logs (one-site kernel), steps 1-3 are paired plain steps, step 4 logs again, ...
    a7 = _run(p, ic, 7, 2, tile, march)
    b7 = _run(p, ic, 7, 3, tile, march)
    assert np.max(np.abs(a7[0] - b7[0])) <= 2e-6 and np.max(np.abs(a7[1] - b7[1])) <= 2e-6
    for ra, rb in zip(a7[2], b7[2]):
        assert ra["time_iter"] == rb["time_iter"]
        for k in ("energy", "magnetic", "electric", "kinetic", "plaq_su2", "plaq_u1", "phi_sq"):
            assert abs(ra[k] - rb[k]) <= 1e-6 * max(1.0, abs(ra[k])), k
    b10 = _run(p, ic, 10, 3, tile, march)
    o_sc, o_ve = oracle_mod.init_fields(op, oracle_mod.ICSpec(**ic), np.float64)
    oracle_mod.evolve(op, o_sc, o_ve, 10)
    assert np.max(np.abs(b10[0].astype(np.float64) - o_sc)) <= 6e-6
    assert np.max(np.abs(b10[1].astype(np.float64) - o_ve)) <= 6e-6


def test_pair_step_is_refused_where_not_built(oracle_mod):
    from gftevolver_b200 import Evolver, GftError, LatticeParams
    cases = [dict(model=2, nx=4, ny=8, nz=32),             # 2HDM
             dict(model=1, nx=4, ny=8, nz=32, fixed_axes=1),  # Fixed faces
             ]
    for c in cases:
        with Evolver(LatticeParams(**c), form="mixed") as ev:
            with pytest.raises(GftError):
                ev.set_kernel(3, 0, 8)
    with Evolver(LatticeParams(nx=4, ny=8, nz=32), form="mixed") as ev:
        with pytest.raises(GftError):
            ev.set_kernel(3, 1, 8)  # 4 x 32 tiles: not built with two sites per thread
