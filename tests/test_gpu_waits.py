"""The tiled kernel's bounded waits: the error path runs, and nothing hangs (GPU).

Every wait of the TMA plane ring is bounded (2 s of %globaltimer).  A wait that
gives up makes the tile drain its copies still in flight (with the 2 s bound)
and return; the step then reports GFT_E_TIMEOUT.  Here the limit is shortened
to 1 ns with gft_set_wait_limit, which turns each plane wait into one
non-blocking test: it fails while the copies it waits for are still landing,
and the copies themselves complete, so the drain ends and no wait is left
unfinished.  After the error the handle is usable again: a re-upload and a
step with the default limit reproduce a fresh handle bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form,shape", [
    ("mixed", (16, 16, 64)),  # every tile wraps: one CTA barrier per plane
    ("fp64", (8, 24, 96)),    # an interior 8 x 32 tile: the FP64 march without per-plane barriers
])
def test_plane_wait_gives_up_and_the_handle_recovers(oracle_mod, form, shape):
    from gftevolver_b200 import Evolver, GftError, LatticeParams
    from gftevolver_b200 import _lib
    nx, ny, nz = shape
    op = oracle_mod.Params(model=oracle_mod.MODEL_SM, nx=nx, ny=ny, nz=nz, energy_every=2, gauss_every=2)
    p = LatticeParams(**op.__dict__)
    ic = oracle_mod.ICSpec(seed=77, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float64 if form == "fp64" else np.float32)
    with Evolver(p, form=form) as ev:
        ev.set_kernel(2, 0, 8)
        ev.set_wait_limit(1)
        ev.upload(sc, ve, 0)
        with pytest.raises(GftError) as err:
            ev.evolve(1)
        assert err.value.code == _lib.GFT_E_TIMEOUT
        # the default limit again: the next steps succeed from a fresh upload
        ev.set_wait_limit(0)
        ev.upload(sc, ve, 0)
        rows = ev.evolve(5)
        assert ev.last_warnings == 0
        a_sc, a_ve = ev.download()
    with Evolver(p, form=form) as ev:
        ev.set_kernel(2, 0, 8)
        ev.upload(sc, ve, 0)
        rows_ref = ev.evolve(5)
        b_sc, b_ve = ev.download()
    np.testing.assert_array_equal(a_sc, b_sc)
    np.testing.assert_array_equal(a_ve, b_ve)
    assert [r["energy"] for r in rows] == [r["energy"] for r in rows_ref]


def test_long_wait_limit_leaves_results_unchanged(oracle_mod):
    """A limit well above any copy's latency (10 ms) changes nothing: the waits succeed."""
    from gftevolver_b200 import Evolver, LatticeParams
    op = oracle_mod.Params(model=oracle_mod.MODEL_SM, nx=8, ny=16, nz=64, energy_every=3, gauss_every=3)
    p = LatticeParams(**op.__dict__)
    ic = oracle_mod.ICSpec(seed=78, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(op, ic, np.float32)
    out = []
    for limit in (0, 10_000_000):
        with Evolver(p, form="mixed") as ev:
            ev.set_kernel(2, 0, 8)
            ev.set_wait_limit(limit)
            ev.upload(sc, ve, 0)
            ev.evolve(4)
            out.append(ev.download())
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
