"""x-slabs on the GPU: ghost planes, interior-only observables, exchange after
every step (gftevolver_b200.slab over gft_set_slab / gft_set_exchange /
gft_level_planes).

One GPU is available, so multi-rank runs are emulated in one process: (1) one
slab that is the whole lattice, its ghosts refreshed by the library's exchange
callback (the lattice is periodic onto itself); (2) two slabs on the same GPU
stepped alternately, ghosts copied between them after each step.  The
interior equals the whole-lattice evolution: bit for bit in the FP64 form
(the one-thread-per-site kernel reads the same neighbour values), within the
tiled-kernel contraction bound (2e-6 after 7 steps) in the mixed form, whose
x-chunks start at different planes.  Observables over the own planes equal the
whole lattice's to 1e-12 relative (FP64; summation order differs) -- 1e-6 for
the mixed form.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(model=1, shape=(12, 8, 32), every=(2, 3)):
    from gftevolver_b200 import LatticeParams
    nx, ny, nz = shape
    return LatticeParams(model=model, nx=nx, ny=ny, nz=nz, energy_every=every[0], gauss_every=every[1])


IC = dict(seed=23, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)


def _rows_close(a, b, tol):
    assert [r["time_iter"] for r in a] == [r["time_iter"] for r in b]
    for x, y in zip(a, b):
        for k in ("energy", "potential", "gradient", "kinetic", "magnetic", "electric", "plaq_su2", "plaq_u1",
                  "phi_sq"):
            assert abs(x[k] - y[k]) <= tol * max(abs(y[k]), 1e-300), (k, x[k], y[k])


@pytest.mark.parametrize("form,ftol,rtol", [("fp64", 0.0, 1e-12), ("mixed", 2e-6, 1e-6)])
@pytest.mark.parametrize("model", [1, 2])
def test_single_slab_equals_whole_lattice(form, ftol, rtol, model):
    from gftevolver_b200 import Evolver, InitialData
    from gftevolver_b200.slab import SlabEvolver
    p = _params(model)
    ic = InitialData(**IC)
    with Evolver(p, form=form) as ev:
        ev.init_fields(ic)
        g0 = ev.download()
        g_rows = ev.evolve(7)
        g_sc, g_ve = ev.download()
    slab = SlabEvolver(p, form=form)
    try:
        slab.init_fields(ic)
        s0 = slab.download_own()
        assert np.array_equal(s0[0], g0[0]) and np.array_equal(s0[1], g0[1])  # global random keys
        rows = slab.evolve(7)
        s_sc, s_ve = slab.download_own()
    finally:
        slab.close()
    assert np.max(np.abs(s_sc - g_sc)) <= ftol and np.max(np.abs(s_ve - g_ve)) <= ftol
    _rows_close(rows, g_rows, rtol)
    if form == "fp64":  # Gauss residual over the own planes only, after the ghost refresh
        for a, b in zip(rows, g_rows):
            if b["has_gauss"]:
                assert np.allclose(a["gauss_max"], b["gauss_max"], rtol=1e-12, atol=1e-300)
                assert np.allclose(a["gauss_int"], b["gauss_int"], rtol=1e-12, atol=1e-300)


def test_two_slabs_on_one_gpu_equal_whole_lattice():
    import torch

    from gftevolver_b200 import Evolver, InitialData
    from gftevolver_b200.slab import SlabEvolver
    p = _params(1, (10, 8, 32), every=(2, 0))  # Gauss off: its ghosts are refreshed only between calls here
    ic = InitialData(**IC)
    with Evolver(p, form="fp64") as ev:
        ev.init_fields(ic)
        g_rows = ev.evolve(6)
        g_sc, g_ve = ev.download()
    a = SlabEvolver(p, form="fp64", rank=0, world=2, auto_exchange=False)
    b = SlabEvolver(p, form="fp64", rank=1, world=2, auto_exchange=False)
    try:
        for s in (a, b):
            s.init_fields(ic)
        rows_a, rows_b = [], []
        for t in range(6):
            rows_a += a.evolve(1)
            rows_b += b.evolve(1)
            lvl = t % 2  # the level step t wrote
            for d, s_ in zip(a.planes(lvl, 0), b.planes(lvl, b.nloc)):
                d.copy_(s_)
            for d, s_ in zip(a.planes(lvl, a.nloc + 1), b.planes(lvl, 1)):
                d.copy_(s_)
            for d, s_ in zip(b.planes(lvl, 0), a.planes(lvl, a.nloc)):
                d.copy_(s_)
            for d, s_ in zip(b.planes(lvl, b.nloc + 1), a.planes(lvl, 1)):
                d.copy_(s_)
            torch.cuda.synchronize()
        sa, va = a.download_own()
        sb, vb = b.download_own()
    finally:
        a.close()
        b.close()
    assert np.array_equal(np.concatenate([sa, sb], axis=1), g_sc)
    assert np.array_equal(np.concatenate([va, vb], axis=1), g_ve)
    for ra, rb, rg in zip(rows_a, rows_b, g_rows):
        assert abs(ra["energy"] + rb["energy"] - rg["energy"]) <= 1e-12 * abs(rg["energy"])
        plaq = (ra["plaq_su2"] * a.own_sites + rb["plaq_su2"] * b.own_sites) / (a.own_sites + b.own_sites)
        assert abs(plaq - rg["plaq_su2"]) <= 1e-12


@pytest.mark.parametrize("form,kind,ftol,rtol", [
    ("fp64", 0, 0.0, 1e-12),     # one thread per site: exchange after each whole step, bit for bit
    ("mixed", 2, 2e-6, 1e-6),    # tiled: boundary planes, exchange overlapped with the interior planes
    ("mixed", 3, 2e-6, 1e-6),    # tiled, two sites per thread on plain steps
])
def test_library_exchange_over_nccl_equals_whole_lattice(form, kind, ftol, rtol):
    """exchange='library': gft_evolve posts the ghost-plane exchange over NCCL itself (here one rank,
    which sends its boundary planes to itself).  The slab equals the whole lattice as with the
    callback exchange; in the tiled kernels the x-chunks start at other planes (contraction bound)."""
    from gftevolver_b200 import Evolver, InitialData
    from gftevolver_b200.slab import SlabEvolver
    p = _params(1, (12, 8, 32), every=(3, 3))
    ic = InitialData(**IC)
    with Evolver(p, form=form) as ev:
        ev.init_fields(ic)
        g_rows = ev.evolve(8)
        g_sc, g_ve = ev.download()
    slab = SlabEvolver(p, form=form, exchange="library")
    try:
        if kind:  # march 4: boundary chunks of 4 planes at each end, 4 interior planes
            slab.local.set_kernel(kind, 0, 4)
        slab.init_fields(ic)
        l0 = slab.local.launch_count
        rows = slab.evolve(8)
        launches = slab.local.launch_count - l0
        s_sc, s_ve = slab.download_own()
    finally:
        slab.close()
    assert np.max(np.abs(s_sc - g_sc)) <= ftol and np.max(np.abs(s_ve - g_ve)) <= ftol
    _rows_close(rows, g_rows, rtol)
    if kind:  # the plain steps were split into boundary and interior launches
        with Evolver(p, form=form) as ev:
            ev.set_kernel(kind, 0, 4)
            ev.init_fields(ic)
            l1 = ev.launch_count
            ev.evolve(8)
            whole = ev.launch_count - l1
        assert launches == whole + 2 * 5  # 5 plain steps of 8 (logging every 3), two more launches each
