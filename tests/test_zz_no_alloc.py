"""gft_observe_static: the allocation-free observables entry point (GPU).

Some callers cannot allocate device memory where they need the observables
(a memory budget fixed up front, a region that must stay asynchronous since
cudaMalloc/cudaFree synchronise the device, or fields owned by another
framework's allocator).  gft_observe_static computes the same numbers as the
handle-based gft_observe from the caller's own device buffers, using a fixed
scratch array compiled into the library.  This file is collected last so that
a stopped run has already exercised everything else; it passes both alone in
a fresh process and after the other tests.

Tolerance: the mixed-form energies agree to 1e-6 relative (the tolerance the
other mixed-form tests use), plaquette means and <phi^dag phi> to 1e-7.
"""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# 2HDM couplings beyond the default: the U(N/2)-breaking terms and the energy offset
COUPLED_2HDM = dict(m12i=0.03, l5i=0.02, l6i=-0.015, l7i=0.01, l6r=0.012, l7r=-0.008, apply_norm=1,
                    energy_offset=0.37)


def _state(model, shape, steps, extra=None):
    from gftevolver_b200 import Evolver, InitialData, LatticeParams
    nx, ny, nz = shape
    p = LatticeParams(model=model, nx=nx, ny=ny, nz=nz, energy_every=1, **(extra or {}))
    ic = InitialData(seed=4242, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                     eps_sigma=0.1)
    with Evolver(p, form="mixed") as ev:
        ev.init_fields(ic)
        ev.evolve(steps)  # nonzero electric field and scalar velocity
        ref = ev.observe()
        sc, ve = ev.download(np.float32)
        ti = ev.time_iter
    return p, ref, sc, ve, ti


KEYS = ("energy", "potential", "gradient", "kinetic", "magnetic", "electric", "plaq_su2", "plaq_u1", "phi_sq")


@pytest.mark.parametrize("model,shape,extra", [(1, (24, 16, 32), None), (2, (12, 10, 18), None),
                                               (2, (10, 12, 14), COUPLED_2HDM),
                                               (2, (10, 12, 16), dict(higgs_family=1, gpp=0.45)),
                                               (2, (12, 10, 14), dict(higgs_family=2, gpp=0.55))],
                         ids=["sm", "2hdm", "2hdm_coupled", "2hdm_family_u1", "2hdm_family_su2"])
def test_observe_static_matches_observe_twice(model, shape, extra):
    import torch
    from gftevolver_b200 import _lib
    from gftevolver_b200.evolver import make_config
    lib = _lib.load()
    p, ref, sc, ve, ti = _state(model, shape, 3, extra)
    cfg = make_config(p, "mixed", 0)
    d_sc = torch.from_numpy(sc).cuda()
    d_ve = torch.from_numpy(ve).cuda()
    out = torch.empty(9, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share the scratch array
        out.fill_(float("nan"))
        rc = lib.gft_observe_static(ctypes.byref(cfg), ctypes.c_void_p(d_sc.data_ptr()),
                                    ctypes.c_void_p(d_ve.data_ptr()), ti, ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_void_p(stream))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = dict(zip(KEYS, out.cpu().tolist()))
        for k in KEYS[:6]:
            assert math.isfinite(got[k])
            assert abs(got[k] - ref[k]) <= 1e-6 * max(abs(ref["energy"]), 1.0), (k, got[k], ref[k])
        for k in KEYS[6:]:
            assert abs(got[k] - ref[k]) <= 1e-7 * max(abs(ref[k]), 1.0), (k, got[k], ref[k])


def test_observe_static_rejects_lattices_beyond_its_scratch():
    from gftevolver_b200 import LatticeParams, _lib
    from gftevolver_b200.evolver import make_config
    lib = _lib.load()
    cfg = make_config(LatticeParams(nx=448, ny=448, nz=448), "mixed", 0)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.gft_observe_static(ctypes.byref(cfg), dummy, dummy, 0, dummy, None)
    assert rc == _lib.GFT_E_UNSUPPORTED
    assert "67108864" in _lib.last_error()


def test_observe_static_rejects_an_invalid_configuration_with_a_message():
    import dataclasses

    from gftevolver_b200 import LatticeParams, _lib
    from gftevolver_b200.evolver import make_config
    lib = _lib.load()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the configuration check comes first
    for bad in (dict(dx=0.0), dict(dt=float("nan")), dict(nx=0)):
        cfg = make_config(dataclasses.replace(LatticeParams(nx=8, ny=8, nz=8), **bad), "mixed", 0)
        rc = lib.gft_observe_static(ctypes.byref(cfg), dummy, dummy, 0, dummy, None)
        assert rc == _lib.GFT_E_INVALID, bad
        assert _lib.last_error().startswith("gft_observe_static: "), _lib.last_error()


def test_observe_static_is_captured_and_replayed_in_a_cuda_graph():
    """The property the entry point exists for: after one call outside any capture
    (which loads the library's module and looks up its scratch array), a call is
    captured in a CUDA graph in global capture mode -- where any device allocation,
    by this thread or another, fails the capture -- and its replay gives the same
    numbers bit for bit."""
    import torch
    from gftevolver_b200 import _lib
    from gftevolver_b200.evolver import make_config
    lib = _lib.load()
    p, ref, sc, ve, ti = _state(1, (16, 12, 32), 2)
    cfg = make_config(p, "mixed", 0)
    d_sc = torch.from_numpy(sc).cuda()
    d_ve = torch.from_numpy(ve).cuda()
    out = torch.empty(9, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()

    def call(stream):
        return lib.gft_observe_static(ctypes.byref(cfg), ctypes.c_void_p(d_sc.data_ptr()),
                                      ctypes.c_void_p(d_ve.data_ptr()), ti, ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(stream.cuda_stream))

    with torch.cuda.stream(side):
        assert call(side) == 0, _lib.last_error()
    torch.cuda.synchronize()
    first = out.clone()
    out.fill_(float("nan"))
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side, capture_error_mode="global"):
        rc = call(torch.cuda.current_stream())
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert torch.isnan(out).all()  # capturing ran nothing
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, first)
    assert abs(first[0].item() - ref["energy"]) <= 1e-6 * abs(ref["energy"])
    del graph
