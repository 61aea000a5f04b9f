"""The C-ABI library: loads and exports every entry point include/gft.h declares (CPU only, no compute)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gft.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(gft_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from gftevolver_b200 import build
    build.build()
    from gftevolver_b200 import _lib
    return _lib.load()


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("gft_create", "gft_destroy", "gft_upload_f32", "gft_upload_f64", "gft_download_f32",
                     "gft_download_f64", "gft_evolve", "gft_observe", "gft_init_fields", "gft_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"symbols declared in include/gft.h but not exported: {missing}"


def test_binding_covers_every_declared_symbol():
    from gftevolver_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_struct_layouts_match_header():
    """ctypes mirrors of the header structs have the sizes the C compiler gives them."""
    import subprocess
    import tempfile
    from gftevolver_b200 import _lib
    prog = r'''
#include <stdio.h>
#include "gft.h"
int main(void){printf("%zu %zu %zu\n", sizeof(gft_config), sizeof(gft_observables), sizeof(gft_ic));return 0;}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        exe = os.path.join(d, "s")
        open(c, "w").write(prog)
        subprocess.check_call(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe])
        sizes = [int(v) for v in subprocess.check_output([exe]).split()]
    assert sizes == [ctypes.sizeof(_lib.GftConfig), ctypes.sizeof(_lib.GftObservables), ctypes.sizeof(_lib.GftIC)]


def test_create_rejects_invalid_config_without_gpu(lib):
    """Argument validation happens before any device call (reference: std::runtime_error at construction)."""
    from gftevolver_b200 import _lib
    cfg = _lib.GftConfig()
    cfg.model = 5
    cfg.nx = cfg.ny = cfg.nz = 4
    cfg.dx = cfg.dy = cfg.dz = 1.0
    cfg.dt = 0.05
    h = ctypes.c_void_p()
    assert lib.gft_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.GFT_E_UNSUPPORTED
    assert b"model" in lib.gft_last_error(None)
    cfg.model = 1
    cfg.nx = 0
    assert lib.gft_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.GFT_E_INVALID
    # a Higgs-family gauge field exists in the 2HDM only (WilsonLoops::TwoHDM); 0..2
    cfg.nx = 4
    cfg.form = _lib.GFT_FORM_MIXED
    cfg.higgs_family = _lib.GFT_HF_U1
    assert lib.gft_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.GFT_E_INVALID
    assert b"2HDM" in lib.gft_last_error(None)
    cfg.model = _lib.GFT_MODEL_2HDM
    cfg.higgs_family = 3
    assert lib.gft_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.GFT_E_INVALID
    cfg.higgs_family = 0
    cfg.generator_rep = 2
    assert lib.gft_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.GFT_E_INVALID
    assert b"generator_rep" in lib.gft_last_error(None)
    assert not h.value


def test_batch_create_validates_members_without_gpu(lib):
    """Ensemble members must share model, form (mixed), device and logging cadence; checked before any device call."""
    from gftevolver_b200 import LatticeParams, _lib
    from gftevolver_b200.evolver import make_config
    a = LatticeParams(nx=8, ny=4, nz=16, energy_every=2)
    b = LatticeParams(nx=8, ny=4, nz=16, energy_every=2, model=_lib.GFT_MODEL_2HDM)
    h = ctypes.c_void_p()
    cfgs = (_lib.GftConfig * 2)(make_config(a), make_config(b))
    assert lib.gft_batch_create(cfgs, 2, ctypes.byref(h)) == _lib.GFT_E_INVALID
    assert b"model" in lib.gft_last_error(None)
    c = LatticeParams(nx=8, ny=4, nz=16, energy_every=3)
    cfgs = (_lib.GftConfig * 2)(make_config(a), make_config(c))
    assert lib.gft_batch_create(cfgs, 2, ctypes.byref(h)) == _lib.GFT_E_INVALID
    cfgs = (_lib.GftConfig * 1)(make_config(a, "fp64"))
    assert lib.gft_batch_create(cfgs, 1, ctypes.byref(h)) == _lib.GFT_E_UNSUPPORTED
    d = LatticeParams(nx=8, ny=6, nz=16, energy_every=2)  # ny % 4 != 0: no tile shape fits
    cfgs = (_lib.GftConfig * 2)(make_config(a), make_config(d))
    assert lib.gft_batch_create(cfgs, 2, ctypes.byref(h)) == _lib.GFT_E_UNSUPPORTED
    assert lib.gft_batch_create(cfgs, 0, ctypes.byref(h)) == _lib.GFT_E_INVALID
    # members with a Higgs-family field must share it (gaugeNum)
    e = LatticeParams(nx=8, ny=4, nz=16, energy_every=2, model=_lib.GFT_MODEL_2HDM, higgs_family=_lib.GFT_HF_SU2)
    e1 = LatticeParams(nx=8, ny=4, nz=16, energy_every=2, model=_lib.GFT_MODEL_2HDM, higgs_family=_lib.GFT_HF_U1)
    cfgs = (_lib.GftConfig * 2)(make_config(e), make_config(e1))
    assert lib.gft_batch_create(cfgs, 2, ctypes.byref(h)) == _lib.GFT_E_INVALID
    assert b"Higgs-family" in lib.gft_last_error(None)
    f = LatticeParams(nx=8, ny=4, nz=16, energy_every=2, generator_rep=1)
    cfgs = (_lib.GftConfig * 1)(make_config(f))
    assert lib.gft_batch_create(cfgs, 1, ctypes.byref(h)) == _lib.GFT_E_UNSUPPORTED
    assert not h.value
