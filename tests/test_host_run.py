"""gft_run -- GFTEvolver's main() over the C ABI: reads the reference's
positional .cfg tree and writes the analysers' .dat files.

CPU: the configuration a reference run would see is parsed into gft_config
(no device call).  GPU: the same configuration tree and initial data run
through the reference binary (oracle/_ref/ref32, its own analysers writing
Data/*.dat) and through gft_run in the reference-arithmetic form; the .dat
rows agree to the printed precision (6 significant digits; 2e-5 relative
allows one unit in the last printed digit where the reference's float running
sums and the FP64 sums round differently) and the final fields to the ref32
bound (8 float ulps, at most 1 % of words different).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GFT_RUN = os.path.join(ROOT, "gftevolver_b200", "gft_run")


@pytest.fixture(scope="module")
def gft_run():
    if not os.path.exists(GFT_RUN):
        from gftevolver_b200 import build
        build.build()
        build.build_host()
    return GFT_RUN


def _params(orc, model, fixed_axes=0, higgs_family=0, generator_rep=0):
    return orc.Params(model=model, nx=6, ny=5, nz=8, dt=0.05, damping=0.3, nt_damped=2, energy_every=2,
                      gauss_every=3, g=0.61, gp=0.33, fixed_axes=fixed_axes, higgs_family=higgs_family, gpp=0.47,
                      generator_rep=generator_rep)


@pytest.mark.parametrize("model", [1, 2])
def test_config_tree_is_parsed_like_the_reference(tmp_path, oracle_mod, gft_run, model):
    from oracle import refrun
    p = _params(oracle_mod, model)
    refrun.write_configs(str(tmp_path), p, 7)
    out = subprocess.run([gft_run, str(tmp_path), "--print-config", "--form", "ref32"], capture_output=True,
                         text=True, check=True).stdout.split()
    kv = {out[i]: out[i + 1] for i in range(0, len(out) - 1, 2)}
    assert int(kv["model"]) == model and int(kv["nt"]) == 7
    assert (int(kv["nx"]), int(kv["ny"]), int(kv["nz"])) == (6, 5, 8)
    assert float(kv["dt"]) == 0.05 and float(kv["g"]) == 0.61 and float(kv["gp"]) == 0.33
    assert float(kv["damping"]) == float(np.float32(0.3)) and int(kv["nt_damped"]) == 2
    assert int(kv["energy_every"]) == 2 and int(kv["gauss_every"]) == 3 and int(kv["fixed_axes"]) == 0
    if model == 1:
        assert float(kv["lambda"]) == p.lam and float(kv["eta_sqr"]) == p.eta_sqr
    else:
        assert float(kv["m12r"]) == p.m12r and float(kv["l4p5"]) == p.l4p5 and int(kv["break_son"]) == 1


def test_unsupported_reference_configuration_is_refused(tmp_path, oracle_mod, gft_run):
    from oracle import refrun
    p = _params(oracle_mod, 1)
    refrun.write_configs(str(tmp_path), p, 7)
    lat = tmp_path / "Core" / "Config" / "Lattice.cfg"
    lat.write_text(lat.read_text().replace("faces                          : 3 3 3 3 3 3",
                                           "faces                          : 1 3 3 3 3 3"))
    r = subprocess.run([gft_run, str(tmp_path), "--print-config"], capture_output=True, text=True)
    assert r.returncode == 1 and "pairs" in r.stderr


@pytest.mark.parametrize("hf", [0, 1, 2])
def test_higgs_family_is_read_from_the_vector_width(tmp_path, oracle_mod, gft_run, hf):
    """5, 6 or 9 vector components per direction select gaugeNum 4, 5 or 7
    (WilsonLoops/Source/TwoHDM.cpp:229-241); g'' comes from TwoHDM.cfg."""
    from oracle import refrun
    refrun.write_configs(str(tmp_path), _params(oracle_mod, 2, higgs_family=hf), 7)
    out = subprocess.run([gft_run, str(tmp_path), "--print-config"], capture_output=True, text=True,
                         check=True).stdout.split()
    assert int(out[out.index("higgs_family") + 1]) == hf
    assert float(out[out.index("gpp") + 1]) == 0.47
    if hf:
        refrun.write_configs(str(tmp_path), _params(oracle_mod, 1), 7)
        lat = tmp_path / "Core" / "Config" / "Lattice.cfg"
        lat.write_text(lat.read_text().replace("vector components per direction: 5",
                                               "vector components per direction: " + ("6" if hf == 1 else "9")))
        r = subprocess.run([gft_run, str(tmp_path), "--print-config"], capture_output=True, text=True)
        assert r.returncode == 1 and "StandardModel needs 4 or 5" in r.stderr


@pytest.mark.parametrize("model,hf", [(1, 0), (2, 0), (2, 1), (2, 2)])
def test_generator_representation_is_parsed(tmp_path, oracle_mod, gft_run, model, hf):
    """SM: 4 vector components per direction mean generators (WilsonLoops/Source/StandardModel.cpp:195-210);
    TwoHDM: the flag in TwoHDM.cfg with 4, 5 or 7 components."""
    from oracle import refrun
    refrun.write_configs(str(tmp_path), _params(oracle_mod, model, higgs_family=hf, generator_rep=1), 7)
    out = subprocess.run([gft_run, str(tmp_path), "--print-config"], capture_output=True, text=True,
                         check=True).stdout.split()
    assert int(out[out.index("generator_rep") + 1]) == 1
    assert int(out[out.index("higgs_family") + 1]) == hf


def test_fixed_faces_are_parsed(tmp_path, oracle_mod, gft_run):
    from oracle import refrun
    refrun.write_configs(str(tmp_path), _params(oracle_mod, 1, fixed_axes=5), 7)
    out = subprocess.run([gft_run, str(tmp_path), "--print-config"], capture_output=True, text=True,
                         check=True).stdout.split()
    assert out[out.index("fixed_axes") + 1] == "5"


def _numbers(path):
    return [[float(v) for v in line.split()] for line in open(path) if line.strip()]


@pytest.mark.gpu
@pytest.mark.parametrize("model,fixed_axes,hf,gen", [(1, 0, 0, 0), (2, 0, 0, 0), (1, 5, 0, 0), (2, 0, 1, 0),
                                                     (2, 0, 2, 0), (1, 0, 0, 1), (2, 0, 2, 1)])
def test_dat_rows_and_fields_match_the_reference_run(tmp_path, oracle_mod, gft_run, model, fixed_axes, hf, gen):
    from oracle import refrun
    if not refrun.available(False):
        pytest.skip("oracle/_ref/ref32 not built")
    p = _params(oracle_mod, model, fixed_axes, hf, gen)
    ic = oracle_mod.ICSpec(seed=5, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                           eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(p, ic, np.float32)
    ref_dir, gpu_dir = tmp_path / "ref", tmp_path / "gpu"
    ref_dir.mkdir()
    r_sc, r_ve, _, _ = refrun.run(p, sc, ve, 7, workdir=str(ref_dir))
    shutil.copytree(ref_dir, gpu_dir, ignore=shutil.ignore_patterns("Data", "final.bin", "rows.txt", "timing.txt"))
    subprocess.run([gft_run, str(gpu_dir), "--form", "ref32", "--ic", str(gpu_dir / "ic.bin"), "--final-bin",
                    str(gpu_dir / "final.bin")], check=True, capture_output=True, text=True)
    for name in ("global_quantities.dat", "global_quantities_gauge.dat"):
        a, b = _numbers(gpu_dir / "Data" / name), _numbers(ref_dir / "Data" / name)
        assert len(a) == len(b) and len(a) > 0
        for ra, rb in zip(a, b):
            assert len(ra) == len(rb)
            np.testing.assert_allclose(ra, rb, rtol=2e-5, atol=1e-12)
    raw = np.fromfile(gpu_dir / "final.bin", dtype=np.float32)
    g_sc, g_ve = raw[:sc.size].reshape(sc.shape), raw[sc.size:].reshape(ve.shape)
    for g, r in ((g_sc, r_sc), (g_ve, r_ve)):
        tol = 8 * np.spacing(np.maximum(np.abs(g), np.abs(r)))
        assert np.all(np.abs(g.astype(np.float64) - r) <= tol + 1e-30)
        assert np.mean(g != r) <= 0.01


@pytest.mark.parametrize("ic_types,random_uniform", [((1, 0), (42, -1.0, 1.0, 1)), ((0, 1), (7, -0.5, 0.25, 0)),
                                                     ((1, 1), (-3, 0.0, 2.0, 1)), ((0, 0), (42, -1.0, 1.0, 1))])
@pytest.mark.parametrize("model,hf,gen", [(1, 0, 0), (2, 0, 0), (2, 2, 0), (1, 0, 1)])
def test_configured_initial_condition_matches_the_reference(tmp_path, oracle_mod, gft_run, model, hf, gen, ic_types,
                                                            random_uniform):
    """Zero scalars / identity links and RandomUniform (Core/Source/Lattice.cpp:358-401,
    InitialConditions/Source/RandomUniform.cpp:60-77), bit for bit against the
    initial fields the reference binary built from the same configuration tree."""
    from oracle import refrun
    if not refrun.available(False):
        pytest.skip("oracle/_ref/ref32 not built")
    p = _params(oracle_mod, model, higgs_family=hf, generator_rep=gen)
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    refrun.run(p, None, None, 1, workdir=str(ref_dir), ic_types=ic_types, random_uniform=random_uniform)
    want = np.fromfile(ref_dir / "initial.bin", dtype=np.float32)
    out = subprocess.run([gft_run, str(ref_dir), "--print-config"], capture_output=True, text=True,
                         check=True).stdout.split()
    assert (int(out[out.index("ic_scalar") + 1]), int(out[out.index("ic_gauge") + 1])) == ic_types
    for form, dtype in (("ref32", np.float32), ("fp64", np.float64)):
        path = tmp_path / f"initial_{form}.bin"
        subprocess.run([gft_run, str(ref_dir), "--form", form, "--initial-bin", str(path), "--initial-only"],
                       check=True, capture_output=True, text=True)
        got = np.fromfile(path, dtype=dtype)
        assert got.size == want.size
        np.testing.assert_array_equal(got, want.astype(dtype))


def test_initial_only_refuses_device_initial_data(tmp_path, oracle_mod, gft_run):
    from oracle import refrun
    refrun.write_configs(str(tmp_path), _params(oracle_mod, 1), 7)
    r = subprocess.run([gft_run, str(tmp_path), "--device-ic", "3", "--initial-bin", str(tmp_path / "x.bin"),
                        "--initial-only"], capture_output=True, text=True)
    assert r.returncode == 1 and "--device-ic" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("model,hf", [(1, 0), (2, 2)])
def test_local_analyser_files_match_the_reference(tmp_path, oracle_mod, gft_run, model, hf):
    """Energy's and GaugeCondition's local files (Continual/local_quantities_<step>.dat: option-major
    densities; Continual/local_quantities_gauge_<step>.dat: gaugeNum violations per site) of every
    local-output step, against the reference run's own files."""
    from oracle import refrun
    if not refrun.available(False):
        pytest.skip("oracle/_ref/ref32 not built")
    p = _params(oracle_mod, model, higgs_family=hf)
    p.energy_local_every, p.gauss_local_every = 3, 2
    ic = oracle_mod.ICSpec(seed=9, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                           eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(p, ic, np.float32)
    ref_dir, gpu_dir = tmp_path / "ref", tmp_path / "gpu"
    ref_dir.mkdir()
    refrun.run(p, sc, ve, 7, workdir=str(ref_dir), energy_local=(0, 2, 5))
    shutil.copytree(ref_dir, gpu_dir, ignore=shutil.ignore_patterns("Data", "final.bin", "rows.txt", "timing.txt"))
    subprocess.run([gft_run, str(gpu_dir), "--form", "ref32", "--ic", str(gpu_dir / "ic.bin")], check=True,
                   capture_output=True, text=True)
    ref_files = sorted(os.listdir(ref_dir / "Data" / "Continual"))
    assert ref_files == sorted(os.listdir(gpu_dir / "Data" / "Continual"))
    assert "local_quantities_6.dat" in ref_files and "local_quantities_gauge_6.dat" in ref_files
    for name in ref_files:
        a = np.loadtxt(gpu_dir / "Data" / "Continual" / name)
        b = np.loadtxt(ref_dir / "Data" / "Continual" / name)
        assert a.shape == b.shape, name
        np.testing.assert_allclose(a, b, rtol=2e-5, atol=1e-6 * max(np.abs(b).max(), 1e-3), err_msg=name)
    for name in ("global_quantities.dat", "global_quantities_gauge.dat"):
        a, b = _numbers(gpu_dir / "Data" / name), _numbers(ref_dir / "Data" / name)
        assert len(a) == len(b)
        for ra, rb in zip(a, b):
            np.testing.assert_allclose(ra, rb, rtol=2e-5, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("both", [0, 1])
def test_output_fields_dumps_match_the_reference(tmp_path, oracle_mod, gft_run, both):
    """OutputFields (Analysers/Source/OutputFields.cpp:63-200): the initial, every continual
    (after steps 3 and 6) and the final dump, one or both time levels, against the reference
    run's own files.  Values print with 6 significant digits; where the ref32 fields differ
    from the reference's in the last float bits the printed digit may differ by one."""
    from oracle import refrun
    if not refrun.available(False):
        pytest.skip("oracle/_ref/ref32 not built")
    p = _params(oracle_mod, 2, higgs_family=1)
    ic = oracle_mod.ICSpec(seed=8, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    sc, ve = oracle_mod.init_fields(p, ic, np.float32)
    ref_dir, gpu_dir = tmp_path / "ref", tmp_path / "gpu"
    ref_dir.mkdir()
    refrun.run(p, sc, ve, 7, workdir=str(ref_dir), output_fields=(both, 1, 1, 1, 3))
    shutil.copytree(ref_dir, gpu_dir, ignore=shutil.ignore_patterns("Data", "final.bin", "rows.txt", "timing.txt"))
    subprocess.run([gft_run, str(gpu_dir), "--form", "ref32", "--ic", str(gpu_dir / "ic.bin")], check=True,
                   capture_output=True, text=True)
    names = ["initial_fields.dat", "Continual/fields_3.dat", "Continual/fields_6.dat", "final_fields.dat"]
    for name in names:
        a, b = _numbers(gpu_dir / "Data" / name), _numbers(ref_dir / "Data" / name)
        assert len(a) == len(b) == p.nsite * (2 if both else 1), name
        a, b = np.array(a), np.array(b)
        assert a.shape == b.shape == (len(b), p.nsc + p.nve), name
        np.testing.assert_allclose(a, b, rtol=2e-5, atol=1e-6, err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("model", [1, 2])
def test_configured_initial_condition_run_matches_the_reference(tmp_path, oracle_mod, gft_run, model):
    """The whole job from the configured initial condition (RandomUniform scalars,
    identity links): no initial-data file on either side."""
    from oracle import refrun
    if not refrun.available(False):
        pytest.skip("oracle/_ref/ref32 not built")
    p = _params(oracle_mod, model)
    ref_dir, gpu_dir = tmp_path / "ref", tmp_path / "gpu"
    ref_dir.mkdir()
    r_sc, r_ve, _, _ = refrun.run(p, None, None, 7, workdir=str(ref_dir), ic_types=(1, 0),
                                  random_uniform=(42, -0.5, 0.5, 1))
    shutil.copytree(ref_dir, gpu_dir, ignore=shutil.ignore_patterns("Data", "*.bin", "rows.txt", "timing.txt"))
    subprocess.run([gft_run, str(gpu_dir), "--form", "ref32", "--initial-bin", str(gpu_dir / "initial.bin"),
                    "--final-bin", str(gpu_dir / "final.bin")], check=True, capture_output=True, text=True)
    np.testing.assert_array_equal(np.fromfile(gpu_dir / "initial.bin", dtype=np.float32),
                                  np.fromfile(ref_dir / "initial.bin", dtype=np.float32))
    for name in ("global_quantities.dat", "global_quantities_gauge.dat"):
        a, b = _numbers(gpu_dir / "Data" / name), _numbers(ref_dir / "Data" / name)
        assert len(a) == len(b) and len(a) > 0
        for ra, rb in zip(a, b):
            np.testing.assert_allclose(ra, rb, rtol=2e-5, atol=1e-12)
    raw = np.fromfile(gpu_dir / "final.bin", dtype=np.float32)
    g_sc, g_ve = raw[:r_sc.size].reshape(r_sc.shape), raw[r_sc.size:].reshape(r_ve.shape)
    for g, r in ((g_sc, r_sc), (g_ve, r_ve)):
        tol = 8 * np.spacing(np.maximum(np.abs(g), np.abs(r)))
        assert np.all(np.abs(g.astype(np.float64) - r) <= tol + 1e-30)
        assert np.mean(g != r) <= 0.01
