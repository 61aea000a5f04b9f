"""TEST INFRASTRUCTURE ONLY -- runs the reference itself (oracle/_ref/ref32|ref64).

The binaries are the unmodified GFTEvolver sources compiled by
``oracle/build_ref.sh`` with ``oracle/ref_harness.cpp`` as ``main``.  This
module writes the reference's positional ``.cfg`` files for a run (in the
line structure each ``configure`` function parses, e.g.
``Core/Source/Lattice.cpp:33-145``, ``Core/Source/Model.cpp:145-222``,
``Potentials/Source/Double_SO_N.cpp:122-213``), writes the initial data, runs
the binary and reads back the final fields and the analysers' sums.

Used to generate the golden fixtures (tests/golden/make_golden.py), by the
parity tests when the binaries exist, and as the timed CPU baseline of
bench.py (``cpu_baseline.kind = "reference"``).
"""
from __future__ import annotations

import os
import subprocess
import tempfile
import time

import numpy as np

from . import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def binary(fp64: bool) -> str:
    return os.path.join(REF_DIR, "ref64" if fp64 else "ref32")


def available(fp64: bool = False) -> bool:
    return os.access(binary(fp64), os.X_OK)


def _num(v) -> str:
    if isinstance(v, (bool, np.bool_)):
        return "1" if v else "0"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def _header(n: int, title: str) -> list[str]:
    """n description lines without ':' (each configure() skips a fixed count)."""
    lines = [f"{title} (written for a reference run; positional format)"]
    while len(lines) < n:
        lines.append("")
    return lines


def _write(path: str, lines: list[str]) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_configs(work: str, p: orc.Params, nt: int, ic_types=(0, 0), random_uniform=(42, -1.0, 1.0, 1),
                  output_fields=None, energy_local=(0, 1, 2, 3, 4, 5)) -> None:
    """ic_types: Lattice.cfg initial-condition types (0 zero / identity links, 1 RandomUniform);
    random_uniform: InitialConditions/Config/RandomUniform.cfg (seed, min, max, equal time levels);
    output_fields: None (OutputFields off) or (both levels, initial, final, continual, frequency)
    for Analysers/Config/OutputFields.cfg; energy_local: the Energy local options written when
    p.energy_local_every > 0 (0 energy, 1 potential, 2 gradient, 3 kinetic, 4 magnetic, 5 electric)."""
    sm = p.model == orc.MODEL_SM
    # Core/Config/Lattice.cfg -- Lattice::configure (Lattice.cpp:47-143)
    lat = _header(10, "Lattice")
    lat += [
        f"grid points (nx ny nz)         : {p.nx} {p.ny} {p.nz}",
        f"spacings (dx dy dz)            : {_num(p.dx)} {_num(p.dy)} {_num(p.dz)}",
        f"timesteps                      : {nt}",
        f"timestep size                  : {_num(p.dt)}",
        "",
        f"scalar components              : {p.nsc}",
        f"vector components per direction: {p.dw}",
        "",
        "override nt by light crossings",
        "flag                           : 0",
        "crossings                      : 1",
        "",
        "initial condition types for",
        "scalar fields and gauge fields",
        "(zero, loaded by the harness)",
        f"types                          : {ic_types[0]} {ic_types[1]}",
        "",
        "analysis options",
        f"output fields                  : {0 if output_fields is None else 1}",
        f"calculate energy               : {1 if p.energy_every > 0 or p.energy_local_every > 0 else 0}",
        f"calculate gauge condition      : {1 if p.gauss_every > 0 or p.gauss_local_every > 0 else 0}",
        "",
        "boundary conditions",
        "six faces",
        "periodic [3]",
        "all faces periodic",
        "(-x) (+x) (-y) (+y) (-z) (+z)",
        "in this order",
        "faces                          : " + " ".join("1 1" if (p.fixed_axes >> a) & 1 else "3 3"
                                                         for a in range(3)),
        "",
        "progress reports               : 0",
        "report frequency               : 1000000",
    ]
    _write(os.path.join(work, "Core", "Config", "Lattice.cfg"), lat)

    # InitialConditions/Config/RandomUniform.cfg -- RandomUniform::configure (RandomUniform.cpp:14-34)
    ru = _header(12, "RandomUniform")
    ru += [f"seed                           : {int(random_uniform[0])}",
           f"range (min max)                : {_num(random_uniform[1])} {_num(random_uniform[2])}",
           f"equal time levels              : {int(random_uniform[3])}"]
    _write(os.path.join(work, "InitialConditions", "Config", "RandomUniform.cfg"), ru)

    # Core/Config/Model.cfg -- Model::configure (Model.cpp:173-221)
    mod = _header(11, "Model")
    mod += [
        f"potential type                 : {1 if sm else 2}",
        "gradient type",
        f"type                           : {2 if sm else 3}",
        "wilson loop type",
        f"type                           : {1 if sm else 2}",
        "",
        f"damping factor                 : {_num(p.damping)}",
        f"damped timesteps               : {p.nt_damped}",
        "override by time              : 0",
        "time                           : 0",
    ]
    _write(os.path.join(work, "Core", "Config", "Model.cfg"), mod)

    # WilsonLoops/Config/{StandardModel,TwoHDM}.cfg (StandardModel.cpp:17-31, TwoHDM.cpp:17-39)
    wl = _header(12, "Wilson loops")
    wl += [f"g                              : {_num(p.g)}", f"gp                             : {_num(p.gp)}"]
    if sm:
        wl += ["", f"division tolerance             : {_num(p.div_tol)}"]
        _write(os.path.join(work, "WilsonLoops", "Config", "StandardModel.cfg"), wl)
    else:
        wl += [f"gpp                            : {_num(p.gpp)}", "",
               f"generator representation       : {1 if p.generator_rep else 0}", "",
               f"division tolerance             : {_num(p.div_tol)}"]
        _write(os.path.join(work, "WilsonLoops", "Config", "TwoHDM.cfg"), wl)

    # Gradients/Config/{StandardModel,TwoHDM}.cfg (Gradients StandardModel.cpp:54-57)
    gr = _header(12, "Gradients") + [f"division tolerance             : {_num(p.div_tol)}"]
    _write(os.path.join(work, "Gradients", "Config", "StandardModel.cfg" if sm else "TwoHDM.cfg"), gr)

    if sm:
        # Potentials/Config/SO_N.cfg (SO_N.cpp:21-27)
        so = _header(15, "SO_N") + [f"lambda                         : {_num(p.lam)}",
                                     f"eta squared                    : {_num(p.eta_sqr)}"]
        _write(os.path.join(work, "Potentials", "Config", "SO_N.cfg"), so)
    else:
        # Potentials/Config/Double_SO_N.cfg (Double_SO_N.cpp:131-210)
        d = _header(40, "Double_SO_N")
        d += [
            "components in f1               : 4",
            "",
            f"apply normalisation            : {p.apply_norm}",
            f"energy offset                  : {_num(p.energy_offset)}",
            "",
            f"m1 m2                          : {_num(p.m1)} {_num(p.m2)}",
            f"l1 l2                          : {_num(p.l1)} {_num(p.l2)}",
            f"l3                             : {_num(p.l3)}",
            "",
            "",
            "terms breaking to one SO(N)",
            "need equal component counts",
            f"break to SO(N)                 : {p.break_son}",
            "",
            f"m12r                           : {_num(p.m12r)}",
            f"l4p5                           : {_num(p.l4p5)}",
            f"l6r l7r                        : {_num(p.l6r)} {_num(p.l7r)}",
            "",
            "",
            "terms breaking to U(N/2)",
            "need equal even counts",
            "in f1 and f2",
            f"break to U(N/2)                : {p.break_uhalfn}",
            "",
            f"m12i                           : {_num(p.m12i)}",
            f"l4m5 l5i                       : {_num(p.l4m5)} {_num(p.l5i)}",
            f"l6i l7i                        : {_num(p.l6i)} {_num(p.l7i)}",
        ]
        _write(os.path.join(work, "Potentials", "Config", "Double_SO_N.cfg"), d)

    # Analysers/Config/OutputFields.cfg (OutputFields.cpp:5-49)
    if output_fields is not None:
        both, initial, final, continual, freq = output_fields
        of = _header(13, "OutputFields")
        of += [f"both time levels               : {int(both)}", f"initial                        : {int(initial)}",
               f"final                          : {int(final)}", "",
               f"continual                      : {int(continual)}", f"frequency                      : {int(freq)}", "",
               "initial path                   : initial_fields.dat",
               "continual path                 : Continual/fields",
               "final path                     : final_fields.dat"]
        _write(os.path.join(work, "Analysers", "Config", "OutputFields.cfg"), of)

    # Analysers/Config/Energy.cfg (Energy.cpp:14-47)
    ef = max(p.energy_every, 1)
    en = _header(13, "Energy")
    en += ["global path                    : global_quantities.dat"]
    en += [f"global option {k}                : {1 if p.energy_every > 0 else 0}" for k in range(6)]
    el = max(p.energy_local_every, 1)
    en += [f"global frequency               : {ef}", "",
           "local path                     : Continual/local_quantities"]
    en += [f"local option {k}                 : {1 if p.energy_local_every > 0 and k in energy_local else 0}"
           for k in range(6)]
    en += [f"local frequency                : {el}"]
    _write(os.path.join(work, "Analysers", "Config", "Energy.cfg"), en)

    # Analysers/Config/GaugeCondition.cfg (GaugeCondition.cpp:14-47)
    gf = max(p.gauss_every, 1)
    ga = _header(13, "GaugeCondition")
    ga += ["global path                    : global_quantities_gauge.dat",
           f"integrated                     : {1 if p.gauss_every > 0 else 0}",
           f"maximum                        : {1 if p.gauss_every > 0 else 0}",
           f"global frequency               : {gf}", "",
           "local path                     : Continual/local_quantities_gauge",
           f"local violation                : {1 if p.gauss_local_every > 0 else 0}",
           f"local frequency                : {max(p.gauss_local_every, 1)}"]
    _write(os.path.join(work, "Analysers", "Config", "GaugeCondition.cfg"), ga)


def run(p: orc.Params, scalars: np.ndarray | None, vectors: np.ndarray | None, nt: int, fp64: bool = False,
        workdir: str | None = None, timeout: float = 600.0, ic_types=(0, 0), random_uniform=(42, -1.0, 1.0, 1),
        output_fields=None, energy_local=(0, 1, 2, 3, 4, 5)):
    """Run the reference binary from the given two-level initial data, or (scalars
    None) from its own configured initial condition (ic_types, random_uniform).

    Returns (final_scalars, final_vectors, rows, seconds) where rows lists the
    analysers' raw sums per logged step (float in ref32) and seconds is the
    wall time of Lattice::evolve.  The initial fields the run started from are
    left in <workdir>/initial.bin.
    """
    dtype = np.float64 if fp64 else np.float32
    own = workdir is None
    tmp = tempfile.TemporaryDirectory(prefix="gftref_") if own else None
    work = tmp.name if own else workdir
    given = scalars is not None
    if not given:
        scalars = np.zeros((2, p.nx, p.ny, p.nz, p.nsc), dtype)
        vectors = np.zeros((2, p.nx, p.ny, p.nz, p.nve), dtype)
    try:
        write_configs(work, p, nt, ic_types, random_uniform, output_fields, energy_local)
        icp = os.path.join(work, "ic.bin")
        if given:
            with open(icp, "wb") as f:
                f.write(np.ascontiguousarray(scalars, dtype=dtype).tobytes())
                f.write(np.ascontiguousarray(vectors, dtype=dtype).tobytes())
        elif os.path.exists(icp):
            os.remove(icp)
        env = dict(os.environ, GFT_REF_WORKDIR=work)
        t0 = time.perf_counter()
        res = subprocess.run([binary(fp64)], env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                             timeout=timeout)
        wall = time.perf_counter() - t0
        if res.returncode != 0:
            raise RuntimeError(f"reference run failed ({res.returncode}): {res.stderr.decode()[-2000:]}")
        raw = np.fromfile(os.path.join(work, "final.bin"), dtype=dtype)
        nsc_words = scalars.size
        sc = raw[:nsc_words].reshape(scalars.shape)
        ve = raw[nsc_words:].reshape(vectors.shape)
        rows = []
        with open(os.path.join(work, "rows.txt")) as f:
            for line in f:
                t = line.split()
                if not t:
                    continue
                vals = [float(v) for v in t[3:]]
                k = orc.MAX_EQ
                rows.append({"time_iter": int(t[0]), "has_energy": t[1] == "1", "has_gauss": t[2] == "1",
                             "ref_energy": vals[0:6], "ref_gauss_int": vals[6:6 + p.neq],
                             "gauss_max": vals[6 + k:6 + k + p.neq]})
        with open(os.path.join(work, "timing.txt")) as f:
            secs = float(f.read().split()[0])
        return sc, ve, rows, secs if secs > 0 else wall
    finally:
        if tmp is not None:
            tmp.cleanup()
