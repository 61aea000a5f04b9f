"""x-slab decomposition host logic on CPU: gloo ranks (world size 2 and 3)
exchanging ghost planes through gftevolver_b200.slab, the oracle as the
per-rank step.

Each rank evolves its planes plus one ghost plane on each side as a periodic
lattice of its own (the oracle's per-site loop, one step at a time) and
refreshes the ghosts of the level just written after every step.  The
interior then equals the whole-lattice oracle evolution bit for bit: every
site reads only planes x - 1, x, x + 1 of the "now" level.  combine_rows is
checked on synthetic rows (sums, maxima, site-weighted means).
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, shape, model, nt, out_dir, hf=0):
    import datetime

    import torch
    import torch.distributed as dist

    from gftevolver_b200.slab import DistTransport, HaloExchange, combine_rows, partition
    from oracle import oracle as orc

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nx, ny, nz = shape
        op = orc.Params(model=model, nx=nx, ny=ny, nz=nz, higgs_family=hf)
        ic = orc.ICSpec(seed=17, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                        eps_sigma=0.1)
        g_sc, g_ve = orc.init_fields(op, ic, np.float64)
        x0, x1 = partition(nx, world, rank)
        nloc = x1 - x0
        idx = [x % nx for x in range(x0 - 1, x1 + 1)]
        sc = np.ascontiguousarray(g_sc[:, idx])
        ve = np.ascontiguousarray(g_ve[:, idx])
        lp = orc.Params(model=model, nx=nloc + 2, ny=ny, nz=nz, higgs_family=hf)

        def planes(level, x):
            return [torch.from_numpy(sc[level, x]), torch.from_numpy(ve[level, x])]

        halo = HaloExchange(planes, nloc, DistTransport())
        for t in range(nt):
            orc.evolve(lp, sc, ve, 1, t)
            halo(t % 2)  # the level step t wrote: 1 - (t + 1) % 2
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), sc=sc[:, 1:nloc + 1], ve=ve[:, 1:nloc + 1],
                 x0=x0, x1=x1)

        # combine_rows: rank r contributes energy r+1, means (r+1)/10 over (r+1)*10 sites, max 2r
        own = (rank + 1) * 10
        extra = [0.5, float(rank), 3.0][:op.neq - 4]  # Higgs-family constraints (gaugeNum 5 or 7)
        rows = [{"time_iter": 4, "has_energy": True, "has_gauss": True, "energy": rank + 1.0, "potential": 1.0,
                 "gradient": 0.0, "kinetic": 0.0, "magnetic": 0.0, "electric": 0.0,
                 "plaq_su2": (rank + 1) / 10.0, "plaq_u1": 1.0, "phi_sq": 2.0,
                 "gauss_int": [1.0, 0.0, 0.0, float(rank)] + extra,
                 "gauss_max": [2.0 * rank, 0.0, 1.0, 0.0] + extra}]
        tot = combine_rows(rows, own)[0]
        np.savez(os.path.join(out_dir, f"rows{rank}.npz"), energy=tot["energy"], potential=tot["potential"],
                 plaq_su2=tot["plaq_su2"], plaq_u1=tot["plaq_u1"], gauss_int=tot["gauss_int"],
                 gauss_max=tot["gauss_max"])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,shape,model,hf", [(2, (8, 4, 6), 1, 0), (3, (7, 3, 5), 1, 0), (2, (6, 4, 4), 2, 0),
                                                 (2, (6, 3, 4), 2, 2)])
def test_slab_ranks_match_whole_lattice(tmp_path, oracle_mod, world, shape, model, hf):
    import torch.multiprocessing as mp

    nt = 5
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, shape, model, nt, str(tmp_path), hf), nprocs=world, join=True,
                       start_method="spawn")
    nx, ny, nz = shape
    op = oracle_mod.Params(model=model, nx=nx, ny=ny, nz=nz, higgs_family=hf)
    ic = oracle_mod.ICSpec(seed=17, mean=[1.0 if model == 1 else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                           eps_sigma=0.1)
    g_sc, g_ve = oracle_mod.init_fields(op, ic, np.float64)
    oracle_mod.evolve(op, g_sc, g_ve, nt, 0)
    covered = []
    for r in range(world):
        z = np.load(tmp_path / f"rank{r}.npz")
        x0, x1 = int(z["x0"]), int(z["x1"])
        covered += list(range(x0, x1))
        assert np.array_equal(z["sc"], g_sc[:, x0:x1])
        assert np.array_equal(z["ve"], g_ve[:, x0:x1])
    assert covered == list(range(nx))
    sites = [(r + 1) * 10 for r in range(world)]
    for r in range(world):
        z = np.load(tmp_path / f"rows{r}.npz")
        assert float(z["energy"]) == sum(r2 + 1.0 for r2 in range(world))
        assert float(z["potential"]) == float(world)
        assert abs(float(z["plaq_su2"]) - sum(s * (i + 1) / 10.0 for i, s in enumerate(sites)) / sum(sites)) < 1e-15
        assert abs(float(z["plaq_u1"]) - 1.0) < 1e-15
        extra_sum = [0.5 * world, float(sum(range(world))), 3.0 * world][:op.neq - 4]
        extra_max = [0.5, float(world - 1), 3.0][:op.neq - 4]
        assert list(z["gauss_int"]) == [float(world), 0.0, 0.0, float(sum(range(world)))] + extra_sum
        assert list(z["gauss_max"]) == [2.0 * (world - 1), 0.0, 1.0, 0.0] + extra_max


def test_partition_covers_every_plane_once():
    from gftevolver_b200.slab import partition
    for nx in (1, 2, 7, 64, 257):
        for world in range(1, min(nx, 9) + 1):
            parts = [partition(nx, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == nx
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        partition(3, 4, 0)


def _share_worker(rank, world, port, out_dir):
    import datetime
    import os

    import torch.distributed as dist

    from gftevolver_b200.slab import share_id
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        calls = []

        def make_id():
            calls.append(1)
            return os.urandom(128)

        got = share_id(make_id, rank, world)
        with open(os.path.join(out_dir, f"id{rank}.bin"), "wb") as f:
            f.write(got)
        with open(os.path.join(out_dir, f"calls{rank}.txt"), "w") as f:
            f.write(str(len(calls)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_communicator_id_is_made_once_and_shared(tmp_path, world):
    """The library-side slab exchange joins one NCCL communicator per group of ranks: rank 0
    alone makes the 128-byte id, and every rank ends up with the same bytes (gloo ranks on CPU)."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_share_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    ids = [(tmp_path / f"id{r}.bin").read_bytes() for r in range(world)]
    assert len(ids[0]) == 128 and all(x == ids[0] for x in ids)
    assert [int((tmp_path / f"calls{r}.txt").read_text()) for r in range(world)] == [1] + [0] * (world - 1)
