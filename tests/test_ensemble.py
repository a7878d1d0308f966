"""The batched ensemble: scene partitioning across ranks (CPU, gloo) and, on the
GPU, per-scene densities bit-exact against the same scene run alone, forces
within FP32 tolerance, one graph launch per step, and an autotuner that leaves
the scenes' state untouched."""
import os

import numpy as np
import pytest

from stardust_b200 import _lib as L
from stardust_b200.ensemble import partition


def _members():
    from stardust_b200.scenes import ensemble_members

    return ensemble_members(64, 4)


def test_members_follow_recipe():
    ms = _members()
    assert len(ms) == 64
    for m in ms:
        assert 16_384 <= m["n"] <= 1_048_576 or m["kind"] == "zeldovich"
        assert m["grid"] in (32, 64, 128)
    assert {m["kind"] for m in ms} == {"disk", "zeldovich"}


def test_partition_is_balanced_and_complete():
    ms = _members()
    for ranks in (1, 2, 4, 8):
        parts = partition(ms, ranks)
        assert sorted(i for p in parts for i in p) == list(range(len(ms)))
        cost = [sum(184 * ms[i]["n"] + 40 * ms[i]["grid"] ** 3 for i in p) for p in parts]
        biggest = max(184 * m["n"] + 40 * m["grid"] ** 3 for m in ms)
        assert max(cost) - min(cost) <= biggest


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = _members()
    mine = partition(ms, world)[rank]
    import torch

    t = torch.tensor([len(mine), sum(ms[i]["n"] for i in mine)], dtype=torch.int64)
    allt = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(allt, t)
    out.put((rank, mine, [a.tolist() for a in allt]))
    dist.destroy_process_group()


def test_two_rank_partition_covers_every_scene_once():
    import multiprocessing as mp
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    scenes = sorted(i for _, mine, _ in res for i in mine)
    assert scenes == list(range(64))
    totals = res[0][2]
    assert sum(t[1] for t in totals) == sum(m["n"] for m in _members())


def _small_members():
    from stardust_b200.scenes import disk_galaxy, zeldovich

    out = []
    for kind, n, G, seed in (("disk", 20_000, 32, 1), ("zeldovich", 32 ** 3, 32, 2), ("disk", 70_000, 64, 3),
                             ("zeldovich", 48 ** 3, 64, 4), ("disk", 150_000, 128, 5)):
        p, v = disk_galaxy(n, seed) if kind == "disk" else zeldovich(round(n ** (1 / 3)), seed)
        out.append(({"n": len(p), "grid": G}, p, v))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("tune", [False, True])
def test_ensemble_density_bit_exact_against_solo_runs(cuda, tune):
    from stardust_b200.ensemble import Ensemble, member_config
    from stardust_b200.sim import Sim

    dt = 1e-3
    members = _small_members()
    with Ensemble(0) as ens:
        for m, p, v in members:
            ens.add(member_config(m, keep_density=1), p, v)
        orders = [L.SD_ORDER_TILED] * len(members)
        if tune:
            tun = ens.autotune(dt)
            assert all(t["step_ms"] > 0 for t in tun)
            # the fused deposit's share size is tuned too (at least 2048 window particles per CTA)
            assert all((t["deposit_split"] >= 2048) == (t["order"] == "tiled") for t in tun)
            orders = [{"tiled": L.SD_ORDER_TILED, "rowmajor": L.SD_ORDER_ROWMAJOR}[t["order"]] for t in tun]
        ens.steps(dt, 1)
        ens.synchronize()
        dens = [ens.scene(i).density() for i in range(len(members))]
        ens.steps(dt, 3)
        ens.synchronize()
        acc = [ens.scene(i).accel() for i in range(len(members))]
        parts = [ens.scene(i).get_particles() for i in range(len(members))]
    for i, (m, p, v) in enumerate(members):
        with Sim(0) as s:
            cfg = member_config(m, keep_density=1)
            cfg.order = orders[i]  # the tuned sort order, so particles line up slot by slot
            s.init(cfg)
            s.set_particles(p, v)
            s.step(dt)
            assert np.array_equal(s.density(), dens[i]), f"scene {i}: density differs"
            for _ in range(3):
                s.step(dt)
            a = s.accel()
            sp, _ = s.get_particles()
        # the same particles in the same sorted order; forces within FP32 tolerance
        live = sp[:, 0] >= 0
        assert np.abs(parts[i][0][live, :3] - sp[live, :3]).max() < 1e-5
        scale = np.abs(a[:, :3]).max()
        assert np.abs(acc[i][:, :3] - a[:, :3]).max() <= 1e-4 * scale


@pytest.mark.gpu
def test_ensemble_one_graph_launch_per_step(cuda):
    from stardust_b200.ensemble import Ensemble, member_config
    from stardust_b200.sim import Sim

    members = _small_members()[:3]
    with Ensemble(0) as ens:
        for m, p, v in members:
            ens.add(member_config(m), p, v)
        ens.steps(1e-3, 2)  # builds the graphs
        k = ens.graph_kernels()
        assert k >= 10 * len(members)
        before = Sim.kernel_launches()
        ens.steps(1e-3, 5)
        ens.synchronize()
        assert Sim.kernel_launches() - before == 5 * k
        assert all(ens.scene(i).step_count() == 7 for i in range(len(members)))
