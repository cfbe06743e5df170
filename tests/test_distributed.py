"""Multi-GPU host logic on CPU: two gloo ranks play two GGEMS devices.

Each rank takes its share of the primaries and its own random streams
(ggems_b200.distributed), runs it (here through the CPU oracle, standing in
for the rank's GPU), and the tallies are summed by one all-reduce.  The
result must equal GGEMS's two-device run: device d's share simulated with
device d's streams, detector histograms summed.
"""

import os
import socket

import numpy as np
import pytest

import parity
import scenes
from ggems_b200 import abi, distributed


def test_primaries_split_like_ggems():
    for total, world in ((10, 3), (1_000_000, 8), (7, 8), (2 ** 20 * 3 + 5, 2)):
        counts = [distributed.primaries_of_rank(total, world, r) for r in range(world)]
        assert sum(counts) == total
        assert max(counts) - min(counts) <= 1 and counts == sorted(counts, reverse=True)
    # device balancing: float-weighted, rounding loss to device 0
    counts = [distributed.primaries_of_rank(1000001, 3, r, balance=[0.5, 0.25, 0.25]) for r in range(3)]
    assert sum(counts) == 1000001 and counts[1] == counts[2] == 250000
    with pytest.raises(ValueError):
        distributed.primaries_of_rank(10, 2, 2)


def test_random_streams_follow_device_order():
    for rank in (0, 1, 3):
        st = distributed.random_states_of_rank(777, rank).reshape(5, -1)
        ref = scenes.seed_states(777, skip=rank * abi.GG_MAXIMUM_PARTICLES)
        assert np.array_equal(st, ref)


def _scene():
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    sc.set_world((20, 16, 10), (120.0, 100.0, 80.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    return sc, src


def _rank_main(rank, world, port, total, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        sc, src = _scene()
        n = distributed.primaries_of_rank(total, world, rank)
        states = distributed.random_states_of_rank(777, rank).reshape(5, -1)
        _, T, _ = parity.run_oracle(sc, src, n, states=states, threads=2)
        distributed.reduce_tallies(T)
        np.save(os.path.join(out_dir, "h%d.npy" % rank), np.concatenate(T.histograms))
        np.save(os.path.join(out_dir, "w%d.npy" % rank), T.world["photon_tracking"])
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_two_ggems_devices(tmp_path):
    import torch.multiprocessing as mp
    total, world = 120001, 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, total, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    h0 = np.load(tmp_path / "h0.npy")
    h1 = np.load(tmp_path / "h1.npy")
    assert np.array_equal(h0, h1)  # every rank holds the sum
    # GGEMS with two devices: device d simulates its share with its streams; histograms summed.
    sc, src = _scene()
    expected = None
    world_expected = None
    for d in range(world):
        n = total // world + (1 if d < total % world else 0)
        _, T, _ = parity.run_oracle(sc, src, n, states=scenes.seed_states(777, skip=d * abi.GG_MAXIMUM_PARTICLES))
        h = np.concatenate(T.histograms).astype(np.int64)
        expected = h if expected is None else expected + h
        w = T.world["photon_tracking"].astype(np.int64)
        world_expected = w if world_expected is None else world_expected + w
    assert np.array_equal(h0.astype(np.int64), expected)
    assert expected.sum() > 0
    w0, w1 = np.load(tmp_path / "w0.npy"), np.load(tmp_path / "w1.npy")
    assert np.array_equal(w0, w1) and np.array_equal(w0.astype(np.int64), world_expected)
    assert world_expected.sum() > 0
