"""The multi-GPU tally exchange on the device (GPU test, one GPU): the
buffers gg_device_tallies lists are aliased by torch tensors without a copy,
and reduce_device_tallies sums them in place over NCCL.  On one GPU the group
has one rank, so the sum must leave every tally exactly as the run left it;
the arithmetic over several ranks is the same all-reduce (the host-side
reduction over two ranks is checked bit-exact against GGEMS's two-device run
in tests/test_distributed.py)."""

import os
import socket

import numpy as np
import pytest

import parity
import scenes
from ggems_b200 import abi

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_device_tallies_reduce_in_place():
    import datetime
    import torch
    import torch.distributed as dist
    from ggems_b200 import _native, distributed
    ctx = _native.Context(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
        sc.solids[0].dose_map = sc._add_dose(sc.solids[0], {"photon_tracking": True})
        sc.set_world((20, 20, 20), (50.0, 50.0, 50.0))
        src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
        _, T0, _ = parity.run_gpu(ctx, sc, src, 300_000)
        tensors = distributed.device_tallies(ctx.handle)
        # 2 histograms; edep, edep^2, hit, photon tracking; world count, energy, energy^2, momentum
        assert len(tensors) == 10
        assert [t.dtype for t in tensors[:6]] == [torch.int32, torch.int32, torch.int64, torch.float64, torch.int32,
                                                  torch.int32]
        # aliasing: the tensor is the context's histogram
        h0 = tensors[0].cpu().numpy()
        assert np.array_equal(h0, T0.histograms[0]) and h0.sum() > 0
        assert distributed.reduce_device_tallies(ctx.handle) == 10
        T1 = sc.tallies()
        ctx.read_tallies(T1)
        for a, b in zip(T0.histograms, T1.histograms):
            assert np.array_equal(a, b)
        for k in ("edep", "edep_squared", "hit", "photon_tracking"):
            assert np.array_equal(getattr(T0, k)[0], getattr(T1, k)[0]), k
        for k, v in T0.world.items():
            assert np.array_equal(v, T1.world[k]), k
    finally:
        dist.destroy_process_group()
        ctx.close()
