"""Scatter surrogate on the GPU: the U-Net kernels against the numpy oracle
(forward and gradients), the line-integral projector against an independent
ray sampling, the projector's primary against the MC primary (total minus
scatter histogram), and a small end-to-end training run showing what the
network gains over a plain low-count MC estimate of the scatter."""

import ctypes as C
import os
import sys
import tempfile

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import unet_oracle as uo  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def _inputs(seed, batch, side):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:side, 0:side] / side
    base = np.stack([np.exp(-2.0 * ((x - 0.5) ** 2 + (y - 0.5) ** 2)), 3.0 * x * y], -1)
    inp = np.stack([base + rng.uniform(0, 0.3, base.shape) for _ in range(batch)]).astype(np.float32)
    tgt = (0.5 * inp[..., 0] + 0.2 * inp[..., 1] ** 2 + rng.uniform(0, 0.05, inp.shape[:3])).astype(np.float32)
    return inp, tgt


def test_unet_forward_and_gradients_match_oracle(torch):
    from ggems_b200.scatter import UNet
    net = UNet(2, 64, seed=5)
    p = net.parameters()
    assert len(p) == uo.parameter_count()
    inp, tgt = _inputs(1, 2, 64)
    x, t = torch.from_numpy(inp).cuda(), torch.from_numpy(tgt).cuda()
    y = net.forward(x).cpu().numpy()
    y_ref, _ = uo.forward(p.astype(np.float64), inp.astype(np.float64))
    fwd_err = np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref)
    loss, g = net.gradients(x, t)
    loss_ref, g_ref = uo.loss_and_gradients(p.astype(np.float64), inp.astype(np.float64), tgt.astype(np.float64))
    print("U-Net forward relative error %.4f, loss %.6f vs %.6f" % (fwd_err, loss, loss_ref))
    assert fwd_err < 0.02
    assert abs(loss - loss_ref) <= 0.03 * loss_ref
    layers_g, wo_g, _, _ = uo.unpack(g.astype(np.float64))
    layers_r, wo_r, _, _ = uo.unpack(g_ref)
    for i, ((wg, bg), (wr, br)) in enumerate(zip(layers_g, layers_r)):
        if i == 0:
            wg, wr = wg[:, :, :uo.INPUT_CHANNELS], wr[:, :, :uo.INPUT_CHANNELS]  # padded input channels carry no signal
        for a, b in ((wg, wr), (bg, br)):
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            cos = float((a * b).sum() / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))
            assert rel < 0.08 and cos > 0.995, (i, rel, cos)
    rel = np.linalg.norm(wo_g - wo_r) / np.linalg.norm(wo_r)
    assert rel < 0.03
    net.close()


def test_unet_training_lowers_the_loss(torch):
    from ggems_b200.scatter import UNet
    net = UNet(4, 64, seed=7)
    inp, tgt = _inputs(2, 4, 64)
    x, t = torch.from_numpy(inp).cuda(), torch.from_numpy(tgt).cuda()
    first = net.train_step(x, t, 1e-3)
    for _ in range(60):
        last = net.train_step(x, t, 1e-3)
    print("U-Net loss %.5f -> %.5f after 60 Adam steps" % (first, last))
    assert last < 0.2 * first
    net.close()


@pytest.fixture(scope="module")
def geometry():
    from ggems_b200.scatter import Geometry
    return Geometry(64, tempfile.mkdtemp())


def _sampled_line_integral(geo, src, ph, det, i, j, step=0.02):
    """Independent check: integrate mu along the ray by fine sampling."""
    m = np.array(list(det.obb.matrix), np.float64).reshape(4, 4)
    es = np.array(list(det.box_size)) / np.array(list(det.virtual_element_number))
    local = np.array([det.obb.border_min[0] + (i + 0.5) * es[0], det.obb.border_min[1] + (j + 0.5) * es[1], 0.0, 1.0])
    pixel = (m @ local)[:3]
    s = np.array([src.matrix[3], src.matrix[7], src.matrix[11]], np.float64)
    pm = np.array(list(ph.obb.matrix), np.float64).reshape(4, 4)
    inv = np.linalg.inv(pm)
    a = (inv @ np.append(s, 1.0))[:3]
    b = (inv @ np.append(pixel, 1.0))[:3]
    n = np.array(list(ph.number_of_voxels))
    vs = np.array(list(ph.voxel_sizes))
    bmin = np.array(list(ph.obb.border_min))
    labels = np.ctypeslib.as_array(ph.labels, (int(n.prod()),))
    length = np.linalg.norm(b - a)
    ts = (np.arange(int(length / step)) + 0.5) / int(length / step)
    pts = a[None, :] + ts[:, None] * (b - a)[None, :]
    idx = np.floor((pts - bmin) / vs).astype(np.int64)
    ok = np.all((idx >= 0) & (idx < n), axis=1)
    lab = labels[idx[ok, 0] + idx[ok, 1] * n[0] + idx[ok, 2] * n[0] * n[1]]
    return float(geo.mu[lab].sum() * length / len(ts))


def test_line_integrals_match_ray_sampling(geometry):
    from ggems_b200.scatter import random_phantom
    rng = np.random.default_rng(4)
    labels = random_phantom(rng)
    src, ph, det = geometry.projection(37.0, labels, 0)
    L = geometry.line_integrals(src, ph, det)
    assert L.max() > 1.0
    for i, j in ((32, 32), (10, 40), (50, 20), (31, 5), (0, 0)):
        ref = _sampled_line_integral(geometry, src, ph, det, i, j)
        assert abs(L[j, i] - ref) <= 0.01 * max(ref, 0.05), (i, j, L[j, i], ref)


def test_batched_inputs_match_single_projections(geometry):
    """gg_line_integrals_batch (one phantom, several angles) writes (exp(-L), L)
    equal to the single-projection projector's L."""
    from ggems_b200.scatter import random_phantom
    labels = random_phantom(np.random.default_rng(8))
    projs = [(a, labels) for a in (0.0, 33.0, 90.0, 211.5)]
    x = geometry.network_inputs(projs)
    for k, (angle, lab) in enumerate(projs):
        L = geometry.line_integrals(*geometry.projection(angle, lab, 0))
        assert np.array_equal(x[k, ..., 1], L)
        np.testing.assert_allclose(x[k, ..., 0], np.exp(-L), rtol=2e-6, atol=0)


def test_projector_primary_matches_mc_primary(geometry):
    """exp(-L) (projector) vs total - scatter (MC) at 60 keV: same shape."""
    from ggems_b200.scatter import random_phantom
    rng = np.random.default_rng(5)
    projs = [(float(a), random_phantom(rng)) for a in (0.0, 120.0)]
    total, scatter = geometry.simulate(projs, 4_000_000)
    for k, (angle, labels) in enumerate(projs):
        src, ph, det = geometry.projection(angle, labels, 0)
        T = np.exp(-geometry.line_integrals(src, ph, det))
        primary = total[k] - scatter[k]
        assert scatter[k].sum() > 0 and primary.sum() > 0
        c = np.corrcoef(T.ravel(), primary.ravel())[0, 1]
        print("projection %d: corr(exp(-L), MC primary) = %.4f" % (k, c))
        assert c > 0.97


def test_surrogate_beats_low_count_mc(geometry, torch):
    """A network trained on MC pairs predicts the scatter of new phantoms closer
    to a high-count reference than a low-count plain MC does; the 5 % judge keeps
    or replaces it per projection."""
    from ggems_b200 import scatter as S
    rng = np.random.default_rng(6)
    side = 64
    train = [(float(rng.uniform(0, 360)), S.random_phantom(rng)) for _ in range(128)]
    _, s_train = geometry.simulate(train, 20_000_000, seed=21)
    x_train = S.make_inputs(geometry, train)
    y_train = S.normalise(s_train, 20_000_000, side)
    net = S.UNet(8, side, seed=2)
    losses = S.train(net, x_train, y_train, epochs=30, lr=1e-3)
    test = [(float(rng.uniform(0, 360)), S.random_phantom(rng)) for _ in range(8)]
    _, s_ref = geometry.simulate(test, 400_000_000, seed=22)
    _, s_low = geometry.simulate(test, 1_000_000, seed=23)
    ref = S.normalise(s_ref, 400_000_000, side)
    low = S.normalise(s_low, 1_000_000, side)
    pred = S.predict(net, S.make_inputs(geometry, test))
    final, used = S.judge(pred, low)
    e_net = np.mean([S.relative_error(p, r) for p, r in zip(pred, ref)])
    e_low = np.mean([S.relative_error(m, r) for m, r in zip(low, ref)])
    e_fin = np.mean([S.relative_error(f, r) for f, r in zip(final, ref)])
    print("surrogate: loss %.4f -> %.4f; error vs reference: network %.3f, low-count MC %.3f, judged %.3f "
          "(kept %d/8)" % (losses[0], np.mean(losses[-10:]), e_net, e_low, e_fin, (used == S.JUDGE_NETWORK).sum()))
    assert np.mean(losses[-10:]) < losses[0]
    assert e_net < 0.5 * e_low
    assert e_fin <= e_low + 1e-9
    net.close()


def test_device_inputs_match_host_inputs(geometry, torch):
    """The projector writes the same network inputs into device memory as into
    a host array."""
    from ggems_b200 import scatter as S
    rng = np.random.default_rng(10)
    projs = [(float(rng.uniform(0, 360)), S.random_phantom(rng)) for _ in range(3)]
    projs += [(float(rng.uniform(0, 360)), projs[0][1]) for _ in range(2)]
    host = S.make_inputs(geometry, projs)
    dev = S.make_inputs(geometry, projs, device=True)
    assert torch.is_tensor(dev) and dev.is_cuda
    assert np.array_equal(dev.cpu().numpy(), host)


def test_device_judge_matches_host_judge(geometry, torch):
    """The scan's device path (histograms read on the GPU, normalised, judged
    there) gives the host path's counts, estimates and verdicts."""
    from ggems_b200 import scatter as S
    rng = np.random.default_rng(9)
    side = 64
    projs = [(float(rng.uniform(0, 360)), S.random_phantom(rng)) for _ in range(6)]
    run = geometry.start_simulation(projs, 200_000, seed=31, totals=False)
    _, low_d = geometry.finish_simulation_device(run)
    _, low_h = geometry.simulate(projs, 200_000, seed=31, totals=False)
    assert np.array_equal(low_d.cpu().numpy(), low_h)
    low_h = S.normalise(low_h, 200_000, side)
    low_d = S.normalise(low_d, 200_000, side)
    # estimates 2 % off the MC (kept) and 10 % off (replaced), clear of the 5 % band
    pred = np.stack([low_h[k] * (1.02 if k % 2 == 0 else 1.10) for k in range(len(projs))]).astype(np.float32)
    out_h, used_h = S.judge(pred, low_h)
    out_d, used_d = S.judge_device(torch.from_numpy(pred).cuda(), low_d)
    assert np.array_equal(used_h, used_d)
    assert list(used_h) == [S.JUDGE_NETWORK, S.JUDGE_MC] * 3
    assert np.array_equal(out_d.cpu().numpy(), out_h)


def test_committed_network_predicts_new_phantoms(tmp_path):
    """The trained network shipped with the package (ggems_b200/data/
    unet_scatter256.npz, loaded by bench.py's surrogate measurement) at its own
    size: on new phantoms at random angles its scatter projection is within 3 %
    of the truth on the 16x16 block grid and within 6 % per element at full
    resolution (errors against 2e8-primary MC references with the references'
    own counting noise removed).  In a process of its own: the GGEMS API's
    managers are process-wide and this module's fixture holds a 64^2 geometry."""
    import subprocess
    import textwrap
    code = textwrap.dedent(r'''
        import json, os, sys, tempfile
        import numpy as np
        import torch
        from ggems_b200 import scatter as S
        geo = S.Geometry(256, tempfile.mkdtemp())
        net = S.UNet(4, 256, seed=1)
        S.load_network(net, os.path.join(sys.argv[1], "ggems_b200", "data", "unet_scatter256.npz"))
        rng = np.random.default_rng(31)
        projs = [(float(rng.uniform(0, 360)), S.random_phantom(rng)) for _ in range(4)]
        n_ref = 200_000_000
        _, s_ref = geo.simulate(projs, n_ref, seed=77)
        ref = S.normalise(s_ref, n_ref, 256)
        pred = S.predict(net, S.make_inputs(geo, projs))
        print(json.dumps(S._summary(S._errors(pred, ref, n_ref))))
        net.close()
    ''')
    (tmp_path / "case.py").write_text(code)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, str(tmp_path / "case.py"), root], capture_output=True, text=True,
                         timeout=600, env=dict(os.environ, PYTHONPATH=root))
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-3000:]
    import json
    err = json.loads(out.stdout.strip().splitlines()[-1])
    print("committed network on 4 new phantoms:", err)
    assert err["blocks16"]["mean"] < 0.03
    assert err["full"]["mean"] < 0.06
