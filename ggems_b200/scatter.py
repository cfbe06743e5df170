"""Learned scatter surrogate for CBCT projections (no counterpart in GGEMS).

A 4-level BF16 U-Net (include/ggems_b200.h, gg_unet_*; kernels in
csrc/gg_unet.cu) maps two deterministic maps of a projection -- the primary
transmission exp(-L) and the line integral L through the phantom
(gg_line_integrals) -- to its scatter projection.  The network's fixed input
stage adds wide box means and whole-image means of both maps, so every pixel
sees the phantom-scale context that scatter depends on.  Training pairs come from
the Monte Carlo itself: random phantoms at random angles, all run as the jobs
of ONE batched launch (gg_run_jobs); each job's detector keeps a total and a
scatter histogram, the scatter histogram is the target and
total - scatter the MC primary.  At inference every projection also gets a
low-count plain-MC scatter estimate, which judges the network: when the two
integrated scatter signals differ by more than 5 %, the MC estimate replaces
the network's output.

Geometry (the small water-phantom configuration): 64^3 voxels of 2 mm, random
water ellipsoid with bone and air inserts, 60 keV cone (10 deg) at 1000 mm,
flat GOS panel of side x side elements covering 256 mm at 1500 mm.

    python -m ggems_b200.scatter --pairs 2000 --primaries 1e8 --save net.npz   # train + evaluate, JSON line
    python -m ggems_b200.scatter --load net.npz                                # evaluate a trained network
"""

import argparse
import ctypes as C
import json
import os
import tempfile
import time

import numpy as np

from . import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MATERIALS = os.path.join(ROOT, "ggems_b200", "data", "materials.txt")
PHANTOM_N, PHANTOM_VOXEL = 64, 2.0
ENERGY_MEV = 0.060
JUDGE_TOLERANCE = 0.05
# Launch shape of the judge MC, a persistent kernel that holds its SMs for the
# whole scan: transport CTAs per SM and the photon stash's register budget (0:
# off); GGEMS_B200_JUDGE="blocks,registers" overrides both.  Measured on the
# 360-angle scan (projections/s): 3 CTAs with the 80-register stash 1,030, with
# the 64-register one 906, 4 CTAs with the 64-register stash 893-982, without
# the stash 925; 2 CTAs (more room for the network's kernels beside it) were
# slower still: the network mostly runs after the MC.
JUDGE_BLOCKS_PER_SM, JUDGE_STASH_REGISTERS = (
    tuple(int(v) for v in os.environ["GGEMS_B200_JUDGE"].split(",")) if "GGEMS_B200_JUDGE" in os.environ else (3, 80))


def _lib():
    from ._native import lib
    P = C.POINTER
    sig = {
        "gg_unet_create": (C.c_int, [C.c_int32, C.c_int32, C.c_uint64, P(C.c_void_p)]),
        "gg_unet_destroy": (C.c_int, [C.c_void_p]),
        "gg_unet_parameter_count": (C.c_int64, [C.c_void_p]),
        "gg_unet_get_parameters": (C.c_int, [C.c_void_p, P(C.c_float)]),
        "gg_unet_set_parameters": (C.c_int, [C.c_void_p, P(C.c_float)]),
        "gg_unet_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "gg_unet_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, P(C.c_float), P(C.c_float)]),
        "gg_unet_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, P(C.c_float)]),
        "gg_unet_last_error": (C.c_char_p, []),
        "gg_line_integrals": (C.c_int, [C.c_void_p, P(abi.gg_solid), P(abi.gg_solid), P(C.c_float), P(C.c_float),
                                        C.c_int32, P(C.c_float)]),
        "gg_line_integrals_batch": (C.c_int, [C.c_void_p, P(abi.gg_solid), P(abi.gg_solid), P(C.c_float), C.c_int32,
                                              P(C.c_float), C.c_int32, P(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


class UNet:
    """The surrogate network on the GPU (device arrays: torch CUDA tensors)."""

    def __init__(self, batch, side, seed=1):
        self.lib = _lib()
        self.batch, self.side = batch, side
        h = C.c_void_p()
        self._check(self.lib.gg_unet_create(batch, side, seed, C.byref(h)))
        self.handle = h

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("U-Net: " + self.lib.gg_unet_last_error().decode())

    def close(self):
        if self.handle:
            self.lib.gg_unet_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def parameter_count(self):
        return int(self.lib.gg_unet_parameter_count(self.handle))

    def parameters(self):
        p = np.zeros(self.parameter_count(), np.float32)
        self._check(self.lib.gg_unet_get_parameters(self.handle, abi.ptr(p, C.c_float)))
        return p

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.gg_unet_set_parameters(self.handle, abi.ptr(p, C.c_float)))

    @staticmethod
    def _ready(*tensors):
        """The network runs on its own stream: wait for the work of torch's
        current stream (e.g. the copies that filled the inputs) first."""
        import torch
        torch.cuda.current_stream(tensors[0].device).synchronize()

    def forward(self, x):
        """x: CUDA float32 [batch, side, side, 2] -> CUDA float32 [batch, side, side]."""
        import torch
        y = torch.empty((self.batch, self.side, self.side), dtype=torch.float32, device=x.device)
        self._ready(x, y)
        self._check(self.lib.gg_unet_forward(self.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())))
        return y

    def gradients(self, x, t):
        self._ready(x, t)
        g = np.zeros(self.parameter_count(), np.float32)
        loss = C.c_float()
        self._check(self.lib.gg_unet_gradients(self.handle, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()),
                                               C.byref(loss), abi.ptr(g, C.c_float)))
        return loss.value, g

    def train_step(self, x, t, lr):
        self._ready(x, t)
        loss = C.c_float()
        self._check(self.lib.gg_unet_train_step(self.handle, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()), lr,
                                                C.byref(loss)))
        return loss.value


# ---------------------------------------------------------------- geometry --
def random_phantom(rng, n=PHANTOM_N, voxel=PHANTOM_VOXEL):
    """uint8 labels (z, y, x): 0 air, 1 water, 2 bone 1.85 -- a water ellipsoid
    of random size with 2-6 random bone or air inserts."""
    c = (np.arange(n, dtype=np.float32) + 0.5) * voxel - n * voxel / 2.0
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    half = n * voxel / 2.0
    ax = rng.uniform(0.55, 0.95, 3) * half
    labels = np.zeros((n, n, n), np.uint8)
    labels[(x / ax[0]) ** 2 + (y / ax[1]) ** 2 + (z / ax[2]) ** 2 <= 1.0] = 1
    for _ in range(int(rng.integers(2, 7))):
        r = rng.uniform(0.08, 0.3, 3) * half
        ctr = rng.uniform(-0.5, 0.5, 3) * ax
        inside = ((x - ctr[0]) / r[0]) ** 2 + ((y - ctr[1]) / r[1]) ** 2 + ((z - ctr[2]) / r[2]) ** 2 <= 1.0
        labels[inside & (labels > 0)] = 2 if rng.uniform() < 0.7 else 0
    return labels


def _rot_z(deg):
    a = np.deg2rad(deg)
    r = np.eye(4, dtype=np.float32)
    r[0, 0], r[0, 1], r[1, 0], r[1, 1] = np.cos(a), -np.sin(a), np.sin(a), np.cos(a)
    return r


class Geometry:
    """Base scene (phantom + flat panel + 60 keV cone) built once through the
    GGEMS API; per-projection geometry = rotation about z + a new phantom."""

    def __init__(self, side, workdir):
        import ggems_b200 as gg
        from .api import lib
        from . import workloads
        self.side = side
        labels = random_phantom(np.random.default_rng(0))
        mhd = workloads.write_mhd(os.path.join(workdir, "phantom.mhd"), labels, (PHANTOM_VOXEL,) * 3)
        rng_file = os.path.join(workdir, "range.txt")
        with open(rng_file, "w") as f:
            f.write("0 0 Air\n1 1 Water\n2 2 Bone185\n")
        gg.GGEMSVerbosity(0)
        gg.GGEMSMaterialsDatabaseManager().set_materials(MATERIALS)
        ph = gg.GGEMSVoxelizedPhantom("phantom")
        ph.set_phantom(mhd, rng_file)
        ph.set_rotation(0.0, 0.0, 0.0, "deg")
        ph.set_position(0.0, 0.0, 0.0, "mm")
        ct = gg.GGEMSCTSystem("panel")
        ct.set_ct_type("flat")
        ct.set_number_of_modules(1, 1)
        ct.set_number_of_detection_elements(side, side, 1)
        es = 256.0 / side
        ct.set_size_of_detection_elements(es, es, 10.0, "mm")
        ct.set_material("GOS")
        ct.set_source_detector_distance(1500.0, "mm")
        ct.set_source_isocenter_distance(1000.0, "mm")
        ct.set_rotation(0.0, 0.0, 0.0, "deg")
        ct.set_threshold(10.0, "keV")
        ct.save(os.path.join(workdir, "projection.mhd"))
        ct.store_scatter(True)
        pm = gg.GGEMSProcessesManager()
        for process in ("Compton", "Photoelectric", "Rayleigh"):
            pm.add_process(process, "gamma", "all")
        pm.set_cross_section_table_number_of_bins(220)
        pm.set_cross_section_table_energy_min(1.0, "keV")
        pm.set_cross_section_table_energy_max(1.0, "MeV")
        gg.GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
        src = gg.GGEMSXRaySource("xray")
        src.set_source_particle_type("gamma")
        src.set_number_of_particles(1000)
        src.set_position(-1000.0, 0.0, 0.0, "mm")
        src.set_rotation(0.0, 0.0, 0.0, "deg")
        src.set_beam_aperture(10.0, "deg")
        src.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
        src.set_monoenergy(ENERGY_MEV * 1000.0, "keV")
        self.gg = gg
        self.ggems = gg.GGEMS()
        self.ggems.initialize(777)
        self.lib = lib
        self.ctx = lib.ggems_device_context(self.ggems.obj, 0)
        # the projector works in a context of its own: its stream does not queue
        # behind the transport launches of self.ctx
        from ._native import lib as native, check
        h = C.c_void_p()
        check(native.gg_context_create(0, C.byref(h)), "gg_context_create")
        self.projector_ctx = h
        self.scene = lib.ggems_scene(self.ggems.obj).contents
        self.source = abi.gg_source()
        assert lib.ggems_source_descriptor(0, C.byref(self.source), None) == 0
        assert self.scene.number_of_solids == 2
        self.phantom = abi.gg_solid()
        C.pointer(self.phantom)[0] = self.scene.solids[0]
        self.detector = abi.gg_solid()
        C.pointer(self.detector)[0] = self.scene.solids[1]
        self.mu = self._mu(self.scene.tables[0])

    @staticmethod
    def _mu(t):
        """Total attenuation per material (mm^-1) at ENERGY_MEV from the navigator's tables."""
        nb, nm = t.number_of_bins, t.number_of_materials
        e = np.ctypeslib.as_array(t.energy_bins, (nb,)).astype(np.float64)
        cs = np.ctypeslib.as_array(t.cross_sections, (3 * nm * nb,)).reshape(3, nm, nb).astype(np.float64)
        total = cs.sum(axis=0)
        return np.array([np.interp(ENERGY_MEV, e, total[m]) for m in range(nm)], np.float32)

    def projection(self, angle, labels, hist_base):
        """(source, phantom solid, detector solid) of one projection; histograms hist_base, +1."""
        base = self.__dict__.get("_base_matrices")
        if base is None:  # the unrotated source and detector frames, as float32 4x4
            base = self._base_matrices = (np.array(list(self.source.matrix), np.float32).reshape(4, 4),
                                          np.array(list(self.detector.obb.matrix), np.float32).reshape(4, 4))
        src = abi.gg_source()
        C.pointer(src)[0] = self.source
        r = _rot_z(angle)
        m = np.ascontiguousarray((r @ base[0]).astype(np.float32))
        C.memmove(src.matrix, m.ctypes.data, 64)
        ph = abi.gg_solid()
        C.pointer(ph)[0] = self.phantom
        ph.labels = abi.ptr(labels, C.c_uint8)
        det = abi.gg_solid()
        C.pointer(det)[0] = self.detector
        m = np.ascontiguousarray((r @ base[1]).astype(np.float32))
        C.memmove(det.obb.matrix, m.ctypes.data, 64)
        det.histogram, det.scatter_histogram = hist_base, hist_base + 1
        return src, ph, det

    def line_integrals(self, src, ph, det):
        out = np.zeros(self.side * self.side, np.float32)
        pos = np.array([src.matrix[3], src.matrix[7], src.matrix[11]], np.float32)
        lib = _lib()
        rc = lib.gg_line_integrals(self.projector_ctx, C.byref(ph), C.byref(det), abi.ptr(pos, C.c_float),
                                   abi.ptr(self.mu, C.c_float), len(self.mu), abi.ptr(out, C.c_float))
        if rc != 0:
            raise RuntimeError(lib.gg_last_error().decode())
        return out.reshape(self.side, self.side)

    def network_inputs(self, projections, device=False):
        """[n, side, side, 2] FP32 network inputs (exp(-L), L): one batched
        projector call per run of projections that share a phantom; a CUDA
        tensor written in place with device=True, else a host array."""
        if device:
            import torch
            out = torch.empty((len(projections), self.side, self.side, 2), dtype=torch.float32, device="cuda")
        else:
            out = np.empty((len(projections), self.side, self.side, 2), np.float32)
        lib = _lib()
        k = 0
        while k < len(projections):
            labels = projections[k][1]
            e = k
            while e < len(projections) and projections[e][1] is labels:
                e += 1
            dets = (abi.gg_solid * (e - k))()
            pos = np.empty((e - k, 3), np.float32)
            ph = None
            for j in range(k, e):
                src, ph, det = self.projection(projections[j][0], labels, 0)
                dets[j - k] = det
                pos[j - k] = (src.matrix[3], src.matrix[7], src.matrix[11])
            target = C.cast(C.c_void_p(out[k:e].data_ptr()), C.POINTER(C.c_float)) if device \
                else abi.ptr(out[k:e], C.c_float)
            rc = lib.gg_line_integrals_batch(self.projector_ctx, C.byref(ph), dets, abi.ptr(pos, C.c_float), e - k,
                                             abi.ptr(self.mu, C.c_float), len(self.mu), target)
            if rc != 0:
                raise RuntimeError(lib.gg_last_error().decode())
            k = e
        return out

    def _states(self, seed):
        """JKISS states of `seed` (seeded once per seed; std::mt19937 over 2^20 slots)."""
        cache = self.__dict__.setdefault("_state_cache", {})
        if seed not in cache:
            import torch  # page-locked, so that the per-launch upload runs at DMA speed
            st = torch.zeros(5 * abi.GG_MAXIMUM_PARTICLES, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
            self.lib.gg_seed_random_states(abi.ptr(st, C.c_uint32), abi.GG_MAXIMUM_PARTICLES, seed, 0)
            cache.clear()
            cache[seed] = st
        return cache[seed]

    def start_simulation(self, projections, primaries, seed=777, totals=True):
        """Launch the projections (list of (angle, labels)) as the jobs of one
        asynchronous launch; finish_simulation() waits and reads the histograms.
        The random streams are GGEMS's seeding of `seed`, or with seed=None
        those the context's previous run left.
        With totals=False every job's total histogram is one shared scratch
        histogram (the 5 % check needs scatter only)."""
        from ._native import _job_array, check
        n = len(projections)
        keep, jobs = [], []
        for k, (angle, labels) in enumerate(projections):
            src, ph, det = self.projection(angle, labels, 2 * k if totals else 0)
            if not totals:
                det.scatter_histogram = 1 + k
            arr = (abi.gg_solid * 2)(ph, det)
            keep.append((src, arr, labels))
            jobs.append((src, primaries, arr))
        nh = 2 * n if totals else n + 1
        sizes = np.full(nh, self.side * self.side, np.int32)
        sc = abi.gg_scene()
        C.pointer(sc)[0] = self.scene
        sc.number_of_histograms = nh
        sc.histogram_sizes = abi.ptr(sizes, C.c_int32)
        lib = self.lib
        check(lib.gg_upload_scene(self.ctx, C.byref(sc)), "gg_upload_scene")
        if seed is not None:  # else the context's streams carry on from its previous run, as GGEMS's do
            states = self._states(seed)
            check(lib.gg_set_random_states(self.ctx, abi.ptr(states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES), "states")
        arr, kp = _job_array(jobs)
        check(lib.gg_run_jobs(self.ctx, arr, n), "gg_run_jobs")
        return dict(n=n, nh=nh, totals=totals, keep=(keep, jobs, arr, kp, sizes, sc))

    def finish_simulation(self, run):
        """(total, scatter) histograms [n, side, side] as float32 counts (total
        None without totals)."""
        from ._native import check
        lib, n, side = self.lib, run["n"], self.side
        check(lib.gg_synchronize(self.ctx), "gg_synchronize")
        hist = np.zeros((run["nh"], side * side), np.int32)
        rows = (C.POINTER(C.c_int32) * run["nh"])(*[abi.ptr(hist[i], C.c_int32) for i in range(run["nh"])])
        tb = abi.gg_tally_buffers()
        tb.histograms = C.cast(rows, C.POINTER(C.POINTER(C.c_int32)))
        check(lib.gg_read_tallies(self.ctx, C.byref(tb)), "gg_read_tallies")
        ms, la = C.c_float(), C.c_int64()
        lib.gg_last_run_stats(self.ctx, C.byref(ms), C.byref(la))
        self.last_ms = ms.value
        if not run["totals"]:
            return None, hist[1:].reshape(n, side, side).astype(np.float32)
        h = hist.reshape(n, 2, side, side)
        return h[:, 0].astype(np.float32), h[:, 1].astype(np.float32)

    def finish_simulation_device(self, run):
        """finish_simulation without the copy to the host: CUDA float32 tensors
        [n, side, side] built from the context's histogram buffers."""
        import torch
        from ._native import check
        from .distributed import device_tallies
        lib, n, side = self.lib, run["n"], self.side
        check(lib.gg_synchronize(self.ctx), "gg_synchronize")
        ms, la = C.c_float(), C.c_int64()
        lib.gg_last_run_stats(self.ctx, C.byref(ms), C.byref(la))
        self.last_ms = ms.value
        hist = device_tallies(self.ctx)[:run["nh"]]
        if not run["totals"]:
            return None, torch.stack(hist[1:]).to(torch.float32).view(n, side, side)
        h = torch.stack(hist).to(torch.float32).view(n, 2, side, side)
        return h[:, 0], h[:, 1]

    def simulate(self, projections, primaries, seed=777, totals=True):
        """start_simulation + finish_simulation."""
        return self.finish_simulation(self.start_simulation(projections, primaries, seed, totals))


def normalise(counts, primaries, side):
    """Counts -> per-primary signal times the number of elements."""
    return counts * (float(side * side) / float(primaries))


def block_mean(img, blocks=16):
    """Scatter is a low-frequency signal: mean over a blocks x blocks grid."""
    img = np.asarray(img, np.float64)
    n = img.shape[-1]
    b = n // blocks
    return img.reshape(img.shape[:-2] + (blocks, b, blocks, b)).mean(axis=(-3, -1))


def smooth(img, blocks=32):
    """Block mean expanded back to full resolution (training targets)."""
    n = np.asarray(img).shape[-1]
    b = n // blocks
    return np.repeat(np.repeat(block_mean(img, blocks), b, axis=-2), b, axis=-1).astype(np.float32)


def make_inputs(geometry, projections, device=False):
    """[n, side, side, 2]: primary transmission exp(-L) and line integral L
    (a CUDA tensor with device=True, else a host array)."""
    return geometry.network_inputs(projections, device)


# Verdicts of the judge, per projection.
JUDGE_MC, JUDGE_RESCALED, JUDGE_NETWORK = 0, 1, 2


def judge(predicted, low_count_mc, tolerance=JUDGE_TOLERANCE):
    """The judge as specified, per projection against the low-count plain-MC
    estimate: JUDGE_NETWORK when the network's integrated scatter is within
    `tolerance` of the MC's (the network's output is kept), else JUDGE_MC (the
    MC estimate replaces it).  Returns (outputs, verdicts)."""
    out, verdict = [], []
    for p, m in zip(predicted, low_count_mc):
        sp, sm = float(p.sum()), float(m.sum())
        keep = abs(sp - sm) <= tolerance * max(sm, 1e-12)
        out.append(p if keep else m)
        verdict.append(JUDGE_NETWORK if keep else JUDGE_MC)
    return np.stack(out), np.array(verdict)


def judge_device(predicted, low_count_mc, tolerance=JUDGE_TOLERANCE):
    """judge() on CUDA tensors [n, side, side] (integrated scatter summed in
    FP64): (outputs as a CUDA tensor, verdicts as a host array)."""
    import torch
    sp = predicted.to(torch.float64).sum(dim=(1, 2))
    sm = low_count_mc.to(torch.float64).sum(dim=(1, 2))
    keep = (sp - sm).abs() <= tolerance * sm.clamp(min=1e-12)
    out = torch.where(keep[:, None, None], predicted, low_count_mc)
    return out, np.where(keep.cpu().numpy(), JUDGE_NETWORK, JUDGE_MC)


def judge_rescaled(predicted, low_count_mc, primaries, side=None, tolerance=JUDGE_TOLERANCE, shape_blocks=4,
                   shape_p=1e-3):
    """A variant of the judge with a third verdict (reported beside the judge
    as specified, not in its place): a projection outside the 5 % band whose
    network shape agrees with the MC's counts on a shape_blocks x shape_blocks
    grid (chi-square of the MC's counts per block against the network rescaled
    to the MC's integral, Poisson variances, shape_blocks^2 - 1 degrees of
    freedom, p >= shape_p) gets the network rescaled to the MC's integral
    (JUDGE_RESCALED) instead of the MC estimate; the MC's integral carries
    ~1/sqrt(counts) noise, about 2 % at 1e6 primaries.  Returns (outputs,
    verdicts)."""
    from scipy.stats import chi2
    out, verdict = [], []
    limit = chi2.isf(shape_p, shape_blocks * shape_blocks - 1)
    final, used = judge(predicted, low_count_mc, tolerance)
    for p, m, f, v in zip(predicted, low_count_mc, final, used):
        sp, sm = float(p.sum()), float(m.sum())
        if v == JUDGE_NETWORK or sp <= 0.0 or sm <= 0.0:
            out.append(f)
            verdict.append(v)
            continue
        n = side if side is not None else p.shape[-1]
        to_counts = float(primaries) / float(n * n)  # inverse of normalise()
        counts = block_mean(m, shape_blocks) * (n // shape_blocks) ** 2 * to_counts
        expected = block_mean(p, shape_blocks) * (n // shape_blocks) ** 2 * to_counts * (sm / sp)
        stat = float((((counts - expected) ** 2) / np.maximum(expected, 1.0)).sum())
        if stat <= limit:
            out.append(p * (sm / sp))
            verdict.append(JUDGE_RESCALED)
        else:
            out.append(m)
            verdict.append(JUDGE_MC)
    return np.stack(out), np.array(verdict)


def relative_error(a, ref, blocks=16):
    """Relative L2 error of a scatter projection, on a blocks x blocks grid of
    block means (blocks=None: per element, at full resolution)."""
    if blocks is not None:
        a, ref = block_mean(a, blocks), block_mean(ref, blocks)
    a, ref = np.asarray(a, np.float64), np.asarray(ref, np.float64)
    return float(np.linalg.norm(a - ref) / max(np.linalg.norm(ref), 1e-30))


def reference_noise(ref, primaries, blocks=16):
    """Relative L2 norm of a reference's own counting noise, in the units of
    relative_error: a reference of `primaries` primaries (normalised counts
    `ref`) has Poisson variance counts x (side^2 / primaries)^2 per element;
    block means divide it by the block's element count."""
    ref = np.asarray(ref, np.float64)
    side = ref.shape[-1]
    scale = float(side * side) / float(primaries)
    var = ref * scale  # = counts * scale^2
    if blocks is not None:
        b = side // blocks
        var = block_mean(var, blocks) / (b * b)
        ref = block_mean(ref, blocks)
    return float(np.sqrt(var.sum()) / max(np.linalg.norm(ref), 1e-30))


def error_vs_truth(err, floor):
    """An estimate's error against the (unknown) true scatter image, from its
    error against a reference whose own noise is `floor`: the two errors are
    independent, so err^2 = true_err^2 + floor^2."""
    return float(np.sqrt(max(err * err - floor * floor, 0.0)))


def learning_rate(step, total, lr, warmup=100, floor=0.01):
    """Linear warm-up over `warmup` steps, then cosine decay to floor * lr."""
    if step < warmup:
        return lr * (step + 1) / warmup
    t = (step - warmup) / max(total - warmup, 1)
    return lr * (floor + (1.0 - floor) * 0.5 * (1.0 + np.cos(np.pi * min(t, 1.0))))


def train(net, inputs, targets, epochs, lr=1e-3, seed=0):
    """Adam on (inputs, smoothed targets / their mean) with a warm-up + cosine
    learning-rate schedule; the mean is kept in net.target_scale and applied by
    predict()."""
    import torch
    n = len(inputs)
    B = net.batch
    rng = np.random.default_rng(seed)
    targets = smooth(targets)
    net.target_scale = float(max(targets.mean(), 1e-30))
    X = torch.from_numpy(inputs).cuda()
    Y = torch.from_numpy((targets / net.target_scale).astype(np.float32)).cuda()
    losses = []
    per_epoch = n // B
    total = epochs * per_epoch
    for epoch in range(epochs):
        order = rng.permutation(n)
        for s in range(0, n - B + 1, B):
            idx = torch.from_numpy(order[s:s + B]).cuda()
            xb = X.index_select(0, idx).contiguous()
            yb = Y.index_select(0, idx).contiguous()
            losses.append(net.train_step(xb, yb, learning_rate(len(losses), total, lr)))
    return losses


def predict_device(net, inputs):
    """The network's scatter estimates of `inputs` [n, side, side, 2] (a host
    array, copied up once, or a CUDA tensor) as a CUDA tensor: the forward
    passes back to back over batches of net.batch."""
    import torch
    B, n = net.batch, len(inputs)
    X = inputs if torch.is_tensor(inputs) else torch.from_numpy(np.ascontiguousarray(inputs, np.float32)).cuda()
    out = torch.empty((n, net.side, net.side), dtype=torch.float32, device=X.device)
    for s in range(0, n, B):
        m = min(B, n - s)
        xb = X[s:s + B] if m == B else torch.cat([X[s:], X.new_zeros((B - m,) + tuple(X.shape[1:]))])
        out[s:s + m] = net.forward(xb)[:m]
    return out * getattr(net, "target_scale", 1.0)


def predict(net, inputs):
    """predict_device, copied to the host."""
    return predict_device(net, inputs).cpu().numpy()


# (C_in, C_out, down-sampling factor) of the 14 3x3 convolutions (csrc/gg_unet.cu)
LAYERS = [(16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 128, 4), (128, 128, 4), (128, 256, 8),
          (256, 256, 8), (384, 128, 4), (128, 128, 4), (192, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1)]


def forward_flops(side, batch):
    """Tensor-core FLOPs of one forward pass: sum over the convolutions of
    2 * 9 * C_in * C_out * pixels (the first layer's 16 input channels are the
    padded width the tensor cores compute)."""
    return sum(2 * 9 * ci * co * batch * (side // d) ** 2 for ci, co, d in LAYERS)


def time_network(side=256, batch=8, repeats=20):
    """Device time of the forward pass (CUDA events) and its TFLOP/s."""
    import torch
    net = UNet(batch, side, seed=1)
    x = torch.rand((batch, side, side, 2), device="cuda")
    for _ in range(3):
        net.forward(x)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(repeats):
        net.forward(x)
    stop.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / repeats
    # one training step: forward, backward (data and weight gradients: twice the
    # forward's FLOP) and the Adam update
    t = torch.rand((batch, side, side), device="cuda")
    for _ in range(3):
        net.train_step(x, t, 1e-4)
    torch.cuda.synchronize()
    start.record()
    for _ in range(repeats):
        net.train_step(x, t, 1e-4)
    stop.record()
    torch.cuda.synchronize()
    train_ms = start.elapsed_time(stop) / repeats
    net.close()
    return ms, forward_flops(side, batch) / (ms * 1e-3) / 1e12, train_ms


def _conv_weight_mask(count):
    """True at the 3x3 convolution weights of the parameter vector (layer by
    layer: weights [9][C_out][C_in], then biases; then the 1x1 output layer)."""
    mask = np.zeros(count, bool)
    off = 0
    for ci, co, _ in LAYERS:
        mask[off:off + 9 * ci * co] = True
        off += 9 * ci * co + co
    return mask


def save_network(net, path):
    """The trained network: the convolution weights as BF16 bits (the forward
    pass rounds the FP32 master weights to BF16 the same way, round to nearest
    even, so inference is unchanged), biases and the output layer in FP32."""
    p = net.parameters()
    mask = _conv_weight_mask(len(p))
    bits = p[mask].view(np.uint32).astype(np.uint64)
    bf16 = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)
    np.savez_compressed(path, conv_weights_bf16=bf16, other_fp32=p[~mask],
                        target_scale=np.float64(getattr(net, "target_scale", 1.0)))


def load_network(net, path):
    z = np.load(path)
    if "parameters" in z.files:
        p = z["parameters"]
    else:
        p = np.zeros(net.parameter_count(), np.float32)
        mask = _conv_weight_mask(len(p))
        p[mask] = (z["conv_weights_bf16"].astype(np.uint32) << 16).view(np.float32)
        p[~mask] = z["other_fp32"]
    net.set_parameters(p)
    net.target_scale = float(z["target_scale"])


def surrogate_pipeline(geo, net, projections, judge_primaries, seed):
    """The surrogate at inference: per projection the deterministic inputs and
    the network's scatter estimate, the low-count plain-MC estimate of all
    projections (one batched launch per chunk of jobs) and the 5 % judge.
    The judge MC seeds its streams with `seed`, or continues the transport
    context's streams with seed=None.  Returns (final, prediction, low-count
    MC, verdicts, seconds); the variant with rescaling (judge_rescaled) is
    left in geo.last_rescaled."""
    import torch
    torch.cuda.synchronize()
    t = [time.perf_counter()]
    # The network's inputs first: the projector's many small kernels run alone
    # on the GPU in milliseconds, where beside the persistent judge MC they
    # would crawl (they could take 0.3-0.9 s of a 0.35 s scan, depending on
    # which kernels reached the SMs first).  Then the judge MC, a persistent
    # launch that holds the SMs (JUDGE_BLOCKS_PER_SM, JUDGE_STASH_REGISTERS);
    # the network's kernels follow it.
    x = make_inputs(geo, projections, device=True)
    t.append(time.perf_counter())
    from ._native import check
    bps, lanes, ratio4 = C.c_int32(), C.c_int32(), C.c_int32()
    stash, swap, rnd = C.c_int32(), C.c_int32(), C.c_int32()
    check(geo.lib.gg_get_transport_tuning(geo.ctx, C.byref(bps), C.byref(lanes), C.byref(ratio4)), "tuning")
    check(geo.lib.gg_get_transport_stash(geo.ctx, C.byref(stash), C.byref(swap), C.byref(rnd)), "stash")
    check(geo.lib.gg_set_transport_tuning(geo.ctx, JUDGE_BLOCKS_PER_SM, lanes.value, ratio4.value), "tuning")
    check(geo.lib.gg_set_transport_stash(geo.ctx, JUDGE_STASH_REGISTERS, swap.value, rnd.value), "stash")
    try:
        run = geo.start_simulation(projections, int(judge_primaries), seed=seed, totals=False)
    finally:
        check(geo.lib.gg_set_transport_tuning(geo.ctx, bps.value, lanes.value, ratio4.value), "tuning")
        check(geo.lib.gg_set_transport_stash(geo.ctx, stash.value, swap.value, rnd.value), "stash")
    t.append(time.perf_counter())
    pred_d = predict_device(net, x)
    t.append(time.perf_counter())
    _, low_d = geo.finish_simulation_device(run)
    low_d = normalise(low_d, judge_primaries, geo.side)
    t.append(time.perf_counter())
    final_d, used = judge_device(pred_d, low_d)
    # the scan's output, on the host (page-locked: torch's host allocator keeps
    # the block for the next scan once this one is released)
    final = torch.empty(final_d.shape, dtype=final_d.dtype, pin_memory=True)
    final.copy_(final_d)
    final = final.numpy()
    t.append(time.perf_counter())
    pred, low = pred_d.cpu().numpy(), low_d.cpu().numpy()
    geo.last_rescaled = judge_rescaled(pred, low, judge_primaries, geo.side)
    geo.last_breakdown = {"inputs": t[1] - t[0], "judge_mc_launch": t[2] - t[1], "network": t[3] - t[2],
                          "judge_mc_wait": t[4] - t[3], "judge": t[5] - t[4]}
    return final, pred, low, used, t[-1] - t[0]


METRIC = "scatter projections/s (surrogate + 1e6-primary MC judge vs plain MC at <=5% error)"
ERROR_GRIDS = (("blocks16", 16), ("full", None))


def _errors(est, refs, ref_primaries):
    """Per projection: error against the reference and against the truth (the
    reference's counting noise removed), on the 16x16 block grid and at full
    resolution."""
    out = {}
    for name, blocks in ERROR_GRIDS:
        raw = [relative_error(e, r, blocks) for e, r in zip(est, refs)]
        floor = [reference_noise(r, ref_primaries, blocks) for r in refs]
        out[name] = {"raw": raw, "floor": floor, "truth": [error_vs_truth(a, b) for a, b in zip(raw, floor)]}
    return out


def _summary(err):
    return {name: {"mean": float(np.mean(e["truth"])), "max": float(np.max(e["truth"])),
                   "mean_raw": float(np.mean(e["raw"])), "reference_noise": float(np.mean(e["floor"]))}
            for name, e in err.items()}


def evaluate(geo, net, rng, args, simulate_all):
    """The surrogate's measurement: a CBCT scan of a new phantom at args.angles
    angles through the whole pipeline (timed), its errors against
    reference_primaries-primary references on every args.reference_every-th
    angle, and plain MC timed at the primaries that give 5 % error on the same
    metric.  Optionally args.test new phantoms at random angles as well."""
    import torch
    side = geo.side
    out = {"metric": METRIC, "unit": "projections/s", "higher_is_better": True}
    if args.test > 0:
        test_projs = [(float(rng.uniform(0, 360)), random_phantom(rng)) for _ in range(args.test)]
        _, s_ref, _ = simulate_all(test_projs, args.reference_primaries)
        ref = normalise(s_ref, args.reference_primaries, side)
        final, pred, low, used, _ = surrogate_pipeline(geo, net, test_projs, args.judge_primaries, 1234 + args.seed)
        resc, _ = geo.last_rescaled
        out["new_phantoms"] = {
            "projections": args.test, "network_kept": float((used == JUDGE_NETWORK).mean()),
            "judged": _summary(_errors(final, ref, args.reference_primaries)),
            "network": _summary(_errors(pred, ref, args.reference_primaries)),
            "judge_mc": _summary(_errors(low, ref, args.reference_primaries)),
            "judged_with_rescaling": _summary(_errors(resc, ref, args.reference_primaries))}
    phantom = random_phantom(rng)
    scan = [(360.0 * k / args.angles, phantom) for k in range(args.angles)]
    # warm-up at the scan's own size: device pools, job tables and pinned buffers
    # reach their working sizes before the timed scan, whose judge MC then
    # continues the warm-up's random streams on the device (a simulation seeds
    # once, as GGEMS::Initialize does)
    surrogate_pipeline(geo, net, scan, args.judge_primaries, 4321 + args.seed)
    s_final, s_pred, s_low, s_used, t_scan = surrogate_pipeline(geo, net, scan, args.judge_primaries, None)
    s_resc, s_resc_used = geo.last_rescaled
    breakdown = {k: v / args.angles * 1e3 for k, v in geo.last_breakdown.items()}
    picked = list(range(0, args.angles, args.reference_every))
    _, s_ref_scan, _ = simulate_all([scan[k] for k in picked], args.reference_primaries)
    ref_scan = normalise(s_ref_scan, args.reference_primaries, side)
    e_final = _errors([s_final[k] for k in picked], ref_scan, args.reference_primaries)
    e_pred = _errors([s_pred[k] for k in picked], ref_scan, args.reference_primaries)
    e_low = _errors([s_low[k] for k in picked], ref_scan, args.reference_primaries)
    e_resc = _errors([s_resc[k] for k in picked], ref_scan, args.reference_primaries)
    sur_per_s = args.angles / t_scan
    # Plain MC at 5 %: it is unbiased, so its error against the truth falls as
    # 1/sqrt(primaries) from the judge MC's (measured on the same angles).  Its
    # rate is the device time of one batched launch of plain_angles angles at
    # the block-grid count (no host overhead counted against it); the
    # full-resolution count is far larger and uses that measured rate.
    n_plain = {name: float(args.judge_primaries * (float(np.mean(e_low[name]["truth"])) / 0.05) ** 2)
               for name, _ in ERROR_GRIDS}
    angles = [scan[k] for k in picked[:args.plain_angles]]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, s_plain, plain_ms = simulate_all(angles, n_plain["blocks16"])
    t_plain = time.perf_counter() - t0
    rate = len(angles) * n_plain["blocks16"] / (plain_ms * 1e-3)
    e_plain = _errors(normalise(s_plain, n_plain["blocks16"], side), ref_scan[:len(angles)],
                      args.reference_primaries)
    plain = {"mc_primaries_per_s": rate, "projections_timed": len(angles),
             "wall_projections_per_s": len(angles) / t_plain}
    for name, _ in ERROR_GRIDS:
        per_s = rate / n_plain[name]
        plain[name] = {"primaries_for_5pct": n_plain[name], "projections_per_s": per_s,
                       "speedup": sur_per_s / per_s,
                       "error_mean": float(np.mean(e_plain[name]["truth"])) if name == "blocks16" else None}

    def integral_errors(est, refs):
        return [abs(float(e.sum()) - float(r.sum())) / float(r.sum()) for e, r in zip(est, refs)]
    net_int = integral_errors([s_pred[k] for k in picked], ref_scan)
    low_int = integral_errors([s_low[k] for k in picked], ref_scan)
    out.update({
        "value": sur_per_s,
        "judge": "as specified: network kept within 5 % of the judge MC's integrated scatter, else replaced by it",
        "scan": {"angles": args.angles, "seconds": t_scan, "network_kept": float((s_used == JUDGE_NETWORK).mean()),
                 "replaced_by_mc": float((s_used == JUDGE_MC).mean()), "reference_angles": len(picked),
                 "ms_per_projection": breakdown,
                 "error": _summary(e_final), "network_error": _summary(e_pred), "judge_mc_error": _summary(e_low)},
        "plain_mc": plain,
        "with_rescaling": {"judge": "judge_rescaled: outside the 5 % band, a network of the right shape is rescaled "
                                    "to the MC's integral instead of replaced",
                           "network_kept": float((s_resc_used == JUDGE_NETWORK).mean()),
                           "rescaled": float((s_resc_used == JUDGE_RESCALED).mean()),
                           "error": _summary(e_resc)},
        "integrated_scatter_error": {"network_rms": float(np.sqrt(np.mean(np.square(net_int)))),
                                     "network_max": float(np.max(net_int)),
                                     "judge_mc_rms": float(np.sqrt(np.mean(np.square(low_int)))),
                                     "projections": len(net_int)},
        "errors": "relative L2 against the truth: error against the reference with the reference's own counting "
                  "noise removed in quadrature (raw errors beside); 'blocks16' on a 16x16 grid of block means, "
                  "'full' per detector element at full resolution; the network's training targets are 32x32 "
                  "block means"})
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--side", type=int, default=256)
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--primaries", type=float, default=1e8, help="primaries per training target")
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--test", type=int, default=16, help="test projections (new phantoms, random angles)")
    ap.add_argument("--angles", type=int, default=360, help="inference angles of one new phantom")
    ap.add_argument("--reference-every", type=int, default=10, help="1e9-primary reference on every n-th angle")
    ap.add_argument("--judge-primaries", type=float, default=1e6)
    ap.add_argument("--reference-primaries", type=float, default=1e9)
    ap.add_argument("--chunk", type=int, default=64, help="projections per batched MC launch")
    ap.add_argument("--save", help="write the trained network (.npz)")
    ap.add_argument("--load", help="skip data generation and training: load a trained network (.npz)")
    ap.add_argument("--seed", type=int, default=11, help="seed of the phantoms, angles and MC streams")
    ap.add_argument("--network-only", action="store_true", help="time the network's forward pass and training step only")
    ap.add_argument("--plain-angles", type=int, default=16, help="scan angles plain MC is timed on")
    ap.add_argument("--json-out", help="also write the JSON line to this file")
    args = ap.parse_args(argv)
    if args.network_only:
        ms, tflops, train_ms = time_network(args.side, args.batch)
        peaks = None
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        peak = peaks["bf16_tflops"] if peaks else 1590.0
        print(json.dumps({"metric": "U-Net forward TFLOP/s", "side": args.side, "batch": args.batch,
                          "ms_per_forward": ms, "ms_per_projection": ms / args.batch,
                          "gflop_per_forward": forward_flops(args.side, args.batch) / 1e9,
                          "tflops": tflops, "peak_tflops": peak, "frac": tflops / peak,
                          "ms_per_train_step": train_ms,
                          "train_tflops": 3 * forward_flops(args.side, args.batch) / (train_ms * 1e-3) / 1e12,
                          "peak_source": "measured" if peaks else "fallback"}), flush=True)
        return 0
    import torch  # (CUDA memory for the network's device arrays)
    work = tempfile.mkdtemp(prefix="ggems_scatter_")
    geo = Geometry(args.side, work)
    rng = np.random.default_rng(args.seed)
    side = args.side

    def simulate_all(projs, primaries):
        tot, sca, ms = [], [], 0.0
        for s in range(0, len(projs), args.chunk):
            t, sc = geo.simulate(projs[s:s + args.chunk], int(primaries), seed=int(rng.integers(1, 2 ** 31)))
            tot.append(t)
            sca.append(sc)
            ms += geo.last_ms
        return np.concatenate(tot), np.concatenate(sca), ms

    net = UNet(args.batch, side, seed=3)
    t_data = t_train = mc_ms = 0.0
    losses = []
    if args.load:
        load_network(net, args.load)
    else:
        t0 = time.time()
        train_projs = [(float(rng.uniform(0, 360)), random_phantom(rng)) for _ in range(args.pairs)]
        _, s_train, mc_ms = simulate_all(train_projs, args.primaries)
        x_train = make_inputs(geo, train_projs)
        y_train = normalise(s_train, args.primaries, side)
        t_data = time.time() - t0
        del train_projs
        t0 = time.time()
        losses = train(net, x_train, y_train, args.epochs)
        t_train = time.time() - t0
        del x_train, y_train
        if args.save:
            save_network(net, args.save)
    out = evaluate(geo, net, rng, args, simulate_all)
    out["config"] = {"side": side, "pairs": args.pairs, "target_primaries": args.primaries, "epochs": args.epochs,
                     "judge_primaries": args.judge_primaries, "reference_primaries": args.reference_primaries,
                     "loaded": bool(args.load), "network": os.path.basename(args.load) if args.load else None}
    out["times_s"] = {"data": t_data, "train": t_train, "train_mc_ms": mc_ms}
    out["final_loss"] = float(np.mean(losses[-20:])) if losses else None
    line = json.dumps(out)
    print(line, flush=True)
    if args.json_out:
        with open(args.json_out, "w") as f:
            f.write(line + "\n")
    net.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
