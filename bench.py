#!/usr/bin/env python
"""Benchmark of the GGEMS photon path on B200: primaries/s on the 256^3 CBCT
projection (120 kVp polyenergetic cone beam, 1e8 primaries, flat 512x512 GOS
panel of 0.8 mm at SDD 1500 mm / SID 1000 mm, Compton + photoelectric +
Rayleigh, primary and scatter histograms).

One step = one full CBCT projection of 1e8 primaries (96 batches of up to
2^20 random slots, exactly as GGEMS splits them).  Inputs are synthetic
(seeded phantom generator, synthetic spectrum) in GGEMS's file formats and go
through the GGEMS-compatible API (materials database, voxelized phantom, CT
system, X-ray source, processes, range cuts, initialize).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
For N > 1, launch with torch.distributed.run; every rank runs its own
projection with its own random streams (weak scaling).
"""

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PRIMARIES = 100_000_000
WORKLOAD = "cbct256_120kVp_flat512"


def _rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _ensure_built():
    from ggems_b200 import build
    if not os.path.exists(build.LIB):
        build.build()


def _configure(files, primaries, seed_offset_slots=0):
    """Build the CBCT simulation through the GGEMS-compatible Python API."""
    import ggems_b200 as gg
    mhd, rng_file, spectrum = files
    gg.GGEMSVerbosity(0)
    gg.GGEMSMaterialsDatabaseManager().set_materials(os.path.join(ROOT, "ggems_b200", "data", "materials.txt"))
    phantom = gg.GGEMSVoxelizedPhantom("phantom")
    phantom.set_phantom(mhd, rng_file)
    phantom.set_rotation(0.0, 0.0, 0.0, "deg")
    phantom.set_position(0.0, 0.0, 0.0, "mm")
    ct = gg.GGEMSCTSystem("flat_panel")
    ct.set_ct_type("flat")
    ct.set_number_of_modules(1, 1)
    ct.set_number_of_detection_elements(512, 512, 1)
    ct.set_size_of_detection_elements(0.8, 0.8, 10.0, "mm")
    ct.set_material("GOS")
    ct.set_source_detector_distance(1500.0, "mm")
    ct.set_source_isocenter_distance(1000.0, "mm")
    ct.set_rotation(0.0, 0.0, 0.0, "deg")
    ct.set_threshold(10.0, "keV")
    ct.save(os.path.join(os.path.dirname(mhd), "projection.mhd"))
    ct.store_scatter(True)
    pm = gg.GGEMSProcessesManager()
    pm.add_process("Compton", "gamma", "all")
    pm.add_process("Photoelectric", "gamma", "all")
    pm.add_process("Rayleigh", "gamma", "all")
    pm.set_cross_section_table_number_of_bins(220)
    pm.set_cross_section_table_energy_min(1.0, "keV")
    pm.set_cross_section_table_energy_max(1.0, "MeV")
    gg.GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
    src = gg.GGEMSXRaySource("xray")
    src.set_source_particle_type("gamma")
    src.set_number_of_particles(primaries)
    src.set_position(-1000.0, 0.0, 0.0, "mm")
    src.set_rotation(0.0, 0.0, 0.0, "deg")
    src.set_beam_aperture(11.0, "deg")
    src.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
    src.set_polyenergy(spectrum)
    return gg


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _smi_device(local=0):
    """The nvidia-smi id (index or UUID) of this process's CUDA device `local`."""
    vis = [d.strip() for d in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if d.strip()]
    return vis[local] if local < len(vis) else str(local)


def _profile_value(key):
    """A figure from the committed ncu summary of the transport kernel ("key: value" lines)."""
    path = os.path.join(ROOT, "profiles", "transport_kernel_cbct256.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(key + ":"):
            try:
                return float(line.split(":")[1].split()[0])
            except (IndexError, ValueError):
                return None
    return None


def _profile_traffic():
    """DRAM bytes per transport launch from the committed ncu summary, if present."""
    return _profile_value("dram_bytes_per_full_launch")


def _issue_roofline(primaries_per_s, clocks):
    """The transport kernel's real limit: warp instructions issued per second
    (warp instructions per primary, from the committed ncu summary of this
    workload, x primaries/s) against the issue ceiling of one warp instruction
    per scheduler per cycle (SMs x 4 schedulers x median SM clock sampled during
    the timed region)."""
    per_primary = _profile_value("warp_instructions_per_primary")
    if not per_primary or not clocks or not clocks.get("sm_mhz"):
        return None
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    ceiling = sms * 4 * clocks["sm_mhz"] * 1e6
    achieved = per_primary * primaries_per_s
    return {"bound": "issue", "achieved": achieved / 1e12, "peak": ceiling / 1e12, "unit": "T warp-inst/s",
            "frac": achieved / ceiling, "warp_instructions_per_primary": per_primary, "sms": sms,
            "sm_mhz": clocks["sm_mhz"]}


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return None


def cpu_reference_run(scene_ptr, source, n, threads, kind, states):
    """Run n primaries of the workload on the host with the reference kernels
    (oracle/_ref, GGEMS's own device code compiled for the host) or the oracle
    port, from a copy of `states` (5 x 2^20 JKISS words).  Returns (seconds,
    counts per primary or None)."""
    from ggems_b200 import abi
    import numpy as np
    if kind == "reference":
        lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libgg_ref.so"))
        fn = lib.gg_ref_run
    else:
        lib = C.CDLL(os.path.join(ROOT, "oracle", "_build", "libgg_oracle.so"))
        fn = lib.gg_oracle_run
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.gg_scene), C.POINTER(abi.gg_source), C.c_uint64, C.POINTER(C.c_uint32),
                   C.POINTER(abi.gg_particle_buffers), C.POINTER(abi.gg_tally_buffers), C.c_int]
    sc = scene_ptr.contents
    st = np.array(states, np.uint32, copy=True)
    hs = [int(sc.histogram_sizes[i]) for i in range(sc.number_of_histograms)]
    ds = [int(sc.dose_maps[i].total_number_of_dosels) for i in range(sc.number_of_dose_maps)]
    tallies = abi.Tallies(hs, ds)
    counts = None
    if kind != "reference":
        lib.gg_oracle_counts.argtypes = [C.POINTER(C.c_uint64), C.c_int]
        lib.gg_oracle_counts(None, 1)
    t0 = time.perf_counter()
    rc = fn(scene_ptr, C.byref(source), n, abi.ptr(st, C.c_uint32), None, C.byref(tallies.struct), threads)
    dt = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError("CPU run failed: %d" % rc)
    if kind != "reference":
        cnt = (C.c_uint64 * 5)()
        lib.gg_oracle_counts(cnt, 1)
        counts = [cnt[i] / max(n, 1) for i in range(4)]
    return dt, counts


def _cpu_sample(scene_ptr, source, what):
    """About 10 s of the reference kernels on every host thread for `scene`."""
    kind = _cpu_kind()
    threads = os.cpu_count() or 1
    st = _seed_states(777)
    m = _sample_size(scene_ptr, source, threads, kind, 10.0, st)
    dt, _ = cpu_reference_run(scene_ptr, source, m, threads, kind, st)
    return {"value": m / dt, "unit": "primaries/s", "cores": threads, "kind": kind,
            "sample": "%d primaries of %s (seed 777) on %d host threads, %.1f s, in a process that has not imported "
                      "torch" % (m, what, threads, dt)}


def _cpu_leg_process(args):
    """_cpu_sample of this workload's scene in a process of its own that builds
    the scene through the GGEMS API and imports no torch (it does hold a CUDA
    context: the volume creator and GGEMS::Initialize need one)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--workload", args.workload, "--cpu-leg", "--primaries",
           str(args.primaries)]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE")}
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900, env=env)
    for line in r.stdout.splitlines():
        if line.startswith("{"):
            d = json.loads(line).get("cpu_baseline")
            if d:
                return d
    return {"unavailable": "CPU baseline process failed: " + (r.stderr.strip().splitlines() or ["?"])[-1]}


def _cpu_kind():
    ref = os.path.join(ROOT, "oracle", "_ref", "libgg_ref.so")
    return "reference" if os.path.exists(ref) else "port"


def _ensure_oracle():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "libgg_oracle.so")):
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "build.py")])


def _seed_states(seed=777):
    """GGEMS's seeding (std::mt19937(seed), 4 words per slot) from the oracle side."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import scenes
    return scenes.seed_states(seed)


def _sample_size(scene_ptr, source, threads, kind, budget_s, states):
    """Primaries for about budget_s seconds of host work (pilot run first)."""
    pilot = 20000
    while True:
        dt, _ = cpu_reference_run(scene_ptr, source, pilot, threads, kind, states)
        # a pilot shorter than a second is dominated by thread start-up: grow it
        if dt >= 1.0 or pilot >= 4 * 1048576:
            break
        pilot = min(pilot * max(2, int(1.0 / max(dt, 1e-3))), 4 * 1048576)
    n = int(pilot * budget_s / max(dt, 1e-3))
    return max(pilot, min(n, 64 * 1048576))


def _batch_sizes(primaries):
    """GGEMSSource::OrganizeParticlesInBatch: ceil(n / 2^20) batches, the first
    n mod batches of them one primary larger."""
    nb = -(-primaries // 1048576)
    q, r = divmod(primaries, nb)
    return [q + 1 if i < r else q for i in range(nb)]


def _cbct_sample(scene_ptr, source, threads, kind, budget_s, states, primaries=PRIMARIES):
    """A bounded sample of the projection: its first k whole batches (the same
    slots and random streams as the projection's first k batches), k chosen so
    that one run takes about budget_s on these threads.  Returns (k, primaries)."""
    sizes = _batch_sizes(primaries)
    dt, _ = cpu_reference_run(scene_ptr, source, sizes[0], threads, kind, states)
    k = max(1, min(len(sizes), int(round(budget_s / max(dt, 1e-3)))))
    return k, sum(sizes[:k])


SURROGATE_NET = os.path.join(ROOT, "ggems_b200", "data", "unet_scatter256.npz")


def surrogate_measurement(tmp, angles=360, reference_every=10):
    """The second metric: scatter projections/s of the learned surrogate (the
    committed trained network + the 1e6-primary plain-MC judge, as specified)
    against plain MC at <= 5 % error, on a 360-angle CBCT scan of a new phantom,
    errors against 1e9-primary references on every `reference_every`-th angle.
    Run by ggems_b200.scatter in a process of its own (the GGEMS API's managers
    are process-wide).  Returns the summary dict, or None without the network."""
    if not os.path.exists(SURROGATE_NET):
        return None
    out = os.path.join(tmp, "surrogate.json")
    cmd = [sys.executable, "-m", "ggems_b200.scatter", "--load", SURROGATE_NET, "--test", "0", "--angles",
           str(angles), "--reference-every", str(reference_every), "--batch", "40", "--json-out", out]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=1200)
    if r.returncode != 0:
        return {"error": (r.stdout + r.stderr)[-800:]}
    d = json.load(open(out))
    scan, plain = d["scan"], d["plain_mc"]
    return {"metric": d["metric"], "value": d["value"], "unit": "projections/s",
            "plain_mc_projections_per_s": {k: plain[k]["projections_per_s"] for k in ("blocks16", "full")},
            "speedup_vs_plain_mc": {k: plain[k]["speedup"] for k in ("blocks16", "full")},
            "plain_mc_primaries_for_5pct": {k: plain[k]["primaries_for_5pct"] for k in ("blocks16", "full")},
            "plain_mc_error_blocks16": plain["blocks16"]["error_mean"],
            "plain_mc_primaries_per_s": plain["mc_primaries_per_s"],
            "error": scan["error"], "network_error": scan["network_error"], "judge_mc_error": scan["judge_mc_error"],
            "network_kept": scan["network_kept"], "replaced_by_mc": scan["replaced_by_mc"],
            "judge": d["judge"], "with_rescaling": d["with_rescaling"],
            "integrated_scatter_error": d["integrated_scatter_error"],
            "scan": {"angles": scan["angles"], "seconds": scan["seconds"], "reference_angles": scan["reference_angles"],
                     "ms_per_projection": scan["ms_per_projection"]},
            "errors": d["errors"], "network": os.path.basename(SURROGATE_NET),
            "config": {"phantom": "64^3 x 2 mm random water/bone/air, 60 keV, 256^2 panel", "judge_primaries": 1e6,
                       "reference_primaries": 1e9, "training": "2000 MC pairs at 1e8 primaries, 60 epochs"}}


def _pinned(n, dtype):
    """A zeroed page-locked host array (torch's host allocator), so that the
    end-to-end copies run at DMA speed as a caller with pinned buffers gets."""
    import numpy as np
    import torch
    dtype = np.dtype(dtype)
    tdt = {np.dtype(np.int32): torch.int32, np.dtype(np.uint32): torch.int32, np.dtype(np.float64): torch.float64,
           np.dtype(np.float32): torch.float32, np.dtype(np.int16): torch.int16}[dtype]
    return torch.zeros(int(n), dtype=tdt, pin_memory=True).numpy().view(dtype)


def _transport_launch(lib, ctx):
    """The transport kernel's launch knobs on this context."""
    v = [C.c_int32() for _ in range(8)]
    lib.gg_get_transport_tuning(ctx, C.byref(v[0]), C.byref(v[1]), C.byref(v[2]))
    lib.gg_get_transport_launch(ctx, C.byref(v[3]), C.byref(v[4]))
    lib.gg_get_transport_stash(ctx, C.byref(v[5]), C.byref(v[6]), C.byref(v[7]))
    return {"blocks_per_sm": v[0].value or "as many as fit", "regroup_ratio4": v[2].value, "block_threads": v[3].value,
            "slots_per_claim": v[4].value, "stash_registers": v[5].value, "stash_swap_lanes": v[6].value,
            "stash_round_photons": v[7].value}


def _cbct_config(primaries, batches, world):
    """The workload both arms report (same dict on the product and the reference arm)."""
    return {"workload": WORKLOAD, "phantom": "256x256x256 uint8, 1 mm, air/water/bone(1.85)",
            "primaries_per_step": primaries, "batches_per_step": batches,
            "detector": "flat 512x512 GOS, 0.8 mm, SDD 1500 / SID 1000",
            "processes": "Compton, photoelectric, Rayleigh",
            "parallelism": ("%d ranks, independent histories, one tally all-reduce per run" % world) if world > 1
            else "single GPU",
            "l2": "256 MB buffer written between timed steps (inputs 17 MB < L2)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--primaries", type=int, default=PRIMARIES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass (profiling runs)")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned-surrogate measurement")
    ap.add_argument("--cpu-leg", action="store_true",
                    help="water / curved: print only the CPU baseline of the workload's scene (run by the bench "
                         "itself in a process that imports no torch)")
    ap.add_argument("--workload", default="cbct",
                    choices=["cbct", "water", "batched", "mesh", "volume", "curved", "surrogate"],
                    help="cbct: the CBCT projection (default); water: 64^3 water dosimetry, 1e6 primaries; "
                         "batched: 360 angles + 16 phantoms in one launch; mesh: meshed-phantom dosimetry; "
                         "volume: CT image -> material labels on the device; surrogate: learned scatter "
                         "projections/s vs plain MC (also part of the cbct line)")
    ap.add_argument("--mesh-subdivisions", type=int, default=6, help="icosphere subdivisions of the mesh body")
    ap.add_argument("--primaries-per-job", type=int, default=10_000_000)
    args = ap.parse_args()
    rank, world, local = _rank()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    _ensure_built()
    _ensure_oracle()
    tmp = tempfile.mkdtemp(prefix="ggems_bench_")
    from ggems_b200 import workloads
    files = workloads.cbct_files(tmp, 256, 1.0, seed=1)
    if args.workload == "batched":
        return run_batched(args, tmp, rank)
    if args.workload == "mesh":
        return run_mesh(args, tmp, rank)
    if args.workload == "volume":
        return run_volume(args, rank)
    if args.workload == "water":
        return run_water(args, tmp, rank)
    if args.workload == "curved":
        return run_curved(args, tmp, rank)
    # The CBCT line's CPU baseline is taken first, the way the reference arm
    # takes it: on the B200 hosts it was measured on, the same host code ran
    # ~1.6x slower (1.6x the user CPU time) once any process on the host had
    # imported torch, even an idle one, and the timed GPU steps below need torch.
    args.cpu_baseline_early = None
    if args.workload == "cbct" and not args.no_cpu_baseline and rank == 0 and world == 1:
        m = _reference_measurement(args.primaries, 2, 1)
        m["cpu_baseline"]["sample"] += (", 1 warm-up and 2 timed runs before this process imports torch (the "
                                        "reference arm's measurement)")
        args.cpu_baseline_early = m["cpu_baseline"]
    if args.workload == "surrogate":
        if rank == 0:
            print(json.dumps(surrogate_measurement(tmp) or {"unavailable": "no trained network"}), flush=True)
        return 0

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    gg = _configure(files, args.primaries)
    from ggems_b200 import abi, distributed
    from ggems_b200.api import lib
    if world > 1:
        gg.GGEMSOpenCLManager().set_device_index(local)
    ggems = gg.GGEMS()
    # Every rank seeds 777; rank r then takes the random streams after those of
    # ranks < r (device order of GGEMSPseudoRandomGenerator), set just below.
    ggems.initialize(777)
    ctx = lib.ggems_device_context(ggems.obj, 0)
    import numpy as np
    rank_states = None  # this rank's initial streams (rank 0: GGEMS's own seeding above)
    if rank > 0:
        rank_states = np.zeros(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
        lib.gg_seed_random_states(abi.ptr(rank_states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES, 777,
                                  rank * abi.GG_MAXIMUM_PARTICLES)
        lib.gg_set_random_states(ctx, abi.ptr(rank_states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES)
    src = abi.gg_source()
    n_src = C.c_uint64()
    assert lib.ggems_source_descriptor(0, C.byref(src), C.byref(n_src)) == 0
    scene_ptr = lib.ggems_scene(ggems.obj)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def check(rc, what):
        if rc != 0:
            raise RuntimeError("%s: %s" % (what, lib.gg_last_error().decode()))

    def step():
        check(lib.gg_run_source(ctx, C.byref(src), args.primaries), "gg_run_source")
        check(lib.gg_synchronize(ctx), "gg_synchronize")
        ms, launches = C.c_float(), C.c_int64()
        lib.gg_last_run_stats(ctx, C.byref(ms), C.byref(launches))
        return ms.value, launches.value

    for _ in range(args.warmup):
        flush.zero_()
        torch.cuda.synchronize()
        step()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-timed region (inputs resident in HBM) ----
    times, launches = [], 0
    barrier()
    with ClockSampler(_smi_device(local)) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ms, n = step()
            times.append(ms)
            launches += n
    barrier()
    total_ms = sum(times)
    if dist is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.primaries * args.steps / (total_ms * 1e-3)

    # ---- end to end through the C ABI: host scene -> device, run, tallies -> host ----
    sc = scene_ptr.contents
    hs = [int(sc.histogram_sizes[i]) for i in range(sc.number_of_histograms)]
    # inputs and results in page-locked host memory
    tallies = abi.Tallies(hs, [], alloc=_pinned)
    states = _pinned(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
    states[:] = rank_states if rank_states is not None else np.frombuffer(
        C.string_at(lib.ggems_initial_random_states(ggems.obj, 0), 5 * abi.GG_MAXIMUM_PARTICLES * 4), np.uint32)
    h2d = sum(int(sc.solids[i].number_of_voxels[0]) * sc.solids[i].number_of_voxels[1] * sc.solids[i].number_of_voxels[2]
              for i in range(sc.number_of_solids) if sc.solids[i].type == abi.GG_SOLID_VOXELIZED)
    for i in range(sc.number_of_tables):
        t = sc.tables[i]
        h2d += 4 * (t.number_of_bins + 3 * t.number_of_materials * t.number_of_bins + 101 * t.number_of_bins + 4 * t.number_of_materials)
    h2d += states.nbytes + 2 * 4 * (int(src.number_of_energy_bins) + 1)
    d2h = sum(4 * h for h in hs)
    e2e_times = []
    for k in range(0 if args.no_e2e else args.steps + 1):
        barrier()
        t0 = time.perf_counter()
        check(lib.gg_upload_scene(ctx, scene_ptr), "gg_upload_scene")
        check(lib.gg_set_random_states(ctx, abi.ptr(states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES), "random states")
        step()
        if world > 1:  # the run's one exchange: sum the device tallies over ranks (NCCL, in place, exact)
            distributed.reduce_device_tallies(ctx)
        check(lib.gg_read_tallies(ctx, C.byref(tallies.struct)), "gg_read_tallies")
        t1 = time.perf_counter()
        if k > 0:  # first pass warms the host allocations
            e2e_times.append(t1 - t0)
    e2e_total = sum(e2e_times) if e2e_times else float("nan")
    if dist is not None:
        t = torch.tensor([e2e_total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * args.primaries * args.steps / e2e_total

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    nb = C.c_int64()
    lib.gg_batch_plan(args.primaries, None, 0, C.byref(nb))
    batches = int(nb.value)

    # ---- CPU baseline and roofline (rank 0, N = 1 only) ----
    # The same sample the reference arm times: the projection's first whole
    # batches from GGEMS's seeding of 777, on every host thread.
    cpu_baseline, counts = None, None
    kind = _cpu_kind()
    ref_states = _seed_states(777)
    if not args.no_cpu_baseline and world == 1:
        cpu_baseline = args.cpu_baseline_early
    _, counts = cpu_reference_run(scene_ptr, src, 20000 if args.no_cpu_baseline else 100000, os.cpu_count() or 1,
                                  "port", ref_states)
    S, box, D, H = counts
    # algorithmic bytes per primary: source state 40 B + 1 B label per voxel step + 20 B per dose
    # deposit + 8 B per detector count + 28 B final state
    bytes_per_primary = 40 + S + 20 * D + 8 * H + 28
    peaks = _peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    achieved = value / world * bytes_per_primary / 1e9
    per_launch_traffic = _profile_traffic()
    clocks = clk.summary()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": per_launch_traffic,
                "peak_source": "measured" if peaks else "fallback",
                "bytes_per_primary": bytes_per_primary,
                "voxel_steps_per_primary": S, "box_steps_per_primary": box, "detector_counts_per_primary": H,
                # issue-bound kernel: what the ncu summary says about the issue slots and lanes
                "l2_hit_rate_pct": _profile_value("l2_hit_rate_pct"),
                "issue_active_pct": _profile_value("issue_active_pct"),
                "lanes_active_pct": _profile_value("lanes_active_pct"),
                "issue": _issue_roofline(value / world, clocks)}
    line = {
        "metric": "primaries/s (CBCT 256^3, 120 kVp)", "value": value, "unit": "primaries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom generator, synthetic 120 kVp spectrum)",
        "config": _cbct_config(args.primaries, batches, world),
        "e2e": {"value": e2e_value, "unit": "primaries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roofline,
        "cpu_baseline": cpu_baseline,
        "clocks": clocks,
        "transport": _transport_launch(lib, ctx),
    }
    if not args.no_surrogate and world == 1:
        line["surrogate"] = surrogate_measurement(tmp)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _configure_water(files, primaries):
    """The 64^3 water phantom with a dose map and a 60 keV cone source, through the GGEMS API."""
    import ggems_b200 as gg
    mhd, rng_file = files
    gg.GGEMSVerbosity(0)
    gg.GGEMSMaterialsDatabaseManager().set_materials(os.path.join(ROOT, "ggems_b200", "data", "materials.txt"))
    phantom = gg.GGEMSVoxelizedPhantom("phantom")
    phantom.set_phantom(mhd, rng_file)
    phantom.set_rotation(0.0, 0.0, 0.0, "deg")
    phantom.set_position(0.0, 0.0, 0.0, "mm")
    dose = gg.GGEMSDosimetryCalculator()
    dose.attach_to_navigator("phantom")
    dose.set_output_basename(os.path.join(os.path.dirname(mhd), "dose"))
    dose.edep(True)
    dose.hit(True)
    dose.edep_squared(True)
    dose.uncertainty(True)
    pm = gg.GGEMSProcessesManager()
    for process in ("Compton", "Photoelectric", "Rayleigh"):
        pm.add_process(process, "gamma", "all")
    pm.set_cross_section_table_number_of_bins(220)
    pm.set_cross_section_table_energy_min(1.0, "keV")
    pm.set_cross_section_table_energy_max(1.0, "MeV")
    gg.GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
    src = gg.GGEMSXRaySource("xray")
    src.set_source_particle_type("gamma")
    src.set_number_of_particles(primaries)
    src.set_position(-1000.0, 0.0, 0.0, "mm")
    src.set_rotation(0.0, 0.0, 0.0, "deg")
    src.set_beam_aperture(10.0, "deg")
    src.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
    src.set_monoenergy(60.0, "keV")
    return gg, dose


def run_batched(args, tmp, rank):
    """Batched workload: 360 projection angles of the 64^3 water phantom and 16
    phantoms of uneven size (96-320 voxels per side) x primaries-per-job, as the
    jobs of one persistent launch captured in a CUDA graph, launch shape from the
    autotuner.  One step = one replay of the graph (every job once)."""
    import torch
    from ggems_b200 import abi, workloads, _native
    from ggems_b200.api import lib
    gg, dose = _configure_water(workloads.water_files(tmp, 64, 2.0), args.primaries_per_job)
    ggems = gg.GGEMS()
    ggems.initialize(777)
    ctx = lib.ggems_device_context(ggems.obj, 0)
    base = lib.ggems_scene(ggems.obj).contents
    src = abi.gg_source()
    assert lib.ggems_source_descriptor(0, C.byref(src), None) == 0
    w = workloads.BatchedWorkload(lib, base, src, os.path.join(ROOT, "ggems_b200", "data", "materials.txt"),
                                  primaries=args.primaries_per_job)

    def check(rc, what):
        if rc != 0:
            raise RuntimeError("%s: %s" % (what, lib.gg_last_error().decode()))

    check(lib.gg_upload_scene(ctx, C.byref(w.scene)), "gg_upload_scene")
    # tune on a sample of the job mix itself: every 12th angle and every 4th
    # phantom, 2e6 primaries each
    sample = [(s, min(n, 2_000_000), solids) for s, n, solids in w.jobs[:360:12] + w.jobs[360::4]]
    sarr, skeep = _native._job_array(sample)
    ms = C.c_float()
    check(lib.gg_autotune_jobs(ctx, sarr, len(skeep), C.byref(ms)), "gg_autotune_jobs")
    bps, lanes, ratio = C.c_int32(), C.c_int32(), C.c_int32()
    lib.gg_get_transport_tuning(ctx, C.byref(bps), C.byref(lanes), C.byref(ratio))
    threads, grain = C.c_int32(), C.c_int32()
    lib.gg_get_transport_launch(ctx, C.byref(threads), C.byref(grain))
    stash, swap, round_photons = C.c_int32(), C.c_int32(), C.c_int32()
    lib.gg_get_transport_stash(ctx, C.byref(stash), C.byref(swap), C.byref(round_photons))
    arr, keep = _native._job_array(w.jobs)
    graph = C.c_void_p()
    check(lib.gg_capture_jobs(ctx, arr, len(keep), C.byref(graph)), "gg_capture_jobs")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def step():
        flush.zero_()
        torch.cuda.synchronize()
        check(lib.gg_graph_launch(graph), "gg_graph_launch")
        check(lib.gg_synchronize(ctx), "gg_synchronize")
        t, n = C.c_float(), C.c_int64()
        lib.gg_last_run_stats(ctx, C.byref(t), C.byref(n))
        return t.value, n.value

    for _ in range(args.warmup):
        step()
    times, launches = [], 0
    with ClockSampler(_smi_device()) as clk:
        for _ in range(args.steps):
            t, n = step()
            times.append(t)
            launches += n
    lib.gg_graph_destroy(graph)
    total_ms = sum(times)
    value = w.total_primaries * args.steps / (total_ms * 1e-3)
    if rank == 0:
        print(json.dumps({
            "metric": "primaries/s (batched: 360 angles + 16 phantoms, one launch)", "value": value,
            "unit": "primaries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (64^3 water phantom; seeded ellipsoid phantoms)",
            "config": {"workload": "batched_360x%d_16phantoms" % args.primaries_per_job,
                       "jobs": len(w.jobs), "primaries_per_step": w.total_primaries,
                       "phantom_edges": w.phantom_edges,
                       "tuning": {"blocks_per_sm": bps.value, "regroup_ratio4": ratio.value,
                                  "block_threads": threads.value, "slots_per_claim": grain.value,
                                  "stash_registers": stash.value, "stash_round_photons": round_photons.value,
                                  "tuned_on": "%d sampled jobs of the mix, 2e6 primaries each" % len(sample)},
                       "launch": "one persistent kernel per step, replayed CUDA graph",
                       "l2": "256 MB buffer written between timed steps"},
            "gpu_launches": launches, "clocks": clk.summary()}), flush=True)
    return 0


def run_mesh(args, tmp, rank):
    """Meshed dosimetry: an STL body (ellipsoid 120/100/150 mm) with 8 inner
    ellipsoids, one material (water), 80 keV cone, dose on 2 mm dosels, through
    the GGEMS API (GGEMSMeshedPhantom).  One step = one run of --primaries."""
    import torch
    import ggems_b200 as gg
    from ggems_b200 import abi, workloads
    from ggems_b200.api import lib
    stl = os.path.join(tmp, "body.stl")
    tris = workloads.body_mesh(args.mesh_subdivisions, max(args.mesh_subdivisions - 1, 0), 8, seed=1)
    workloads.write_stl(stl, tris)
    gg.GGEMSVerbosity(0)
    gg.GGEMSMaterialsDatabaseManager().set_materials(os.path.join(ROOT, "ggems_b200", "data", "materials.txt"))
    mesh = gg.GGEMSMeshedPhantom("phantom_mesh")
    mesh.set_phantom(stl)
    mesh.set_rotation(0.0, 0.0, 0.0, "deg")
    mesh.set_position(0.0, 0.0, 0.0, "mm")
    mesh.set_mesh_octree_depth(4)
    mesh.set_material("Water")
    dose = gg.GGEMSDosimetryCalculator()
    dose.attach_to_navigator("phantom_mesh")
    dose.set_output_basename(os.path.join(tmp, "mesh_dose"))
    dose.set_dosel_size(2.0, 2.0, 2.0, "mm")
    dose.edep(True)
    dose.hit(True)
    dose.edep_squared(True)
    pm = gg.GGEMSProcessesManager()
    for process in ("Compton", "Photoelectric", "Rayleigh"):
        pm.add_process(process, "gamma", "all")
    gg.GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
    src = gg.GGEMSXRaySource("xray")
    src.set_source_particle_type("gamma")
    src.set_number_of_particles(args.primaries)
    src.set_position(-1000.0, 0.0, 0.0, "mm")
    src.set_rotation(0.0, 0.0, 0.0, "deg")
    src.set_beam_aperture(8.0, "deg")
    src.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
    src.set_monoenergy(80.0, "keV")
    ggems = gg.GGEMS()
    ggems.initialize(777)
    ctx = lib.ggems_device_context(ggems.obj, 0)
    s = abi.gg_source()
    assert lib.ggems_source_descriptor(0, C.byref(s), None) == 0
    sc = lib.ggems_scene(ggems.obj).contents
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def step():
        flush.zero_()
        torch.cuda.synchronize()
        if lib.gg_run_source(ctx, C.byref(s), args.primaries) != 0 or lib.gg_synchronize(ctx) != 0:
            raise RuntimeError(lib.gg_last_error().decode())
        t, n = C.c_float(), C.c_int64()
        lib.gg_last_run_stats(ctx, C.byref(t), C.byref(n))
        return t.value, n.value

    for _ in range(args.warmup):
        step()
    times, launches = [], 0
    with ClockSampler(_smi_device()) as clk:
        for _ in range(args.steps):
            t, n = step()
            times.append(t)
            launches += n
    total_ms = sum(times)
    d = sc.dose_maps[0]
    if rank == 0:
        print(json.dumps({
            "metric": "primaries/s (meshed dosimetry)", "value": args.primaries * args.steps / (total_ms * 1e-3),
            "unit": "primaries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (icosphere ellipsoid meshes)",
            "config": {"workload": "mesh_%dtri_80keV" % len(tris), "triangles": len(tris),
                       "navigation": "BVH" if (os.environ.get("GGEMS_B200_MESH_BVH", "1" if len(tris) > 4096 else "0")
                                               != "0") else "octree scan",
                       "primaries_per_step": args.primaries, "dose_grid": list(d.number_of_dosels),
                       "l2": "256 MB buffer written between timed steps"},
            "gpu_launches": launches, "clocks": clk.summary()}), flush=True)
    return 0


def run_curved(args, tmp, rank):
    """The CT-scanner configuration of GGEMS's example 2: a 10 mm water box drawn by
    the volume creator into a 120^3 x 0.1 mm MET_INT volume, a curved detector of
    46 modules of 64 x 16 x 1 GOS elements (0.6 mm; SDD 1085.6 mm, SID 595 mm, 10 keV
    threshold), a 120 kVp cone of 12.5 deg from (-595, 0, 0) mm, through the GGEMS
    API.  One step = one projection of --primaries; `cpu_baseline` = the same scene
    on the host cores."""
    import numpy as np
    import ggems_b200 as gg
    from ggems_b200 import abi, workloads
    from ggems_b200.api import lib
    gg.GGEMSVerbosity(0)
    gg.GGEMSMaterialsDatabaseManager().set_materials(os.path.join(ROOT, "ggems_b200", "data", "materials.txt"))
    vc = gg.GGEMSVolumeCreatorManager()
    vc.set_dimensions(120, 120, 120)
    vc.set_element_sizes(0.1, 0.1, 0.1, "mm")
    vc.set_output(os.path.join(tmp, "phantom.mhd"))
    vc.set_range_output(os.path.join(tmp, "range_phantom.txt"))
    vc.set_material("Air")
    vc.set_data_type("MET_INT")
    vc.initialize()
    box = gg.GGEMSBox(10.0, 10.0, 10.0, "mm")
    box.set_position(0.0, 0.0, 0.0, "mm")
    box.set_label_value(1)
    box.set_material("Water")
    box.initialize()
    box.draw()
    box.delete()
    vc.write()
    phantom = gg.GGEMSVoxelizedPhantom("phantom")
    phantom.set_phantom(os.path.join(tmp, "phantom.mhd"), os.path.join(tmp, "range_phantom.txt"))
    phantom.set_rotation(0.0, 0.0, 0.0, "deg")
    phantom.set_position(0.0, 0.0, 0.0, "mm")
    ct = gg.GGEMSCTSystem("Stellar")
    ct.set_ct_type("curved")
    ct.set_number_of_modules(1, 46)
    ct.set_number_of_detection_elements(64, 16, 1)
    ct.set_size_of_detection_elements(0.6, 0.6, 0.6, "mm")
    ct.set_material("GOS")
    ct.set_source_detector_distance(1085.6, "mm")
    ct.set_source_isocenter_distance(595.0, "mm")
    ct.set_rotation(0.0, 0.0, 0.0, "deg")
    ct.set_threshold(10.0, "keV")
    ct.save(os.path.join(tmp, "projection.mhd"))
    pm = gg.GGEMSProcessesManager()
    for process in ("Compton", "Photoelectric", "Rayleigh"):
        pm.add_process(process, "gamma", "all")
    pm.set_cross_section_table_number_of_bins(220)
    pm.set_cross_section_table_energy_min(1.0, "keV")
    pm.set_cross_section_table_energy_max(1.0, "MeV")
    gg.GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
    src = gg.GGEMSXRaySource("point_source")
    src.set_source_particle_type("gamma")
    src.set_number_of_particles(args.primaries)
    src.set_position(-595.0, 0.0, 0.0, "mm")
    src.set_rotation(0.0, 0.0, 0.0, "deg")
    src.set_beam_aperture(12.5, "deg")
    src.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
    src.set_polyenergy(workloads.write_spectrum(os.path.join(tmp, "spectrum_120kVp.dat")))
    ggems = gg.GGEMS()
    ggems.initialize(777)
    ctx = lib.ggems_device_context(ggems.obj, 0)
    s = abi.gg_source()
    assert lib.ggems_source_descriptor(0, C.byref(s), None) == 0
    scene_ptr = lib.ggems_scene(ggems.obj)
    sc = scene_ptr.contents
    if args.cpu_leg:
        print(json.dumps({"cpu_baseline": _cpu_sample(scene_ptr, s, "the same projection")}), flush=True)
        return 0
    import torch
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def step():
        flush.zero_()
        torch.cuda.synchronize()
        if lib.gg_run_source(ctx, C.byref(s), args.primaries) != 0 or lib.gg_synchronize(ctx) != 0:
            raise RuntimeError(lib.gg_last_error().decode())
        t, n = C.c_float(), C.c_int64()
        lib.gg_last_run_stats(ctx, C.byref(t), C.byref(n))
        return t.value, n.value

    for _ in range(args.warmup):
        step()
    times, launches = [], 0
    with ClockSampler(_smi_device()) as clk:
        for _ in range(args.steps):
            t, n = step()
            times.append(t)
            launches += n
    total_ms = sum(times)
    cpu = None if args.no_cpu_baseline else _cpu_leg_process(args)
    if rank == 0:
        print(json.dumps({
            "metric": "primaries/s (curved 46-module CT)", "value": args.primaries * args.steps / (total_ms * 1e-3),
            "unit": "primaries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (volume-creator water box, synthetic 120 kVp spectrum)",
            "config": {"workload": "ct_scanner_curved46_120kVp", "solids": int(sc.number_of_solids),
                       "phantom": "120^3 MET_INT, 0.1 mm, 10 mm water box", "primaries_per_step": args.primaries,
                       "detector": "46 modules x 64 x 16 GOS, 0.6 mm, SDD 1085.6 / SID 595",
                       "l2": "256 MB buffer written between timed steps"},
            "gpu_launches": launches, "cpu_baseline": cpu, "clocks": clk.summary()}), flush=True)
    return 0


def run_water(args, tmp, rank):
    """Water dosimetry: 64^3 water of 2 mm voxels, 60 keV cone, edep / E^2 / hit
    tallies and the dose + uncertainty finalisation, 1e6 primaries per step,
    through the GGEMS API.  `value` = device-timed primaries/s of the transport
    launch; `e2e` = scene and random states uploaded, run, dose finalised and
    tallies read back to host memory, wall-clocked."""
    import numpy as np
    from ggems_b200 import abi, workloads
    from ggems_b200.api import lib
    n = 1_000_000 if args.primaries == PRIMARIES else args.primaries
    files = workloads.water_files(tmp, 64, 2.0)
    gg, _ = _configure_water(files, n)
    ggems = gg.GGEMS()
    ggems.initialize(777)
    ctx = lib.ggems_device_context(ggems.obj, 0)
    src = abi.gg_source()
    assert lib.ggems_source_descriptor(0, C.byref(src), None) == 0
    scene_ptr = lib.ggems_scene(ggems.obj)
    sc = scene_ptr.contents
    if args.cpu_leg:
        print(json.dumps({"cpu_baseline": _cpu_sample(scene_ptr, src, "the same run")}), flush=True)
        return 0
    import torch
    dm = sc.dose_maps[0]
    nd = int(dm.total_number_of_dosels)
    dose, unc = _pinned(nd, np.float32), _pinned(nd, np.float32)  # page-locked results
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def check(rc, what):
        if rc != 0:
            raise RuntimeError("%s: %s" % (what, lib.gg_last_error().decode()))

    def step():
        check(lib.gg_run_source(ctx, C.byref(src), n), "gg_run_source")
        check(lib.gg_synchronize(ctx), "gg_synchronize")
        t, k = C.c_float(), C.c_int64()
        lib.gg_last_run_stats(ctx, C.byref(t), C.byref(k))
        return t.value, k.value

    for _ in range(args.warmup):
        step()
    times, launches = [], 0
    with ClockSampler(_smi_device()) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t, k = step()
            times.append(t)
            launches += k
    total_ms = sum(times)
    value = n * args.steps / (total_ms * 1e-3)
    states = _pinned(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
    states[:] = np.frombuffer(C.string_at(lib.ggems_initial_random_states(ggems.obj, 0),
                                          5 * abi.GG_MAXIMUM_PARTICLES * 4), np.uint32)
    tallies = abi.Tallies([], [nd], alloc=_pinned)
    e2e = []
    for k in range(args.steps + 1):
        t0 = time.perf_counter()
        check(lib.gg_upload_scene(ctx, scene_ptr), "gg_upload_scene")
        check(lib.gg_set_random_states(ctx, abi.ptr(states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES), "states")
        step()
        check(lib.gg_compute_dose(ctx, 0, 0, C.c_float(1.0), 0, C.c_float(0.0), abi.ptr(dose, C.c_float),
                                  abi.ptr(unc, C.c_float)), "gg_compute_dose")
        check(lib.gg_read_tallies(ctx, C.byref(tallies.struct)), "gg_read_tallies")
        if k:
            e2e.append(time.perf_counter() - t0)
    cpu = None if args.no_cpu_baseline else _cpu_leg_process(args)
    if rank == 0:
        print(json.dumps({
            "metric": "primaries/s (64^3 water dosimetry, 60 keV)", "value": value, "unit": "primaries/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (uniform water phantom)",
            "config": {"workload": "water64_2mm_60keV_dose", "primaries_per_step": n,
                       "tallies": "edep, edep^2, hit; dose + uncertainty in e2e",
                       "l2": "256 MB buffer written between timed steps"},
            "e2e": {"value": n * len(e2e) / sum(e2e), "unit": "primaries/s",
                    "h2d_bytes_per_step": 64 ** 3 + states.nbytes, "d2h_bytes_per_step": nd * (4 + 4 + 8 + 8 + 4)},
            "gpu_launches": launches, "cpu_baseline": cpu, "clocks": clk.summary()}), flush=True)
    return 0


# HU ranges -> materials of a CT range file (first <= HU < last)
CT_RANGES = [(-1100, -950), (-950, -700), (-700, -100), (-100, -20), (-20, 40), (40, 200), (200, 800), (800, 3100)]


def run_volume(args, rank):
    """Range-table label conversion of a CT image (512^3 int16 HU) on the
    device (gg_volume_labels, GGEMSVoxelizedSolid::ConvertImageToLabel).  One
    step = one conversion of the whole image; `value` = voxels/s of the kernel
    with the image resident, `e2e` = upload of the image from host memory +
    conversion + labels back to host memory through the C ABI."""
    import numpy as np
    import torch
    from ggems_b200 import abi
    from ggems_b200._native import Volume
    dims = (512, 512, 512)
    n = int(np.prod(dims))
    rng = np.random.default_rng(5)
    # body-like HU image: blocks of tissue classes with noise
    classes = np.array([-1000, -800, -400, -60, 10, 100, 500, 1500], np.int16)
    coarse = rng.integers(0, len(classes), (dims[2] // 8, dims[1] // 8, dims[0] // 8))
    img = np.repeat(np.repeat(np.repeat(classes[coarse], 8, 0), 8, 1), 8, 2)
    img = (img + rng.integers(-30, 30, img.shape).astype(np.int16)).reshape(-1)
    first = np.array([r[0] for r in CT_RANGES], np.float32)
    last = np.array([r[1] for r in CT_RANGES], np.float32)
    v = Volume(abi.GG_MET_SHORT, dims, (1.0, 1.0, 1.0))
    v.upload(img)
    out = np.empty(n, np.uint8)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    missing = C.c_int64()

    def step():
        flush.zero_()
        torch.cuda.synchronize()
        from ggems_b200._native import lib as nlib, check
        check(nlib.gg_volume_labels(v.handle, abi.ptr(first, C.c_float), abi.ptr(last, C.c_float), len(first),
                                    abi.ptr(out, C.c_uint8), C.byref(missing)), "gg_volume_labels")
        return v.last_kernel_ms()

    for _ in range(args.warmup):
        step()
    times = []
    with ClockSampler(_smi_device()) as clk:
        for _ in range(args.steps):
            times.append(step())
    total_ms = sum(times)
    value = n * args.steps / (total_ms * 1e-3)
    e2e = []
    for k in range(args.steps + 1):
        t0 = time.perf_counter()
        v.upload(img)
        lab, miss = v.labels(first, last)
        if k:
            e2e.append(time.perf_counter() - t0)
    assert miss == 0
    # oracle parity on the timed output, then the CPU baseline on a slab
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import scenes
    ref = np.empty(n, np.uint8)
    m = C.c_int64()
    scenes.oracle().gg_oracle_labels(img.ctypes.data_as(C.c_void_p), abi.GG_MET_SHORT, n, abi.ptr(first, C.c_float),
                                     abi.ptr(last, C.c_float), len(first), abi.ptr(ref, C.c_uint8), C.byref(m))
    assert np.array_equal(ref, lab) and np.array_equal(ref, out), "labels differ from the oracle"
    slab = n // 8
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < 10.0:
        scenes.oracle().gg_oracle_labels(img.ctypes.data_as(C.c_void_p), abi.GG_MET_SHORT, slab,
                                         abi.ptr(first, C.c_float), abi.ptr(last, C.c_float), len(first),
                                         abi.ptr(ref, C.c_uint8), C.byref(m))
        reps += 1
    cpu_dt = time.perf_counter() - t0
    peaks = _peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    bytes_per_voxel = 2 + 1  # int16 read + uint8 label written
    achieved = value * bytes_per_voxel / 1e9
    v.close()
    if rank == 0:
        print(json.dumps({
            "metric": "voxels/s (CT image -> material labels)", "value": value, "unit": "voxels/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16",
            "data": "synthetic (seeded blocky HU image)",
            "config": {"workload": "ct_labels_512x512x512_int16_8ranges", "ranges": len(CT_RANGES),
                       "l2": "256 MB buffer written between timed steps; image 268 MB > L2"},
            "e2e": {"value": n * len(e2e) / sum(e2e), "unit": "voxels/s", "h2d_bytes_per_step": img.nbytes,
                    "d2h_bytes_per_step": n},
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "bytes_per_voxel": bytes_per_voxel,
                         "peak_source": "measured" if peaks else "fallback"},
            "cpu_baseline": {"value": slab * reps / cpu_dt, "unit": "voxels/s", "cores": 1, "kind": "port",
                             "sample": "%d passes over 64 of the 512 slices (GGEMS's one pass per range line), %.1f s"
                                       % (reps, cpu_dt)},
            "clocks": clk.summary()}), flush=True)
    return 0


def _reference_measurement(primaries, steps, warmup):
    """GGEMS's kernels built for the host (oracle/_ref; else the oracle port)
    on all host threads, replaying GGEMS::RunOnDevice batch by batch on the
    CBCT scene built from the oracle side, `warmup` untimed and `steps` timed
    runs, each of the projection's first whole batches."""
    _ensure_oracle()
    kind = _cpu_kind()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import scenes
    # tables from GGEMS's own host code when it was built here (bit-identical to the oracle's)
    builder = "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libgg_ref_tables.so")) else "oracle"
    scene, source = scenes.cbct_api_scene(256, 1.0, seed=1, builder=builder)
    ss = scene.struct()
    scene_ptr = C.pointer(ss)
    src = source.struct
    states = scenes.seed_states(777)
    threads = os.cpu_count() or 1
    budget = min(8.0, max(1.0, 150.0 / max(steps + warmup, 1)))
    k, n = _cbct_sample(scene_ptr, src, threads, kind, budget, states, primaries)
    for _ in range(warmup):
        cpu_reference_run(scene_ptr, src, n, threads, kind, states)
    times = [cpu_reference_run(scene_ptr, src, n, threads, kind, states)[0] for _ in range(steps)]
    value = n * steps / sum(times)
    batches = len(_batch_sizes(primaries))
    sample = ("each step: the projection's first %d of %d batches (%d primaries, seed 777) on %d host threads"
              % (k, batches, n, threads))
    return {"value": value, "times": times, "batches": batches,
            "cpu_baseline": {"value": value, "unit": "primaries/s", "cores": threads, "kind": kind, "sample": sample}}


def run_reference_arm(args, rank, world):
    """The reference's CPU implementation of the path on all host threads:
    GGEMS's own kernels built for the host (oracle/_ref) when available, else
    the oracle port, replaying GGEMS::RunOnDevice batch by batch.  The scene,
    tables and random streams come from the oracle side (tests/scenes.py:
    GGEMS's own host table builders, oracle/_ref/libgg_ref_tables.so, else the
    oracle's restatement; GGEMS's mt19937 seeding), so nothing of the product
    library is loaded.  Each step is a bounded sample of the projection
    (its first whole batches, the same slots and streams as the projection);
    `config` is the product arm's."""
    if rank != 0:
        return 0
    m = _reference_measurement(args.primaries, args.steps, args.warmup)
    value, times, batches = m["value"], m["times"], m["batches"]
    print(json.dumps({
        "impl": "reference", "metric": "primaries/s (CBCT 256^3, 120 kVp)", "value": value, "unit": "primaries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded phantom generator, synthetic 120 kVp spectrum)",
        "config": _cbct_config(args.primaries, batches, world),
        "cpu_baseline": m["cpu_baseline"],
        "e2e": {"value": value, "unit": "primaries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
