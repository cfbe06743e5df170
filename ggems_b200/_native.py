"""Loader for ``libggems.so`` (CUDA transport layer + C++ host API).

There is no fallback: if the library is missing or was not built, importing
this module raises, so nothing can silently run on the CPU instead.
"""

import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libggems.so")


class GGEMSNativeError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise GGEMSNativeError("libggems.so is not built: run `python -m ggems_b200.build` (%s)" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    sig = {
        "gg_device_count": (C.c_int, [P(C.c_int32)]),
        "gg_context_create": (C.c_int, [C.c_int32, P(C.c_void_p)]),
        "gg_context_destroy": (C.c_int, [C.c_void_p]),
        "gg_last_error": (C.c_char_p, []),
        "gg_set_random_states": (C.c_int, [C.c_void_p, P(C.c_uint32), C.c_int64]),
        "gg_get_random_states": (C.c_int, [C.c_void_p, P(C.c_uint32), C.c_int64]),
        "gg_seed_random_states": (C.c_int, [P(C.c_uint32), C.c_int64, C.c_uint32, C.c_int64]),
        "gg_upload_scene": (C.c_int, [C.c_void_p, P(abi.gg_scene)]),
        "gg_reset_tallies": (C.c_int, [C.c_void_p]),
        "gg_read_tallies": (C.c_int, [C.c_void_p, P(abi.gg_tally_buffers)]),
        "gg_read_particles": (C.c_int, [C.c_void_p, P(abi.gg_particle_buffers), C.c_int64]),
        "gg_run_source": (C.c_int, [C.c_void_p, P(abi.gg_source), C.c_uint64]),
        "gg_synchronize": (C.c_int, [C.c_void_p]),
        "gg_batch_plan": (C.c_int, [C.c_uint64, P(C.c_uint64), C.c_int64, P(C.c_int64)]),
        "gg_compute_dose": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_int32, C.c_float,
                                      P(C.c_float), P(C.c_float)]),
        "gg_last_run_stats": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_int64)]),
        "gg_run_jobs": (C.c_int, [C.c_void_p, P(abi.gg_job), C.c_int32]),
        "gg_capture_jobs": (C.c_int, [C.c_void_p, P(abi.gg_job), C.c_int32, P(C.c_void_p)]),
        "gg_graph_launch": (C.c_int, [C.c_void_p]),
        "gg_graph_destroy": (C.c_int, [C.c_void_p]),
        "gg_set_transport_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
        "gg_get_transport_tuning": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
        "gg_autotune": (C.c_int, [C.c_void_p, P(abi.gg_source), C.c_uint64, P(C.c_float)]),
        "gg_autotune_jobs": (C.c_int, [C.c_void_p, P(abi.gg_job), C.c_int32, P(C.c_float)]),
        "gg_set_transport_launch": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
        "gg_get_transport_launch": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32)]),
        "gg_set_transport_stash": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
        "gg_get_transport_stash": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
        "gg_device_tallies": (C.c_int, [C.c_void_p, P(abi.gg_device_tally), C.c_int32, P(C.c_int32)]),
        "gg_set_tracking": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
        "gg_read_tracking": (C.c_int, [C.c_void_p, P(abi.gg_track_point), C.c_int32, P(C.c_int32)]),
        "gg_volume_create": (C.c_int, [C.c_int32, C.c_int32, P(C.c_int32), P(C.c_float), P(C.c_void_p)]),
        "gg_volume_destroy": (C.c_int, [C.c_void_p]),
        "gg_volume_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
        "gg_volume_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
        "gg_volume_draw": (C.c_int, [C.c_void_p, P(abi.gg_shape), C.c_int32]),
        "gg_volume_labels": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_int32, P(C.c_uint8),
                                       P(C.c_int64)]),
        "gg_volume_last_kernel_ms": (C.c_int, [C.c_void_p, P(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(rc, what=""):
    if rc != 0:
        msg = lib.gg_last_error().decode(errors="replace")
        raise GGEMSNativeError("%s failed (%s): %s" % (what or "ggems call", abi.STATUS.get(rc, rc), msg))


class Context:
    """One GPU context of the transport layer."""

    def __init__(self, device=0):
        h = C.c_void_p()
        check(lib.gg_context_create(device, C.byref(h)), "gg_context_create")
        self.handle = h

    def close(self):
        if self.handle:
            lib.gg_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_random_states(self, states):
        check(lib.gg_set_random_states(self.handle, abi.ptr(states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES),
              "gg_set_random_states")

    def get_random_states(self, states):
        check(lib.gg_get_random_states(self.handle, abi.ptr(states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES),
              "gg_get_random_states")

    def upload_scene(self, scene_struct):
        self._scene = scene_struct
        check(lib.gg_upload_scene(self.handle, C.byref(scene_struct)), "gg_upload_scene")

    def reset_tallies(self):
        check(lib.gg_reset_tallies(self.handle), "gg_reset_tallies")

    def run(self, source_struct, n, sync=True):
        check(lib.gg_run_source(self.handle, C.byref(source_struct), n), "gg_run_source")
        if sync:
            self.synchronize()

    def synchronize(self):
        check(lib.gg_synchronize(self.handle), "gg_synchronize")

    def read_tallies(self, tallies):
        check(lib.gg_read_tallies(self.handle, C.byref(tallies.struct)), "gg_read_tallies")

    def read_particles(self, particles):
        check(lib.gg_read_particles(self.handle, C.byref(particles.struct), particles.n), "gg_read_particles")

    def last_run_stats(self):
        ms, n = C.c_float(), C.c_int64()
        check(lib.gg_last_run_stats(self.handle, C.byref(ms), C.byref(n)), "gg_last_run_stats")
        return ms.value, n.value

    def run_jobs(self, jobs):
        """jobs: sequence of (gg_source, number_of_particles, solids array or None); one launch."""
        arr, keep = _job_array(jobs)
        check(lib.gg_run_jobs(self.handle, arr, len(keep)), "gg_run_jobs")

    def capture_jobs(self, jobs):
        """The same batched launch as a CUDA graph (ggems_b200._native.Graph)."""
        arr, keep = _job_array(jobs)
        g = C.c_void_p()
        check(lib.gg_capture_jobs(self.handle, arr, len(keep), C.byref(g)), "gg_capture_jobs")
        return Graph(g, keep)

    def set_tuning(self, blocks_per_sm=0, regroup_lanes=32, regroup_ratio4=4):
        check(lib.gg_set_transport_tuning(self.handle, blocks_per_sm, regroup_lanes, regroup_ratio4),
              "gg_set_transport_tuning")

    def tuning(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib.gg_get_transport_tuning(self.handle, C.byref(a), C.byref(b), C.byref(c)), "gg_get_transport_tuning")
        return a.value, b.value, c.value

    def set_launch(self, block_threads=256, slots_per_claim=1):
        check(lib.gg_set_transport_launch(self.handle, block_threads, slots_per_claim), "gg_set_transport_launch")

    def launch(self):
        """(block threads, slots per claim) of the transport launch."""
        a, b = C.c_int32(), C.c_int32()
        check(lib.gg_get_transport_launch(self.handle, C.byref(a), C.byref(b)), "gg_get_transport_launch")
        return a.value, b.value

    def set_stash(self, registers=80, swap_lanes=4, round_photons=40):
        """Photon stash of the transport kernel: 0 (off), 64 or 80 registers."""
        check(lib.gg_set_transport_stash(self.handle, registers, swap_lanes, round_photons), "gg_set_transport_stash")

    def stash(self):
        """(registers, swap lanes, round photons) of the photon stash; 0 registers = off."""
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib.gg_get_transport_stash(self.handle, C.byref(a), C.byref(b), C.byref(c)), "gg_get_transport_stash")
        return a.value, b.value, c.value

    def autotune(self, source, number_of_particles):
        ms = C.c_float()
        check(lib.gg_autotune(self.handle, C.byref(source), number_of_particles, C.byref(ms)), "gg_autotune")
        return ms.value

    def autotune_jobs(self, jobs):
        """gg_autotune on a batched launch of `jobs` (as run_jobs takes them)."""
        arr, keep = _job_array(jobs)
        ms = C.c_float()
        check(lib.gg_autotune_jobs(self.handle, arr, len(keep), C.byref(ms)), "gg_autotune_jobs")
        return ms.value

    def set_tracking(self, slot, capacity=4096):
        check(lib.gg_set_tracking(self.handle, slot, capacity), "gg_set_tracking")

    def read_tracking(self, capacity=4096):
        """The tracked slot's points of the last run (list of abi.gg_track_point), and how many were recorded."""
        pts = (abi.gg_track_point * capacity)()
        count = C.c_int32()
        check(lib.gg_read_tracking(self.handle, pts, capacity, C.byref(count)), "gg_read_tracking")
        return list(pts[:min(count.value, capacity)]), count.value

    def compute_dose(self, dose_map, solid, n, scale=1.0, water_reference=False, minimum_density=0.0,
                     uncertainty=True):
        import numpy as np
        dose = np.zeros(n, np.float32)
        unc = np.zeros(n, np.float32) if uncertainty else None
        check(lib.gg_compute_dose(self.handle, dose_map, solid, scale, 1 if water_reference else 0, minimum_density,
                                  abi.ptr(dose, C.c_float), abi.ptr(unc, C.c_float)), "gg_compute_dose")
        return dose, unc


def _job_array(jobs):
    keep = []
    for source, n, solids in jobs:
        j = abi.gg_job()
        j.source = source
        j.number_of_particles = n
        j.solids = C.cast(solids, C.POINTER(abi.gg_solid)) if solids is not None else C.cast(None, C.POINTER(abi.gg_solid))
        keep.append((j, solids))
    arr = (abi.gg_job * len(keep))(*[k[0] for k in keep])
    return arr, keep


class Graph:
    """A captured batched launch (gg_capture_jobs); launch() replays it."""

    def __init__(self, handle, keep):
        self.handle = handle
        self._keep = keep

    def launch(self):
        check(lib.gg_graph_launch(self.handle), "gg_graph_launch")

    def close(self):
        if self.handle:
            lib.gg_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Volume:
    """A phantom image on the device (gg_volume_*): analytic shapes drawn into
    it, or an MHD image uploaded and converted to labels by a range table."""

    def __init__(self, met_type, dimensions, element_sizes, device=0):
        import numpy as np
        self.met_type = met_type
        self.dimensions = tuple(int(d) for d in dimensions)
        self.dtype = np.dtype(abi.MET_DTYPES[met_type])
        dims = (C.c_int32 * 3)(*self.dimensions)
        es = (C.c_float * 3)(*[float(e) for e in element_sizes])
        h = C.c_void_p()
        check(lib.gg_volume_create(device, met_type, dims, es, C.byref(h)), "gg_volume_create")
        self.handle = h

    @property
    def elements(self):
        return self.dimensions[0] * self.dimensions[1] * self.dimensions[2]

    def close(self):
        if getattr(self, "handle", None):
            lib.gg_volume_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def draw(self, shapes):
        arr = (abi.gg_shape * len(shapes))(*shapes)
        check(lib.gg_volume_draw(self.handle, arr, len(shapes)), "gg_volume_draw")

    def upload(self, image):
        import numpy as np
        a = np.ascontiguousarray(image, self.dtype).reshape(-1)
        if a.size != self.elements:
            raise ValueError("image has %d elements, the volume %d" % (a.size, self.elements))
        check(lib.gg_volume_upload(self.handle, a.ctypes.data_as(C.c_void_p), a.nbytes), "gg_volume_upload")

    def download(self):
        import numpy as np
        a = np.empty(self.elements, self.dtype)
        check(lib.gg_volume_download(self.handle, a.ctypes.data_as(C.c_void_p), a.nbytes), "gg_volume_download")
        return a

    def labels(self, first, last):
        """uint8 labels of every element and the number left unconverted (255)."""
        import numpy as np
        f = np.ascontiguousarray(first, np.float32)
        l_ = np.ascontiguousarray(last, np.float32)
        out = np.empty(self.elements, np.uint8)
        missing = C.c_int64()
        check(lib.gg_volume_labels(self.handle, abi.ptr(f, C.c_float), abi.ptr(l_, C.c_float), len(f),
                                   abi.ptr(out, C.c_uint8), C.byref(missing)), "gg_volume_labels")
        return out, missing.value

    def last_kernel_ms(self):
        ms = C.c_float()
        check(lib.gg_volume_last_kernel_ms(self.handle, C.byref(ms)), "gg_volume_last_kernel_ms")
        return ms.value
