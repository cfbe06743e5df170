"""One GGEMS run over several GPUs: one process per GPU, ``torch.distributed``.

Histories are independent, so the transport itself needs no exchange.  Ranks
play the roles of GGEMS's activated devices:

* rank r simulates its share of a source's primaries, split as
  GGEMSSource::OrganizeParticlesInBatch does (src/sources/GGEMSSource.cc:379-400:
  N / devices each with the remainder to the first devices, or the
  float-weighted device balancing with the rounding loss added to device 0);
* rank r uses the random streams GGEMS gives device r: the std::mt19937
  sequence of the seed after 4 * 2^20 draws per preceding device
  (src/randoms/GGEMSPseudoRandomGenerator.cc:140-167);
* at the end one collective sums the tallies over ranks: detector histograms
  as GGEMSSystem::SaveResults sums its devices' histograms
  (src/navigators/GGEMSSystem.cc:183-200), and dose tallies likewise
  (GGEMS overwrites the hit and energy-squared maps per device instead of
  summing them, GGEMSDosimetryCalculator.cc:623,713; that is not reproduced).

On GPUs the reduction runs on the device tallies themselves
(reduce_device_tallies): every buffer a context tallies into (gg_device_tallies)
is all-reduced in place over NCCL, the energy maps as the int64 fixed-point
integers the kernels add (LSB 2^-32 MeV), so the sums are exact at any size
and independent of the rank order, and nothing crosses to the host before
gg_read_tallies.  reduce_tallies does the same on host copies (gloo ranks,
CPU tests); there the energy arrives as doubles, exact while a dosel holds
less than 2^21 MeV.
"""

import ctypes as C

import numpy as np

from . import abi


def primaries_of_rank(total, world, rank, balance=None):
    """Primaries simulated by `rank` of `world` for a source of `total` primaries."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    if balance is None:
        return total // world + (1 if rank < total % world else 0)
    if len(balance) != world:
        raise ValueError("one balance weight per rank is needed")
    counts = [int(np.float32(total) * np.float32(w)) for w in balance]
    lost = total - sum(counts)
    counts[0] += abs(lost)
    return counts[rank]


def random_states_of_rank(seed, rank):
    """JKISS states (5 x 2^20 uint32, SoA) of GGEMS device `rank` for `seed`."""
    from ._native import lib
    states = np.zeros(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
    rc = lib.gg_seed_random_states(abi.ptr(states, C.c_uint32), abi.GG_MAXIMUM_PARTICLES, seed,
                                   rank * abi.GG_MAXIMUM_PARTICLES)
    if rc != 0:
        raise RuntimeError(lib.gg_last_error().decode())
    return states


def _all_reduce_sum(array, dist, group):
    import torch
    if array is None:
        return
    dtype = torch.int64 if array.dtype.kind in "iu" else torch.float64
    t = torch.from_numpy(np.ascontiguousarray(array)).to(dtype)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy()
    if array.dtype.kind in "iu" and (out > np.iinfo(array.dtype).max).any():
        raise OverflowError("tally sum exceeds %s" % array.dtype)
    array[...] = out.astype(array.dtype)


class _DeviceArray:
    """A device buffer seen through __cuda_array_interface__ (zero copy)."""

    TYPESTR = {abi.GG_TALLY_INT32: "<i4", abi.GG_TALLY_INT64: "<i8", abi.GG_TALLY_FP64: "<f8"}

    def __init__(self, tally):
        self.__cuda_array_interface__ = {"shape": (int(tally.count),), "typestr": self.TYPESTR[tally.type],
                                         "data": (int(tally.address), False), "version": 3, "strides": None}


def device_tallies(context):
    """The context's device tally buffers (gg_device_tallies) as torch tensors
    that alias them."""
    import torch
    from ._native import lib, check
    n = C.c_int32()
    check(lib.gg_device_tallies(context, None, 0, C.byref(n)), "gg_device_tallies")
    arr = (abi.gg_device_tally * max(n.value, 1))()
    check(lib.gg_device_tallies(context, arr, n.value, C.byref(n)), "gg_device_tallies")
    return [torch.as_tensor(_DeviceArray(arr[i]), device="cuda") for i in range(n.value)]


def reduce_device_tallies(context, group=None):
    """Sum the tallies of `context` (a gg_context handle) over all ranks of
    `group`, in place on every rank's GPU (NCCL): call after the run has
    finished (gg_synchronize), then read them with gg_read_tallies."""
    import torch
    import torch.distributed as dist
    tensors = device_tallies(context)
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    torch.cuda.synchronize()
    return len(tensors)


def reduce_tallies(tallies, group=None):
    """Sum an ``abi.Tallies`` (histograms, edep, edep^2, hits, photon tracking)
    over all ranks of `group`, in place on every rank."""
    import torch.distributed as dist
    for arrays in (tallies.histograms, tallies.edep, tallies.edep_squared, tallies.hit, tallies.photon_tracking):
        for a in arrays:
            _all_reduce_sum(a, dist, group)
    # world grid (GGEMSWorld::SaveResults sums its devices' grids, GGEMSWorld.cc:423-602)
    for a in (tallies.world or {}).values():
        _all_reduce_sum(a, dist, group)
    return tallies
