"""ggems_b200: GGEMS's photon-transport hot path on NVIDIA B200 (sm_100a).

``from ggems_b200 import *`` gives the GGEMS Python API (GGEMS,
GGEMSXRaySource, GGEMSVoxelizedPhantom, GGEMSCTSystem,
GGEMSDosimetryCalculator, ...) backed by ``libggems.so``.  The native library
is loaded on first use of an API name; ``ggems_b200.abi`` (the ctypes mirror
of include/ggems_b200.h) can be imported without it.
"""

_API = ("GGEMSError", "GGEMSVerbosity", "GGEMS", "GGEMSOpenCLManager", "GGEMSMaterialsDatabaseManager",
        "GGEMSMaterials", "GGEMSCrossSections", "GGEMSAttenuations", "GGEMSProcessesManager", "GGEMSRangeCutsManager",
        "GGEMSSourceManager", "GGEMSXRaySource", "GGEMSVoxelizedSource", "GGEMSVoxelizedPhantom", "GGEMSMeshedPhantom",
        "GGEMSWorld", "GGEMSVolumeCreatorManager", "GGEMSBox", "GGEMSTube", "GGEMSSphere",
        "GGEMSCTSystem", "GGEMSDosimetryCalculator", "GGEMSProfilerManager", "GGEMSRAMManager", "clean_safely")

__all__ = list(_API)


def __getattr__(name):
    if name in _API:
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
