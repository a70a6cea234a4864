"""piko-public_b200: Piko's binned raster and Reyes pipelines on one B200.

The product is libpiko_b200.so (C ABI: include/piko_b200.h), built from
csrc/ by build.py: hand-written sm_100a kernels for every stage phase and a
C++ host runtime.  This package adds the ctypes binding (runtime), a Python
mirror of the reference's pipeline classes (pipes), seeded synthetic
workloads (scenes) and host camera matrices (camera).

Import it as ``piko_b200`` (the directory name is not an identifier):

    import importlib.util, sys
    spec = importlib.util.spec_from_file_location(
        "piko_b200", "piko-public_b200/__init__.py",
        submodule_search_locations=["piko-public_b200"])
"""
from . import camera, scenes  # noqa: F401
from .runtime import (Asset, Batch, Context, Pipe, PikoError, Scene, Server, Tuner, const_state,  # noqa: F401
                      load_library, tune_bucket, write_bmp, LIB_PATH)
from .pipes import (ConstantState, MutableState, PikoScreen, RasterPipe, ReyesPipe,  # noqa: F401
                    piko_patch, raster_wtri)

__all__ = ["camera", "scenes", "Asset", "Batch", "Context", "Pipe", "PikoError", "Scene", "Server", "Tuner", "const_state",
           "load_library", "tune_bucket", "write_bmp",
           "ConstantState", "MutableState", "PikoScreen", "RasterPipe", "ReyesPipe", "piko_patch", "raster_wtri"]
