"""The C ABI: libpiko_b200.so loads and exports every entry point that
include/*.h declares; host-only calls behave without a GPU."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(piko_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ["piko_ctx_create", "piko_pipe_create", "piko_scene_create", "piko_frame_prepare",
              "piko_frame_run", "piko_frame_read", "piko_scene_destroy", "piko_batch_run"]:
        assert n in names


def test_library_exports_every_declared_symbol(pk):
    lib = pk.load_library()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol(pk):
    from piko_b200 import runtime
    assert set(declared_symbols()) <= set(runtime.SIGNATURES)


def test_pipeline_descriptors_match_reference_stages(pk):
    from piko_b200 import runtime as rt
    lib = pk.load_library()
    d = rt.PipeDesc()
    lib.piko_pipe_desc_raster(ctypes.byref(d))
    assert d.n_stages == 2 and d.n_links == 1
    assert (d.stages[0].bin_size_x, d.stages[0].threads_per_tile) == (32, 512)   # vertexShader.pikostage:18
    assert (d.stages[1].bin_size_x, d.stages[1].threads_per_tile) == (8, 32)     # raster.pikostage:14,26
    lib.piko_pipe_desc_reyes(ctypes.byref(d))
    assert d.n_stages == 3 and d.n_links == 3
    assert [d.stages[i].bin_size_x for i in range(3)] == [0, 64, 64]
    links = {(d.links[i].out_stage, d.links[i].in_stage, d.links[i].out_port, d.links[i].in_port) for i in range(3)}
    assert (0, 0, 1, 1) in links   # pikoConnect(split, split, 1, 1), reyesPipe.h:31


def test_version_and_null_handling(pk):
    lib = pk.load_library()
    assert lib.piko_version().startswith(b"piko-b200")
    assert lib.piko_ctx_destroy(None) == 1          # PIKO_ERR_INVALID
    assert lib.piko_frame_run(None, None) == 1
    assert lib.piko_last_error(None) == b"no context"


def test_context_without_device_reports_no_device(pk):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from piko_b200 import runtime as rt
    lib = pk.load_library()
    h = ctypes.c_void_p()
    assert lib.piko_ctx_create(None, ctypes.byref(h)) == rt.ERR_NO_DEVICE
