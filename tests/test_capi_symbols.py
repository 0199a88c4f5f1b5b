"""The C-ABI library builds, loads without a GPU and exports every function
include/scmc_gpu.h declares (no compute calls here)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "scmc_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(scmc_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("scmc_field", "scmc_cov", "scmc_field_device", "scmc_cov_device", "scmc_export_records",
              "scmc_last_error", "scmc_philox_stream"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from mcspeckle_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    lib.scmc_abi_version.restype = ctypes.c_int
    assert lib.scmc_abi_version() == 2


def test_python_struct_matches_header_layout():
    """The ctypes mirror has the C struct's field order and count."""
    from mcspeckle_b200 import _abi
    src = open(HEADER).read()
    body = src[src.index("typedef struct {\n    int32_t dim;"):]
    body = body[:body.index("} scmc_mc_args;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = re.findall(r"(\w+)(?:\[\d+\])?;", body)
    py = [f[0].rstrip("_") for f in _abi.McArgs._fields_]
    assert py == [f.rstrip("_") for f in fields]


def _header_fields(name):
    src = open(HEADER).read()
    body = src[:src.index("} %s;" % name)]
    body = body[body.rindex("typedef struct {"):]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    return re.findall(r"(\w+)(?:\[\d+\])?;", body)


def test_serving_structs_match_header_layout():
    from mcspeckle_b200 import _abi
    assert [f[0] for f in _abi.RequestInfo._fields_] == _header_fields("scmc_request_info")
    assert [f[0] for f in _abi.ServerStats._fields_] == _header_fields("scmc_server_stats")
    assert [f[0] for f in _abi.StageTimes._fields_] == _header_fields("scmc_stage_times")
    assert [f[0].rstrip("_") for f in _abi.FqArgs._fields_] == [f.rstrip("_") for f in _header_fields("scmc_fq_args")]


def test_server_create_without_gpu_fails_loudly():
    """No CPU fallback: without a visible sm_100 device the server refuses."""
    import torch
    if torch.cuda.is_available():
        return
    import ctypes as C
    from mcspeckle_b200 import _abi, _lib
    h = C.c_void_p()
    st = _lib.lib().scmc_server_create(0, 2, 0, C.byref(h))
    assert st in (_abi.SCMC_ERR_NODEVICE, _abi.SCMC_ERR_CUDA)
    assert not h.value
