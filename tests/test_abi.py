"""The C-ABI library without a GPU: it loads, exports every function that
include/*.h declares, and a context on a machine without a usable device
reports an error instead of crashing."""
import ctypes
import glob
import importlib
import os
import re

import pytest

from conftest import REPO

HEADERS = sorted(glob.glob(os.path.join(REPO, "include", "*.h")))
DECL = re.compile(r"^(?:LVC|TKE|OP)_API\s+[^(]*?\b([A-Za-z_][A-Za-z_0-9]*)\s*\(", re.M)
# which library implements each header
HEADER_LIB = {"LocVolCalib.h": "liblvc.so", "tridiag.h": "liblvc.so", "tke.h": "libtke.so", "op.h": "libop.so"}


def declared_functions(lib_name: str = "liblvc.so"):
    names = []
    for h in HEADERS:
        assert os.path.basename(h) in HEADER_LIB, h
        if HEADER_LIB[os.path.basename(h)] != lib_name:
            continue
        with open(h) as f:
            names += DECL.findall(f.read())
    return names


def test_headers_declare_the_generated_api():
    names = set(declared_functions())
    for required in ("futhark_context_config_new", "futhark_context_new", "futhark_entry_main",
                     "futhark_values_f32_1d", "futhark_shape_f32_1d", "futhark_free_f32_1d",
                     "futhark_context_sync", "futhark_context_get_error", "futhark_context_free",
                     "futhark_context_config_free", "futhark_context_config_set_device"):
        assert required in names


@pytest.mark.parametrize("lib_name", sorted(set(HEADER_LIB.values())))
def test_library_exports_every_declared_symbol(lib_name):
    lib = ctypes.CDLL(os.path.join(REPO, "futhark-benchmarks_b200", lib_name))
    names = declared_functions(lib_name)
    assert names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_symbol(pkg):
    pkg.load_library()  # raises if a signature names a missing symbol


def test_tke_mirror_binds_every_declared_symbol(tke):
    # every function of include/tke.h has its C signature declared in the mirror
    lib = tke.load_library()
    unbound = [n for n in declared_functions("libtke.so") if getattr(lib, n).argtypes is None]
    assert not unbound, unbound


def test_op_mirror_binds_every_declared_symbol():
    op = importlib.import_module("futhark-benchmarks_b200.op")
    lib = op.load_library()
    unbound = [n for n in declared_functions("libop.so") if getattr(lib, n).argtypes is None]
    assert not unbound, unbound
    # struct op_args: seven int32 sizes, then nine pointers
    assert ctypes.sizeof(op._OpArgs) == 8 * 4 + 9 * 8


def test_tke_context_without_gpu_reports_error(tke, pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.FutharkError) as ei:
        tke.TkeContext()
    assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR


def test_op_context_without_gpu_reports_error(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    op = importlib.import_module("futhark-benchmarks_b200.op")
    with pytest.raises(pkg.FutharkError) as ei:
        op.OpContext()
    assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR


def test_tke_step_args_layout(tke):
    # struct tke_step_args: three int64 dimensions, then 27 pointers
    assert ctypes.sizeof(tke._StepArgs) == 3 * 8 + (len(tke.STEP_INPUTS) + len(tke.STEP_OUTPUTS) + 1) * 8
    assert len(tke.INPUT_NAMES) == 25 and len(tke.OUTPUT_NAMES) == 7


def test_context_without_gpu_reports_error(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.FutharkError) as ei:
        pkg.Context()
    assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR


def test_config_api_is_callable_without_gpu(pkg):
    lib = pkg.load_library()
    cfg = lib.futhark_context_config_new()
    assert cfg
    lib.futhark_context_config_set_device(cfg, b"#0")
    lib.futhark_context_config_set_debugging(cfg, 1)
    lib.futhark_context_config_set_cache_file(cfg, b"/nonexistent")
    lib.futhark_context_config_free(cfg)


def test_tuning_parameters_by_name(pkg):
    # the Futhark-generated API's tuning-parameter surface; no device needed
    lib = pkg.load_library()
    names = [lib.futhark_get_tuning_param_name(i).decode() for i in range(lib.futhark_get_tuning_param_count())]
    assert names == ["lvc.streams", "lvc.grid"]
    assert lib.futhark_get_tuning_param_name(len(names)) is None
    cfg = lib.futhark_context_config_new()
    try:
        assert lib.futhark_context_config_set_tuning_param(cfg, b"lvc.streams", 2) == 0
        assert lib.futhark_context_config_set_tuning_param(cfg, b"lvc.grid", 1) == 0
        assert lib.futhark_context_config_set_tuning_param(cfg, b"lvc.streams", 0) == 1
        assert lib.futhark_context_config_set_tuning_param(cfg, b"lvc.streams", 9) == 1
        assert lib.futhark_context_config_set_tuning_param(cfg, b"lvc.grid", 2) == 0
        assert lib.futhark_context_config_set_tuning_param(cfg, b"lvc.grid", 3) == 1
        assert lib.futhark_context_config_set_tuning_param(cfg, b"no.such.param", 1) == 1
    finally:
        lib.futhark_context_config_free(cfg)
