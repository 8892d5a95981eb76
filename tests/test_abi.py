"""CPU checks of the C-ABI boundary: the library loads, exports every
function include/swdk.h declares, and the product path fails loudly without
a GPU instead of falling back to the CPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(swdk_\w+)\s*\(", txt)))


def _lib():
    from jdsurfg_b200 import build as B
    B.build()
    return C.CDLL(os.path.join(ROOT, "jdsurfg_b200", "libswdk.so"))


def test_library_exports_every_declared_symbol():
    lib = _lib()
    names = _declared("swdk.h")
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from jdsurfg_b200 import Engine, SwdkError
    with pytest.raises(SwdkError):
        Engine()


def test_config_defaults_and_arg_checks():
    lib = _lib()
    from jdsurfg_b200.engine import Config
    cfg = Config()
    assert lib.swdk_config_default(C.byref(cfg)) == 0
    assert cfg.refine == 1 and cfg.sngl == 1 and cfg.sphere == 1 and abs(cfg.rtol - 1e-10) < 1e-20
    # node-rebuilt layers on; no call splits into column halves unless asked
    assert cfg.node_layers == 1 and cfg.split_cols == 0 and cfg.block_roots == 0
    assert lib.swdk_config_default(None) == -1
    assert lib.swdk_create(None, None) == -1
    assert lib.swdk_kmax(None) == 0
    # proposals: a null context is refused before any CUDA call
    lib.swdk_set_proposal_shift.argtypes = [C.c_void_p, C.c_double]
    assert lib.swdk_set_proposal_shift(None, 0.1) == -1
    lib.swdk_set_proposal.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double]
    assert lib.swdk_set_proposal(None, None, None, 1.0, 1.0) == -1


def test_fmst_entry_points_check_arguments_without_gpu():
    """swdk_fmst_*: bad arguments are refused with SWDK_E_ARG before any CUDA
    call, and creating a handle without a GPU fails instead of falling back."""
    import torch
    lib = _lib()
    from jdsurfg_b200.fmst import Grid
    vp = C.c_void_p
    lib.swdk_fmst_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(Grid)]
    lib.swdk_fmst_set_options.argtypes = [vp, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.swdk_fmst_pairs.argtypes = [vp, C.c_int] + [vp] * 9 + [C.c_int] + [vp] * 4
    h = vp()
    assert lib.swdk_fmst_create(None, 0, None) == -1
    assert lib.swdk_fmst_create(C.byref(h), 0, C.byref(Grid(3, 10, 40.0, 100.0, 0.3, 0.3))) == -1
    assert lib.swdk_fmst_create(C.byref(h), 0, C.byref(Grid(10, 10, 40.0, 100.0, 0.0, 0.3))) == -1
    assert lib.swdk_fmst_set_options(None, 0, 8, 12, -1, 4) == -1
    assert lib.swdk_fmst_pairs(None, 1, *([None] * 9), 1, None, None, None, None) == -1
    if not torch.cuda.is_available():
        rc = lib.swdk_fmst_create(C.byref(h), 0, C.byref(Grid(10, 12, 40.0, 100.0, 0.3, 0.3)))
        assert rc != 0 and not h.value
