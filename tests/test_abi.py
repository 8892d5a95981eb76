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
    assert lib.swdk_config_default(None) == -1
    assert lib.swdk_create(None, None) == -1
    assert lib.swdk_kmax(None) == 0
