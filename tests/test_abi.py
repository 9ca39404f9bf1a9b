"""The C ABI library loads on a machine without a GPU, exports every entry point
include/rbgpu.h declares, and reports the absence of a device as an error."""
import ctypes
import os
import re

import rainbow_b200 as rb
from rainbow_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "rbgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:rb_status|void|int32_t|char\s*\*|const char\s*\*)\s*\*?\s*(rb_[a-z_0-9]+)\s*\(",
                                 text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_native.SIGNATURES), sorted(set(names) - set(_native.SIGNATURES))


def test_abi_version_and_status_strings():
    assert rb.lib().rb_abi_version() == 10
    for code in range(12):
        assert rb.lib().rb_status_string(code)
    assert rb.lib().rb_status_string(999) == b"unknown status"


def test_context_without_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    assert rb.lib().rb_context_create(ctypes.byref(h), 0) == 11  # RB_ERR_NO_DEVICE
    assert rb.lib().rb_context_create(None, 0) == 1


def test_cpp_program_on_the_c_abi_reports_no_device_without_a_gpu():
    """tests/native/c_abi_example drives the C ABI from C++; without a GPU the
    library reports RB_ERR_NO_DEVICE (there is no CPU fallback)."""
    import subprocess
    import torch
    if torch.cuda.is_available():
        return
    exe = os.path.join(ROOT, "tests", "native", "c_abi_example")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.startswith("no device"), out.stdout + out.stderr
