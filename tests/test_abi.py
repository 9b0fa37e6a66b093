"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

from conftest import REPO


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(s2l_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_symbols()
    for must in ("s2l_gpu_apply", "s2l_gpu_gmres", "s2l_gpu_bicgstab", "s2l_gpu_spmv", "s2l_gpu_setup_end"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from s2l_b200 import capi
    assert os.path.exists(capi.LIB_PATH), "libs2l_gpu.so was not built (run __graft_entry__.build())"
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(capi.EXPORTED) <= set(declared_symbols()) | {"s2l_gpu_setup_bytes"}


def test_create_without_device_fails_cleanly():
    """On a host without a GPU the library reports an error instead of falling back to the CPU."""
    import torch
    from s2l_b200 import capi
    if torch.cuda.is_available():
        return
    lib = capi.load()
    h = ctypes.c_void_p()
    rc = lib.s2l_gpu_create(0, 0, ctypes.byref(h))
    assert rc != capi.S2L_OK
