"""The C ABI library loads and exports every entry point include/gccu.h
declares (no device calls)."""
import os
import re
import subprocess

import gccu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "gccu.h")).read()
    return sorted(set(re.findall(r"\bint\s+(gccu_\w+)\s*\(", text)))


def test_header_and_binding_agree(built):
    assert declared() == gccu.exported_symbols()


def test_library_exports_all_symbols(built):
    lib = gccu.lib()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", gccu.LIB_PATH], capture_output=True,
                         text=True).stdout
    for name in declared():
        assert re.search(r"\bT\s+" + name + r"\b", out), name


def test_build_targets_sm100a():
    # the engine is compiled for sm_100a only (the tcgen05 kernels need the
    # architecture-specific target); the device-side check is in
    # tests/test_gpu_device.py
    text = open(os.path.join(ROOT, "gecco-public_b200", "Makefile")).read()
    arch = re.search(r"^ARCH\s*:=\s*(.*)$", text, re.M).group(1).split()
    assert arch == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "$(ARCH)" in re.search(r"^NVFLAGS\s*:=.*(?:\n\s+.*)*", text, re.M).group(0)


def test_errors_are_reported(built):
    import pytest
    with pytest.raises(gccu.GccuError, match="gccu_init has not been called"):
        gccu._call("gccu_sync")
