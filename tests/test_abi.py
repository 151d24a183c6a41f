"""CPU checks of the C ABI library: it loads and exports every symbol that
include/gemsgpu.h declares (no compute call; no GPU needed)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    with open(os.path.join(ROOT, "include", "gemsgpu.h")) as f:
        return set(re.findall(r"\b(gemsgpu_\w+)\s*\(", f.read()))


def test_library_exports_header_symbols():
    import gems_b200
    gems_b200.lib()  # loads (cudart is linked statically)
    out = subprocess.run(["nm", "-D", "--defined-only", gems_b200.gemsgpu.LIBPATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = header_symbols() - exported
    assert not missing, missing


def test_binding_covers_header():
    import gems_b200
    assert header_symbols() == set(gems_b200.declared_symbols())


def test_library_built_for_sm100a():
    import gems_b200
    out = subprocess.run(["cuobjdump", "--list-elf", gems_b200.gemsgpu.LIBPATH],
                         capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_no_device_errors_cleanly():
    """Without a GPU, creating a context returns an error code, not a crash."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import gems_b200
    with pytest.raises(gems_b200.GemsGpuError):
        gems_b200.Context()
