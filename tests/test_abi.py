"""The C-ABI library loads and exports every entry point include/stwo_b200.h declares (no GPU needed)."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "stwo_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(stwo_b200_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "stwo_b200_prove_wide_fibonacci" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    import stwo_b200
    out = subprocess.run(["nm", "-D", "--defined-only", stwo_b200.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(stwo_b200.lib(), n)  # resolvable through ctypes


def test_binding_covers_header():
    import stwo_b200
    assert set(declared_functions()) <= set(stwo_b200.EXPORTED_SYMBOLS) | {"stwo_b200_telemetry_snapshot"}


def test_status_strings_and_telemetry_without_device():
    import stwo_b200
    assert stwo_b200.lib().stwo_b200_status_string(stwo_b200.E_CONSTRAINTS) == b"constraints not satisfied"
    assert stwo_b200.lib().stwo_b200_version().startswith(b"stwo_b200")
    assert stwo_b200.kernel_launches() >= 0
