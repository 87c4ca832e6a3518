"""CPU tests of the C ABI library: it builds for sm_100a, loads without a GPU,
and exports every entry point include/uc.h declares."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(uc_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["uc_ctx_create", "uc_pack", "uc_minimizers", "uc_find_edges", "uc_contract", "uc_emit",
                 "uc_compact_device", "uc_compact_host", "uc_job_submit", "uc_compact_file"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from unitigcoarsening_b200 import build as B
    lib = B.build()
    out = subprocess.check_output(["nm", "-D", "--defined-only", lib], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    L = ctypes.CDLL(lib)  # loads on a machine without a GPU
    for n in declared_functions():
        assert getattr(L, n) is not None


def test_status_strings_without_gpu():
    from unitigcoarsening_b200 import lib
    L = lib()
    assert L.uc_status_str(0) == b"ok"
    assert L.uc_status_str(1) == b"invalid input"
    assert int(L.uc_output_bound(1000, 31)) >= 1000


def test_build_targets_sm100a_only():
    from unitigcoarsening_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
