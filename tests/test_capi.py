"""CPU tests of the C ABI library: it builds for sm_100a, loads without a GPU,
and exports every entry point include/uc.h declares."""
import ctypes
import os
import re
import subprocess

import pytest

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


# The three config files the reference ships (base, cond, fourpart), written
# out in their form: six numeric lines, then one word (no final newline).
# The reference's code never reads them; the CLI accepts this form and
# rejects others without touching a GPU (--check).
REFERENCE_CONFIGS = {
    "base_config.txt": "4\n0\n0\n2\n10\n1e-10\nnone",
    "cond_config.txt": "2\n0\n0\n2\n10\n1e-10\nnone",
    "fourpart_config.txt": "4\n0\n0\n4\n10\n1e-10\nnone",
}


def _cli(tmp_path, *extra):
    from unitigcoarsening_b200 import build as B
    B.build()
    inp = tmp_path / "in.txt"
    inp.write_text("3\nACG\nCGT\nGTA\n")
    return subprocess.run([B.CLI, str(inp), "3", "2", str(tmp_path / "out.txt"), "--check", *extra],
                          capture_output=True, text=True)


def test_cli_accepts_reference_config_files(tmp_path):
    ref_dir = os.environ.get("UC_REFERENCE_DIR", "")
    for name, body in REFERENCE_CONFIGS.items():
        p = tmp_path / name
        p.write_text(body)
        r = _cli(tmp_path, "--config", str(p))
        assert r.returncode == 0, r.stderr
        assert "ok: 3 k-mers" in r.stdout
        # the reference's own copy, where its tree is at hand
        q = os.path.join(ref_dir, name)
        if ref_dir and os.path.exists(q):
            r = _cli(tmp_path, "--config", q)
            assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("body", ["4\n0\nx\n2\n10\n1e-10\nnone", "4\n0\n0\n2\n10\n1e-10", "4\n0\n0\n2\n10\n1e-10\nno ne",
                                  "4\n0\n0\n2\n10\n1e-10\nnone\n7\n", "4 5\n0\n0\n2\n10\n1e-10\nnone", ""])
def test_cli_rejects_other_config_files(tmp_path, body):
    p = tmp_path / "cfg.txt"
    p.write_text(body)
    r = _cli(tmp_path, "--config", str(p))
    assert r.returncode != 0
    assert "config" in r.stderr


def test_cli_check_rejects_bad_arguments(tmp_path):
    assert _cli(tmp_path).returncode == 0
    from unitigcoarsening_b200 import build as B
    r = subprocess.run([B.CLI, "in.txt", "3", "2"], capture_output=True, text=True)
    assert r.returncode != 0 and "Usage" in r.stderr
    inp = tmp_path / "in.txt"
    inp.write_text("3\nACG\nCGT\nGTA\n")
    r = subprocess.run([B.CLI, str(inp), "3", "3", str(tmp_path / "o.txt"), "--check"], capture_output=True, text=True)
    assert r.returncode != 0  # l must be below k


def test_binding_structs_match_the_header(tmp_path):
    """The ctypes structures of the Python binding have the sizes and field
    offsets of the C structs in include/uc.h (compiled and printed by the
    host compiler; a field renamed or reordered on one side fails here)."""
    from unitigcoarsening_b200 import api
    structs = {"uc_stats": api.Stats, "uc_tuning": api.Tuning, "uc_faults": api.Faults,
               "uc_server_config": api.ServerConfig, "uc_server_job_info": api.JobInfo,
               "uc_server_totals": api.ServerTotals}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "uc.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        name, field, value = ln.split()
        got[(name, field)] = int(value)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
