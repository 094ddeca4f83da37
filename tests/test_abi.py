"""CPU checks of the C ABI: the library loads without a GPU and exports every
entry point include/dpa_b200.h declares. No compute is called here."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import dpa_b200
from dpa_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "dpa_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(dpa_\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("dpa_curve_sink")))


def test_header_declares_the_bound_functions():
    names = declared_functions()
    assert len(names) >= 15
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = N.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIBRARY_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (dpa_\w+)", out))
    for name in declared_functions():
        assert name in exported, name
        assert getattr(lib, name) is not None


def test_version_and_names_without_gpu():
    lib = N.load()
    assert b"sm_100a" in lib.dpa_version()
    code = C.c_int32(-1)
    for name, want in N.INTEGRATORS.items():
        assert lib.dpa_integrator_from_name(name.encode(), C.byref(code)) == 0
        assert code.value == want
    assert lib.dpa_integrator_from_name(b"rk4", C.byref(code)) == 1


def test_null_arguments_are_rejected():
    lib = N.load()
    assert lib.dpa_context_destroy(None) == 1
    assert lib.dpa_context_synchronize(None) == 1
    assert lib.dpa_advect_round(None, None, None, 0, None, None, None, N.CURVE_SINK(), None) == 1
    assert lib.dpa_last_error(None) == b"no context"
    assert lib.dpa_context_create(0, None) == 1


def test_device_count_and_context_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = N.load()
    n = C.c_int(-1)
    assert lib.dpa_device_count(C.byref(n)) == 0
    assert n.value == 0
    with pytest.raises(dpa_b200.DpaError):
        dpa_b200.Context(0)


# ctypes mirrors of the header's structures, by typedef name.
STRUCTS = {
    "dpa_advect_options": N.AdvectOptions,
    "dpa_curve_chunk": N.CurveChunk,
    "dpa_tuning": N.Tuning,
    "dpa_server_options": N.ServerOptions,
    "dpa_request": N.Request,
    "dpa_response": N.Response,
    "dpa_server_stats": N.ServerStats,
}


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes structure has the size and field offsets that a C compiler
    gives the header's typedef (a field added on one side only would shift
    the fields after it)."""
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "dpa_b200.h"',
             "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(HEADER.parent), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        cname, what, value = line.split()
        got[(cname, what)] = int(value)
    for cname, py in STRUCTS.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
