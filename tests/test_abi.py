"""The C ABI: the library loads without a GPU, exports every function that
include/*.h declares, and the ctypes mirror in crushrs_b200/abi.py has the
same struct sizes and field offsets as a C compiler gives the headers."""
import ctypes as C
import os
import re
import shutil
import subprocess
import tempfile

import pytest

from crushrs_b200 import abi
from crushrs_b200.native import LIB_PATH, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
HEADERS = sorted(f for f in os.listdir(INCLUDE) if f.endswith(".h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**\s*(crush_[a-z0-9_]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_every_declared_function():
    handle = lib()
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(handle, n)]
    assert not missing, missing
    assert os.path.exists(LIB_PATH)


def test_last_error_is_a_string_before_any_call():
    assert isinstance(lib().crush_last_error(), bytes)


STRUCTS = {
    "crush_material": abi.Material, "crush_contact": abi.Contact, "crush_settings": abi.Settings, "crush_vehicle": abi.Vehicle,
    "crush_model_desc": abi.ModelDesc, "crush_vehicle_result": abi.VehicleResult, "crush_results": abi.Results,
    "crush_vehicle_spec": abi.VehicleSpec, "crush_scenario": abi.Scenario, "crush_tuning": abi.Tuning,
    "crush_contact_stats": abi.ContactStats, "crush_server_config": abi.ServerConfig, "crush_server_result": abi.ServerResult,
    "crush_server_stats": abi.ServerStats,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_the_headers():
    lines = ['#include <stdio.h>', '#include <stddef.h>'] + [f'#include "{h}"' for h in HEADERS] + ["int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} __sizeof__ %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-I", INCLUDE, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            parts = line.split()
            got[tuple(parts[:-1])] = int(parts[-1])
    for cname, py in STRUCTS.items():
        assert got[(cname, "__sizeof__")] == C.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])


def test_batch_solve_rejects_bad_arguments_before_touching_a_device():
    """crush_batch_solve checks its arguments first: no models, a null
    model or a null output array is CRUSH_ERR_INVALID with a message."""
    import ctypes as C

    from crushrs_b200 import scenarios as S
    from crushrs_b200.native import lib

    L = lib()
    m = S.Model.build(S.batch_headon(0))
    arr = (C.POINTER(abi.ModelDesc) * 1)(C.pointer(m.desc))
    out = (abi.Results * 1)()
    assert L.crush_batch_solve(arr, 0, 0, out) == abi.CRUSH_ERR_INVALID
    assert L.crush_batch_solve(arr, 1, 0, None) == abi.CRUSH_ERR_INVALID
    nulls = (C.POINTER(abi.ModelDesc) * 1)()
    assert L.crush_batch_solve(nulls, 1, 0, out) == abi.CRUSH_ERR_INVALID
    assert L.crush_last_error().decode()
