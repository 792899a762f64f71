"""The ctypes mirrors of the C ABI structures (cellbasedmodels.jl_b200/_abi.py)
have the layout of include/cbm_b200.h: the same size, and every field at the
same offset with the same size.  A small C program built with gcc against the
header prints sizeof/offsetof; no CUDA call is made."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

import conftest

abi = conftest.cbm._abi

STRUCTS = {
    "cbm_config": abi.CbmConfig,
    "cbm_state_view": abi.CbmStateView,
    "cbm_community_desc": abi.CbmCommunityDesc,
    "cbm_batch_tuning": abi.CbmBatchTuning,
    "cbm_medium_config": abi.CbmMediumConfig,
    "cbm_rods_config": abi.CbmRodsConfig,
}


def _c_layout(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "cbm_b200.h"',
             "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} . %zu %zu\\n", sizeof({cname}), (size_t)0);')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu %zu\\n", '
                         f"offsetof({cname}, {fname}), sizeof((({cname}*)0)->{fname}));")
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(conftest.ROOT, "include"), "-o",
                    str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        cname, fname, a, b = line.split()
        table[(cname, fname)] = (int(a), int(b))
    return table


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header(tmp_path):
    table = _c_layout(tmp_path)
    for cname, cls in STRUCTS.items():
        assert table[(cname, ".")][0] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            field = getattr(cls, fname)
            assert table[(cname, fname)] == (field.offset, field.size), (cname, fname)


JULIA_TYPES = {"Int32": C.c_int32, "Int64": C.c_int64, "UInt32": C.c_uint32,
               "UInt64": C.c_uint64, "Float64": C.c_double}


def _julia_structs():
    """name -> [(field, Julia type)] of the `struct Cbm... end` blocks of the
    Julia stubs."""
    import re
    text = open(os.path.join(conftest.ROOT, "INTEGRATION.md")).read()
    out = {}
    for m in re.finditer(r"^(?:mutable )?struct (Cbm\w+)\n(.*?)^end", text, flags=re.S | re.M):
        fields = []
        for part in re.split(r"[;\n]", m.group(2)):
            part = part.strip()
            if part:
                name, typ = part.split("::")
                fields.append((name.strip(), typ.strip()))
        out[m.group(1)] = fields
    return out


def _ctype_of(julia):
    import re
    m = re.fullmatch(r"NTuple\{(\d+),(\w+)\}", julia)
    if m:
        return JULIA_TYPES[m.group(2)] * int(m.group(1))
    return JULIA_TYPES[julia]


def test_julia_stub_structs_match_the_mirrors():
    """The Julia mirrors in the ccall stubs list the C fields in order, with
    types of the same size (Julia cannot run here, so the text is checked)."""
    jl = _julia_structs()
    for name in ("CbmConfig", "CbmCommunityDesc", "CbmBatchTuning", "CbmMediumConfig",
                 "CbmRodsConfig"):
        cls = getattr(abi, name)
        assert [f for f, _ in jl[name]] == [f for f, _ in cls._fields_], name
        for (f, jt), (_, ct) in zip(jl[name], cls._fields_):
            assert C.sizeof(_ctype_of(jt)) == C.sizeof(ct), (name, f)
