"""The Python mirror's ctypes structures match the C ABI's struct layouts (no GPU).

A small C program, compiled with gcc against include/dualres_b200.h, prints sizeof
and offsetof of every field of every public struct; each must equal the ctypes
mirror's (dualres_b200/api.py). A drift between the header and the mirror would
otherwise pass garbage across the boundary without an error."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

from dualres_b200 import api

MIRRORS = {
    "dr_volume_desc": api.VolumeDesc,
    "dr_volume_info": api.VolumeInfo,
    "dr_hmc_opts": api.HmcOpts,
    "dr_chain_stats": api.ChainStats,
    "dr_server_opts": api.ServerOpts,
    "dr_job_status": api.JobStatus,
    "dr_server_stats": api.ServerStats,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "dualres_b200.h"', "int main(void) {"]
    for cname, cls in MIRRORS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        cname, field, value = line.split()
        layout[(cname, field)] = int(value)
    return layout


@pytest.mark.parametrize("cname", sorted(MIRRORS))
def test_ctypes_mirror_matches_header(c_layout, cname):
    cls = MIRRORS[cname]
    assert c_layout[(cname, "sizeof")] == ctypes.sizeof(cls), cname
    for f, _ in cls._fields_:
        assert c_layout[(cname, f)] == getattr(cls, f).offset, (cname, f)


def _header_prototypes():
    import re
    src = open(os.path.join(ROOT, "include", "dualres_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for ret, name, args in re.findall(r"\b([A-Za-z_][\w\s\*]*?)\b(dr_\w+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
        args = " ".join(args.split())
        out[name] = (ret.strip(), [] if args in ("", "void") else [a.strip() for a in args.split(",")])
    return out


def _c_kind(decl):
    """Coarse kind of one C parameter declaration."""
    if "*" in decl:
        return "ptr"
    t = decl.split()[:-1] if len(decl.split()) > 1 else decl.split()
    t = " ".join(w for w in t if w != "const")
    return {"int": "i32", "int64_t": "i64", "uint64_t": "u64", "float": "f32", "double": "f64"}.get(t, t)


def _ctypes_kind(t):
    if t in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(t, type) and issubclass(t, ctypes._Pointer)):
        return "ptr"
    for kind, ct in (("i32", ctypes.c_int), ("i64", ctypes.c_int64), ("u64", ctypes.c_uint64),
                     ("f32", ctypes.c_float), ("f64", ctypes.c_double)):
        if t is ct:
            return kind
    return repr(t)


def test_ctypes_signatures_match_header_prototypes():
    protos = _header_prototypes()
    L = api.lib(build_if_missing=False)
    checked = 0
    for name, (_, params) in sorted(protos.items()):
        fn = getattr(L, name, None)
        if fn is None or fn.argtypes is None:
            continue
        assert len(fn.argtypes) == len(params), (name, params, fn.argtypes)
        for decl, t in zip(params, fn.argtypes):
            assert _c_kind(decl) == _ctypes_kind(t), (name, decl, t)
        checked += 1
    assert checked >= 30, checked
