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
