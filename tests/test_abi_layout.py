"""The ctypes binding's struct layouts equal the C header's: a small C
program compiled against include/hfg.h prints every struct's size and field
offsets, which must match the ctypes mirrors (no GPU needed)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from hfgpu import lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "hfg_basis": L.HfgBasis,
    "hfg_jk_opts": L.JKOptions,
    "hfg_jk_stats": L.JKStats,
    "hfg_scf_opts": L.SCFOptions,
    "hfg_scf_result": L.SCFResult,
    "hfg_autotune_opts": L.AutotuneOptions,
    "hfg_autotune_result": L.AutotuneResult,
    "hfg_job": L.Job,
    "hfg_job_result": L.JobResult,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_the_header(tmp_path):
    lines = ['#include "hfg.h"', "#include <stdio.h>", "#include <stddef.h>", "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append('  printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for field, _ in cls._fields_:
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, field, cname, field))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = {}
    for ln in subprocess.check_output([str(exe)], text=True).splitlines():
        name, field, val = ln.split()
        got[(name, field)] = int(val)
    for cname, cls in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
