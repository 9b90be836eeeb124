"""The ctypes layouts of imagestackalignator_b200/isa.py against the C
structs of include/isa.h, without a GPU: a small C program compiled with gcc
prints sizeof and offsetof of every field; each must equal the ctypes
structure's size and field offset, so that a host binding built from the
header and the tests' binding pass the same bytes."""
import ctypes
import os
import subprocess

import pytest

from imagestackalignator_b200 import isa

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "isa_level": isa.IsaLevel,
    "isa_prealign": isa.IsaPrealign,
    "isa_track_pair": isa.IsaTrackPair,
    "isa_post_params": isa.IsaPostParams,
    "isa_raw_info": isa.IsaRawInfo,
    "isa_params": isa.IsaParams,
    "isa_dng_layout": isa.IsaDngLayout,
    "isa_dng_color_tags": isa.IsaDngColorTags,
    "isa_dng_level_tags": isa.IsaDngLevelTags,
    "isa_raw_levels": isa.IsaRawLevels,
    "isa_pef_info": isa.IsaPefInfo,
    "isa_burst": isa.IsaBurst,
    "isa_tuning": isa.IsaTuning,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "isa.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0; }")
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    return got


@pytest.mark.parametrize("cname", list(STRUCTS))
def test_ctypes_layout_matches_header(c_layout, cname):
    cls = STRUCTS[cname]
    assert ctypes.sizeof(cls) == c_layout[(cname, "size")]
    for fname, _ in cls._fields_:
        assert getattr(cls, fname).offset == c_layout[(cname, fname)], fname
