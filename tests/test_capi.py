"""The C ABI without a GPU: the library loads, exports every entry point that
include/*.h declares, and the ctypes mirrors of its structs have the C
layout.  No compute calls are made."""
import ctypes
import glob
import os
import re
import subprocess
import tempfile

import pytest

import pbbsbench_b200 as pb
from pbbsbench_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(pbg_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = pb.lib()
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(L, name), name
    bound = {s[0] for s in _capi.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_library_is_sm100a_build():
    # the build recipe targets sm_100a only
    assert "arch=compute_100a,code=sm_100a" in " ".join(_capi.NVCC_FLAGS)
    assert os.path.exists(_capi.LIB_PATH)


def test_struct_layouts_match_c():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "pbbs_bfs.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(pbg_bfs_opts), sizeof(pbg_bfs_stats), sizeof(pbg_gen_params),
         offsetof(pbg_bfs_stats, visited), offsetof(pbg_bfs_stats, device_ms), offsetof(pbg_gen_params, a),
         offsetof(pbg_gen_params, perm_seed), sizeof(pbg_mis_stats), offsetof(pbg_mis_stats, device_ms));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_capi.BfsOpts), ctypes.sizeof(_capi.BfsStats), ctypes.sizeof(_capi.GenParams),
            _capi.BfsStats.visited.offset, _capi.BfsStats.device_ms.offset, _capi.GenParams.a.offset,
            _capi.GenParams.perm_seed.offset, ctypes.sizeof(_capi.MisStats), _capi.MisStats.device_ms.offset]
    assert got == want


def test_error_message_is_empty_initially_and_bad_args_report():
    L = pb.lib()
    # argument checks that return before touching the device
    h = ctypes.c_void_p()
    rc = L.pbg_graph_upload(None, None, 0, 0, 0, ctypes.byref(h))
    assert rc == 1
    assert b"NULL" in L.pbg_last_error()
    with pytest.raises(pb.PbgError):
        _capi.check(L.pbg_bfs_stats_get(None, None))


def test_default_opts():
    o = _capi.default_opts()
    assert (o.parent_mode, o.direction, o.alpha, o.beta) == (0, 0, 20, 20)
