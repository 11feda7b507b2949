"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/tbg.h declares, its struct layouts match the reference's and the
Python binding's, and error paths return the documented status codes."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(tbg):
    L = tbg.lib()
    names = tbg.exported_symbols()
    assert {"RHO", "RHT", "RSM", "PSM", "tbg_join_device", "tbg_find"} <= set(names)
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/tbg.h but not exported"


LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include "tbg.h"
#define P(T) printf(#T " %zu\n", sizeof(T))
#define O(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
  P(struct row_t); P(struct table_t); P(struct output_list_t); P(struct threadresult_t);
  P(struct result_t); P(algorithm_t); P(tbg_config); P(tbg_stats); P(tbg_row_out);
  O(struct table_t, num_tuples); O(struct table_t, sorted); O(struct output_list_t, next);
  O(struct threadresult_t, threadid); O(struct result_t, nthreads); O(algorithm_t, join);
  O(tbg_config, seed); O(tbg_config, timing); O(tbg_stats, ms_total); O(tbg_stats, kernel_launches);
  P(tbg_batch_join); O(tbg_batch_join, nS);
  return 0;
}
"""


def test_struct_layouts(tbg):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(src, "w").write(LAYOUT_C)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = dict(l.rsplit(" ", 1) for l in subprocess.run([exe], capture_output=True, text=True,
                                                            check=True).stdout.splitlines())
    out = {k: int(v) for k, v in out.items()}
    # the reference's layouts on LP64 (Include/data-types.h:44-93)
    assert out["struct row_t"] == 8
    assert out["struct table_t"] == 24 and out["struct table_t.num_tuples"] == 8
    assert out["struct output_list_t"] == 24 and out["struct output_list_t.next"] == 16
    assert out["struct threadresult_t"] == 24 and out["struct result_t"] == 24
    assert out["algorithm_t"] == 136 and out["algorithm_t.join"] == 128
    assert out["tbg_row_out"] == 12
    # the Python binding mirrors the C structs
    assert C.sizeof(tbg.Table) == out["struct table_t"]
    assert C.sizeof(tbg.Result) == out["struct result_t"]
    assert C.sizeof(tbg.ThreadResult) == out["struct threadresult_t"]
    assert C.sizeof(tbg.OutputList) == out["struct output_list_t"]
    assert C.sizeof(tbg.Algorithm) == out["algorithm_t"]
    assert C.sizeof(tbg.Config) == out["tbg_config"]
    assert tbg.Config.seed.offset == out["tbg_config.seed"]
    assert C.sizeof(tbg.Stats) == out["tbg_stats"]
    assert tbg.Stats.ms_total.offset == out["tbg_stats.ms_total"]
    assert C.sizeof(tbg.BatchJoin) == out["tbg_batch_join"] == 32
    assert tbg.BatchJoin.nS.offset == out["tbg_batch_join.nS"]


def test_registry(tbg):
    L = tbg.lib()
    for name in ("RHO", "RHT", "RSM", "PSM", "LRN"):
        a = L.tbg_find(name.encode())
        assert a and a.contents.name.decode() == name
    assert not L.tbg_find(b"NPO_st")
    assert L.tbg_last_error() == tbg.ERR_UNKNOWN_ALGO
    with pytest.raises(tbg.TbgError):
        tbg.find("MWAY")


def test_device_api_argument_errors(tbg):
    L = tbg.lib()
    cfg = tbg.config("RHO")
    m = C.c_uint64()
    # null relation with rows
    assert L.tbg_join_device(C.byref(cfg), None, 10, None, 10, None, 0, C.byref(m), None, None) == tbg.ERR_ARG
    # misaligned pointers
    assert L.tbg_join_device(C.byref(cfg), 4, 10, 8, 10, None, 0, C.byref(m), None, None) == tbg.ERR_ARG
    # unknown algorithm id
    bad = tbg.config("RHO")
    bad.algo = 42
    assert L.tbg_join_device(C.byref(bad), 8, 1, 8, 1, None, 0, C.byref(m), None, None) == tbg.ERR_ARG
    assert L.tbg_join_device(None, 8, 1, 8, 1, None, 0, C.byref(m), None, None) == tbg.ERR_ARG


def test_dropin_slice_setting(tbg):
    """tbg_set_dropin_slices returns the previous setting and clamps to
    0 (automatic) .. 16; it needs no device."""
    prev = tbg.set_dropin_slices(3)
    try:
        assert tbg.set_dropin_slices(40) == 3
        assert tbg.set_dropin_slices(-5) == 16
        assert tbg.set_dropin_slices(1) == 0
        assert tbg.set_dropin_slices(0) == 1
    finally:
        tbg.set_dropin_slices(prev)


def test_dropin_without_gpu_returns_status(tbg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    R = np.zeros(4, dtype=tbg.ROW)
    with pytest.raises(tbg.TbgError) as e:
        tbg.find("RHO").join(R, R, 2)
    assert e.value.code == tbg.ERR_NO_DEVICE


def test_dropin_exit_mode_mirrors_reference(tbg):
    """Default error mode exits with EXIT_FAILURE like Include/util.c:11-18."""
    code = f"""
import ctypes as C, importlib, sys, numpy as np
sys.path.insert(0, {ROOT!r})
t = importlib.import_module('tee-bench_b200')
L = t.lib()
L.tbg_set_error_mode(t.ERRMODE_EXIT)
R = np.zeros(4, dtype=t.ROW)
tr = t.table(R)
# null relation pointer: an argument error, reported before any device use
L.RHO(None, C.byref(tr), 1)
print('not reached')
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode == 1, r.stderr
    assert "[ERROR]" in r.stderr and "not reached" not in r.stdout


def test_shard_of_matches_the_host_rule(tbg):
    """tbg_shard_of (a host function of the library) and the package's numpy
    shard_of give every key the same shard."""
    import numpy as np
    L = tbg.lib()
    keys = np.random.default_rng(3).integers(0, 2 ** 32, 2000, dtype=np.uint64).astype(np.uint32)
    keys[:3] = [0, 1, 0xFFFFFFFF]
    for n in (1, 2, 3, 7, 8, 256):
        want = tbg.shard_of(keys, n)
        got = [L.tbg_shard_of(int(k), n) for k in keys]
        assert list(want) == got
        assert want.min() >= 0 and want.max() < n
