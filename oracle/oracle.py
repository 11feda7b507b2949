"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this module, and only as the checker or as the timed CPU
reference.  Two libraries sit behind it:

* ``_build/libtbo.so``  -- tbo.c, a plain-C restatement of the reference's
  generators (App/Lib/generator.cpp, App/Lib/genzipf.c) and its RHO / RHT
  radix join (Joins/radix_join.c);
* ``_ref/libtbref[_mat].so`` -- the reference's own join sources compiled by
  oracle/Makefile (present wherever they were built; absent otherwise).

Relations are numpy arrays of dtype ``ROW`` (uint32 key, uint32 payload), the
layout of ``struct row_t`` (Include/data-types.h:44-47).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROW = np.dtype([("key", "<u4"), ("payload", "<u4")])

_lib = None
_ref = {}


def build():
    """Compile the restatement (and the reference, when its tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_build", "libtbo.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P, U64, I64, I, D = C.c_void_p, C.c_uint64, C.c_int64, C.c_int, C.c_double
        L.tbo_seed.argtypes = [C.c_uint]
        L.tbo_gen_pk.argtypes = [P, U64]
        L.tbo_gen_fk.argtypes = [P, U64, I64]
        L.tbo_gen_fk_sel.argtypes = [P, U64, I64]
        L.tbo_gen_zipf.argtypes = [P, U64, C.c_uint32, D]
        L.tbo_fill_payloads.argtypes = [P, U64, I]
        for f in (L.tbo_rho, L.tbo_rht):
            f.argtypes = [P, U64, P, U64, I, I, P, U64]
            f.restype = I64
        L.tbo_radix_hist.argtypes = [P, U64, I, I, P]
        L.tbo_row_hash.argtypes = [C.c_uint32] * 3
        L.tbo_row_hash.restype = U64
        L.tbo_rows_checksum.argtypes = [P, U64]
        L.tbo_rows_checksum.restype = U64
        L.tbo_join_direct.argtypes = [P, U64, P, U64, I, C.POINTER(I64), C.POINTER(U64)]
        L.tbo_join_direct.restype = I
        L.tbo_mlp_loss_grad.argtypes = [I, P, P, P, U64, P]
        L.tbo_mlp_loss_grad.restype = D
        L.tbo_mlp_forward.argtypes = [I, P, P, U64, P]
        _lib = L
    return _lib


def ref(materialize: bool = False):
    """The reference's own join library, or None where it was never built."""
    name = "libtbref_mat.so" if materialize else "libtbref.so"
    if name not in _ref:
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            _ref[name] = None
        else:
            L = C.CDLL(path)
            L.tbref_seed.argtypes = [C.c_uint]
            L.tbref_gen.argtypes = [C.c_int, C.c_void_p, C.c_uint64, C.c_int64, C.c_double]
            L.tbref_gen.restype = C.c_int
            L.tbref_join.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                     C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_int64),
                                     C.POINTER(C.c_double)]
            L.tbref_join.restype = C.c_int64
            _ref[name] = L
    return _ref[name]


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


# ---------------------------------------------------------------- generators
def seed(s: int):
    lib().tbo_seed(s)


def gen(kind: str, n: int, maxid: int = 0, zipf: float = 0.0, payload_kind: int | None = None):
    """Generate a relation with the restated reference generator.

    kind: 'pk' | 'fk' | 'fk_sel' | 'zipf'.  Uses the glibc rand() stream that
    the last seed() call set, exactly as the reference does."""
    rows = np.zeros(n, dtype=ROW)
    L = lib()
    if kind == "pk":
        L.tbo_gen_pk(_p(rows), n)
    elif kind == "fk":
        L.tbo_gen_fk(_p(rows), n, maxid)
    elif kind == "fk_sel":
        L.tbo_gen_fk_sel(_p(rows), n, maxid)
    elif kind == "zipf":
        L.tbo_gen_zipf(_p(rows), n, maxid, zipf)
    else:
        raise ValueError(kind)
    if payload_kind is not None:
        L.tbo_fill_payloads(_p(rows), n, payload_kind)
    return rows


def fill_payloads(rows, kind: int):
    lib().tbo_fill_payloads(_p(rows), len(rows), kind)
    return rows


def ref_gen(kind: str, n: int, maxid: int = 0, zipf: float = 0.0):
    """Same as gen() but through the reference's own generator sources."""
    L = ref()
    if L is None:
        raise RuntimeError("reference library not built")
    rows = np.zeros(n, dtype=ROW)
    k = {"pk": 0, "fk": 1, "fk_sel": 2, "zipf": 3}[kind]
    if L.tbref_gen(k, _p(rows), n, maxid, zipf) != 0:
        raise RuntimeError("reference generator failed")
    return rows


def ref_seed(s: int):
    ref().tbref_seed(s)


# -------------------------------------------------------------------- joins
def rho(R, S, radix_bits=14, passes=2, materialize=False, algo="RHO"):
    """Restated RHO (or RHT): returns count, or (count, rows[n,3]) when materialising."""
    L = lib()
    f = L.tbo_rho if algo == "RHO" else L.tbo_rht
    if not materialize:
        return int(f(_p(R), len(R), _p(S), len(S), radix_bits, passes, None, 0))
    cnt = int(f(_p(R), len(R), _p(S), len(S), radix_bits, passes, None, 0))
    out = np.zeros((max(cnt, 1), 3), dtype=np.uint32)
    cnt2 = int(f(_p(R), len(R), _p(S), len(S), radix_bits, passes, _p(out), cnt))
    assert cnt2 == cnt
    return cnt, out[:cnt]


def ref_join(name, R, S, nthreads=1, materialize=False):
    """The reference's own join: (count, rows or None, runtime_us)."""
    L = ref(materialize)
    if L is None:
        raise RuntimeError("reference library not built")
    nrows = C.c_int64(0)
    rt = C.c_double(0)
    cap = 0
    out = None
    if materialize:
        cap = len(S) * 4 + 16
        out = np.zeros((cap, 3), dtype=np.uint32)
    cnt = int(L.tbref_join(name.encode(), _p(R), len(R), _p(S), len(S), nthreads, _p(out), cap,
                           C.byref(nrows), C.byref(rt)))
    rows = out[: min(nrows.value, cap)] if materialize else None
    return cnt, rows, rt.value


def radix_hist(rows, radix_bits=14, passes=2):
    h = np.zeros(1 << radix_bits, dtype=np.uint64)
    lib().tbo_radix_hist(_p(rows), len(rows), radix_bits, passes, _p(h))
    return h


def rows_checksum(rows3):
    rows3 = np.ascontiguousarray(rows3, dtype=np.uint32)
    return int(lib().tbo_rows_checksum(_p(rows3), len(rows3)))


def join_direct(R, S, nthreads=None):
    """Count and row checksum of the equi-join by direct key addressing."""
    nthreads = nthreads or min(64, os.cpu_count() or 1)
    c = C.c_int64(0)
    s = C.c_uint64(0)
    rv = lib().tbo_join_direct(_p(R), len(R), _p(S), len(S), nthreads, C.byref(c), C.byref(s))
    if rv != 0:
        raise MemoryError("tbo_join_direct")
    return int(c.value), int(s.value)


def sort_rows(rows3):
    """Canonical order of materialised rows: by (key, Rpayload, Spayload)."""
    rows3 = np.asarray(rows3, dtype=np.uint32).reshape(-1, 3)
    order = np.lexsort((rows3[:, 2], rows3[:, 1], rows3[:, 0]))
    return rows3[order]


# ------------------------------------------------------------- learned model
def mlp_loss_grad(H, params, x, y):
    params = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    g = np.zeros(params.size, dtype=np.float64)
    loss = lib().tbo_mlp_loss_grad(H, _p(params), _p(x), _p(y), len(x), _p(g))
    return float(loss), g


def mlp_forward(H, params, x):
    params = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(len(x), dtype=np.float64)
    lib().tbo_mlp_forward(H, _p(params), _p(x), len(x), _p(out))
    return out
