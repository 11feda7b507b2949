"""tee-bench-b200: Python front end of libtbg.so, the B200 equi-join library.

The C ABI (include/tbg.h) is the product; this module binds it with ctypes
and mirrors the reference's plugin interface for tests and benchmarks:

* ``algorithms`` / ``find(name)``: the name registry of native.cpp:34-46;
  ``find("RHO").join(R, S, nthreads)`` calls the drop-in entry point with
  ``struct table_t`` arguments exactly like native.cpp:125 does;
* ``join_device(...)``: the device-resident entry point on raw device
  pointers and a CUDA stream handle (any allocator: torch, cupy, cudaMalloc);
* ``gen_pk / gen_fk / gen_zipf``: on-GPU seeded generators.

The package directory name contains a hyphen, so import it with
``importlib.import_module("tee-bench_b200")``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libtbg.so")
ROW = np.dtype([("key", "<u4"), ("payload", "<u4")])
OUT_ROW = np.dtype([("key", "<u4"), ("Rpayload", "<u4"), ("Spayload", "<u4")])

# status codes (include/tbg.h)
OK, ERR_ARG, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_CAPACITY, ERR_UNKNOWN_ALGO, ERR_NO_DEVICE = range(8)
RHO_ID, RHT_ID, RSM_ID, PSM_ID, LRN_ID = range(5)
ALGO_IDS = {"RHO": RHO_ID, "RHT": RHT_ID, "RSM": RSM_ID, "PSM": PSM_ID, "LRN": LRN_ID}
MODEL_MLP, MODEL_SAMPLE, MODEL_UNTRAINED, MODEL_UNIFORM = range(4)
ERRMODE_EXIT, ERRMODE_RETURN = 0, 1


class Row(C.Structure):
    _fields_ = [("key", C.c_uint32), ("payload", C.c_uint32)]


class Table(C.Structure):  # struct table_t, Include/data-types.h:49-54
    _fields_ = [("tuples", C.POINTER(Row)), ("num_tuples", C.c_uint64),
                ("ratio_holes", C.c_int), ("sorted", C.c_int)]


class OutputList(C.Structure):  # struct output_list_t, Include/data-types.h:56-61
    pass


OutputList._fields_ = [("key", C.c_uint32), ("Rpayload", C.c_uint32), ("Spayload", C.c_uint32),
                       ("next", C.POINTER(OutputList))]


class ThreadResult(C.Structure):  # Include/data-types.h:74-78
    _fields_ = [("nresults", C.c_int64), ("results", C.POINTER(OutputList)),
                ("threadid", C.c_uint32)]


class Result(C.Structure):  # Include/data-types.h:81-85
    _fields_ = [("totalresults", C.c_int64), ("resultlist", C.POINTER(ThreadResult)),
                ("nthreads", C.c_int)]


JOINFN = C.CFUNCTYPE(C.POINTER(Result), C.POINTER(Table), C.POINTER(Table), C.c_int)


class Algorithm(C.Structure):  # Include/data-types.h:68-71
    _fields_ = [("name", C.c_char * 128), ("join", JOINFN)]


class Config(C.Structure):
    _fields_ = [("algo", C.c_int), ("radix_bits", C.c_int), ("passes", C.c_int),
                ("materialize", C.c_int), ("skew_split", C.c_int), ("model", C.c_int),
                ("train_steps", C.c_int), ("heavy_bypass", C.c_int),
                ("sample_rate", C.c_double), ("imbalance_limit", C.c_double),
                ("seed", C.c_uint64), ("timing", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("matches", C.c_uint64), ("partitions", C.c_uint64), ("work_items", C.c_uint64),
                ("max_part_R", C.c_uint64), ("max_part_S", C.c_uint64),
                ("mean_part_R", C.c_double), ("mean_part_S", C.c_double),
                ("imbalance", C.c_double), ("predicted_imbalance", C.c_double),
                ("radix_bits", C.c_int), ("passes", C.c_int), ("used_fallback", C.c_int),
                ("heavy_keys", C.c_uint64), ("heavy_rows_S", C.c_uint64),
                ("train_steps", C.c_int), ("train_loss", C.c_float),
                ("kernel_launches", C.c_uint32),
                ("ms_hist", C.c_float), ("ms_pass1", C.c_float), ("ms_pass2", C.c_float),
                ("ms_join", C.c_float), ("ms_learn", C.c_float), ("ms_total", C.c_float),
                ("heavy_rows_predicted", C.c_double), ("heavy_rows_sampled", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchJoin(C.Structure):
    _fields_ = [("dR", C.c_void_p), ("nR", C.c_uint64), ("dS", C.c_void_p), ("nS", C.c_uint64)]


class TbgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tbg status {code}: {msg}")
        self.code = code


_lib = None


def build(force: bool = False):
    """Compile libtbg.so in-tree (nvcc, sm_100a)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_tbg_build", os.path.join(HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


def lib():
    """Load libtbg.so; fails loudly when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} missing: run tee-bench_b200/build.py (nvcc) first")
    L = C.CDLL(LIB_PATH)
    P, U64, I, D = C.c_void_p, C.c_uint64, C.c_int, C.c_double
    for name in ("RHO", "RHT", "RSM", "PSM", "LRN", "RHO_mat", "RHT_mat", "RSM_mat", "PSM_mat", "LRN_mat"):
        f = getattr(L, name)
        f.argtypes = [C.POINTER(Table), C.POINTER(Table), I]
        f.restype = C.POINTER(Result)
    L.tbg_find.argtypes = [C.c_char_p]
    L.tbg_find.restype = C.POINTER(Algorithm)
    L.tbg_result_free.argtypes = [C.POINTER(Result)]
    L.tbg_set_error_mode.argtypes = [I]
    L.tbg_set_error_mode.restype = I
    L.tbg_last_error.restype = I
    L.tbg_last_error_string.restype = C.c_char_p
    L.tbg_config_init.argtypes = [C.POINTER(Config)]
    L.tbg_join_device.argtypes = [C.POINTER(Config), P, U64, P, U64, P, U64, C.POINTER(U64),
                                  C.POINTER(Stats), P]
    L.tbg_join_device.restype = I
    L.tbg_join_device_async.argtypes = [C.POINTER(Config), P, U64, P, U64, P, U64, P, P]
    L.tbg_join_device_async.restype = I
    L.tbg_sync_status.argtypes = [P]
    L.tbg_sync_status.restype = I
    L.tbg_kernel_launches.restype = U64
    L.tbg_gen_pk.argtypes = [P, U64, U64, P]
    L.tbg_gen_fk.argtypes = [P, U64, U64, U64, P]
    L.tbg_gen_zipf.argtypes = [P, U64, U64, D, I, U64, P]
    for f in (L.tbg_gen_pk, L.tbg_gen_fk, L.tbg_gen_zipf):
        f.restype = I
    L.tbg_rows_checksum.argtypes = [P, U64, C.POINTER(U64), P]
    L.tbg_rows_checksum.restype = I
    L.tbg_rows_to_relation.argtypes = [P, U64, P, P]
    L.tbg_rows_to_relation.restype = I
    L.tbg_join_three_way.argtypes = [C.POINTER(Config), P, U64, P, U64, P, U64, P, U64, C.POINTER(U64),
                                     C.POINTER(U64), P]
    L.tbg_join_three_way.restype = I
    L.tbg_batch_create.argtypes = [C.POINTER(BatchJoin), I, C.POINTER(Config), P, C.POINTER(P)]
    L.tbg_batch_create.restype = I
    L.tbg_batch_run.argtypes = [P, P, P]
    L.tbg_batch_run.restype = I
    L.tbg_batch_sync.argtypes = [P]
    L.tbg_batch_sync.restype = I
    L.tbg_batch_describe.argtypes = [P, C.c_char_p, C.c_size_t]
    L.tbg_batch_describe.restype = I
    L.tbg_batch_destroy.argtypes = [P]
    L.tbg_last_transfer_bytes.argtypes = [C.POINTER(U64), C.POINTER(U64)]
    L.tbg_set_dropin_slices.argtypes = [I]
    L.tbg_set_dropin_slices.restype = I
    L.tbg_mlp_param_count.restype = I
    L.tbg_mlp_feature.argtypes = [C.c_uint32]
    L.tbg_mlp_feature.restype = C.c_float
    L.tbg_mlp_init.argtypes = [P, U64]
    L.tbg_mlp_init.restype = I
    L.tbg_mlp_grad.argtypes = [P, P, P, U64, P, P]
    L.tbg_mlp_grad.restype = I
    L.tbg_mlp_train.argtypes = [P, P, P, U64, I, C.c_float, U64]
    L.tbg_mlp_train.restype = I
    L.tbg_shard_split.argtypes = [P, U64, I, P, C.POINTER(U64), P]
    L.tbg_shard_split.restype = I
    L.tbg_shard_of.argtypes = [C.c_uint32, I]
    L.tbg_shard_of.restype = C.c_uint32
    L.tbg_set_error_mode(ERRMODE_RETURN)  # Python callers get exceptions, not exit()
    _lib = L
    return L


def _check(rc):
    if rc != OK:
        L = lib()
        raise TbgError(rc, L.tbg_last_error_string().decode(errors="replace"))


def exported_symbols():
    """Names include/tbg.h declares with TBG_API."""
    import re
    hdr = open(os.path.join(os.path.dirname(HERE), "include", "tbg.h")).read()
    names = re.findall(r"TBG_API[^;(]*?\**\s*(\w+)\s*(?:\(|\[|;)", hdr)
    return sorted(n for n in set(names) if not n.startswith("__"))


# ------------------------------------------------------------------ drop-in
def table(rows: np.ndarray) -> Table:
    rows = np.ascontiguousarray(rows, dtype=ROW)
    t = Table()
    t.tuples = rows.ctypes.data_as(C.POINTER(Row)) if len(rows) else C.POINTER(Row)()
    t.num_tuples = len(rows)
    t._keep = rows
    return t


def result_rows(res) -> np.ndarray:
    """Walks resultlist[t].results for nresults nodes per thread."""
    r = res.contents
    out = []
    for t in range(r.nthreads):
        tr = r.resultlist[t]
        node = tr.results
        for _ in range(tr.nresults):
            n = node.contents
            out.append((n.key, n.Rpayload, n.Spayload))
            node = n.next
    return np.array(out, dtype=np.uint32).reshape(-1, 3)


class JoinAlgorithm:
    """One registry entry: ``join(R, S, nthreads)`` like algorithm_t.join."""

    def __init__(self, name):
        self.name = name

    def join(self, R, S, nthreads=1, materialize=False):
        L = lib()
        tR, tS = table(R), table(S)
        fn = getattr(L, self.name + ("_mat" if materialize else ""))
        res = fn(C.byref(tR), C.byref(tS), nthreads)
        if not res:
            _check(L.tbg_last_error() or ERR_CUDA)
        try:
            count = int(res.contents.totalresults)
            rows = result_rows(res) if materialize else None
        finally:
            L.tbg_result_free(res)
        return (count, rows) if materialize else count


algorithms = [JoinAlgorithm(n) for n in ("RHO", "RHT", "RSM", "PSM", "LRN")]


def find(name: str) -> JoinAlgorithm:
    L = lib()
    if not L.tbg_find(name.encode()):
        raise TbgError(ERR_UNKNOWN_ALGO, f"unknown algorithm {name!r}")
    return JoinAlgorithm(name)


# ------------------------------------------------------------------ device API
def config(algo="RHO", **kw) -> Config:
    c = Config()
    lib().tbg_config_init(C.byref(c))
    c.algo = ALGO_IDS[algo] if isinstance(algo, str) else int(algo)
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c


def join_device(cfg: Config, dR: int, nR: int, dS: int, nS: int, d_rows: int = 0, rows_cap: int = 0,
                stream: int = 0, check: bool = True):
    """Returns (status, matches, Stats)."""
    L = lib()
    m = C.c_uint64(0)
    st = Stats()
    rc = L.tbg_join_device(C.byref(cfg), dR, nR, dS, nS, d_rows or None, rows_cap, C.byref(m),
                           C.byref(st), stream or None)
    if check:
        _check(rc)
    return rc, int(m.value), st


def join_device_async(cfg, dR, nR, dS, nS, d_matches, d_rows=0, rows_cap=0, stream=0):
    _check(lib().tbg_join_device_async(C.byref(cfg), dR, nR, dS, nS, d_rows or None, rows_cap,
                                       d_matches, stream or None))


def gen_pk(d: int, n: int, seed: int, stream: int = 0):
    _check(lib().tbg_gen_pk(d, n, seed, stream or None))


def gen_fk(d: int, n: int, maxid: int, seed: int, stream: int = 0):
    _check(lib().tbg_gen_fk(d, n, maxid, seed, stream or None))


def gen_zipf(d: int, n: int, alphabet: int, z: float, scatter: int, seed: int, stream: int = 0):
    _check(lib().tbg_gen_zipf(d, n, alphabet, z, scatter, seed, stream or None))


def rows_checksum(d_rows: int, n: int, stream: int = 0) -> int:
    v = C.c_uint64(0)
    _check(lib().tbg_rows_checksum(d_rows, n, C.byref(v), stream or None))
    return int(v.value)


def rows_to_relation(d_rows: int, n: int, d_out: int, stream: int = 0):
    _check(lib().tbg_rows_to_relation(d_rows or None, n, d_out or None, stream or None))


def join_three_way(cfg: Config, dR, nR, dS, nS, dT, nT, d_rows2=0, rows2_cap=0, stream=0):
    """(matches of R x S, matches of T x to_relation(R x S))."""
    m1, m2 = C.c_uint64(), C.c_uint64()
    _check(lib().tbg_join_three_way(C.byref(cfg), dR, nR, dS, nS, dT, nT, d_rows2 or None, rows2_cap,
                                    C.byref(m1), C.byref(m2), stream or None))
    return int(m1.value), int(m2.value)


def set_dropin_slices(k: int) -> int:
    """S slices the drop-in RHO/RHT copy and join one by one (0: automatic,
    1: copy all, then join).  Returns the previous setting."""
    return lib().tbg_set_dropin_slices(int(k))


def last_transfer_bytes():
    h, d = C.c_uint64(), C.c_uint64()
    lib().tbg_last_transfer_bytes(C.byref(h), C.byref(d))
    return int(h.value), int(d.value)


# ------------------------------------------------------------------ several GPUs
def shard_of(keys, nshards: int) -> np.ndarray:
    """Shard of each key for a join split over nshards ranks (tbg_shard_of):
    the top bits of the multiplicative hash key * 0x9E3779B1 (mod 2^32),
    range-reduced to [0, nshards) by a multiply-shift."""
    h = (np.asarray(keys, dtype=np.uint64) * np.uint64(0x9E3779B1)) & np.uint64(0xFFFFFFFF)
    return ((h * np.uint64(nshards)) >> np.uint64(32)).astype(np.int64)


def shard_split(d_in: int, n: int, nshards: int, d_out: int, stream: int = 0) -> list:
    """Groups n device rows by shard into d_out (tbg_shard_split); returns
    the nshards + 1 row offsets of the groups."""
    offs = (C.c_uint64 * (nshards + 1))()
    _check(lib().tbg_shard_split(d_in or None, n, nshards, d_out or None, offs, stream or None))
    return [int(x) for x in offs]


def distributed_join_count(dist, R, S, split, join, new_rows):
    """Count of one equi-join whose relations are spread over the ranks of the
    process group `dist` (NCCL on GPUs, gloo in CPU tests); every rank calls
    it with its own rows of R and of S (1-D int64 tensors, one row each).

    Every rank splits its rows by shard (``split(rows, nshards) -> (grouped
    rows, offsets)``), the pieces move to their shards' ranks with an
    all-to-all (counts first, then rows), each rank joins what it received
    (``join(R_recv, S_recv) -> count``) and the counts are summed.  Keys never
    meet across shards, so the sum is the join's count, which every rank
    returns.  ``new_rows(n)`` allocates a receive buffer of n rows.  With one
    rank the rows are joined as they are.  This replaces the reference's
    per-thread chunking of one join (Joins/radix_join.c:1285-1306) by a split
    across GPUs by key."""
    import torch
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    if world == 1:
        return int(join(R, S))
    received = []
    for rows in (R, S):
        grouped, offs = split(rows, world)
        send = [offs[d + 1] - offs[d] for d in range(world)]
        sc = torch.tensor(send, dtype=torch.int64, device=rows.device)
        rc = torch.empty_like(sc)
        dist.all_to_all_single(rc, sc)
        recv = [int(x) for x in rc.tolist()]
        out = new_rows(sum(recv))
        dist.all_to_all_single(out, grouped, output_split_sizes=recv, input_split_sizes=send)
        received.append(out)
    c = torch.tensor([int(join(received[0], received[1]))], dtype=torch.int64, device=R.device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return int(c.item())


# ------------------------------------------------------------------ model
def mlp_init(seed: int) -> np.ndarray:
    L = lib()
    p = np.zeros(L.tbg_mlp_param_count(), dtype=np.float32)
    _check(L.tbg_mlp_init(p.ctypes.data, seed))
    return p


def mlp_grad(params, x, y):
    """(loss, grad) of the MSE over the points, computed by the GPU kernels."""
    L = lib()
    params = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    g = np.zeros_like(params)
    loss = C.c_float()
    _check(L.tbg_mlp_grad(params.ctypes.data, x.ctypes.data, y.ctypes.data, len(x), g.ctypes.data,
                          C.addressof(loss)))
    return float(loss.value), g


def mlp_train(params, x, y, steps, lr=0.01, seed=1):
    L = lib()
    p = np.ascontiguousarray(params, dtype=np.float32).copy()
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    _check(L.tbg_mlp_train(p.ctypes.data, x.ctypes.data, y.ctypes.data, len(x), steps, lr, seed))
    return p


def mlp_feature(ranks) -> np.ndarray:
    """Model input of sample ranks: log2(rank + 1) / 16 - 1 (what LRN feeds
    the MLP; rank 1 is the key the sample saw most often)."""
    return (np.log2(np.asarray(ranks, dtype=np.float64) + 1.0) / 16.0 - 1.0).astype(np.float32)


# ------------------------------------------------------------------ batches
class Batch:
    """Many independent joins planned once (autotuned, one CUDA graph) and
    replayed with run(); joins = [(dR, nR, dS, nS), ...] device pointers."""

    def __init__(self, joins, cfg: Config = None, stream: int = 0):
        L = lib()
        self.n = len(joins)
        arr = (BatchJoin * max(1, self.n))()
        for i, (dR, nR, dS, nS) in enumerate(joins):
            arr[i] = BatchJoin(dR or None, nR, dS or None, nS)
        h = C.c_void_p()
        _check(L.tbg_batch_create(arr, self.n, C.byref(cfg) if cfg is not None else None, stream or None,
                                  C.byref(h)))
        self._h = h

    def run(self, d_counts: int = 0, stream: int = 0):
        _check(lib().tbg_batch_run(self._h, d_counts or None, stream or None))

    def sync(self):
        _check(lib().tbg_batch_sync(self._h))

    def describe(self) -> dict:
        import json
        L = lib()
        n = L.tbg_batch_describe(self._h, None, 0)
        buf = C.create_string_buffer(n + 1)
        L.tbg_batch_describe(self._h, buf, n + 1)
        return json.loads(buf.value.decode())

    def close(self):
        if self._h:
            lib().tbg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_launches() -> int:
    return int(lib().tbg_kernel_launches())
