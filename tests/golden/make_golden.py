"""Generates tests/golden/reference_vectors.json from the REFERENCE's own code.

Run in a container where the reference tree was compiled by oracle/Makefile
(oracle/_ref/libtbref*.so):

    python tests/golden/make_golden.py

Every vector comes from the reference sources (App/Lib/generator.cpp,
App/Lib/genzipf.c, Joins/radix_join.c, Joins/radix_sortmerge_join.c,
Joins/psm/*), never from this project's code, so the restated oracle and the
GPU path are both checked against the reference itself.  Payloads follow the
harness policy (R: i * 2654435761 mod 2^32, S: row index), since the
reference generators never write them.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def payloads(rows, kind):
    i = np.arange(len(rows), dtype=np.uint64)
    rows["payload"] = ((i * 2654435761) & 0xFFFFFFFF).astype(np.uint32) if kind == 0 else i.astype(np.uint32)
    return rows


# generator cases: (kind, n, maxid, zipf, seed)
GEN_CASES = [
    ("pk", 64, 0, 0.0, 11111),
    ("pk", 1 << 16, 0, 0.0, 11111),
    ("fk", 100000, 1 << 15, 0.0, 22222),
    ("fk", 1 << 17, 1 << 17, 0.0, 22222),
    ("fk_sel", 1 << 17, 1 << 18, 0.0, 22222),
    ("fk_sel", 1 << 18, 1 << 16, 0.0, 22222),
    ("zipf", 1 << 17, 1 << 15, 0.5, 22222),
    ("zipf", 1 << 17, 1 << 15, 1.0, 22222),
    ("zipf", 1 << 17, 1 << 15, 1.5, 22222),
]

# join cases: name, R spec, S spec (kind, n, maxid, zipf), seeds
JOIN_CASES = [
    ("default_c1", ("pk", 1 << 21, 0, 0.0), ("fk", 1 << 21, 1 << 21, 0.0), 11111, 22222),
    ("fk_8x", ("pk", 1 << 16, 0, 0.0), ("fk", 1 << 19, 1 << 16, 0.0), 11111, 22222),
    ("sel50", ("pk", 1 << 17, 0, 0.0), ("fk_sel", 1 << 19, 1 << 18, 0.0), 11111, 22222),
    ("zipf05", ("pk", 1 << 16, 0, 0.0), ("zipf", 1 << 19, 1 << 16, 0.5), 11111, 22222),
    ("zipf10", ("pk", 1 << 16, 0, 0.0), ("zipf", 1 << 19, 1 << 16, 1.0), 11111, 22222),
    ("zipf15", ("pk", 1 << 16, 0, 0.0), ("zipf", 1 << 19, 1 << 16, 1.5), 11111, 22222),
    ("ragged", ("pk", 12345, 0, 0.0), ("fk", 54321, 12345, 0.0), 3, 4),
    ("tiny", ("pk", 1, 0, 0.0), ("fk", 7, 1, 0.0), 5, 6),
]


def ref_relation(spec, seed):
    kind, n, maxid, z = spec
    O.ref_seed(seed)
    return O.ref_gen(kind, n, maxid, z)


def isolated_join(algo, R, S, nt):
    import multiprocessing as mp
    ctx = mp.get_context("fork")
    q = ctx.Queue()

    def work():
        q.put(O.ref_join(algo, R, S, nthreads=nt)[0])

    p = ctx.Process(target=work)
    p.start()
    p.join(120)
    if p.is_alive():
        p.kill()
        return "timeout"
    if p.exitcode != 0:
        return f"crashed (exit {p.exitcode})"
    return q.get()


def main():
    if O.ref() is None:
        raise SystemExit("oracle/_ref/libtbref.so missing: run `make -C oracle REF=<reference source tree>`")
    out = {"payload_policy": "R.payload = i*2654435761 mod 2^32, S.payload = i",
           "generators": [], "joins": []}
    for kind, n, maxid, z, seed in GEN_CASES:
        O.ref_seed(seed)
        rows = O.ref_gen(kind, n, maxid, z)
        e = {"kind": kind, "n": n, "maxid": maxid, "zipf": z, "seed": seed,
             "keys_sha256": sha(rows["key"]), "first_keys": rows["key"][:16].tolist()}
        if n <= 64:
            e["keys"] = rows["key"].tolist()
        out["generators"].append(e)
        print("gen", kind, n)
    for name, rs, ss, seedR, seedS in JOIN_CASES:
        R = payloads(ref_relation(rs, seedR), 0)
        S = payloads(ref_relation(ss, seedS), 1)
        e = {"name": name, "R": list(rs), "S": list(ss), "seedR": seedR, "seedS": seedS,
             "R_keys_sha256": sha(R["key"]), "S_keys_sha256": sha(S["key"])}
        for algo in ("RHO", "RHT"):
            for nt in (1, 4):
                c, _, _ = O.ref_join(algo, R, S, nthreads=nt)
                e[f"{algo}_n{nt}"] = c
        # The reference's RSM and PSM read past partition ends in merge()
        # (Joins/radix_sortmerge_join.c:40-71, Joins/psm/parallel_sortmerge_join.h:18-51)
        # and can crash; each runs in its own process and is recorded as observed.
        for algo in ("RSM", "PSM"):
            for nt in (1, 4):
                e[f"{algo}_n{nt}_observed"] = isolated_join(algo, R, S, nt)
        c, rows, _ = O.ref_join("RHO", R, S, nthreads=4, materialize=True)
        srt = O.sort_rows(rows)
        e["RHO_mat_rows"] = int(len(rows))
        e["RHO_mat_count"] = c
        e["RHO_mat_checksum"] = O.rows_checksum(rows)
        e["RHO_mat_sorted_sha256"] = sha(srt)
        if len(rows) <= 16:
            e["RHO_mat_sorted_rows"] = srt.tolist()
        out["joins"].append(e)
        print("join", name, e["RHO_n1"], e["RSM_n4_observed"], e["PSM_n1_observed"])
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
