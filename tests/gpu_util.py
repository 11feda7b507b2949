"""Device-buffer helpers for the GPU tests (torch is used only to allocate
memory and name streams; every join goes through the library's C ABI)."""
from __future__ import annotations

import numpy as np


def to_dev(torch, rows: np.ndarray, offset_rows: int = 0):
    """Copies a ROW array to the device; offset_rows > 0 places it that many
    rows into a larger buffer (for misaligned-pointer cases).  Returns
    (keepalive tensor, device pointer)."""
    raw = np.ascontiguousarray(rows).view(np.int64).reshape(-1)
    t = torch.zeros(len(raw) + offset_rows + 1, dtype=torch.int64, device="cuda")
    if len(raw):
        t[offset_rows:offset_rows + len(raw)] = torch.from_numpy(raw.copy()).cuda()
    return t, t.data_ptr() + 8 * offset_rows


def out_rows(torch, cap: int):
    t = torch.zeros(max(cap, 1) * 3, dtype=torch.int32, device="cuda")
    return t, t.data_ptr()


def rows_to_host(t, n: int) -> np.ndarray:
    return t[: n * 3].cpu().numpy().view(np.uint32).reshape(-1, 3)


def run_join(tbg, torch, algo, R, S, materialize=False, cap=None, offset=0, **cfgkw):
    """Device-API join on host arrays.  Returns (count, rows or None, stats)."""
    tR, pR = to_dev(torch, R, offset)
    tS, pS = to_dev(torch, S, offset)
    cfg = tbg.config(algo, materialize=int(materialize), **cfgkw)
    rows = None
    if materialize:
        cap = len(S) * 2 + 16 if cap is None else cap
        tO, pO = out_rows(torch, cap)
        rc, m, st = tbg.join_device(cfg, pR, len(R), pS, len(S), pO, cap,
                                    stream=torch.cuda.current_stream().cuda_stream)
        rows = rows_to_host(tO, min(m, cap))
    else:
        rc, m, st = tbg.join_device(cfg, pR, len(R), pS, len(S),
                                    stream=torch.cuda.current_stream().cuda_stream)
    return m, rows, st


def dev_relation(torch, n: int):
    t = torch.empty(max(n, 1), dtype=torch.int64, device="cuda")
    return t, t.data_ptr()


def dev_to_host_rows(t, n: int) -> np.ndarray:
    return t[:n].cpu().numpy().view(np.uint32).reshape(-1, 2).copy().view(
        np.dtype([("key", "<u4"), ("payload", "<u4")])).reshape(-1)
