"""The binary FP64 checkpoint of simox_checkpoint_write / _read, read and
written with numpy (no GPU needed): little-endian "SIMOXCK1", int32 version 1,
int32 n, int64 step, float64 box[3], int32 id[n], float64 x[n][3], v[n][3],
f[n][3], q[n].  The reference's restart.xyz (PRINT_SNAPSHOT, util.f90:22-81)
keeps 7 significant digits of x and 5 of v and f; this file keeps every bit."""
from __future__ import annotations

import numpy as np

MAGIC = b"SIMOXCK1"
VERSION = 1
HEADER = 48          # magic 8 + version, n 2 x 4 + step 8 + box 24


def write(path: str, ids, x, v, f, q, box, step: int = 0) -> None:
    ids = np.ascontiguousarray(ids, dtype="<i4")
    n = ids.size
    arrays = [np.ascontiguousarray(a, dtype="<f8").reshape(n, 3) for a in (x, v, f)]
    with open(path, "wb") as fh:
        fh.write(MAGIC)
        fh.write(np.array([VERSION, n], dtype="<i4").tobytes())
        fh.write(np.array([step], dtype="<i8").tobytes())
        fh.write(np.ascontiguousarray(box, dtype="<f8").reshape(3).tobytes())
        fh.write(ids.tobytes())
        for a in arrays:
            fh.write(a.tobytes())
        fh.write(np.ascontiguousarray(q, dtype="<f8").reshape(n).tobytes())


def read(path: str) -> dict:
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) < HEADER or data[:8] != MAGIC:
        raise ValueError(f"{path}: not a checkpoint")
    version, n = np.frombuffer(data, "<i4", 2, 8)
    if version != VERSION or n < 0:
        raise ValueError(f"{path}: unsupported version {version} or n {n}")
    n = int(n)
    need = HEADER + 4 * n + 8 * 10 * n
    if len(data) < need:
        raise ValueError(f"{path}: short file ({len(data)} of {need} bytes)")
    step = int(np.frombuffer(data, "<i8", 1, 16)[0])
    box = np.frombuffer(data, "<f8", 3, 24).copy()
    off = HEADER
    ids = np.frombuffer(data, "<i4", n, off).copy()
    off += 4 * n
    out = {"n": n, "step": step, "box": box, "ids": ids}
    for name in ("x", "v", "f"):
        out[name] = np.frombuffer(data, "<f8", 3 * n, off).reshape(n, 3).copy()
        off += 24 * n
    out["q"] = np.frombuffer(data, "<f8", n, off).copy()
    return out
