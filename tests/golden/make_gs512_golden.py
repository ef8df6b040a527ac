"""Generates tests/golden/gs512_oracle.json: digests of the CPU oracle's
Gray-Scott fields on the headline workload (512^3 domain, 8^3 chunks, 40
balls, seed 1; workloads.gray_scott) after 1, 2, 100 and 1000 steps.

For each checkpoint it records the SHA-256 of u and v at the existing points
(float32 bytes in (chunk position, offset) order) plus their float64 sums, so
a GPU run can be checked bit for bit without shipping 53 MB of fields.  At
100 and 1000 steps it also records the error of those FP32 fields against the
same update in double precision (the FP64 oracle): max absolute error and the
normwise relative error ||f32 - f64|| / ||f64|| over the existing points, per
field.  The oracle is the checker only; this script runs it once (FP32: a
few minutes on 8 host threads; FP64: about ten more).

Usage: python tests/golden/make_gs512_golden.py
"""
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from oracle import oracle as O  # noqa: E402
from openfpm_data_b200 import workloads as W  # noqa: E402

CHECKPOINTS = (1, 2, 100, 1000)
OUT = os.path.join(HERE, "gs512_oracle.json")


def field_digest(data_u, data_v, mask, n, bs=512):
    ex = (mask[: n * bs] & 1).astype(bool)
    u = np.ascontiguousarray(data_u[: n * bs][ex], dtype=np.float32)
    v = np.ascontiguousarray(data_v[: n * bs][ex], dtype=np.float32)
    return {"u_sha256": hashlib.sha256(u.tobytes()).hexdigest(), "v_sha256": hashlib.sha256(v.tobytes()).hexdigest(),
            "u_sum": float(u.astype(np.float64).sum()), "v_sum": float(v.astype(np.float64).sum()),
            "points": int(ex.sum())}


def oracle_grid():
    ps = W.gray_scott()
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    o = O.OracleGrid(ps.size, edge=8, ptypes=[O.T_F32] * 4)
    for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
        o.set_background(p, b)
    o.load_map(keys, data + [d.copy() for d in data], mask)
    return o, keys


def fp64_error(f32, f64, ex):
    a = np.asarray(f32, dtype=np.float64)[ex]
    b = np.asarray(f64, dtype=np.float64)[ex]
    return {"max_abs": float(np.max(np.abs(a - b))),
            "normwise_rel": float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))}


def main():
    O.build()
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    o, keys = oracle_grid()
    n = len(keys)
    out = {"workload": "gray_scott_512^3_chunk8^3_40balls_seed1", "params": prm, "chunks": n, "checkpoints": {}}
    _, data0, mask0 = o.export()
    ex = (mask0[: n * 512] & 1).astype(bool)
    u64 = np.asarray(data0[0], dtype=np.float64)
    v64 = np.asarray(data0[1], dtype=np.float64)
    done = 0
    t0 = time.time()
    for cp in CHECKPOINTS:
        # continue the ping-pong from buffer pair (0, 1) or (2, 3) depending on the steps done so far
        src, dst = ((0, 1), (2, 3)) if done % 2 == 0 else ((2, 3), (0, 1))
        o.gs7_steps(src[0], src[1], dst[0], dst[1], *prm, steps=cp - done)
        _, data, mask = o.export()
        fu, fv = (2, 3) if cp % 2 == 1 else (0, 1)
        rec = field_digest(data[fu], data[fv], mask, n)
        if cp >= 100:  # the same steps in double precision, continued from the previous checkpoint
            u64, v64 = o.gs7_f64(u64, v64, *prm[:4], prm[4], 1.0, 0.0, cp - done, threads=os.cpu_count() or 1)
            rec["fp64_error"] = {"u": fp64_error(data[fu][: n * 512], u64[: n * 512], ex),
                                 "v": fp64_error(data[fv][: n * 512], v64[: n * 512], ex)}
        elif cp == 2:
            u64, v64 = o.gs7_f64(u64, v64, *prm[:4], prm[4], 1.0, 0.0, 2, threads=os.cpu_count() or 1)
        done = cp
        out["checkpoints"][str(cp)] = rec
        print(f"step {cp}: {time.time() - t0:.1f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(OUT)


if __name__ == "__main__":
    main()
