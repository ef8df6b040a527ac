"""Generates tests/golden/gs512_oracle.json: digests of the CPU oracle's
Gray-Scott fields on the headline workload (512^3 domain, 8^3 chunks, 40
balls, seed 1; workloads.gray_scott) after 1, 2, 100 and 1000 steps.

For each checkpoint it records the SHA-256 of u and v at the existing points
(float32 bytes in (chunk position, offset) order) plus their float64 sums, so
a GPU run can be checked bit for bit without shipping 53 MB of fields.  The
oracle is the checker only; this script runs it once (a few minutes on 8
host threads).

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


def main():
    O.build()
    prm = [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]
    o, keys = oracle_grid()
    n = len(keys)
    out = {"workload": "gray_scott_512^3_chunk8^3_40balls_seed1", "params": prm, "chunks": n, "checkpoints": {}}
    done = 0
    t0 = time.time()
    for cp in CHECKPOINTS:
        # continue the ping-pong from buffer pair (0, 1) or (2, 3) depending on the steps done so far
        src, dst = ((0, 1), (2, 3)) if done % 2 == 0 else ((2, 3), (0, 1))
        o.gs7_steps(src[0], src[1], dst[0], dst[1], *prm, steps=cp - done)
        done = cp
        _, data, mask = o.export()
        fu, fv = (2, 3) if done % 2 == 1 else (0, 1)
        out["checkpoints"][str(cp)] = field_digest(data[fu], data[fv], mask, n)
        print(f"step {cp}: {time.time() - t0:.1f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(OUT)


if __name__ == "__main__":
    main()
