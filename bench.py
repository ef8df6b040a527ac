#!/usr/bin/env python
"""Headline benchmark: applyStencils throughput on the Gray-Scott 512^3 sparse grid.

Workload (seeded, synthetic, see openfpm_data_b200/workloads.py): a 512^3
SparseGridGpu of 8^3 chunks, occupancy the union of 40 balls (seed 1),
fields u, v (+ ping-pong copies), Du .16 Dv .08 F .035 k .065 dt 1.  One step
is one Gray-Scott 7-point stencil application over every active point.

  value  Gpts/s over the K timed steps, inputs resident in HBM, CUDA events on
         the launching stream, max over ranks; N > 1 runs independent
         replicas (weak scaling, no collective on the data path).
  e2e    the same metric through the C ABI from pinned host buffers: per e2e
         step one full solve (upload keys/u/v/mask, `--solve-steps` stencil
         steps, download u/v).
  roofline  algorithmic bytes of the stencil kernel (17 B per active point:
         u, v read + u, v written + 1 mask byte) / its average launch time,
         against the measured HBM copy bandwidth.

--impl reference times the CPU restatement of the reference's sgrid_cpu
path (oracle/sgrid_cpu_baseline.cpp, all host threads) on the same
workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

L2_BYTES = 126 * 2 ** 20
METRIC = "stencil Gpts/s (Gray-Scott 7-point, 512^3 sparse grid)"
UNIT = "Gpts/s"
ALG_BYTES_PER_PT = 17


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-solves", type=int, default=3)
    ap.add_argument("--solve-steps", type=int, default=1000)
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--stages", type=int, default=0)
    return ap.parse_args()


# ---------------------------------------------------------------- distributed plumbing
class Dist:
    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            backend = "nccl" if _cuda_ok() else "gloo"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            if _cuda_ok():
                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()
            if _cuda_ok():
                torch.cuda.synchronize()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{self.local}" if _cuda_ok() else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, interval_ms: int = 20):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            sel = ["-i", uuid if uuid.startswith("GPU-") else "GPU-" + uuid]
        except Exception:
            sel = ["-i", str(device_index)]
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", str(interval_ms)] + sel, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def _peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic():
    """DRAM bytes per launch of the stencil kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "stencil7_gs7_512.md")
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


def gs_params():
    from openfpm_data_b200 import workloads as W
    return [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]


def cpu_baseline(ps, keys_unused, threads: int, max_steps: int, budget_s: float = 25.0):
    """sgrid_cpu restatement on the host cores: Gray-Scott steps on the full grid."""
    from oracle import oracle as O
    O.build()
    c = O.CpuSgrid(ps.size, 4, [1.0, 0.0, 1.0, 0.0])
    c.insert(ps.coords, ps.values + ps.values)
    prm = gs_params()
    t0 = time.perf_counter()
    c.gs(0, 1, 2, 3, *prm, steps=1, threads=threads)
    one = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, budget_s // max(one, 1e-6))))
    t0 = time.perf_counter()
    c.gs(2, 3, 0, 1, *prm, steps=steps, threads=threads)
    dt = time.perf_counter() - t0
    return len(ps.coords) * steps / dt / 1e9, steps, dt


# ---------------------------------------------------------------- arms
def run_ours(args, dist: Dist):
    import torch

    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import workloads as W

    torch.cuda.set_device(dist.local)
    dev = dist.local
    ps = W.gray_scott()
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    npts = len(ps.coords)
    g = sgb.SparseGridGpu(ps.size, ["f32"] * 4, edge=8, device=dev)
    for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
        g.setBackgroundValue(p, b)
    if args.ctas_per_sm or args.stages:
        g.setLaunchConfig(args.ctas_per_sm, args.stages)
    g.load_map(keys, data + [d.copy() for d in data], mask)
    prm = gs_params()
    stream = torch.cuda.current_stream()
    footprint = g.nchunks * 512 * (4 * 4 + 1)

    # warm-up (W steps), then exactly K timed steps continuing the ping-pong
    g.run_steps(sgb.GS7, [0, 1], [2, 3], prm, args.warmup, use_graph=False)
    src, dst = ([2, 3], [0, 1]) if args.warmup % 2 else ([0, 1], [2, 3])
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    time.sleep(0.05)
    dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    g.run_steps(sgb.GS7, src, dst, prm, args.steps, use_graph=False)
    ev1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    g.check_device_errors()
    t_local = ev0.elapsed_time(ev1) / 1e3
    t_max = dist.max(t_local)
    value = dist.world * npts * args.steps / t_max / 1e9

    # roofline of the stencil kernel (the only kernel of the timed region)
    avg_launch = t_local / args.steps
    alg_bytes = ALG_BYTES_PER_PT * npts
    peak, peak_kind = _peak_hbm()
    achieved = alg_bytes / avg_launch / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": _profile_traffic(),
                "peak_kind": peak_kind, "alg_bytes_per_launch": alg_bytes,
                "chunk_slot_bytes_per_launch": g.nchunks * 512 * 17}

    # end to end through the C ABI from pinned host memory
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    h_keys, h_u, h_v, h_mask = pin(keys), pin(data[0]), pin(data[1]), pin(mask)
    n = len(keys)
    out_u = torch.empty((n + 1) * 512, dtype=torch.float32).pin_memory()
    out_v = torch.empty((n + 1) * 512, dtype=torch.float32).pin_memory()
    e2e_steps = max(1, args.e2e_solves)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fin_dst = False
    for _ in range(e2e_steps):
        g.load_map(h_keys, [h_u, h_v, None, None], h_mask)
        fin_dst = g.run_steps(sgb.GS7, [0, 1], [2, 3], prm, args.solve_steps, use_graph=False)
        su, sv = g.private_get_data_array(2 if fin_dst else 0), g.private_get_data_array(3 if fin_dst else 1)
        out_u.copy_(su, non_blocking=True)
        out_v.copy_(sv, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = dist.max(e0.elapsed_time(e1) / 1e3)
    e2e = {"value": round(dist.world * npts * args.solve_steps * e2e_steps / t_e2e / 1e9, 3), "unit": UNIT,
           "h2d_bytes_per_step": int(h_keys.nbytes + h_u.nbytes + h_v.nbytes + h_mask.nbytes),
           "d2h_bytes_per_step": int(out_u.numel() * 4 + out_v.numel() * 4),
           "step": f"one solve: upload, {args.solve_steps} Gray-Scott steps, download u and v"}
    assert np.isfinite(out_u.numpy()[:1000]).all()

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        v1, st, dt = cpu_baseline(ps, keys, 1, args.cpu_steps)
        cpu = {"value": round(v1, 5), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{st} Gray-Scott steps on the full 512^3 grid ({npts} points), 1 thread, {dt:.1f} s"}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_max / args.steps * 1e3, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, workloads.gray_scott)",
        "config": {"workload": "gray_scott_512^3_chunk8^3_40balls_seed1", "active_points_per_gpu": npts,
                   "chunks": g.nchunks, "fields": "u,v float32 + ping-pong", "parallelism": f"replicas x{dist.world}",
                   "l2": f"inputs {footprint / 2**20:.0f} MiB > L2 {L2_BYTES / 2**20:.0f} MiB, no flush",
                   "launch": {"ctas_per_sm": args.ctas_per_sm or 2, "stages": args.stages or 6}},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps,
        "clocks": clk,
    }
    return line


def run_reference(args, dist: Dist):
    from openfpm_data_b200 import workloads as W
    if dist.rank != 0:
        return None
    threads = os.cpu_count() or 1
    ps = W.gray_scott()
    # warm-up steps are run (not timed) by cpu_baseline's probe step
    v, st, dt = cpu_baseline(ps, None, threads, max(1, args.steps), budget_s=90.0)
    cpu = {"value": round(v, 5), "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"{st} Gray-Scott steps on the full 512^3 grid ({len(ps.coords)} points), {threads} threads"}
    return {"metric": METRIC, "value": round(v, 5), "unit": UNIT, "n_gpus": dist.world, "steps": st,
            "warmup": 1, "ms_per_step": round(dt / st * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, workloads.gray_scott)",
            "config": {"workload": "gray_scott_512^3_chunk8^3_40balls_seed1", "active_points": len(ps.coords)},
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": round(v, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    dist = Dist(args.gpus)
    try:
        line = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
        if line is not None and dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
