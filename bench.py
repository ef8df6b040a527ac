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
# the library's default launch configuration of the pipelined 8^3 kernel (automatic ring depth)
DEFAULT_CTAS_PER_SM, DEFAULT_STAGES = "auto", "auto"
WORKLOADS = ("gs512", "heat128", "insert1024", "batched256", "served", "ghost512", "conv1000", "conv2b")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-solves", type=int, default=3)
    ap.add_argument("--solve-steps", type=int, default=1000)
    ap.add_argument("--cpu-steps", type=int, default=150, help="cap of the CPU baseline sample (10-30 s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--stages", type=int, default=0)
    ap.add_argument("--workload", choices=list(WORKLOADS), default="gs512",
                    help="gs512 (the headline line) or one of the other workloads")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="served: arrival window")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="served: Poisson arrival rate (requests/s)")
    ap.add_argument("--plain-sample", type=int, default=64, help="served: requests solved alone for the baseline")
    ap.add_argument("--no-sub-records", action="store_true",
                    help="gs512: leave out the bounded runs of the other configurations")
    ap.add_argument("--sub-serve-seconds", type=float, default=6.0, help="sub-records: served arrival window")
    ap.add_argument("--sub-sustained-rate", type=float, default=400.0,
                    help="sub-records: an arrival rate the served form keeps up with (requests/s)")
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

    def gather(self, obj) -> list:
        """Every rank's `obj` (a small picklable summary), in rank order."""
        if not self.pg:
            return [obj]
        out = [None] * self.world
        self.pg.all_gather_object(out, obj)
        return out

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
    """SM clock and clock-event reasons of one GPU, sampled during a region: by NVML from a
    background thread every 5 ms (read-only queries), or by `nvidia-smi -lms` where NVML cannot be
    loaded.  stop() returns the median SM clock under load, the maximum, the reasons seen and the
    number of samples."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device_index: int, interval_ms: int = 20):
        self.proc = None
        self.thread = None
        self.samples = []  # (sm MHz, max MHz, reason bits)
        self.uuid = None
        try:
            import torch
            u = str(torch.cuda.get_device_properties(device_index).uuid)
            self.uuid = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            pass
        if self._start_nvml():
            return
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        sel = ["-i", self.uuid] if self.uuid else ["-i", str(device_index)]
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", str(interval_ms)] + sel, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def _start_nvml(self) -> bool:
        try:
            import threading

            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid else None
            if h is None:
                return False
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._stop_flag = False

            def run():
                while not self._stop_flag:
                    try:
                        self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx, int(reasons(h))))
                    except Exception:
                        pass
                    time.sleep(0.005)

            self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx, int(reasons(h))))
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return True
        except Exception:
            return False

    def stop(self):
        if self.thread is not None:
            self._stop_flag = True
            self.thread.join(timeout=5)
            sm = [a for a, _, _ in self.samples]
            mx = self.samples[-1][1] if self.samples else None
            bits = 0
            for _, _, r in self.samples:
                bits |= r
            reasons = sorted(n for n, b in self.REASON_BITS.items() if bits & b)
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                    "samples": len(sm), "source": "nvml"}
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
                "samples": len(sm), "source": "nvidia-smi"}


# ---------------------------------------------------------------- helpers
def _peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic(name="stencil7_gs7_512.md"):
    """DRAM bytes per launch of a kernel from its committed ncu summary under profiles/."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


def gs_params():
    from openfpm_data_b200 import workloads as W
    return [W.GS_PARAMS[k] for k in ("Du", "Dv", "F", "k", "dt")]


def cpu_baseline(ps, keys_unused, threads: int, max_steps: int, budget_s: float = 25.0, warmup: int = 1):
    """sgrid_cpu restatement on the host cores: Gray-Scott steps on the full grid, after `warmup`
    untimed steps (the last of which sizes the timed sample)."""
    from oracle import oracle as O
    O.build()
    c = O.CpuSgrid(ps.size, 4, [1.0, 0.0, 1.0, 0.0])
    c.insert(ps.coords, ps.values + ps.values)
    prm = gs_params()
    one = 0.0
    for _ in range(max(1, warmup)):  # the same input each time: the warm-up result is that of one step
        t0 = time.perf_counter()
        c.gs(0, 1, 2, 3, *prm, steps=1, threads=threads)
        one = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, budget_s // max(one, 1e-6))))
    t0 = time.perf_counter()
    c.gs(2, 3, 0, 1, *prm, steps=steps, threads=threads)
    dt = time.perf_counter() - t0
    return len(ps.coords) * steps / dt / 1e9, steps, dt


def gs512_config(npts: int, nchunks: int, world: int) -> dict:
    """The workload description both arms print (the same dict, so the lines compare)."""
    footprint = nchunks * 512 * (4 * 4 + 1)
    return {"workload": "gray_scott_512^3_chunk8^3_40balls_seed1", "active_points_per_gpu": npts,
            "chunks": nchunks, "fields": "u,v float32 + ping-pong", "parallelism": f"replicas x{world}",
            "l2": f"inputs {footprint / 2**20:.0f} MiB > L2 {L2_BYTES / 2**20:.0f} MiB, no flush"}


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

    # warm-up (W steps), then exactly K timed steps continuing the ping-pong; the clock sampler starts
    # first, so that the GPU goes from the warm-up straight into the timed steps without idling
    clocks = ClockSampler(dev)
    time.sleep(0.05)
    dist.barrier()
    g.run_steps(sgb.GS7, [0, 1], [2, 3], prm, args.warmup, use_graph=False)
    src, dst = ([2, 3], [0, 1]) if args.warmup % 2 else ([0, 1], [2, 3])
    torch.cuda.synchronize()
    dist.barrier()
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

    # end to end through the C ABI from pinned host memory: every solve uploads its inputs, steps and
    # downloads u and v; two device grids on two streams let one solve's copies overlap the other's steps
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    h_keys, h_u, h_v, h_mask = pin(keys), pin(data[0]), pin(data[1]), pin(mask)
    n = len(keys)
    g2 = sgb.SparseGridGpu(ps.size, ["f32"] * 4, edge=8, device=dev)
    for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
        g2.setBackgroundValue(p, b)
    if args.ctas_per_sm or args.stages:
        g2.setLaunchConfig(args.ctas_per_sm, args.stages)
    g2.load_map(h_keys, [h_u, h_v, None, None], h_mask)  # buffers allocated outside the timed region
    g2.run_steps(sgb.GS7, [0, 1], [2, 3], prm, 2, use_graph=False)
    pair = [g, g2]
    streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]
    outs = [(torch.empty((n + 1) * 512, dtype=torch.float32).pin_memory(),
             torch.empty((n + 1) * 512, dtype=torch.float32).pin_memory()) for _ in range(2)]
    out_u, out_v = outs[0]
    e2e_steps = max(1, args.e2e_solves)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for st in streams:
        st.wait_event(e0)
    fin_dst = False
    for k in range(e2e_steps):
        gk, sk = pair[k % 2], streams[k % 2]
        ou, ov = outs[k % 2]
        with torch.cuda.stream(sk):
            gk.load_map(h_keys, [h_u, h_v, None, None], h_mask, stream=sk)
            fin_dst = gk.run_steps(sgb.GS7, [0, 1], [2, 3], prm, args.solve_steps, use_graph=False, stream=sk)
            su = gk.private_get_data_array(2 if fin_dst else 0)
            sv = gk.private_get_data_array(3 if fin_dst else 1)
            ou.copy_(su, non_blocking=True)
            ov.copy_(sv, non_blocking=True)
    for st in streams:
        stream.wait_stream(st)
    e1.record(stream)
    torch.cuda.synchronize()
    out_u, out_v = outs[(e2e_steps - 1) % 2]
    t_e2e = dist.max(e0.elapsed_time(e1) / 1e3)
    e2e = {"value": round(dist.world * npts * args.solve_steps * e2e_steps / t_e2e / 1e9, 3), "unit": UNIT,
           "h2d_bytes_per_step": int(h_keys.nbytes + h_u.nbytes + h_v.nbytes + h_mask.nbytes),
           "d2h_bytes_per_step": int(out_u.numel() * 4 + out_v.numel() * 4),
           "step": f"one solve: upload, {args.solve_steps} Gray-Scott steps, download u and v (solves alternate "
                   "between two device grids on two streams, so copies overlap the other solve's steps)"}
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
        "config": gs512_config(npts, g.nchunks, dist.world),
        "launch": {"ctas_per_sm": args.ctas_per_sm or DEFAULT_CTAS_PER_SM, "stages": args.stages or DEFAULT_STAGES},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps,
        "clocks": clk,
    }
    return line


# ---------------------------------------------------------------- other workloads
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _line(metric, value, unit, dist, args, steps, t, config, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": dist.world, "steps": steps,
         "warmup": args.warmup, "ms_per_step": round(t / max(steps, 1) * 1e3, 5), "higher_is_better": True,
         "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, workloads.py)",
         "config": config}
    d.update(extra)
    return d


def run_heat128(args, dist: Dist):
    """Heat on the 128^3 shell (103,694 points, 379 chunks).  The grid fits in
    L2, so an L2-flushing write (256 MiB) separates the timed steps and only
    the stencil launches are timed (events around each)."""
    import torch

    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import workloads as W
    torch.cuda.set_device(dist.local)
    ps = W.heat_shell()
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    npts = len(ps.coords)
    g = sgb.SparseGridGpu(ps.size, ["f32", "f32"], edge=8, device=dist.local)
    g.load_map(keys, data + [data[0].copy()], mask)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device="cuda")
    for k in range(max(3, args.warmup)):
        g.applyStencils(sgb.HEAT7, [k % 2], [1 - k % 2], [W.HEAT_DT])
    torch.cuda.synchronize()
    clocks = ClockSampler(dist.local)
    dist.barrier()
    evs = []
    for k in range(args.steps):
        flush.fill_(float(k))
        e0, e1 = _events()
        e0.record()
        g.applyStencils(sgb.HEAT7, [k % 2], [1 - k % 2], [W.HEAT_DT])
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    g.check_device_errors()
    t = dist.max(sum(a.elapsed_time(b) for a, b in evs) / 1e3)
    value = dist.world * npts * args.steps / t / 1e9
    peak, pk = _peak_hbm()
    ach = 9 * npts / (t / args.steps) / 1e9
    roof = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
            "traffic": None, "peak_kind": pk, "alg_bytes_per_launch": 9 * npts}
    # e2e: one solve = upload, 100 steps (sgb_run_steps), download
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    hk, hu, hm = pin(keys), pin(data[0]), pin(mask)
    out = torch.empty((len(keys) + 1) * 512, dtype=torch.float32).pin_memory()
    e0, e1 = _events()
    e0.record()
    nsolve = 5
    for _ in range(nsolve):
        g.load_map(hk, [hu, None], hm)
        fin = g.run_steps(sgb.HEAT7, [0], [1], [W.HEAT_DT], 100, use_graph=True)
        out.copy_(g.private_get_data_array(1 if fin else 0), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    te = dist.max(e0.elapsed_time(e1) / 1e3)
    e2e = {"value": round(dist.world * npts * 100 * nsolve / te / 1e9, 3), "unit": "Gpts/s",
           "h2d_bytes_per_step": int(hk.nbytes + hu.nbytes + hm.nbytes), "d2h_bytes_per_step": int(out.numel() * 4),
           "step": "one solve: upload, 100 heat steps (sgb_run_steps: one cooperative launch on this small grid), download"}
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        c = O.CpuSgrid(ps.size, 2, [0.0, 0.0])
        c.insert(ps.coords, [ps.values[0], ps.values[0]])
        t0 = time.perf_counter()
        c.heat(0, 1, W.HEAT_DT, steps=100, threads=1)
        dt = time.perf_counter() - t0
        cpu = {"value": round(npts * 100 / dt / 1e9, 5), "unit": "Gpts/s", "cores": 1, "kind": "port",
               "sample": f"100 heat steps on the 128^3 shell ({npts} points), 1 thread, {dt:.2f} s"}
    return _line("stencil Gpts/s (heat 7-point, 128^3 shell)", round(value, 3), "Gpts/s", dist, args, args.steps, t,
                 {"workload": "heat_128^3_shell_r20-32_chunk8^3_seed0", "active_points_per_gpu": npts,
                  "chunks": g.nchunks, "l2": "256 MiB L2-flushing write between timed steps (grid fits in L2)"},
                 roofline=roof, cpu_baseline=cpu, e2e=e2e, gpu_launches=args.steps, clocks=clk)


def run_insert1024(args, dist: Dist):
    """Insert / flush / tag / 27-point stress, 1024^3: one step = insert 2M
    clustered points (30% duplicates), flush sRight_ (float32 + int32),
    tagBoundaries NNStar, one 27-point box average (NNFull).  Inputs for
    every step are generated beforehand and resident in HBM."""
    import torch

    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import workloads as W
    torch.cuda.set_device(dist.local)
    nsteps = args.steps if args.steps <= 200 else 20
    nwarm = max(3, min(args.warmup, 8))
    size = (1024, 1024, 1024)
    g = sgb.SparseGridGpu(size, ["f32", "i32", "f32"], edge=8, device=dist.local)
    coeff = [1.0 / 27.0] * 27
    inputs = []
    for it in range(nwarm + nsteps):
        pts, fv, iv = W.insert_batch(it + 1000 * dist.rank)
        inputs.append((torch.from_numpy(pts.astype(np.int32)).cuda(), torch.from_numpy(fv).cuda(),
                       torch.from_numpy(iv).cuda()))
    npts = inputs[0][0].shape[0]
    phases = {"insert": 0.0, "flush": 0.0, "tag": 0.0, "box27": 0.0}
    flush_alg = 0.0
    recorded = []  # per timed step: its phase events, read once after the timed region

    def one(inp, timed):
        nonlocal flush_alg
        ev = [_events()[0] for _ in range(5)]
        n_before = g.nchunks
        ev[0].record()
        g.insert(inp[0], [inp[1], inp[2], None])
        ev[1].record()
        g.flush(["sRight_", "sRight_"])
        ev[2].record()
        g.tagBoundaries(sgb.NN_STAR)
        ev[3].record()
        g.applyStencils(sgb.BOX27, [0], [2], coeff)
        ev[4].record()
        if timed:
            recorded.append(ev)
            # staged key + 2 values in, old chunks read, merged chunks written (3 fields + mask)
            flush_alg += 16 * npts + 512 * 13 * (n_before + g.nchunks)

    for it in range(nwarm):
        one(inputs[it], False)
    torch.cuda.synchronize()
    clocks = ClockSampler(dist.local)
    dist.barrier()
    e0, e1 = _events()
    e0.record()
    for it in range(nsteps):
        one(inputs[nwarm + it], True)
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    step_ms, step_phase_ms = [], []
    for ev in recorded:
        per = []
        for k, name in enumerate(phases):
            dt = ev[k].elapsed_time(ev[k + 1])
            phases[name] += dt / 1e3
            per.append(round(dt, 3))
        step_ms.append(round(ev[0].elapsed_time(ev[4]), 3))
        step_phase_ms.append(per)
    g.check_device_errors()
    t = dist.max(e0.elapsed_time(e1) / 1e3)
    value = dist.world * npts * nsteps / t / 1e6
    peak, pk = _peak_hbm()
    ach = flush_alg / phases["flush"] / 1e9
    roof = {"bound": "hbm", "kernel": "flush (sort + merge)", "achieved": round(ach, 1), "peak": peak,
            "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None, "peak_kind": pk,
            "alg_bytes_per_launch": round(flush_alg / nsteps)}
    return _line("insert+flush+tag+box27 Mpts/s (1024^3, 2M points per step)", round(value, 2), "Mpts/s", dist,
                 args, nsteps, t, {"workload": "insert_stress_1024^3_2M_64clusters_sigma24_dup30_seed2",
                                   "points_per_step": npts, "chunks_at_end": g.nchunks,
                                   "phase_seconds": {k: round(v, 4) for k, v in phases.items()},
                                   "step_ms": step_ms,
                                   "step_phase_ms": {"order": list(phases), "steps": step_phase_ms},
                                   "l2": "inputs > L2 (48 MiB of points per step, map > 1 GB)"},
                 roofline=roof, cpu_baseline=None, e2e=None, gpu_launches=None, clocks=clk)


def _batched_specs(n=256):
    from openfpm_data_b200 import autotune as A
    from openfpm_data_b200 import workloads as W
    edges, radii, seeds = W.batch_grids(n)
    return [A.Spec(int(e), np.array([[e / 2.0, e / 2.0, e / 2.0, r]], np.float32), 0, int(s))
            for e, r, s in zip(edges, radii, seeds)]


def _spec_weights(specs):
    """Estimated active points of each batched grid (the ball's volume)."""
    return [4.0 / 3.0 * np.pi * float(sp.balls[0, 3]) ** 3 for sp in specs]


def batched_shard(rank: int, world: int):
    """(all 256 batched grid specs, indices of this rank's grids): the grids are dealt largest-first
    by estimated active points, so every rank computes the same split without talking."""
    from openfpm_data_b200 import shard
    all_specs = _batched_specs()
    return all_specs, shard.shard_weighted(_spec_weights(all_specs), rank, world)


def served_shard(rate: float, seconds: float, rank: int, world: int):
    """(the whole seed-4 request stream, this rank's requests): round-robin by request id."""
    from openfpm_data_b200 import shard
    from openfpm_data_b200 import workloads as W
    all_reqs = W.requests(rate=rate, duration=seconds, seed=4)
    return all_reqs, shard.shard_requests(all_reqs, rank, world)


def run_batched256(args, dist: Dist):
    """256 heat grids of uneven size (edges log-uniform in [32, 384], one
    centred ball of radius 0.25-0.5 edge, seed 3), 200 steps per solve.
    value: solves/s of the batched form (one persistent launch per step over
    the concatenated block maps, each solve's 200 steps one CUDA graph) with
    the autotuned launch; beside it the same solves with per-grid plain
    launches (one applyStencils per grid per step), with the reference's
    one-CTA-per-chunk execution model, and with one sgb_run_steps per grid."""
    import torch

    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import autotune as A
    from openfpm_data_b200 import workloads as W
    torch.cuda.set_device(dist.local)
    # ranks split the 256 grids without any exchange
    all_specs, mine = batched_shard(dist.rank, dist.world)
    specs = [all_specs[i] for i in mine]
    steps_per_solve = 200
    tune = A.autotune(specs[::8], sgb.HEAT7, [W.HEAT_DT], steps=10, device=dist.local)
    nsolves = max(1, min(args.steps, 20))
    nwarm = 1
    b, pts = A.build_batch(specs, sgb.HEAT7, [W.HEAT_DT], steps_per_solve * (nsolves + nwarm), tune.chunk_edge,
                           dist.local)
    b.set_launch_config(tune.ctas_per_sm, tune.stages)
    b.step(steps_per_solve * nwarm, use_graph=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(dist.local)
    dist.barrier()
    e0, e1 = _events()
    e0.record()
    for _ in range(nsolves):
        b.step(steps_per_solve, use_graph=True)
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    t = dist.max(e0.elapsed_time(e1) / 1e3)
    ngr, nch, nbytes = b.info()
    b.close()
    batched = len(all_specs) * nsolves / t
    # per-grid plain launches, the same grids and steps (8^3 chunks, default launch)
    grids = []
    for sp in specs:
        g = sgb.SparseGridGpu((sp.edge,) * 3, ["f32", "f32"], edge=8, device=dist.local)
        g.build_balls(sp.balls, sp.init, sp.seed, [0])
        grids.append(g)
    for g in grids[:4]:
        for k in range(4):
            g.applyStencils(sgb.HEAT7, [k % 2], [1 - k % 2], [W.HEAT_DT])
    torch.cuda.synchronize()
    # plain drop-in use: one applyStencils launch per grid per step (the pipelined kernel)
    p0, p1 = _events()
    p0.record()
    for g in grids:
        for k in range(steps_per_solve):
            g.applyStencils(sgb.HEAT7, [k % 2], [1 - k % 2], [W.HEAT_DT])
    p1.record()
    torch.cuda.synchronize()
    tp = dist.max(p0.elapsed_time(p1) / 1e3)
    # per-grid sgb_run_steps (grids of at most 4 chunks per SM run all steps in one cooperative launch)
    q0, q1 = _events()
    q0.record()
    for g in grids:
        g.run_steps(sgb.HEAT7, [0], [1], [W.HEAT_DT], steps_per_solve, use_graph=False)
    q1.record()
    torch.cuda.synchronize()
    tq = dist.max(q0.elapsed_time(q1) / 1e3)
    # the reference's execution model: one applyStencils launch per grid per step, one CTA per chunk
    # (the generic tile kernel, which gathers the halo per cell as loadGhostBlock does)
    r0, r1 = _events()
    r0.record()
    for g in grids:
        for k in range(steps_per_solve):
            g.applyStencils(sgb.HEAT7, [k % 2], [1 - k % 2], [W.HEAT_DT], tiled=True)
    r1.record()
    torch.cuda.synchronize()
    tr = dist.max(r0.elapsed_time(r1) / 1e3)
    for g in grids:
        g.close()
    plain = len(all_specs) / tp
    plain_ref = len(all_specs) / tr
    per_grid_runs = len(all_specs) / tq
    peak, pk = _peak_hbm()
    ach = 9 * pts * steps_per_solve * nsolves / t / 1e9 if dist.world == 1 else None
    roof = {"bound": "hbm", "achieved": round(ach, 1) if ach else None, "peak": peak, "unit": "GB/s",
            "frac": round(ach / peak, 4) if ach else None, "traffic": None, "peak_kind": pk,
            "alg_bytes_per_launch": 9 * pts}
    return _line("batched solves/s (256 heat grids, 200 steps each)", round(batched, 3), "solves/s", dist, args,
                 nsolves, t, {"workload": "batched_256_heat_grids_edge32-384_logu_seed3", "active_points": pts,
                              "grids_this_rank": len(specs), "split": "grids dealt to ranks by active points",
                              "chunks": nch, "resident_bytes": nbytes,
                              "autotune": {"chunk_edge": tune.chunk_edge, "ctas_per_sm": tune.ctas_per_sm,
                                           "stages": tune.stages, "threads_per_chunk": tune.threads_per_chunk,
                                           "table": tune.table},
                              "plain_solves_per_s": round(plain, 3), "batched_over_plain": round(batched / plain, 2),
                              "plain_one_cta_per_chunk_solves_per_s": round(plain_ref, 3),
                              "batched_over_plain_one_cta_per_chunk": round(batched / plain_ref, 2),
                              "per_grid_run_steps_solves_per_s": round(per_grid_runs, 3),
                              "batched_over_per_grid_run_steps": round(batched / per_grid_runs, 2),
                              "l2": "resident fields >> L2"},
                 roofline=roof, cpu_baseline=None, e2e=None, gpu_launches=steps_per_solve * nsolves, clocks=clk)


def run_served(args, dist: Dist):
    """Served form: Poisson arrivals at 2000 requests/s (seed 4), heat or
    Gray-Scott 50/50, edges log-uniform in [32, 256], 1-8 balls of radius
    0.1-0.3 edge, 50-500 steps; admitted under a 150 GB HBM budget and
    advanced in shared batched launches.  value: completed solves/s over the
    run; p50/p99 latency from arrival to read-back; beside it a sample of the
    same requests solved alone with per-grid plain launches."""
    import torch

    from openfpm_data_b200 import serve as S
    from openfpm_data_b200 import workloads as W
    torch.cuda.set_device(dist.local)
    # one seed-4 stream dealt round-robin to the ranks: each rank serves its share, no exchange
    all_reqs, reqs = served_shard(args.serve_rate, args.serve_seconds, dist.rank, dist.world)
    warm = W.requests(duration=0.05, seed=99)
    srv = S.Server(budget_bytes=150e9, device=dist.local)
    srv.run(warm, realtime=False)
    torch.cuda.synchronize()
    clocks = ClockSampler(dist.local)
    dist.barrier()
    st = srv.run(reqs, realtime=True)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    srv.close()
    summ = st.summary()
    if dist.world > 1:
        # merged latency percentiles and the aggregate over all ranks' requests
        parts = dist.gather({"lat": [d.latency for d in st.done], "wall": st.wall,
                             "pts": sum(d.points * d.steps for d in st.done)})
        lat = np.concatenate([np.asarray(p["lat"], dtype=np.float64) for p in parts]) if parts else np.zeros(1)
        wall = max(p["wall"] for p in parts)
        summ.update({"completed": int(lat.size), "wall_s": round(wall, 3),
                     "solves_per_s": round(lat.size / max(wall, 1e-9), 2),
                     "p50_latency_ms": round(float(np.percentile(lat, 50)) * 1e3, 2) if lat.size else None,
                     "p99_latency_ms": round(float(np.percentile(lat, 99)) * 1e3, 2) if lat.size else None,
                     "gpts_per_s": round(sum(p["pts"] for p in parts) / max(wall, 1e-9) / 1e9, 3),
                     "merged_over_ranks": dist.world})
    sample = reqs[: args.plain_sample]
    t0 = time.perf_counter()
    for r in sample:
        S.solve_alone(r, device=dist.local)
    torch.cuda.synchronize()
    tp = dist.max(time.perf_counter() - t0)
    plain = dist.world * len(sample) / tp  # every rank solves its own sample alone
    served = summ["completed"] / summ["wall_s"] if summ["wall_s"] else 0.0
    return _line(f"served solves/s (heat + Gray-Scott requests, Poisson {args.serve_rate:g}/s)", round(served, 2),
                 "solves/s",
                 dist, args, summ["completed"], summ["wall_s"],
                 {"workload": f"served_poisson{args.serve_rate:g}_{args.serve_seconds:g}s_edge32-256_seed4",
                  "requests": len(all_reqs), "requests_this_rank": len(reqs),
                  "split": "one seed-4 stream dealt round-robin by request id",
                  "serve": summ, "plain_sample": len(sample), "plain_solves_per_s": round(plain, 3),
                  "served_over_plain": round(served / plain, 2), "budget_bytes": 150e9},
                 roofline=None, cpu_baseline=None,
                 e2e={"value": round(served, 2), "unit": "solves/s", "h2d_bytes_per_step": None,
                      "d2h_bytes_per_step": None, "step": "one request: build on device, steps, read back"},
                 gpu_launches=None, clocks=clk)


def run_conv2b(args, dist: Dist):
    """Gray-Scott on the 512^3 benchmark grid written as a conv2_b user lambda against the C++ header
    (the reference's way to write a user stencil), against the library's fixed-function GS7 kernel on the
    same grid: both Gpts/s (CUDA events, `steps` steps after `warmup`) and a one-step bit-for-bit check.
    Runs openfpm_data_b200/bench_conv.cu, built like the drop-in test."""
    from openfpm_data_b200 import build as B
    from openfpm_data_b200 import workloads as W
    exe = B.build_conv_bench()
    ps = W.gray_scott()
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    n = len(keys)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "map.bin")
        with open(path, "wb") as fh:
            fh.write(np.int64(n).tobytes())
            fh.write(keys.astype(np.int64).tobytes())
            for d, b in zip(data, ps.bck):
                fh.write(np.concatenate([d, np.full(512, b, np.float32)]).astype(np.float32).tobytes())
            fh.write(np.concatenate([mask, np.zeros(512, np.uint8)]).tobytes())
        # the program runs on its device 0: this rank's GPU
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(dist.local + 1)]
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=devs[dist.local] if dist.local < len(devs) else str(dist.local))
        clocks = ClockSampler(dist.local)
        r = subprocess.run([exe, path, str(max(1, args.steps)), str(max(3, args.warmup))], capture_output=True,
                           text=True, timeout=900, env=env)
        clk = clocks.stop()
    if r.returncode != 0:
        raise RuntimeError(f"bench_conv failed ({r.returncode}): {r.stderr[-500:]}")
    res = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    steps = res["steps"]
    t = res["active_points"] * steps / (res["conv2_b_gpts"] * 1e9)
    return _line("conv2_b user-lambda Gray-Scott Gpts/s (512^3 sparse grid)", res["conv2_b_gpts"], "Gpts/s", dist,
                 args, steps, t, {"workload": "gray_scott_512^3_chunk8^3_40balls_seed1", "route": "conv2_b lambda",
                                  "fixed_function_gs7_gpts": res["gs7_gpts"],
                                  "conv2_b_over_gs7": res["conv2_b_over_gs7"],
                                  "one_step_bit_equal_to_gs7": res["one_step_bit_equal"]},
                 roofline=None, cpu_baseline=None, e2e=None, gpu_launches=steps, clocks=clk)


def _ghost_boxes(size=512, width=1):
    """The six ghost slabs of a 2x2x2 decomposition of the 512^3 grid: for each
    mid-plane, the `width` layers on either side of it (inclusive boxes)."""
    m, hi = size // 2, size - 1
    boxes = []
    for a in range(3):
        for lo_a, hi_a in ((m - width, m - 1), (m, m + width - 1)):
            lo, up = [0, 0, 0], [hi, hi, hi]
            lo[a], up[a] = lo_a, hi_a
            boxes.append(lo + up)
    return np.array(boxes, dtype=np.int64)


def run_ghost512(args, dist: Dist):
    """Ghost exchange on the Gray-Scott 512^3 grid: one step packs the six
    1-point ghost slabs around the three mid-planes (fields u, v), unpacks
    them into a second grid at the same place and merges them
    (removeAddUnpackFinalize).  Value: exchanged points per second."""
    import torch

    import openfpm_data_b200 as sgb
    from openfpm_data_b200 import workloads as W
    torch.cuda.set_device(dist.local)
    nsteps = args.steps if args.steps <= 500 else 100
    nwarm = max(3, min(args.warmup, 10))
    ps = W.gray_scott()
    keys, data, mask = W.build_block_map(ps.coords, ps.values, ps.size, 8, ps.bck)
    grids = []
    for _ in range(2):
        g = sgb.SparseGridGpu(ps.size, ["f32"] * 4, edge=8, device=dist.local)
        for p, b in enumerate([1.0, 0.0, 1.0, 0.0]):
            g.setBackgroundValue(p, b)
        g.load_map(keys, data + [d.copy() for d in data], mask)
        grids.append(g)
    a, b = grids
    boxes = _ghost_boxes()
    props = [0, 1]
    sizes = a.pack_sizes(boxes, props)
    buf = torch.empty(sum(sizes), dtype=torch.uint8, device=f"cuda:{dist.local}")
    starts = [tuple(int(v) for v in bx[:3]) for bx in boxes]
    phases = {"pack": 0.0, "unpack": 0.0, "merge": 0.0}
    recorded = []

    def one(timed):
        ev = [_events()[0] for _ in range(4)]
        ev[0].record()
        a.pack_boxes(boxes, props, buf)
        ev[1].record()
        b.unpack_boxes(buf, props, starts)
        ev[2].record()
        b.removeAddUnpackFinalize(props)
        ev[3].record()
        if timed:
            recorded.append(ev)

    for _ in range(nwarm):
        one(False)
    torch.cuda.synchronize()
    # packed points and chunks per step, from the buffer's headers
    hb = buf.cpu().numpy().tobytes()
    npnt = ncnk = 0
    pos = 0
    for sz in sizes:
        nc = int(np.frombuffer(hb, "<u8", 1, pos)[0])
        npnt += int(np.frombuffer(hb, "<u4", 1, pos + 32 + 12 * nc)[0])
        ncnk += nc
        pos += sz
    clocks = ClockSampler(dist.local)
    dist.barrier()
    e0, e1 = _events()
    e0.record()
    for _ in range(nsteps):
        one(True)
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    for ev in recorded:
        for k, name in enumerate(phases):
            phases[name] += ev[k].elapsed_time(ev[k + 1]) / 1e3
    a.check_device_errors()
    b.check_device_errors()
    t = dist.max(e0.elapsed_time(e1) / 1e3)
    value = dist.world * npnt * nsteps / t / 1e6
    # pack roofline: the touched chunks' masks once, the packed values read, the packed bytes written
    alg = 512 * ncnk + 8 * npnt + sum(sizes)
    peak, pk = _peak_hbm()
    ach = alg * nsteps / phases["pack"] / 1e9
    roof = {"bound": "hbm", "kernel": "pack (count + scans + emit, one call)", "achieved": round(ach, 1),
            "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None, "peak_kind": pk,
            "alg_bytes_per_launch": alg}

    # end to end: packed bytes to pinned host memory and back (the send / receive of a ghost exchange)
    h_send = torch.empty(buf.numel(), dtype=torch.uint8).pin_memory()
    rbuf = torch.empty_like(buf)
    dist.barrier()
    f0, f1 = _events()
    f0.record()
    for _ in range(nsteps):
        a.pack_boxes(boxes, props, buf)
        h_send.copy_(buf, non_blocking=True)
        rbuf.copy_(h_send, non_blocking=True)
        b.unpack_boxes(rbuf, props, starts)
        b.removeAddUnpackFinalize(props)
    f1.record()
    torch.cuda.synchronize()
    t_e2e = dist.max(f0.elapsed_time(f1) / 1e3)
    e2e = {"value": round(dist.world * npnt * nsteps / t_e2e / 1e6, 3), "unit": "Mpts/s",
           "h2d_bytes_per_step": int(buf.numel()), "d2h_bytes_per_step": int(buf.numel()),
           "step": "pack, packed buffer to pinned host memory and back, unpack, merge"}

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        o = O.OracleGrid(ps.size, edge=8, ptypes=(O.T_F32,) * 4)
        o.load_map(keys, data + [d.copy() for d in data], mask)
        reps, t0 = 0, time.perf_counter()
        while reps < 3 or (time.perf_counter() - t0 < 10 and reps < 50):
            o.pack(boxes, props)
            reps += 1
        dtc = time.perf_counter() - t0
        cpu = {"value": round(npnt * reps / dtc / 1e6, 3), "unit": "Mpts/s", "cores": 1, "kind": "port",
               "sample": f"{reps} packs of the six slabs by the numpy oracle (pack only), {dtc:.1f} s"}
    return _line("ghost exchange Mpts/s (pack + unpack + merge, six 1-point slabs of the Gray-Scott 512^3 grid)",
                 round(value, 2), "Mpts/s", dist, args, nsteps, t,
                 {"workload": "ghost_exchange_gray_scott_512^3_2x2x2_width1", "points_per_step": npnt,
                  "chunks_packed_per_step": ncnk, "packed_bytes_per_step": int(sum(sizes)),
                  "phase_seconds": {k: round(v, 5) for k, v in phases.items()},
                  "l2": "grids 2 x 157 MiB > L2; the packed buffer (a few MB) stays in L2 between pack and unpack"},
                 roofline=roof, cpu_baseline=cpu, e2e=e2e, gpu_launches=None, clocks=clk)


def _shell_1000():
    """The grid of the reference's Conv3x3x3 benchmarks (SparseGridGpu_util_test.cuh:488-680):
    insertSphere3D_radius on 32^3 chunks of 8 from (256, 256, 256), radii 128 / 56 -- the
    points with 56 < sqrtf(|p - (384, 384, 384)|^2) < 128, value x + y + z relative to the
    centre -- in a 1000^3 domain."""
    r = np.arange(256, 512, dtype=np.int64)
    out_c, out_v = [], []
    for z in r:
        y, x = np.meshgrid(r, r, indexing="ij")
        rel = np.stack([x.ravel() - 384, y.ravel() - 384, np.full(x.size, z - 384)], axis=1)
        rad = np.sqrt((rel * rel).sum(axis=1).astype(np.float32))
        keep = (rad < np.float32(128)) & (rad > np.float32(56))
        out_c.append(rel[keep] + 384)
        out_v.append(rel[keep].sum(axis=1).astype(np.float32))
    return np.concatenate(out_c), np.concatenate(out_v)


def run_conv1000(args, dist: Dist):
    """Conv3x3x3 on the reference's benchmark grid, in its four variants: the
    one-chunk-per-CTA tile kernel (STENCIL_MODE_INPLACE) and the point-list kernel
    (STENCIL_MODE_INPLACE_NO_SHARED), on x-fastest and on Morton chunk ids.  GElem/s =
    (existing - boundary points) x applications / time, the reference's measure."""
    import torch

    import openfpm_data_b200 as sgb
    torch.cuda.set_device(dist.local)
    nsteps = args.steps if args.steps <= 500 else 100
    nwarm = max(3, min(args.warmup, 10))
    coords, vals = _shell_1000()
    c_dev = torch.from_numpy(coords.astype(np.int32)).cuda()
    v_dev = torch.from_numpy(vals).cuda()
    coeff = [1.0] * 27
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device="cuda")
    res, clk, nelem, nchunks = {}, None, 0, 0
    peak, pk = _peak_hbm()
    for lin in ("smb", "zmb"):
        g = sgb.SparseGridGpu((1000, 1000, 1000), ["f32", "f32"], edge=8, device=dist.local, linearizer=lin)
        g.insert(c_dev, [v_dev, None])
        g.flush(["smax_", None])
        g.findNeighbours(sgb.NN_FULL)
        g.tagBoundaries(sgb.NN_FULL, calculate_existing_points=True)
        nelem = g.countExistingElements() - g.countBoundaryElements()
        nchunks = g.nchunks
        for mode, kind in (("shared", sgb.BOX27), ("noshared", sgb.BOX27_NS)):
            for _ in range(nwarm):
                g.applyStencils(kind, [0], [1], coeff)
            torch.cuda.synchronize()
            sampler = ClockSampler(dist.local) if (lin, mode) == ("smb", "shared") else None
            dist.barrier()
            evs = []
            for k in range(nsteps):
                flush.fill_(float(k))  # the grid (about 100 MB) would stay in L2 between applications
                e0, e1 = _events()
                e0.record()
                g.applyStencils(kind, [0], [1], coeff)
                e1.record()
                evs.append((e0, e1))
            torch.cuda.synchronize()
            dist.barrier()
            if sampler:
                clk = sampler.stop()
            t = dist.max(sum(a.elapsed_time(b) for a, b in evs) / 1e3)
            res[f"{lin}_{mode}"] = {"gelem_s": round(dist.world * nelem * nsteps / t / 1e9, 3),
                                    "us_per_application": round(t / nsteps * 1e6, 2)}
        g.check_device_errors()
        del g
    head = res["smb_shared"]
    t_one = head["us_per_application"] / 1e6
    ach = 9 * nelem / t_one / 1e9
    roof = {"bound": "hbm", "kernel": "k_box27_e8 (Conv3x3x3, one warp per chunk)",
            "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
            "traffic": _profile_traffic("box27_e8_conv1000.md"),
            "peak_kind": pk, "alg_bytes_per_launch": 9 * nelem}
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        o = O.OracleGrid((1000, 1000, 1000), edge=8, ptypes=[O.T_F32, O.T_F32])
        o.insert_flush(coords, [vals, np.zeros(len(vals), np.float32)], [O.OP_MAX, O.OP_NONE])
        o.tag_boundaries(O.NN_FULL)
        t0 = time.perf_counter()
        o.box27(0, 1, np.ones(27, np.float32))
        dtc = time.perf_counter() - t0
        cpu = {"value": round(nelem / dtc / 1e9, 5), "unit": "GElem/s", "cores": 1, "kind": "port",
               "sample": f"one Conv3x3x3 application on the full grid by the oracle, 1 thread, {dtc:.1f} s"}
    return _line("Conv3x3x3 GElem/s (1000^3 domain, 56 < r < 128 shell, 8^3 chunks)", head["gelem_s"], "GElem/s",
                 dist, args, nsteps, head["us_per_application"] / 1e6 * nsteps,
                 {"workload": "conv3x3x3_1000^3_shell_r56_r128_chunk8", "elements": nelem, "chunks": nchunks,
                  "variants": res, "l2": "256 MiB L2-flushing write before every timed application "
                                         "(the grid fits in L2); events around each application"},
                 roofline=roof, cpu_baseline=cpu, e2e=None, gpu_launches=nsteps, clocks=clk)


def run_reference(args, dist: Dist):
    from openfpm_data_b200 import workloads as W
    if dist.rank != 0:
        return None
    threads = os.cpu_count() or 1
    ps = W.gray_scott()
    nchunks = len(np.unique(((ps.coords[:, 2] // 8) * 64 + ps.coords[:, 1] // 8) * 64 + ps.coords[:, 0] // 8))
    wu = max(1, args.warmup)
    v, st, dt = cpu_baseline(ps, None, threads, max(1, args.steps), budget_s=90.0, warmup=wu)
    cpu = {"value": round(v, 5), "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"{st} Gray-Scott steps on the full 512^3 grid ({len(ps.coords)} points), {threads} threads"}
    return {"metric": METRIC, "value": round(v, 5), "unit": UNIT, "n_gpus": dist.world, "steps": st,
            "warmup": wu, "ms_per_step": round(dt / st * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, workloads.gray_scott)",
            "config": gs512_config(len(ps.coords), nchunks, dist.world),
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": round(v, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


SUB_KEYS = ("metric", "value", "unit", "steps", "ms_per_step", "roofline", "e2e", "cpu_baseline", "clocks",
            "gpu_launches")


def _sub_records(args, dist: Dist) -> dict:
    """The other benchmark configurations, each a bounded run timed like the headline (CUDA events on
    the launching stream, max over ranks, nvidia-smi clocks during its timed region): heat on the
    128^3 shell, the 1024^3 insert / flush / tag / box27 stress, the 256-grid batched form against
    per-grid plain launches, and the served form at 2000 requests/s and at a rate it sustains."""
    import copy
    plans = [
        ("heat128", run_heat128, dict(steps=100, warmup=5)),
        ("insert1024", run_insert1024, dict(steps=10, warmup=8)),
        ("batched256", run_batched256, dict(steps=4, warmup=3)),
        ("conv2b_gs512", run_conv2b, dict(steps=200, warmup=10)),
        ("served_2000rps", run_served, dict(steps=1, warmup=3, serve_rate=2000.0, serve_seconds=args.sub_serve_seconds,
                                            plain_sample=24)),
        ("served_sustained", run_served, dict(steps=1, warmup=3, serve_rate=args.sub_sustained_rate,
                                              serve_seconds=args.sub_serve_seconds, plain_sample=24)),
    ]
    out = {}
    for name, fn, over in plans:
        a = copy.copy(args)
        for k, v in over.items():
            setattr(a, k, v)
        try:
            line = fn(a, dist)
            rec = {k: line.get(k) for k in SUB_KEYS if k in line}
            rec["config"] = line.get("config")
            out[name] = rec
        except Exception as e:  # a failing sub-record is reported, the headline line still prints
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def main():
    args = parse()
    dist = Dist(args.gpus)
    try:
        if args.impl == "reference":
            line = run_reference(args, dist)
        else:
            runners = {"gs512": run_ours, "heat128": run_heat128, "insert1024": run_insert1024,
                       "batched256": run_batched256, "served": run_served, "ghost512": run_ghost512,
                       "conv1000": run_conv1000, "conv2b": run_conv2b}
            line = runners[args.workload](args, dist)
            if args.workload == "gs512" and not args.no_sub_records:
                subs = _sub_records(args, dist)
                if line is not None:
                    line["sub_records"] = subs
        if line is not None and dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
