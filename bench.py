"""Benchmark of the ZFP compress/decompress hot path on B200.

Workload (one step): a 512^3 float64 field -- the smooth field sin(0.10x)cos(0.13y)sin(0.07z) + N(0,1e-3)
scaled by 1e3, with 10% of its 4x4x4 blocks set to exactly zero and 1% of its
values replaced by +-10^U(-30,30) spikes (seeded, synthetic) -- compressed and
decompressed in fixed-accuracy 1e-6 and in fixed-precision 32 (variable-rate,
so block offsets come from the device scan).  Rounding rotates per step over
First/Last x tight_error off/on.  `value` is uncompressed GB coded per second:
4 passes of 1 GiB per step (2 modes x compress + decompress) over the step's
device time, inputs resident in HBM (1 GiB, larger than the 126 MB L2).

`e2e` is the same step through the C ABI (zfp_compress / zfp_decompress)
with host buffers in pinned memory: host->device copies of the field and the
stream, and device->host copies of the stream and the decoded field, inside
the timed region.

Also reported (extra keys): fixed-rate 8 float32 512^3 compress/decompress
GB/s and their roofline fractions; the other workloads (the 64^3 float32
plain array's latency, the 8192^2 float32 Gaussian random field at rates 4,
12 and 24, the 2^28 int32 random walk and the 256^3 uniform int64 field in
fixed-precision and reversible mode); the stream decoded without its block
index; the batched 2,000-array workload and the serving loop.  All inputs
come from tests/workloads.py (seeded, generated on the host).

--impl reference times the CPU restatement of zfp-rs (oracle/; the reference
itself cannot be built here: no Rust toolchain) on all host cores: each step
compresses and decompresses a 64-slice slab of the identical field in both
modes with that step's rounding (chunked compress, reader/worker pipelined
decode, as zfp-rs's Rayon path).
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NX = NY = NZ = 512
ROUNDINGS = [("first", False), ("first", True), ("last", False), ("last", True)]
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=512, help="cube side (default 512)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-fixed", action="store_true", help="skip the fixed-rate float32 measurement")
    ap.add_argument("--no-noindex", action="store_true",
                    help="skip decoding the workload's stream without its block index")
    ap.add_argument("--batched-arrays", type=int, default=2000,
                    help="arrays in the batched workload (0 skips it)")
    ap.add_argument("--batched-max-elems", type=int, default=16_777_216,
                    help="largest array of the batched workload, in elements")
    ap.add_argument("--serve-rates", default="200,1000,5000",
                    help="serving: Poisson arrival rates (req/s), comma separated; empty skips")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="serving: length of each arrival stream")
    ap.add_argument("--clock-csv", default="", help="also write the SM clock samples to this CSV file")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other workloads (64^3 latency, 8192^2 rates, int32 walk, int64 field)")
    ap.add_argument("--serve-small-rate", type=float, default=20000.0,
                    help="serving: rate of a stream of small requests (16 KB..1 MB); 0 skips")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving legs and print their results as one JSON list (the main run "
                         "starts this in a fresh process)")
    return ap.parse_args()


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


SLAB_Z = 64  # z-slices of the field in one reference-arm step (128 MiB of float64 at 512^2)


def host_field(n, seed=0):
    """The variable-rate workload's n^3 float64 field (tests/workloads.py)."""
    from tests import workloads as W

    return W.spiky_f64(n, seed=seed)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons during the timed region,
    read through NVML every 2 ms from a thread (read-only queries); the
    samples also go to a CSV file when a path is given (--clock-csv)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device_index: int, path: Path | None):
        import threading

        self.path = path
        self.samples = []
        self.stop_flag = False
        try:
            import pynvml as nv
            import torch

            nv.nvmlInit()
            h = None
            uuid = getattr(torch.cuda.get_device_properties(device_index), "uuid", None)
            if uuid is not None:
                try:
                    h = nv.nvmlDeviceGetHandleByUUID(("GPU-" + str(uuid)).encode())
                except Exception:
                    h = None
            if h is None:
                h = nv.nvmlDeviceGetHandleByIndex(device_index)
            self.nv, self.h = nv, h
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.get_reasons = get_reasons
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None

    def _run(self):
        nv, h = self.nv, self.h
        while not self.stop_flag:
            try:
                self.samples.append((time.perf_counter(), float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                     int(self.get_reasons(h))))
            except Exception:
                pass
            time.sleep(0.002)

    def stop(self):
        if self.nv is None:
            return None
        self.stop_flag = True
        self.t.join(timeout=5)
        if self.path is not None:
            try:
                with open(self.path, "w") as f:
                    f.write("t_s,sm_mhz,reasons_mask\n")
                    for t, mhz, r in self.samples:
                        f.write(f"{t:.4f},{mhz:.0f},{r:#x}\n")
            except Exception:
                pass
        if not self.samples:
            return None
        reasons = sorted(name for name, bit in self.REASONS.items() if any(r & bit for _, _, r in self.samples))
        return {"sm_mhz": float(np.median([m for _, m, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, every 2 ms"}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(pg, value, device):
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# The two modes of the variable-rate workload as expert parameters
# (minbits, maxbits, maxprec, minexp): fixed_accuracy(1e-6) (min_exp =
# frexp(1e-6).exponent - 1, zfp-rs config.rs:324-333) and fixed_precision(32).
MODES = {"accuracy_1e-6": (1, 16658, 64, -20), "precision_32": (1, 16658, 32, -1074)}


def workload_config(n, ws):
    """The `config` of both arms' lines: the workload itself (each arm states
    separately how it covers it)."""
    return {"workload": f"{n}^3 float64 smooth x1e3 + 10% zero blocks + 1% spikes; fixed-accuracy 1e-6 and "
                        f"fixed-precision 32, rounding First/Last x tight rotating per step",
            "passes_per_step": "2 modes x (compress + decompress) of 1 field",
            "l2": f"inputs ({n ** 3 * 8 / 2 ** 30:.3g} GiB) {'larger' if n ** 3 * 8 > 126e6 else 'not larger'} "
                  f"than the 126 MB L2", "parallelism": f"replicas x{ws}"}


def cpu_steps(slab, threads, steps, first_step=0, gpu_streams=None):
    """Steps of the oracle (the CPU restatement of zfp-rs) on `slab`: per step,
    both modes with the step's rounding, compress (chunked over `threads`) then
    decompress (reader/worker pipeline).  Returns (GB/s of uncompressed data,
    seconds, {(mode, rounding index): stream bytes}); with `gpu_streams` (the
    same keys: the GPU's stream of the same slab) also whether each matched."""
    from oracle import py_oracle as orc

    out = np.empty_like(slab)
    streams = {}
    nbytes = 0
    t0 = time.perf_counter()
    for i in range(first_step, first_step + steps):
        ri = i % len(ROUNDINGS)
        rnd, tight = ROUNDINGS[ri]
        for name, params in MODES.items():
            cfg = orc.config(*params, rnd, tight)
            stream, n = orc.compress(slab, cfg, threads=threads)
            assert n > 0 and orc.decompress(stream, out, cfg, threads=threads) == n
            streams[(name, ri)] = stream
            nbytes += 2 * slab.nbytes
    el = time.perf_counter() - t0
    same = None
    if gpu_streams is not None:
        same = {f"{k[0]}/{ROUNDINGS[k[1]][0]}{'+tight' if ROUNDINGS[k[1]][1] else ''}": gpu_streams.get(k) == v
                for k, v in streams.items()}
    return nbytes / el / 1e9, el, same


def cpu_sample_text(n, threads, steps):
    return (f"{n}x{n}x{SLAB_Z} float64 slab (the first {SLAB_Z} z-slices of the identical {n}^3 field) x {steps} "
            f"steps, fixed-accuracy 1e-6 + fixed-precision 32, rounding First/Last x tight rotating per step; "
            f"compress chunked over {threads} threads with bit concatenation (compress.rs:132-245), decompress "
            f"through the reader/worker pipeline (decompress/pipeline.rs:193-229); C++ restatement of zfp-rs's "
            f"CPU path (oracle/)")


def cpu_baseline(field_np, threads, gpu_streams, steps=8):
    """The CPU baseline beside the GPU arm: `steps` oracle steps on the slab,
    and the byte comparison of its streams with the GPU's streams of the same
    slab (one per mode and rounding)."""
    slab = np.ascontiguousarray(field_np[:SLAB_Z])
    v, el, same = cpu_steps(slab, threads, steps, gpu_streams=gpu_streams)
    return {"value": v, "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": cpu_sample_text(field_np.shape[0], threads, steps), "seconds": el,
            "gpu_stream_identical": same}


def probe_cargo():
    try:
        r = subprocess.run(["cargo", "--version"], capture_output=True, text=True, timeout=20)
        return r.stdout.strip() or f"exit {r.returncode}"
    except Exception as e:  # absent from the image
        return f"absent ({type(e).__name__})"


def run_reference(args):
    ws, rank, local, pg = dist_setup(args)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    threads = os.cpu_count() or 1
    field = host_field(args.size)
    slab = np.ascontiguousarray(field[:SLAB_Z])
    del field
    if args.warmup:
        cpu_steps(slab, threads, args.warmup)
    v, el, _ = cpu_steps(slab, threads, args.steps)
    sample = cpu_sample_text(args.size, threads, args.steps)
    line = {"metric": "compress/decompress GB/s on 1 B200 (bit-exact); batched p50/p99 ms",
            "impl": "reference", "value": v, "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el * 1e3 / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.size, ws), "sample": sample,
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample},
            "reference_toolchain": {"cargo": probe_cargo()},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    ws, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from tests import zfpb

    Z = zfpb.load()
    L = Z.lib()
    if args.serve_only:
        print(json.dumps(serving_legs(Z, dev, args)))
        return
    n = args.size
    field_np = host_field(n, seed=rank)
    field = torch.from_numpy(field_np).to(dev)
    nbytes = field.numel() * 8
    cfgs = {
        "accuracy_1e-6": Z.ZfpConfig.fixed_accuracy(1e-6),
        "precision_32": Z.ZfpConfig.fixed_precision(32),
    }
    cap = max(Z.maximum_size(field.shape, np.float64, c) for c in cfgs.values())
    stream_buf = torch.empty((cap + 7) // 8, dtype=torch.int64, device=dev)
    nblocks = (n // 4) ** 3
    offsets = torch.empty(nblocks + 1, dtype=torch.int64, device=dev)
    out = torch.empty_like(field)
    cs = torch.cuda.current_stream(dev)

    stream_bytes = {}

    def step(i):
        rnd, tight = ROUNDINGS[i % len(ROUNDINGS)]
        for name, cfg in cfgs.items():
            c = cfg.with_rounding(rnd, tight)
            nb = Z.compress_device(field, c, out=stream_buf, offsets=offsets)
            stream_bytes[(name, i % len(ROUNDINGS))] = nb
            Z.decompress_device(stream_buf, nb, out, c, offsets=offsets)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize(dev)
    if pg is not None:
        pg.barrier()
    clocks = ClockSampler(local, Path(args.clock_csv) if args.clock_csv else None) if rank == 0 else None
    Z.timing_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(cs)
    for i in range(args.steps):
        step(i)
    e1.record(cs)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    ktimes = Z.timing_read()
    Z.timing_enable(False)
    clock_info = clocks.stop() if clocks else None
    ms = max_over_ranks(pg, ms, dev)
    if pg is not None:
        pg.barrier()
    ms_per_step = ms / args.steps
    total_bytes = ws * args.steps * 4 * nbytes
    value = total_bytes / (ms / 1e3) / 1e9

    # Roofline of the dominant pass: a compress is encode_var + scan + pack, a
    # decompress is parse + finish (the two halves of the 3D decoder); each
    # moves the field plus the stream (algorithmic bytes).  Per-call time is
    # the pass's summed kernel time over its number of calls, from the event
    # timers above.
    mean_stream = float(np.mean(list(stream_bytes.values())))
    kinds = {k: v for k, v in ktimes.items() if v[1] > 0}
    calls = args.steps * len(cfgs)
    passes = {
        "compress (k_encode_var + k_scan + k_pack)": sum(kinds.get(k, (0, 0))[0] for k in ("encode_var", "scan", "pack")),
        "decompress (k_parse + k_finish)": sum(kinds.get(k, (0, 0))[0] for k in ("parse", "finish", "decode_var")),
    }
    dom = max(passes, key=passes.get)
    algo = nbytes + mean_stream
    peak, peak_kind = hbm_peak()
    call_ms = passes[dom] / calls
    achieved = algo / (call_ms / 1e3) / 1e9
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic_of(dom.split(" ")[0]) if n == 512 else None,
            "algorithmic_bytes_per_launch": algo, "avg_launch_ms": call_ms, "launches": calls,
            "other_pass_ms": {k: v / calls for k, v in passes.items() if k != dom}}
    tr = roof["traffic"]
    if tr and n == 512:
        # profiles/traffic.json holds the measured DRAM bytes of a call at 384^3 scaled to 512^3
        roof["traffic_over_algorithmic"] = tr / algo
        roof["traffic_source"] = "ncu dram__bytes_{read,write}.sum on 384^3, scaled by (512/384)^3"
    launches = int(sum(v[1] for v in ktimes.values()) + 2 * ktimes["scan"][1])  # a scan is 3 kernels

    # End to end through the C ABI with pinned host buffers.
    e2e = None if args.no_e2e else e2e_measure(Z, L, field, cfgs, cap, args, dev)

    # Fixed-rate 8 float32, device resident.
    fr = None if args.no_fixed else fixed_rate_measure(Z, n, dev, args, peak)

    # The same field's fixed-accuracy stream decoded without its block index
    # (a stream from elsewhere): offsets from the speculative parallel walk.
    ni = None if args.no_noindex else no_index_measure(Z, field, out, stream_buf, offsets, cfgs["accuracy_1e-6"], dev)

    # The GPU's streams of the CPU baseline's slab, for the byte comparison.
    slab_streams = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        slab_streams = gpu_slab_streams(Z, field, cfgs, stream_buf)

    # The other workloads: latency of the 64^3 plain array, 8192^2 float32 at
    # fixed rates, the int32 walk and the int64 field.
    del out, stream_buf, field
    torch.cuda.empty_cache()
    oc = None if args.no_configs else configs_measure(Z, dev, args, peak)

    # Batched workload (2,000 mixed arrays) against one call per array.
    bt = batched_measure(Z, dev, args) if args.batched_arrays > 0 else None
    sv = serving_in_child(args, local)

    if rank == 0:
        line = {
            "metric": "compress/decompress GB/s on 1 B200 (bit-exact); batched p50/p99 ms",
            "value": value, "unit": "GB/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": workload_config(n, ws), "mean_stream_bytes": mean_stream,
            "roofline": roof,
            "kernel_ms": {k: {"total_ms": v[0], "launches": v[1]} for k, v in kinds.items()},
            "gpu_launches": launches,
            "e2e": e2e,
            "fixed_rate_f32": fr,
            "other_workloads": oc,
            "no_index_decode": ni,
            "batched": bt,
            "serving": sv,
            "clocks": clock_info,
        }
        if ws == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline(field_np, os.cpu_count() or 1, slab_streams)
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


def gpu_slab_streams(Z, field, cfgs, buf):
    """The GPU streams of the CPU baseline's slab (the first SLAB_Z z-slices of
    the device field), one per mode and rounding, as bytes."""
    import torch

    slab = field[:SLAB_Z]
    got = {}
    for ri, (rnd, tight) in enumerate(ROUNDINGS):
        for name, cfg in cfgs.items():
            nb = Z.compress_device(slab, cfg.with_rounding(rnd, tight), out=buf)
            got[(name, ri)] = buf.view(torch.uint8)[:nb].cpu().numpy().tobytes()
    return got


def timed_calls(fn, reps, dev):
    """CUDA-event times (ms) of `reps` synchronous calls of fn on the current stream."""
    import torch

    cs = torch.cuda.current_stream(dev)
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(cs)
        fn()
        e1.record(cs)
        torch.cuda.synchronize(dev)
        ts.append(e0.elapsed_time(e1))
    return ts


def codec_leg(Z, x, cfg, reps, dev, peak, label):
    """Compress and decompress of the device tensor x: per-call p50/p99 ms
    (CUDA events around each call, host set-up included), GB/s of
    uncompressed data at p50 and the algorithmic roofline fraction (field +
    stream bytes over the p50 time)."""
    import torch

    cap = Z.maximum_size(x.shape, Z._np_dtype(x.dtype), cfg)
    sb = torch.empty((cap + 7) // 8, dtype=torch.int64, device=dev)
    nblk = int(np.prod([(m + 3) // 4 for m in x.shape]))
    offs = torch.empty(nblk + 1, dtype=torch.int64, device=dev)
    y = torch.empty_like(x)
    nb = Z.compress_device(x, cfg, out=sb, offsets=offs)
    for _ in range(3):
        Z.compress_device(x, cfg, out=sb, offsets=offs)
        Z.decompress_device(sb, nb, y, cfg, offsets=offs)
    tc = timed_calls(lambda: Z.compress_device(x, cfg, out=sb, offsets=offs), reps, dev)
    td = timed_calls(lambda: Z.decompress_device(sb, nb, y, cfg, offsets=offs), reps, dev)
    fb = x.numel() * x.element_size()
    pct = lambda v, q: float(np.percentile(v, q))
    res = {"workload": label, "bytes": fb, "stream_bytes": nb, "reps": reps}
    for key, ts in (("compress", tc), ("decompress", td)):
        t = pct(ts, 50) / 1e3
        res[f"{key}_ms_p50"] = pct(ts, 50)
        res[f"{key}_ms_p99"] = pct(ts, 99)
        res[f"{key}_gbs"] = fb / t / 1e9
        res[f"{key}_roofline_frac"] = (fb + nb) / t / 1e9 / peak
    if cfg.min_exp < -1074:
        res["lossless"] = bool(torch.equal(x.view(torch.uint8).reshape(-1), y.view(torch.uint8).reshape(-1)))
    return res


def configs_measure(Z, dev, args, peak):
    """The workloads other than the variable-rate field, device resident."""
    import torch

    from tests import workloads as W

    reps = max(10, min(args.steps, 40))
    out = {}
    x = torch.from_numpy(W.smooth((64, 64, 64), seed=0)).to(dev)
    out["plain_64cubed_f32_rate8"] = codec_leg(
        Z, x, Z.ZfpConfig.fixed_rate(8, np.float32, 3), max(reps, 100), dev, peak,
        "64^3 float32 smooth + N(0,1e-3), fixed-rate 8, rounding Never (launch-bound: latency)")
    x = torch.from_numpy(W.grf_f32(8192)).to(dev)
    for rate in (4, 12, 24):
        out[f"grf_8192sq_f32_rate{rate}"] = codec_leg(
            Z, x, Z.ZfpConfig.fixed_rate(rate, np.float32, 2), reps, dev, peak,
            f"8192^2 float32 Gaussian random field (spectrum k^-3, seed 1), fixed-rate {rate}")
    x = torch.from_numpy(W.random_walk_i32(1 << 28)).to(dev)
    for name, cfg in (("precision20", Z.ZfpConfig.fixed_precision(20)), ("reversible", Z.ZfpConfig.reversible())):
        out[f"walk_2p28_i32_{name}"] = codec_leg(
            Z, x, cfg, reps, dev, peak, f"2^28 int32 random walk (steps U{{-100..100}}), {name}")
    x = torch.from_numpy(W.uniform_i64((256, 256, 256))).to(dev)
    for name, cfg in (("precision32", Z.ZfpConfig.fixed_precision(32)), ("reversible", Z.ZfpConfig.reversible())):
        out[f"uniform_256cubed_i64_{name}"] = codec_leg(
            Z, x, cfg, reps, dev, peak, f"256^3 int64 uniform in +-2^40, {name}")
    del x
    torch.cuda.empty_cache()
    return out


def batched_measure(Z, dev, args):
    """Batched workload through zfpb_compress_batch / zfpb_decompress_batch
    (one plan, replayed as a CUDA graph) against one zfpb_compress_device /
    zfpb_decompress_device call per array, same output checked bit for bit."""
    import torch

    from tests import workloads as W

    specs = W.batched_specs(Z, args.batched_arrays, args.batched_max_elems)
    jobs = [(W.batched_array(sp, i, dev), sp[2]) for i, sp in enumerate(specs)]
    fields = [x for x, _ in jobs]
    cfgs = [c for _, c in jobs]
    total = sum(x.numel() * x.element_size() for x in fields)
    caps = [Z.maximum_size(x.shape, Z._np_dtype(x.dtype), c) for x, c in jobs]
    streams = [torch.empty((cap + 7) // 8, dtype=torch.int64, device=dev) for cap in caps]
    offs = [torch.empty(int(np.prod([(n + 3) // 4 for n in x.shape])) + 1, dtype=torch.int64, device=dev)
            for x in fields]
    outs = [torch.empty_like(x) for x in fields]
    citems = Z.batch_items(fields, cfgs, streams, offsets=offs)
    sizes = Z.compress_batch(citems)  # plans, tunes, captures
    sizes = Z.compress_batch(citems)
    ditems = Z.batch_items(outs, cfgs, streams, nbytes=sizes, offsets=offs)
    Z.decompress_batch(ditems)
    Z.decompress_batch(ditems)
    cs = torch.cuda.current_stream(dev)
    reps = max(5, min(args.steps, 20))

    def timed(fn, n):
        ts = []
        for _ in range(n):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record(cs)
            fn()
            e1.record(cs)
            torch.cuda.synchronize(dev)
            ts.append(e0.elapsed_time(e1))
        return ts

    bc = timed(lambda: Z.compress_batch(citems), reps)
    bd = timed(lambda: Z.decompress_batch(ditems), reps)
    # One call per array, the plain GPU form, into separate buffers.
    s2 = [torch.empty_like(s) for s in streams]
    o2 = [torch.empty_like(x) for x in fields]
    single_sizes = [0] * len(jobs)

    def per_array_compress():
        for i, (x, c) in enumerate(jobs):
            single_sizes[i] = Z.compress_device(x, c, out=s2[i], offsets=offs[i])

    def per_array_decompress():
        for i, (x, c) in enumerate(jobs):
            Z.decompress_device(s2[i], single_sizes[i], o2[i], c, offsets=offs[i])

    per_array_compress()
    per_array_decompress()
    sc = timed(per_array_compress, reps)
    sd = timed(per_array_decompress, reps)
    same = all(sizes[i] == single_sizes[i] and torch.equal(streams[i][: sizes[i] // 8], s2[i][: sizes[i] // 8])
               and torch.equal(outs[i].view(torch.uint8), o2[i].view(torch.uint8)) for i in range(len(jobs)))
    p = lambda v, q: float(np.percentile(v, q))
    res = {
        "workload": f"{len(jobs)} arrays, 60% f32 / 30% f64 / 10% i32, 1D-3D, 64..{args.batched_max_elems} elements "
                    f"log-uniform, sides not multiples of 4, per-array fixed-rate 2-32 / fixed-precision 8-48 / "
                    f"fixed-accuracy 1e-2..1e-9, random rounding",
        "arrays": len(jobs), "bytes": total, "stream_bytes": int(sum(sizes)),
        "compress_ms_p50": p(bc, 50), "compress_ms_p99": p(bc, 99),
        "decompress_ms_p50": p(bd, 50), "decompress_ms_p99": p(bd, 99),
        "compress_gbs": total / (p(bc, 50) / 1e3) / 1e9, "decompress_gbs": total / (p(bd, 50) / 1e3) / 1e9,
        "per_array_compress_ms_p50": p(sc, 50), "per_array_decompress_ms_p50": p(sd, 50),
        "speedup_compress": p(sc, 50) / p(bc, 50), "speedup_decompress": p(sd, 50) / p(bd, 50),
        "identical_to_per_array": bool(same), "reps": reps,
        "timing": "p50 over the same number of repetitions for the batch and for one call per array; "
                  "CUDA events on the calling stream around each whole call (host planning, graph launch, "
                  "per-array launches and synchronisations included)",
    }
    del streams, s2, outs, o2, fields, jobs
    torch.cuda.empty_cache()
    return res


def serving_measure(Z, dev, args, rate, seed=7, max_bytes=256 << 20):
    """Open-loop Poisson requests, 70% decompress / 30% compress, sizes
    log-uniform 16 KB..256 MB of float32/float64 2D/3D data with the batched
    workload's mode mix; through the serving loop (40 GB admission budget,
    4 lanes, 64 MiB batches) and through one synchronous device call per request, on the same
    arrival times.  Requests draw from a pool of resident arrays (requests on
    the same array write the same bytes to its output buffers); a decompress
    request carries its stream's block index, kept from its compression."""
    import torch

    rng = np.random.default_rng(seed)
    pool = []
    for i in range(48):
        nbytes = float(np.exp(rng.uniform(np.log(16 << 10), np.log(max_bytes))))
        dtype = np.float32 if rng.random() < 0.6 else np.float64
        dims = int(rng.integers(2, 4))
        n = nbytes / np.dtype(dtype).itemsize
        base = n ** (1.0 / dims)
        shape = [max(1, int(round(base * rng.uniform(0.8, 1.25)))) for _ in range(dims)]
        noise = torch.randn(shape, device=dev, dtype=torch.float64) * 1e-3
        grid = [torch.arange(m, device=dev, dtype=torch.float64) for m in shape]
        f = torch.ones(shape, device=dev, dtype=torch.float64)
        for ax, (fr, fn) in enumerate(zip([0.10, 0.13, 0.07], [torch.sin, torch.cos, torch.sin])):
            if ax >= dims:
                break
            view = [1] * dims
            view[dims - 1 - ax] = -1
            f = f * fn(fr * grid[dims - 1 - ax]).view(view)
        x = (f + noise).to(torch.float32 if dtype == np.float32 else torch.float64)
        k = int(rng.integers(0, 3))
        if k == 0:
            cfg = Z.ZfpConfig.fixed_rate(float(rng.integers(2, 33)), dtype, dims)
        elif k == 1:
            cfg = Z.ZfpConfig.fixed_precision(int(rng.integers(8, 49)))
        else:
            cfg = Z.ZfpConfig.fixed_accuracy(float(10.0 ** -rng.uniform(2, 9)))
        cfg = cfg.with_rounding(["never", "first", "last"][int(rng.integers(0, 3))], bool(rng.integers(0, 2)))
        cap = Z.maximum_size(x.shape, dtype, cfg)
        stream = torch.empty((cap + 7) // 8, dtype=torch.int64, device=dev)
        index = torch.empty(int(np.prod([(m + 3) // 4 for m in shape])) + 1, dtype=torch.int64, device=dev)
        nb = Z.compress_device(x, cfg, out=stream, offsets=index)  # the stream's block index is kept with it
        cstream = torch.empty_like(stream)
        out = torch.empty_like(x)
        citem = Z.batch_items([x], [cfg], [cstream])[0]
        ditem = Z.batch_items([out], [cfg], [stream], nbytes=[nb], offsets=[index])[0]
        pool.append(dict(x=x, cfg=cfg, stream=stream, nb=nb, index=index, cstream=cstream, out=out, citem=citem,
                         ditem=ditem, bytes=x.numel() * x.element_size()))
    nreq = int(rate * args.serve_seconds)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
    which = rng.integers(0, len(pool), size=nreq)
    dec = rng.random(nreq) < 0.7
    total = sum(pool[w]["bytes"] for w in which)
    torch.cuda.synchronize(dev)

    # Serving loop, warmed with one request per pool array of each kind (its
    # lanes' scratch grows to size), then timed.
    server = Z.Server(40 << 30)
    for j, e in enumerate(pool):
        assert server.submit(e["citem"], False, 2 * j) and server.submit(e["ditem"], True, 2 * j + 1)
    warm = 0
    while warm < 2 * len(pool):
        warm += len(server.poll(256, wait_ms=20))
    lat = np.zeros(nreq)
    queue = np.zeros(nreq)
    got = 0
    bad = 0
    t0 = time.perf_counter()
    for i in range(nreq):
        while time.perf_counter() - t0 < arrivals[i]:
            for tag, res, st, q, l in server.poll(256, wait_ms=0):
                lat[tag], queue[tag] = l, q
                got += 1
                bad += st != 0
        e = pool[which[i]]
        assert server.submit(e["ditem"] if dec[i] else e["citem"], bool(dec[i]), i)
    while got < nreq:
        for tag, res, st, q, l in server.poll(256, wait_ms=20):
            lat[tag], queue[tag] = l, q
            got += 1
            bad += st != 0
    t_serve = time.perf_counter() - t0
    server.close()

    # One synchronous device call per request, same arrival times (warmed the
    # same way: its workspace grows to size first).
    for e in pool:
        Z.compress_device(e["x"], e["cfg"], out=e["cstream"])
        Z.decompress_device(e["stream"], e["nb"], e["out"], e["cfg"], offsets=e["index"])
    torch.cuda.synchronize(dev)
    lat1 = np.zeros(nreq)
    t0 = time.perf_counter()
    for i in range(nreq):
        while time.perf_counter() - t0 < arrivals[i]:
            pass
        e = pool[which[i]]
        if dec[i]:
            Z.decompress_device(e["stream"], e["nb"], e["out"], e["cfg"], offsets=e["index"])
        else:
            Z.compress_device(e["x"], e["cfg"], out=e["cstream"])
        lat1[i] = (time.perf_counter() - t0 - arrivals[i]) * 1e3
    t_single = time.perf_counter() - t0
    pct = lambda v, q: float(np.percentile(v, q))
    res = {
        "workload": f"Poisson {rate:g} req/s for {args.serve_seconds:g} s, 70% decompress / 30% compress, "
                    f"16 KB..{max_bytes >> 20} MB float32/float64 2D/3D, batched mode mix, 40 GB admission budget, "
                    f"4 lanes, 64 MiB batches",
        "requests": nreq, "bytes": int(total),
        "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "gbs": total / t_serve / 1e9, "wall_s": t_serve,
        "queue_p50_ms": pct(queue, 50), "queue_p99_ms": pct(queue, 99), "failed": int(bad),
        "per_request_p50_ms": pct(lat1, 50), "per_request_p99_ms": pct(lat1, 99),
        "per_request_gbs": total / t_single / 1e9, "per_request_wall_s": t_single,
        "timing": "latency = submit to result on the host (wall clock); throughput = request bytes / wall time "
                  "from the first arrival to the last result",
    }
    del pool
    torch.cuda.empty_cache()
    return res


def serving_legs(Z, dev, args):
    """Every serving leg: the Poisson streams of --serve-rates, then the stream of small requests."""
    rates = [float(r) for r in args.serve_rates.split(",") if r.strip()]
    sv = [serving_measure(Z, dev, args, r) for r in rates]
    if args.serve_small_rate > 0:
        sv.append(serving_measure(Z, dev, args, args.serve_small_rate, max_bytes=1 << 20))
    return sv


def serving_in_child(args, local):
    """The serving legs in a fresh process on this rank's GPU, as a serving
    process runs.  Run inside this process after the other legs, the serving
    loop's p99 latency at 200-1,000 req/s was 14-40 ms (mostly time queued
    before launch) against 1.3-1.5 ms in a fresh process; the cause was not
    found (not the loop's own launch, result collection or scratch growth,
    timed inside the library), so the leg gets a process of its own."""
    if not [r for r in args.serve_rates.split(",") if r.strip()] and args.serve_small_rate <= 0:
        return None
    cmd = [sys.executable, str(ROOT / "bench.py"), "--serve-only", "--serve-rates", args.serve_rates,
           "--serve-seconds", str(args.serve_seconds), "--serve-small-rate", str(args.serve_small_rate)]
    # Eager module loading, as a latency-sensitive server should run: with lazy
    # loading (CUDA's default) a kernel's first launch in the process stalls
    # the serving loop 25-36 ms.
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK=str(local), CUDA_MODULE_LOADING="EAGER")
    limit = 600 + 30 * args.serve_seconds * (len(args.serve_rates.split(",")) + 1)
    try:
        r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=limit)
    except subprocess.TimeoutExpired:
        return [{"error": f"serving legs did not finish within {limit:.0f} s"}]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("[")]
    if r.returncode != 0 or not lines:
        # Reported in the line instead of failing the whole benchmark.
        return [{"error": f"serving legs failed (exit {r.returncode}): {r.stderr[-1000:]}"}]
    sv = json.loads(lines[-1])
    for leg in sv:
        leg["process"] = "a fresh process started for the serving legs, CUDA_MODULE_LOADING=EAGER"
    return sv or None


def traffic_of(kind):
    """DRAM bytes per launch of a kernel kind from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    try:
        return json.loads(p.read_text()).get(kind)
    except Exception:
        return None


def e2e_measure(Z, L, field, cfgs, cap, args, dev):
    import torch

    host_field = torch.empty(field.shape, dtype=torch.float64, pin_memory=True)
    host_field.copy_(field.cpu())
    host_out = torch.empty_like(host_field).pin_memory()
    host_stream = torch.empty((cap + 7) // 8 + 1, dtype=torch.int64, pin_memory=True)
    fnp = host_field.numpy()
    onp = host_out.numpy()
    snp = host_stream.numpy()
    bs = L.stream_open(snp.ctypes.data, snp.nbytes)
    zs = L.zfp_stream_open(bs)
    f_in = Z.field_of(fnp)
    f_out = Z.field_of(onp)
    h2d = d2h = 0

    def step(i):
        nonlocal h2d, d2h
        rnd, tight = ROUNDINGS[i % len(ROUNDINGS)]
        for cfg in cfgs.values():
            c = cfg.with_rounding(rnd, tight)
            L.zfp_stream_set_params(zs, c.min_bits, c.max_bits, c.max_prec, c.min_exp)
            L.zfp_stream_set_rounding(zs, c.rounding_code, int(c.tight_error))
            L.zfp_stream_rewind(zs)
            nb = L.zfp_compress(zs, C.byref(f_in))
            assert nb > 0, L.zfpb_last_error()
            L.zfp_stream_rewind(zs)
            assert L.zfp_decompress(zs, C.byref(f_out)) == nb
            h2d += fnp.nbytes + nb
            d2h += nb + onp.nbytes

    for i in range(args.warmup):
        step(i)
    h2d = d2h = 0
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(i)
    torch.cuda.synchronize(dev)
    el = time.perf_counter() - t0
    L.zfp_stream_close(zs)
    L.stream_close(bs)
    total = args.steps * 4 * fnp.nbytes
    return {"value": total / el / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d // args.steps,
            "d2h_bytes_per_step": d2h // args.steps, "ms_per_step": el * 1e3 / args.steps,
            "path": "zfp_compress/zfp_decompress (include/zfp.h) on pinned host buffers"}


def no_index_measure(Z, field, out, stream_buf, offsets, cfg, dev, reps=3):
    """Decompress of the field's stream with and without its block index
    (best of `reps`, CUDA events around each call, the host synchronisations
    of the call included): without one, zfpb_decompress_device finds the block
    offsets by the speculative parallel walk before decoding."""
    import torch

    nb = Z.compress_device(field, cfg, out=stream_buf, offsets=offsets)

    def timed(with_index):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        Z.decompress_device(stream_buf, nb, out, cfg, offsets=offsets if with_index else None)
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1)

    timed(False)
    with_index = min(timed(True) for _ in range(reps))
    without = min(timed(False) for _ in range(reps))
    return {"workload": f"{tuple(field.shape)} float64 fixed-accuracy 1e-6 stream, decompressed without its block index",
            "blocks": int(offsets.numel() - 1), "stream_bytes": nb, "decode_with_index_ms": with_index,
            "decode_without_index_ms": without,
            "path": "zfpb_decompress_device without block offsets: speculative parallel walk, then the decoder"}


def fixed_rate_measure(Z, n, dev, args, peak):
    import torch

    from tests import workloads as W

    x = torch.from_numpy(W.smooth((n, n, n), seed=0)).to(dev)
    cfg = Z.ZfpConfig.fixed_rate(8, np.float32, 3)
    cap = Z.maximum_size(x.shape, np.float32, cfg)
    sb = torch.empty((cap + 7) // 8, dtype=torch.int64, device=dev)
    y = torch.empty_like(x)
    nb = 0
    for _ in range(max(3, args.warmup)):
        nb = Z.compress_device(x, cfg, out=sb)
        Z.decompress_device(sb, nb, y, cfg)
    torch.cuda.synchronize(dev)
    Z.timing_enable(True)
    reps = max(5, args.steps)
    for _ in range(reps):
        Z.compress_device(x, cfg, out=sb)
        Z.decompress_device(sb, nb, y, cfg)
    torch.cuda.synchronize(dev)
    kt = Z.timing_read()
    Z.timing_enable(False)
    fb = x.numel() * 4
    res = {"workload": f"{n}^3 float32 smooth + N(0,1e-3), fixed-rate 8", "stream_bytes": nb}
    for kinds, key in ((("encode_fixed",), "compress"), (("decode_fixed", "parse", "finish"), "decompress")):
        ms = sum(kt[k][0] for k in kinds)
        cnt = reps
        if ms > 0:
            t = ms / cnt / 1e3
            res[f"{key}_gbs"] = fb / t / 1e9
            res[f"{key}_roofline_frac"] = (fb + nb) / t / 1e9 / peak
            res[f"{key}_ms"] = t * 1e3
    return res


if __name__ == "__main__":
    main()
