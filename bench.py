"""Throughput benchmark of the IQM metric path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--metric fsim|ssim|flip|msvd]
                    [--size 1080p|4k] [--batch] [--impl ours|reference] [--pairs B] [--no-cpu-baseline]

One step = one pass of the metric over a batch of B synthetic pairs (1920x1080 by default, 3840x2160
with --size 4k) already resident in HBM (distinct buffers; the batch is larger than the 126 MB L2,
so no flush is needed between steps).  `value` is pairs/s over all ranks; `e2e` is the same metric
through the host API (pinned host images copied in and scores copied out inside the timed region).
With --batch a step is the uneven-size batch instead: 256 pairs with sides uniform in [256, 2048],
SSIM on grey pairs and FSIM on RGB pairs, each metric one CUDA-graph batch plan replay.  With
--impl reference the CPU restatement of the reference's arithmetic (oracle/, all host threads) is
timed on the same workload instead.  Under torchrun each rank evaluates its own batch (independent
pairs, no collective on the data path): weak scaling; with --batch the 256 pairs are sharded
longest-processing-time first over the ranks: strong scaling.
"""
import argparse
import ctypes
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIZES = {"1080p": (1920, 1080), "4k": (3840, 2160)}
W, H = SIZES["1080p"]
SIZE = "1080p"


def set_size(name):
    """1080p, 4k, or WxH (a profiling case; its lines are named by the size)."""
    global W, H, SIZE
    if name in SIZES:
        W, H = SIZES[name]
    else:
        W, H = (int(v) for v in name.lower().split("x"))
    SIZE = name

# metric -> (workload name, synthetic generator name, score count per pair)
WORKLOADS = {
    "fsim": ("fsim_1080p_rgb", "rgb_gain_pair", 2),
    "ssim": ("ssim_1080p_grey", "grey_pair", 1),
    "flip": ("flip_1080p_rgb_67ppd", "rgb_blockquant_pair", 1),
    "msvd": ("msvd_1080p_rgb", "rgb_blockquant_pair", 1),
}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of each metric's dominant
# kernel from an ncu capture of this benchmark, with the pairs that launch processed; the summaries
# under profiles/ give the commands.  Scaled by pairs per launch when the live launch differs.
TRAFFIC = {
    # ssim_kernel, 32 pairs: 568,007,424 B read + 3,266,560 B written (profiles/ssim_kernel_1080p.md)
    "ssim": {"kernel": "ssim_kernel", "bytes_per_launch": 571273984, "pairs_per_launch": 32},
    # fsim_inv_cols_kernel, one chunk of 2 pairs: 10,389,760 + 12,827,904 B (profiles/fsim_inv_cols_kernel_1080p.md)
    "fsim": {"kernel": "fsim_inv_cols_kernel", "bytes_per_launch": 23217664, "pairs_per_launch": 2},
    # flip_vcols_kernel, 16 pairs: 1,628,939,776 + 18,826,752 B (profiles/flip_vcols_kernel_1080p.md)
    "flip": {"kernel": "flip_vcols_kernel", "bytes_per_launch": 1647766528, "pairs_per_launch": 16},
    # msvd_block_kernel, 32 pairs: 528,075,776 + 6,771,712 B (profiles/msvd_block_kernel_1080p.md)
    "msvd": {"kernel": "msvd_block_kernel", "bytes_per_launch": 534847488, "pairs_per_launch": 32},
}
# Executed tensor-core work of the mixed FSIM forms on 480x270 planes (1080p and 4K pairs): per pair
# 32 inverse transforms of each of the 480 columns (270 = 15 x 18: 27 m16n8k16 tiles) and of each
# of the 270 rows (480 = 16 x 30: 48 tiles), 2 * 16 * 8 * 16 = 4096 flops a tile, times the products
# per tile (3 with split-precision operands, 1 with single FP16 operands).
# The mixed SSIM forms run one CTA per 64x64 output tile: 4 warps, each with 5 x 16 horizontal and
# 4 x 16 vertical m16n8k16 tiles (4 moments x 2 n-tiles x 2 k-steps per 16-row block).
MMA_PRODUCTS = {"mixed": 3, "mixed_fast": 1}


def mma_tiles_per_pair(kernel, w, h):
    if kernel == "fsim_inv_cols_mma_kernel":
        return 32 * 480 * 27
    if kernel == "fsim_inv_rows_mma_kernel":
        return 32 * 270 * 48
    if kernel == "ssim_mma_kernel":
        return -(-w // 64) * -(-h // 64) * 4 * (80 + 64)
    return 0


def workload_name(metric):
    return WORKLOADS[metric][0].replace("1080p", SIZE)


def metric_name(metric):
    return "%s image pairs/sec (%s)" % ({"1080p": "1080p", "4k": "4K"}.get(SIZE, SIZE), metric.upper())


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--metric", default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=None, help="pairs per step (default 32 at 1080p, 16 at 4K)")
    ap.add_argument("--size", default="1080p", help="1080p, 4k, or WxH (e.g. 1100x300, a profiling case)")
    ap.add_argument("--batch", action="store_true",
                    help="uneven-size batch: 256 pairs, sides uniform in [256, 2048], SSIM + FSIM through one "
                         "CUDA-graph batch plan")
    ap.add_argument("--distinct", type=int, default=4, help="distinct synthetic pairs (replicated to --pairs)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "mixed_fast"],
                    help="FSIM and SSIM form: FP32, or the tensor-core forms with FP16 operands "
                         "(split-precision hi + lo products, or single products)")
    ap.add_argument("--flip-monitor", default="3840,0.7,0.7",
                    help="FLIP viewing set-up RES,DISTANCE,WIDTH (default 67.02 pixels per degree)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def make_pairs(metric, n):
    from iqm_b200 import synth
    gen = getattr(synth, WORKLOADS[metric][1])
    cfg = {"fsim": 1, "ssim": 0, "flip": 2, "msvd": 2}[metric]
    return [gen(H, W, config=cfg, pair=i) for i in range(n)]


class Clocks:
    """SM clock and throttle reasons sampled through NVML every few ms during the timed region."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device, period=0.005):
        self.device = device
        self.period = period
        self.samples = []
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self.error = None

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report it instead of a number
            self.error = "nvml unavailable: %s" % e
            return
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((mhz, rs))
                except Exception:
                    pass
                self._stop.wait(self.period)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()

    def stop(self):
        if self._thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "not sampled"]}
        self._stop.set()
        self._thread.join()
        mhz = [m for m, _ in self.samples]
        reasons = sorted({name for _, r in self.samples for name, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(mhz)}


def cpu_baseline(metric, pairs, seconds, one_pair_only=False):
    """Times the oracle's reference-faithful FP32 restatement on all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    o = Oracle("f32")
    fn = {"ssim": lambda a, b: o.ssim(a, b), "fsim": lambda a, b: o.fsim(a, b),
          "flip": lambda a, b: o.flip(a, b, ppd=o.flip_ppd(3840.0, 0.7, 0.7)), "msvd": lambda a, b: o.msvd(a, b)}[metric]
    done = 0
    t0 = time.perf_counter()
    while True:
        a, b = pairs[done % len(pairs)]
        fn(a, b)
        done += 1
        el = time.perf_counter() - t0
        if el >= seconds or one_pair_only:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": done / el, "unit": "pairs/s", "cores": cores, "kind": "port",
            "sample": "%d pair(s) of the %s workload (%dx%d), %.1f s, oracle FP32 build, OpenMP" % (
                done, workload_name(metric), W, H, el)}


def oracle_errors(metric, pairs, form_scores):
    """Largest |score - FP64 oracle| over the pairs and their scores, per form (part of the CPU
    baseline leg: the oracle is the checker here)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    o64 = Oracle("f64")
    fn = o64.fsim if metric == "fsim" else o64.ssim
    want = np.array([fn(a, b) for a, b in pairs]).reshape(len(pairs), -1)
    return {name: float(np.abs(s - want).max()) for name, s in form_scores.items()}


def run_reference(args, metric, rank, world):
    """--impl reference: the reference's arithmetic on the host CPU (the oracle port)."""
    if rank != 0:
        return
    pairs = make_pairs(metric, 1)
    for _ in range(max(0, args.warmup)):
        cpu_baseline(metric, pairs, 0.0, one_pair_only=True)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cpu_baseline(metric, pairs, 0.0, one_pair_only=True)
        times.append(time.perf_counter() - t0)
    per = float(np.mean(times))
    value = 1.0 / per
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"impl": "reference", "metric": metric_name(metric), "value": value,
            "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded 1/f^2 noise pairs)",
            "config": {"workload": workload_name(metric), "pairs_per_step": 1, "width": W, "height": H},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "port",
                             "sample": "1 pair per step, oracle FP32 build (reference arithmetic restated), OpenMP"},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batch_pairs(n=256, distinct=2):
    """The uneven-size batch: n pairs, width and height drawn independently and uniformly from
    [256, 2048] (seeded); SSIM pairs grey, FSIM pairs RGB, each a crop of one of `distinct`
    2048x2048 synthetic pairs."""
    from iqm_b200 import synth
    sizes = synth.uneven_sizes(n, seed=3000)
    greys = [synth.grey_pair(2048, 2048, config=3, pair=i) for i in range(distinct)]
    rgbs = [synth.rgb_gain_pair(2048, 2048, config=3, pair=i) for i in range(distinct)]

    def crop(p, w, h):
        return np.ascontiguousarray(p[0][:h, :w]), np.ascontiguousarray(p[1][:h, :w])

    grey = [crop(greys[i % distinct], w, h) for i, (w, h) in enumerate(sizes)]
    rgb = [crop(rgbs[i % distinct], w, h) for i, (w, h) in enumerate(sizes)]
    return sizes, grey, rgb


def run_batch(args, rank, world, local):
    """--batch: 256 uneven pairs per step, SSIM (grey) + FSIM (RGB), each metric one CUDA-graph batch
    plan replay; under torchrun the pairs are LPT-sharded over the ranks (strong scaling)."""
    metric = "uneven-size batch pairs/sec (SSIM+FSIM)"
    sizes, grey, rgb = batch_pairs()
    N = len(sizes)
    total_bytes = sum(8 * w * h for w, h in sizes)  # per metric: both RGBA8 images read once
    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Oracle
        o = Oracle("f32")
        for i in range(max(0, args.warmup)):
            o.ssim(*grey[i]), o.fsim(*rgb[i])
        times = []
        for k in range(args.steps):
            i = (k * 37) % N
            t0 = time.perf_counter()
            o.ssim(*grey[i])
            o.fsim(*rgb[i])
            times.append(time.perf_counter() - t0)
        value = 1.0 / float(np.mean(times))
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": "batch256_ssim_fsim", "pairs_per_step": 1, "sizes": "uniform [256, 2048]"},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "port",
                             "sample": "1 pair of the batch per step (SSIM grey + FSIM RGB), oracle FP32, OpenMP"},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return

    import torch
    import iqm_b200
    from iqm_b200 import parallel

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    costs = [parallel.pair_cost("fsim", w, h) + parallel.pair_cost("ssim", w, h) for w, h in sizes]
    mine = parallel.shard_lpt(costs, world)[rank]
    rt = iqm_b200.Runtime(local)
    stream = torch.cuda.Stream()
    rt.set_stream(stream.cuda_stream)
    bufs = []

    def upload(pairs):
        items = []
        for i in mine:
            a, b = pairs[i]
            da = torch.from_numpy(a.reshape(-1)).cuda()
            db = torch.from_numpy(b.reshape(-1)).cuda()
            bufs.extend([da, db])
            items.append((da.data_ptr(), db.data_ptr(), a.shape[1], a.shape[0], a.shape[1] * 4))
        return items

    g_items, c_items = upload(grey), upload(rgb)
    n = len(mine)
    d_ssim = torch.zeros(max(1, n), dtype=torch.float64, device="cuda")
    d_fsim = torch.zeros(max(1, 2 * n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    plans = []
    if n:
        prec = {"fp32": iqm_b200.IQM_FP32, "mixed": iqm_b200.IQM_MIXED,
                "mixed_fast": iqm_b200.IQM_MIXED_FAST}[args.precision]
        sp = iqm_b200.SSIM(rt)
        sp.precision = prec
        plans.append(iqm_b200.BatchPlan(rt, iqm_b200.METRIC_SSIM, g_items, d_ssim.data_ptr(), ssim=sp.params(),
                                        autotune=False))
        plans.append(iqm_b200.BatchPlan(rt, iqm_b200.METRIC_FSIM, c_items, d_fsim.data_ptr(), precision=prec,
                                        autotune=True))
    launches = sum(p.info()[1] for p in plans)

    def step():
        for p in plans:
            p.run()

    for _ in range(max(3, args.warmup)):
        step()
    stream.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = N / (ms_per_step / 1e3)

    # per-kernel device time from the eager form of the same step (graph replays carry no events)
    ktimes = {}
    if n:
        rt.set_kernel_timing(True)
        fs = iqm_b200.FSIM(rt)
        fs.precision = prec
        for _ in range(2):
            sp.compute_dev(g_items, d_ssim.data_ptr())
            fs.compute_dev(c_items, d_fsim.data_ptr())
        ktimes = rt.kernel_times()
        rt.set_kernel_timing(False)
    ktotal = sum(t for _, t in ktimes.values()) or 1.0
    roof = None
    if ktimes:
        kname, (klaunch, kms) = max(ktimes.items(), key=lambda kv: kv[1][1])
        my_bytes = sum(8 * sizes[i][0] * sizes[i][1] for i in mine)
        alg_launch = 2 * my_bytes / max(1, klaunch)  # two timing steps
        achieved = alg_launch / (kms / max(1, klaunch) / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": None, "kernel": kname, "avg_launch_us": 1e3 * kms / max(1, klaunch),
                "kernel_share": kms / ktotal,
                "pipeline_frac": 2 * total_bytes / world / (ms_per_step / 1e3) / 1e9 / hbm_peak,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "timing": "CUDA events around every launch of an eager pass (graph replays carry none)"}

    # end to end through the host batch API: pinned host images in, scores out, every step
    pin_g = [(torch.from_numpy(grey[i][0]).pin_memory(), torch.from_numpy(grey[i][1]).pin_memory()) for i in mine]
    pin_c = [(torch.from_numpy(rgb[i][0]).pin_memory(), torch.from_numpy(rgb[i][1]).pin_memory()) for i in mine]
    arr_g = iqm_b200._pairs([(a.data_ptr(), b.data_ptr(), a.shape[1], a.shape[0], a.shape[1] * 4) for a, b in pin_g])
    arr_c = iqm_b200._pairs([(a.data_ptr(), b.data_ptr(), a.shape[1], a.shape[0], a.shape[1] * 4) for a, b in pin_c])
    out = np.empty(3 * max(1, n), np.float64)
    outp = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    sp = iqm_b200.SSIM(rt).params()
    fp = iqm_b200.FLIPArguments().c()

    def e2e_step():
        if n:
            rt.check(rt.L.iqm_batch(rt.h, iqm_b200.METRIC_SSIM, arr_g, n, ctypes.byref(sp), ctypes.byref(fp), 0, 0,
                                    outp))
            rt.check(rt.L.iqm_batch(rt.h, iqm_b200.METRIC_FSIM, arr_c, n, ctypes.byref(sp), ctypes.byref(fp), 0, 0,
                                    outp))

    e2e_step()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(2, args.steps // 4)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ems], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    my_in = sum(2 * sizes[i][0] * sizes[i][1] * 4 for i in mine)
    line = {
        "metric": metric, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; crops of 2 distinct 2048x2048 pairs per metric)",
        "config": {"workload": "batch256_ssim_fsim", "pairs_per_step": N, "sizes": "w, h uniform in [256, 2048]",
                   "precision": args.precision, "parallelism": "lpt shards" if world > 1 else "single",
                   "form": "one CUDA-graph batch plan per metric, FSIM shapes autotuned",
                   "l2": "inputs larger than L2 (%.0f MB per metric per step), no flush" % (total_bytes / 1e6)},
        "roofline": roof,
        "kernels": {k: {"launches": c, "avg_us": 1e3 * t / max(1, c), "share": t / ktotal} for k, (c, t) in ktimes.items()},
        "e2e": {"value": N / (ems / e2e_steps / 1e3), "unit": "pairs/s", "h2d_bytes_per_step": 2 * my_in,
                "d2h_bytes_per_step": 3 * 8 * n},
        "gpu_launches": launches * args.steps, "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Oracle
        o = Oracle("f32")
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < args.cpu_seconds:
            i = (done * 37) % N
            o.ssim(*grey[i])
            o.fsim(*rgb[i])
            done += 1
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": done / el, "unit": "pairs/s",
                                "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                                "kind": "port", "sample": "%d pairs of the batch (SSIM + FSIM), %.1f s, oracle FP32, "
                                                          "OpenMP" % (done, el)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for p in plans:
        p.close()
    rt.close()
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    set_size(args.size)
    rank, world, local = dist_env()
    if args.batch:
        run_batch(args, rank, world, local)
        return
    metric = args.metric or "fsim"
    if args.impl == "reference":
        run_reference(args, metric, rank, world)
        return

    import torch
    import iqm_b200

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_note = "measured" if "hbm_gbs" in peaks else "fallback"
    tensor_peak = float(peaks.get("bf16_tflops", 1590.0))
    tensor_note = "measured" if "bf16_tflops" in peaks else "fallback"

    B = args.pairs or (32 if SIZE == "1080p" else 64)
    host_pairs = make_pairs(metric, min(args.distinct if SIZE == "1080p" else min(args.distinct, 2), B))
    rt = iqm_b200.Runtime(local)
    stream = torch.cuda.Stream()
    rt.set_stream(stream.cuda_stream)
    obj = {"fsim": iqm_b200.FSIM, "ssim": iqm_b200.SSIM, "flip": iqm_b200.FLIP, "msvd": iqm_b200.SVD}[metric](rt)
    prec = {"fp32": iqm_b200.IQM_FP32, "mixed": iqm_b200.IQM_MIXED, "mixed_fast": iqm_b200.IQM_MIXED_FAST}[args.precision]
    if metric in ("fsim", "ssim"):
        obj.precision = prec
    nscore = WORKLOADS[metric][2]
    res_x, dist_m, width_m = (float(v) for v in args.flip_monitor.split(","))
    flip_args = iqm_b200.FLIPArguments(res_x, dist_m, width_m)  # default 67.02 pixels per degree

    # device-resident batch: B distinct buffers (replicas of the distinct synthetic pairs)
    img_bytes = H * W * 4
    with torch.cuda.stream(stream):
        dev = torch.empty((B, 2, img_bytes), dtype=torch.uint8, device="cuda")
        for i in range(B):
            a, b = host_pairs[i % len(host_pairs)]
            dev[i, 0].copy_(torch.from_numpy(a.reshape(-1)))
            dev[i, 1].copy_(torch.from_numpy(b.reshape(-1)))
        d_scores = torch.zeros(B * nscore, dtype=torch.float64, device="cuda")
    stream.synchronize()
    base = dev.data_ptr()
    dev_pairs = [(base + (2 * i) * img_bytes, base + (2 * i + 1) * img_bytes, W, H, W * 4) for i in range(B)]

    def step():
        if metric == "flip":
            obj.compute_dev(dev_pairs, d_scores.data_ptr(), flip_args)
        else:
            obj.compute_dev(dev_pairs, d_scores.data_ptr())

    for _ in range(max(3, args.warmup)):
        step()
    launches_per_step = rt.last_launch_count()
    stream.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_per_step = ms / args.steps
    value = world * B / (ms_per_step / 1e3)

    # FSIM and SSIM: the three forms (plain FP32, tensor-core split-precision, tensor-core single
    # products) on the same device buffers, timed the same way, with their scores of the distinct
    # pairs kept for the error against the FP64 oracle (reported with the CPU baseline)
    forms, form_scores = None, {}
    if metric in ("fsim", "ssim"):
        forms = {}
        for fname, fprec in (("fp32", iqm_b200.IQM_FP32), ("mixed", iqm_b200.IQM_MIXED),
                             ("mixed_fast", iqm_b200.IQM_MIXED_FAST)):
            obj.precision = fprec
            for _ in range(3):
                step()
            torch.cuda.synchronize()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            for _ in range(args.steps):
                step()
            f1.record(stream)
            torch.cuda.synchronize()
            fms = f0.elapsed_time(f1)
            if dist:
                t = torch.tensor([fms], device="cuda")
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                fms = float(t.item())
            form_scores[fname] = d_scores[:nscore * len(host_pairs)].cpu().numpy().reshape(-1, nscore)
            forms[fname] = {"value": world * B / (fms / args.steps / 1e3), "ms_per_step": fms / args.steps}
        for fname in forms:
            forms[fname]["vs_fp32"] = forms[fname]["value"] / forms["fp32"]["value"]
            forms[fname]["max_score_diff_vs_fp32"] = float(abs(form_scores[fname] - form_scores["fp32"]).max())
        obj.precision = prec

    # per-kernel device time: the same K steps again with an event after every launch on the
    # library's stream (kept out of the throughput timing above)
    rt.set_kernel_timing(True)
    for _ in range(args.steps):
        step()
    ktimes = rt.kernel_times()
    rt.set_kernel_timing(False)
    ktotal = sum(t for _, t in ktimes.values()) or 1.0
    kname, (klaunch, kms) = max(ktimes.items(), key=lambda kv: kv[1][1])
    kernels = {k: {"launches": n, "avg_us": 1e3 * t / max(1, n), "share": t / ktotal} for k, (n, t) in ktimes.items()}

    # roofline of the dominant kernel: algorithmic bytes (each RGBA8 input read once, 8 B per pixel
    # pair) of the pairs one launch processes / that kernel's average launch duration
    alg_bytes = B * 2 * img_bytes
    pairs_per_launch = B * args.steps / max(1, klaunch)
    alg_launch = pairs_per_launch * 2 * img_bytes
    avg_s = kms / max(1, klaunch) / 1e3
    achieved = alg_launch / avg_s / 1e9
    traffic = None
    if metric in TRAFFIC and TRAFFIC[metric]["kernel"] == kname:
        t = TRAFFIC[metric]
        traffic = t["bytes_per_launch"] * pairs_per_launch / t["pairs_per_launch"]
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "traffic": traffic, "kernel": kname,
            "peak_source": peak_note, "alg_bytes_per_launch": alg_launch, "pairs_per_launch": pairs_per_launch,
            "avg_launch_us": avg_s * 1e6, "kernel_share": ktimes[kname][1] / ktotal,
            "pipeline_frac": alg_bytes / (ms_per_step / 1e3) / 1e9 / hbm_peak,
            "timing": "CUDA events on the library stream around every launch, second pass of the K steps"}
    if metric in ("fsim", "ssim") and args.precision in MMA_PRODUCTS:
        # tensor pipe of the tensor-core kernels: executed MMA flops per launch / average launch time
        tens = {}
        for k in ("fsim_inv_cols_mma_kernel", "fsim_inv_rows_mma_kernel", "ssim_mma_kernel"):
            tiles = mma_tiles_per_pair(k, W, H)
            if k not in ktimes:
                continue
            n_l, t_ms = ktimes[k]
            flops = B * args.steps * tiles * 4096 * MMA_PRODUCTS[args.precision] / max(1, n_l)
            achieved_t = flops / (t_ms / max(1, n_l) / 1e3) / 1e12
            tens[k] = {"achieved": achieved_t, "peak": tensor_peak, "unit": "TFLOP/s", "frac": achieved_t / tensor_peak,
                       "flops_per_launch": flops, "peak_source": tensor_note + " dense bf16 (burst)"}
        roof["tensor"] = tens
    if metric == "flip":
        # FLIP is bound by FP32 arithmetic: the SIMT fraction of its filter taps.  Per pixel pair:
        # the CSF prefilter, 3 channels x 2 images x (horizontal + vertical) taps of 2 rc + 1, and
        # the feature filters, per image 3 horizontal (g, edge, point) and 4 vertical outputs of
        # 2 rf + 1 taps; a multiply-add is 2 flops.  The colour epilogue is not counted.
        ppd = rt.L.iqm_flip_ppd(ctypes.byref(flip_args.c()))
        rf = int(np.ceil(np.float32(3.0) * np.float32(0.5 * 0.082) * np.float32(ppd)))
        rc = int(np.ceil(np.float32(3.0) * np.sqrt(np.float32(0.04) / np.float32(2.0 * np.pi ** 2)) * np.float32(ppd)))
        flops_px = 2 * (12 * (2 * rc + 1) + 14 * (2 * rf + 1))
        sm_max = (clk or {}).get("sm_max_mhz") or 1965
        simt_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12
        simt = flops_px * W * H / (ms_per_step / 1e3 / B) / 1e12
        roof["simt"] = {"achieved": simt, "peak": simt_peak, "unit": "TFLOP/s", "frac": simt / simt_peak,
                        "flops_per_pixel": flops_px, "radii": {"feature": rf, "csf": rc},
                        "scope": "whole step, filter taps only",
                        "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 flops x max SM clock"}

    # end to end: host API with pinned host images and host scores
    e2e = None
    pin = []
    for i in range(B):
        a, b = host_pairs[i % len(host_pairs)]
        pa = torch.from_numpy(a).pin_memory()
        pb = torch.from_numpy(b).pin_memory()
        pin.append((pa, pb))
    items = [(pa.data_ptr(), pb.data_ptr(), W, H, W * 4) for pa, pb in pin]
    arr = iqm_b200._pairs(items)
    out = np.empty(B * nscore, np.float64)
    outp = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    L = rt.L

    def e2e_step():
        if metric == "ssim":
            p = obj.params()
            rt.check(L.iqm_ssim_batch(rt.h, arr, B, ctypes.byref(p), outp))
        elif metric == "msvd":
            rt.check(L.iqm_msvd_batch(rt.h, arr, B, outp))
        elif metric == "flip":
            p = flip_args.c()
            rt.check(L.iqm_flip_batch(rt.h, arr, B, ctypes.byref(p), outp))
        else:
            rt.check(L.iqm_fsim_batch(rt.h, arr, B, obj.precision, obj.energy_mode, outp))

    for _ in range(2):
        e2e_step()
    e2e_steps = max(3, args.steps // 4)
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ems], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e = {"value": world * B / (ems / e2e_steps / 1e3), "unit": "pairs/s",
           "h2d_bytes_per_step": B * 2 * img_bytes, "d2h_bytes_per_step": B * nscore * 8}

    # the host link's own ceiling: the same pinned buffers copied to the device with nothing else
    # running (one plain copy per image, as the e2e step issues), timed like the e2e step
    link = torch.empty(B * 2 * img_bytes, dtype=torch.uint8, device="cuda")

    def link_step():
        off = 0
        for pa, pb in pin:
            for t in (pa, pb):
                n = t.numel() * t.element_size()
                link[off:off + n].copy_(t.view(torch.uint8).reshape(-1), non_blocking=True)
                off += n

    with torch.cuda.stream(stream):
        link_step()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(e2e_steps):
            link_step()
        e1.record(stream)
    torch.cuda.synchronize()
    lms = e0.elapsed_time(e1) / e2e_steps
    del link
    e2e["h2d_gbs"] = B * 2 * img_bytes / (ems / e2e_steps) / 1e6
    e2e["h2d_copy_only_gbs"] = B * 2 * img_bytes / lms / 1e6
    e2e["link_frac"] = e2e["h2d_gbs"] / e2e["h2d_copy_only_gbs"]

    line = {
        "metric": metric_name(metric), "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded 1/f^2 noise pairs, %d distinct replicated to %d device buffers)" % (
            len(host_pairs), B),
        "config": {"workload": workload_name(metric), "pairs_per_step": B, "width": W, "height": H,
                   "precision": args.precision if metric in ("fsim", "ssim") else "fp32",
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (%.0f MB per step), no flush" % (alg_bytes / 1e6)},
        "roofline": roof, "kernels": kernels, "e2e": e2e, "gpu_launches": launches_per_step * args.steps, "clocks": clk,
    }
    if forms:
        line["forms"] = forms
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(metric, host_pairs, args.cpu_seconds)
        if form_scores:
            # the checker: each FSIM form's scores of the distinct pairs against the FP64 oracle
            line["forms_err_vs_fp64"] = oracle_errors(metric, host_pairs, form_scores)
    if rank == 0:
        print(json.dumps(line), flush=True)
    rt.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
