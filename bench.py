#!/usr/bin/env python
"""Benchmark: BC7 (and BC1) encode Mpix/s on B200 against the reference CPU encoder.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (`value`): BC7 of a 2048x2048 RGBA8 texture (colour gradients + 4-octave value noise + 20 hard
rectangles, alpha from 2-octave noise thresholded at 30%), seeded synthetic content. A step encodes one texture
through the device API; steps cycle over a ring of distinct textures whose total size exceeds the 126 MB L2, so no
step reads a texture still resident in L2. Inputs are in HBM when the timed region starts. With N GPUs (torchrun)
every rank encodes its own ring (weak scaling, no collective on the data path); value = all ranks' pixels / max time.

`e2e` is the same workload through the synchronous host C ABI (zap_tex_cuda_bc_encode): pinned host texture in,
host->device copy, encode, device->host copy of the blocks, every step.
`roofline` is the dominant kernel's algorithmic bytes per launch / its CUDA-event duration, against the measured HBM
copy bandwidth. The encoders are compute-bound, so `roofline.alu` adds the bound that binds: the reference
algorithm's counted operations per launch (profiles/alu_ops.json, from oracle/count_ops.py on these textures) over
the same duration, against 128 lanes x SMs x the SM clock sampled during the timed region.
`cpu_baseline` is the reference's own encoder (oracle/_ref, built from zap_tex.h) on this host's cores, using the
reference's band-parallel scheme; `--impl reference` times only that, on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "BC1/BC7 encode Mpix/s on 1 B200 at ref PSNR; batched vs plain launch; vs CPU"
W, H = 2048, 2048
WORKLOAD = "bc7 2048x2048 rgba8, colour gradients + value noise + rectangles, noise alpha"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    p.add_argument("--profile", default=None, choices=["bc7", "bc1", "bc4", "bc5", "bc6h", "astc", "batch", "rdo", "rdo7"],
                   help="profiling case: only that encoder on a ring of 2048x2048 inputs, no e2e / CPU / extras "
                        "(rdo / rdo7: BC1 / BC7 at lambda 30, one chain over a 256x256 texture per step)")
    return p.parse_args()


def run_profile_case(args):
    """A small, self-contained case for ncu: W + K encodes of one format over a ring of distinct 2048^2 textures."""
    import torch

    import zap_b200
    import zap_b200.synth as S
    dev = torch.device("cuda", 0)
    fmt = args.profile
    ring = 10
    if fmt == "batch":  # 256 textures of the batched workload's size / format mix, sides 64..512
        sizes = S.batch_sizes(256, seed=0, lo=6, hi=9)
        fmts = S.batch_formats(256, seed=0)
        texs = [S.colour_texture(w, h, seed=10000 + k, device=dev) for k, (w, h) in enumerate(sizes)]
        b = zap_b200.Batch(texs, fmts)
        ms = time_device(lambda k: b.run(), args.steps, args.warmup, 1)
        print(json.dumps({"profile_case": fmt, "steps": args.steps, "ms_per_step": ms / args.steps,
                          "Mpix_s": args.steps * b.pixels / 1e6 / (ms / 1e3)}))
        b.close()
        return
    if fmt in ("rdo", "rdo7"):  # one serial chain per step: zap_bc_encode(BC1 or BC7, rdo 30) of a 256x256 texture
        tex = S.colour_texture(256, 256, seed=7, alpha="noise", device=dev)
        code = zap_b200.BC1 if fmt == "rdo" else zap_b200.BC7
        out = zap_b200.bc_encode_rdo_dev(tex, code, 30.0)
        ms = time_device(lambda k: zap_b200.bc_encode_rdo_dev(tex, code, 30.0, out=out), args.steps, args.warmup, 1)
        print(json.dumps({"profile_case": fmt, "steps": args.steps, "ms_per_step": ms / args.steps,
                          "Mpix_s": args.steps * 256 * 256 / 1e6 / (ms / 1e3)}))
        return
    if fmt == "bc6h":
        texs = [S.hdr_texture(W, H, seed=k, device=dev) for k in range(ring)]
        enc = lambda t: zap_b200.bc6h_encode_dev(t)  # noqa: E731
    else:
        code = {"bc7": zap_b200.BC7, "bc1": zap_b200.BC1, "bc4": zap_b200.BC4, "bc5": zap_b200.BC5, "astc": zap_b200.ASTC4X4}[fmt]
        if fmt == "bc5":
            texs = [S.normal_map(W, H, seed=k, device=dev) for k in range(ring)]
        else:
            texs = [S.colour_texture(W, H, seed=100 + k, alpha="opaque" if fmt == "bc1" else "noise", device=dev) for k in range(ring)]
            if fmt == "bc4":
                texs = [t[..., :1].contiguous() for t in texs]
        enc = lambda t: zap_b200.bc_encode_dev(t, code)  # noqa: E731
    torch.cuda.synchronize()
    ms = time_device(lambda k: enc(texs[k % ring]), args.steps, args.warmup, 1)
    print(json.dumps({"profile_case": fmt, "steps": args.steps, "ms_per_step": ms / args.steps,
                      "Mpix_s": args.steps * W * H / 1e6 / (ms / 1e3)}))


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":  # CPU only: rank 0 runs the reference, the other ranks exit; no process group
        return world, rank, local
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x, world, device="cuda"):
    """The slowest rank's time: one all_reduce(MAX) after the timed region (the only collective; no data moves)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(max_ms, world, steps, mpix_per_step):
    """Whole-job throughput: every rank encodes its own ring (weak scaling), all ranks' pixels over the max time."""
    return world * steps * mpix_per_step / (max_ms / 1e3)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        # nvidia-smi's start (process launch, NVML set-up) contends with the driver: wait for its first sample, at
        # most 3 s, so it is sampling steadily before the caller's timed work begins (timed regions of a few ms read up
        # to 1 ms slow when they overlapped its start)
        t0 = time.perf_counter()
        while self.proc and not self.rows and self.proc.poll() is None and time.perf_counter() - t0 < 3.0:
            time.sleep(0.01)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def library_md5():
    """First 12 hex digits of the MD5 of the CUDA library this run loaded (which build a line measured)."""
    import hashlib

    import zap_b200
    with open(zap_b200._lib.LIB_PATH, "rb") as f:
        return hashlib.md5(f.read()).hexdigest()[:12]


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# the measured scalar issue rate (instructions per clock per SM), set by measure_alu_peak() before any roofline
ALU_PEAK = {}


def measure_alu_peak(dev, sms, local, seconds=1.0):
    """Measures the SMs' instruction rate for the kinds the encoders are built from (zap_tex_cuda_alu_probe_dev:
    8 CTAs of 256 threads per SM, 8 independent chains per thread of mad.lo.u32, fma.rn.f32, dp4a, or mad/fma
    alternating), each kind one launch of about `seconds`, timed with CUDA events while the SM clock is sampled.
    Rates are in instructions per clock per SM (time x median sampled SM MHz), so a roofline can be scaled to the
    clock of the region it is compared with."""
    import ctypes as C

    import torch

    import zap_b200
    lib = zap_b200.load()
    sink = torch.zeros(4, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    ins = C.c_double()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(kind, iters):
        e0.record()
        zap_b200.check(lib.zap_tex_cuda_alu_probe_dev(kind, iters, sink.data_ptr(), C.c_void_p(stream.cuda_stream), C.byref(ins)),
                       "alu_probe")
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    kinds = {}
    for kind, name in ((0, "imad"), (1, "ffma"), (2, "dp4a"), (3, "imad+ffma")):
        timed(kind, 64)
        ms = timed(kind, 256)
        iters = max(256, min(2_000_000, int(256 * seconds * 1e3 / max(ms, 1e-3))))
        with ClockSampler(local) as clk:
            ms = timed(kind, iters)
        mhz = clk.summary()["sm_mhz"] or clk.summary()["sm_max_mhz"]
        if not mhz:
            continue
        kinds[name] = {"ms": ms, "instructions": ins.value, "sm_mhz": mhz, "G_per_s": ins.value / (ms / 1e3) / 1e9,
                       "per_clk_per_sm": ins.value / (ms / 1e3) / (mhz * 1e6) / sms}
    if kinds:
        best = max((k for k in kinds if k != "dp4a"), key=lambda k: kinds[k]["per_clk_per_sm"])
        ALU_PEAK.update({"per_clk_per_sm": kinds[best]["per_clk_per_sm"], "kind": best, "kinds": kinds})
    return ALU_PEAK


def alu_roofline(kernel, ops_per_launch_ms, sm_mhz, sms):
    """ALU roofline of one kernel: the reference algorithm's counted operations per launch (profiles/alu_ops.json,
    written by oracle/count_ops.py on this workload's textures) over the kernel's average launch time, against the
    measured scalar issue rate (the fastest of mad.lo.u32, fma.rn.f32 and their mix, instructions per clock per SM
    from measure_alu_peak) x SMs x the median SM clock of the timed region; without a measurement, the derived 128
    lanes per SM. The kernels do a texel-to-entry distance (13 counted ops for RGBA) in one dp4a + one multiply-add +
    one min, so a fraction above 1 is possible: it is a throughput figure against scalar issue; the ncu issue-slot
    use of each kernel (profiles/issue_active.json) is the utilisation."""
    ops, ms = ops_per_launch_ms
    table = alu_ops()
    if ops is None or not ms or not sm_mhz:
        return None
    if ALU_PEAK:
        per_clk = ALU_PEAK["per_clk_per_sm"]
        source = (f"measured: {per_clk:.1f} {ALU_PEAK['kind']} instructions per clock per SM (alu probe) x {sms} SMs x "
                  f"{sm_mhz:.0f} MHz (median SM clock, timed region)")
    else:
        per_clk = 128.0
        source = f"derived: {sms} SMs x 128 lanes x {sm_mhz:.0f} MHz (median SM clock, timed region)"
    peak = sms * per_clk * sm_mhz * 1e6 / 1e9
    achieved = ops / (ms / 1e3) / 1e9
    out = {"bound": "alu", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "Gop/s", "frac": achieved / peak,
           "ops_per_launch": ops, "peak_source": source, "ops_definition": table.get("definition") if table else None}
    issue = issue_active().get(kernel)
    if issue is not None:
        out["ncu_issue_active"] = issue
    return out


def issue_active():
    """smsp__issue_active (% of issue slots) per kernel or encode, from the committed ncu captures."""
    try:
        with open(os.path.join(ROOT, "profiles", "issue_active.json")) as f:
            return json.load(f).get("kernels", {})
    except (OSError, ValueError):
        return {}


def alu_ops():
    try:
        with open(os.path.join(ROOT, "profiles", "alu_ops.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def ops_per_texture(kernel):
    table = alu_ops() or {}
    for entry in table.values():
        if isinstance(entry, dict) and kernel in entry.get("ops_per_texture", {}):
            return entry["ops_per_texture"][kernel]
    return None


def reference_cpu(img_np, fmt, reps=3):
    """Best-of-reps wall time of the reference encoder on all host threads (viewer.cpp band scheme)."""
    import oracle_lib
    ref = oracle_lib.reference()
    if ref is None:
        return None
    threads = os.cpu_count() or 1
    best = float("inf")
    out = None
    for _ in range(reps):
        t0 = time.perf_counter()
        out = ref.bc_encode(img_np, fmt, threads=threads)
        best = min(best, time.perf_counter() - t0)
    return {"seconds": best, "threads": threads, "out": out}


def bind_to_gpu_local_cpus(dev):
    """Restrict this process to the CPUs NVML reports as local to the device (read-only queries); returns the
    previous CPU set to restore, or None when NVML or the affinity call is unavailable."""
    try:
        import pynvml
        import torch
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            n = os.cpu_count() or 1
            words = pynvml.nvmlDeviceGetCpuAffinity(h, (n + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * k + b for k, wd in enumerate(words) for b in range(64) if (int(wd) >> b) & 1}
        saved = os.sched_getaffinity(0)
        cpus &= saved
        if not cpus:
            return None
        os.sched_setaffinity(0, cpus)
        return saved
    except Exception:
        return None


def reference_cpu_1core(img_np, fmt, reps=3):
    """Best-of-reps wall time of one reference zap_bc_encode call on one thread (tex_bench.c:208-210)."""
    import oracle_lib
    ref = oracle_lib.reference()
    if ref is None:
        return None
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        ref.bc_encode(img_np, fmt)
        best = min(best, time.perf_counter() - t0)
    return best


def run_reference(args, world, rank):
    """--impl reference: the reference's own CPU encoder, all host threads, same workload and metric."""
    if rank != 0:
        return
    import oracle_lib
    import zap_b200.synth as S
    ref = oracle_lib.reference()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libzapref.so is not built (reference tree absent)"}))
        return
    img = S.colour_texture(W, H, seed=100, alpha="noise").numpy()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        ref.bc_encode(img, 4, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.bc_encode(img, 4, threads=threads)
    dt = time.perf_counter() - t0
    v = args.steps * W * H / 1e6 / dt
    # n_gpus: the N this arm was launched with (rank 0 alone runs it, on the host's cores)
    line = {"metric": METRIC, "value": v, "unit": "Mpix/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "parallelism": f"{threads} host threads, 8-block-row bands"},
            "cpu_baseline": {"value": v, "unit": "Mpix/s", "cores": threads, "kind": "reference",
                             "sample": f"full {W}x{H} texture per step, zap_bc_encode on bands (zap_tex.h at -O2)"},
            "e2e": {"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def time_device(fn, steps, warmup, world, lead_in_ms=0.0):
    """Device time of `steps` calls of fn (CUDA events on the current stream, synchronised on both sides). lead_in_ms:
    a fixed-length spin kernel queued just before the start event, so the host queues the timed work while the GPU
    runs it and the events bracket device work only (a host descheduled for a few ms inside a short timed region
    would otherwise leave the GPU idle inside it: one 20-step headline region read 0.254 ms per step against 0.114)."""
    import torch
    for k in range(warmup):
        fn(k)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if lead_in_ms > 0:
        torch.cuda._sleep(int(lead_in_ms * 2e6))  # about 2e6 cycles per ms at the B200's 1.97 GHz
    e0.record()
    for k in range(steps):
        fn(k)
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    return e0.elapsed_time(e1)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.profile:
        run_profile_case(args)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    import numpy as np
    import torch

    import zap_b200
    import zap_b200.synth as S
    dev = torch.device("cuda", torch.cuda.current_device())
    ring = 10  # 10 x 16 MB > 126 MB L2
    texs = [S.colour_texture(W, H, seed=100 + 1000 * rank + k, alpha="noise", device=dev) for k in range(ring)]
    outs = [torch.empty(zap_b200.bc_size(W, H, zap_b200.BC7), dtype=torch.uint8, device=dev) for _ in range(ring)]
    torch.cuda.synchronize()

    def step(k):
        zap_b200.bc_encode_dev(texs[k % ring], zap_b200.BC7, out=outs[k % ring])

    for k in range(max(3, args.warmup)):
        step(k)
    torch.cuda.synchronize()
    # The timed steps replay CUDA graphs of zap_tex_cuda_bc_encode_dev calls (scratch allocation, counter reset, both
    # kernels): the device work of a step without the host's per-call launch overhead, which on a slow host exceeds
    # the 0.12 ms of GPU work per 2048^2 encode. Whole passes over the ring replay one graph of the ring's 10 steps
    # (one launch per 1.2 ms of GPU work, so a host that stalls between launches does not starve the GPU); the
    # K % 10 steps left over replay one graph per ring slot. e2e keeps the host path.
    graphs = []
    for k in range(ring):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            step(k)
        graphs.append(g)
    ring_graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(ring_graph):
        for k in range(ring):
            step(k)

    def graph_steps(n):  # n consecutive steps from ring slot 0
        for _ in range(n // ring):
            ring_graph.replay()
        for k in range(n % ring):
            graphs[k].replay()

    with ClockSampler(local) as clocks:  # started (and sampling) before the warm-up, so it runs through the timed steps
        graph_steps(max(3, args.warmup))
        torch.cuda.synchronize()
        ms = time_device(lambda k: graph_steps(args.steps), 1, 0, world, lead_in_ms=3.0)
    # per-kernel figures from a second pass of the same steps with the library's event trace on (the trace's own
    # event records stay out of the timed pass above); its launch count is the timed pass's
    zap_b200.trace(True)
    time_device(step, args.steps, 0, world)
    rep = zap_b200.trace_report()
    zap_b200.trace(False)
    ms = max_over_ranks(ms, world)
    mpix = W * H / 1e6
    value = job_value(ms, world, args.steps, mpix)
    launches = sum(v[0] for v in rep.values())

    # dominant kernel roofline: 64 B of texels read + 16 B of block written per 4x4 block processed
    dom = max(rep.items(), key=lambda kv: kv[1][1])
    name, (n, tot_ms, units) = dom
    avg_ms = tot_ms / max(1, n)
    alg_bytes = units / max(1, n) * 80.0
    hbm, peak_kind = peaks()
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(name)
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "peak_source": peak_kind, "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "kernels": {k: {"launches": v[0], "ms": v[1], "units": v[2], "share": v[1] / sum(x[1] for x in rep.values())}
                            for k, v in rep.items()}}
    # the bound that binds: counted algorithmic ops against the SMs' measured issue rate (one launch = one 2048^2
    # texture). The probe runs after every timed workload of the run (its seconds of full load would otherwise warm
    # the GPU before them); the ALU fractions are filled in then.
    csum = clocks.summary()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = csum.get("sm_mhz") or csum.get("sm_max_mhz")

    def fill_alu(extra):
        measure_alu_peak(dev, sms, local)
        roofline["alu"] = alu_roofline(name, (ops_per_texture(name), avg_ms), mhz, sms)
        roofline["alu_kernels"] = {k: alu_roofline(k, (ops_per_texture(k), v[1] / max(1, v[0])), mhz, sms) for k, v in rep.items()}
        for entry in (extra or {}).values():
            counted, ms_enc = entry.pop("_alu_in", (None, None))
            if counted:  # the whole encode (all its kernels) against the ALU roofline
                entry["alu"] = alu_roofline(counted, (ops_per_texture(counted), ms_enc), mhz, sms)

    line = {"metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "l2": f"inputs larger than L2: ring of {ring} distinct {W}x{H} textures",
                       "parallelism": "independent replicas" if world > 1 else "1 gpu",
                       "step": "one zap_tex_cuda_bc_encode_dev call on the next ring texture; the K steps replay CUDA graphs "
                               "of 10 consecutive steps (one pass over the ring), the K % 10 left over one graph each"},
            "roofline": roofline, "gpu_launches": launches, "clocks": clocks.summary(), "library_md5": library_md5()}

    if rank == 0:
        # e2e: host C ABI, pinned host memory, copies inside the timed region. The buffers are allocated and the
        # calls timed on the CPUs local to the GPU (its NUMA node), as a host pipeline would be deployed; pinned
        # pages on the far socket would send every copy across the inter-socket link.
        saved_cpus = bind_to_gpu_local_cpus(dev)
        host_in = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)
        host_in.copy_(texs[0].cpu())
        host_out = torch.empty(zap_b200.bc_size(W, H, zap_b200.BC7), dtype=torch.uint8, pin_memory=True)
        hin, hout = host_in.numpy(), host_out.numpy()
        # the first calls of a run are measurably slower (host clocks and the link warm up, more so on CPUs just
        # bound to): at least 100 calls and one second of calls before timing
        t_warm, n_warm = time.perf_counter(), 0
        while n_warm < 100 or time.perf_counter() - t_warm < 1.0:
            zap_b200.bc_encode(hin, zap_b200.BC7, out=hout)
            n_warm += 1
        # each call is synchronous (copies in, encode, copies out); the steps run as 5 timed segments and the median
        # segment is reported, so a burst of host noise in one segment does not decide the figure
        seg = max(1, args.steps // 5)
        runs = []
        for _ in range(5):
            t0 = time.perf_counter()
            for _ in range(seg):
                zap_b200.bc_encode(hin, zap_b200.BC7, out=hout)
            runs.append((time.perf_counter() - t0) / seg)
        e2e_s = statistics.median(runs)
        line["e2e"] = {"value": mpix / e2e_s, "unit": "Mpix/s", "h2d_bytes_per_step": W * H * 4,
                       "d2h_bytes_per_step": int(hout.size), "api": "zap_tex_cuda_bc_encode (host pointers)",
                       "ms_per_call_segments": [r * 1e3 for r in runs], "timing": "median of 5 segments of wall-clock calls",
                       "host_cpus": "GPU-local (NVML CPU affinity)" if saved_cpus is not None else "unbound"}
        # the copies alone, the bound of a host-pointer call: the texture in and the blocks out over PCIe, pinned
        # buffers, one copy each on one stream (CUDA events), median of 20
        dtex = torch.empty((H, W, 4), dtype=torch.uint8, device=dev)
        dblk = torch.zeros(zap_b200.bc_size(W, H, zap_b200.BC7), dtype=torch.uint8, device=dev)
        scratch_out = torch.empty_like(host_out, pin_memory=True)  # host_out keeps the call's blocks for the parity check
        c0, c1, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        h2d, d2h = [], []
        for _ in range(23):
            c0.record()
            dtex.copy_(host_in, non_blocking=True)
            c1.record()
            scratch_out.copy_(dblk, non_blocking=True)
            c2.record()
            torch.cuda.synchronize()
            h2d.append(c0.elapsed_time(c1))
            d2h.append(c1.elapsed_time(c2))
        h2d_ms, d2h_ms = statistics.median(h2d[3:]), statistics.median(d2h[3:])
        line["e2e"]["copy_bound"] = {"h2d_ms": h2d_ms, "d2h_ms": d2h_ms, "h2d_GB_s": W * H * 4 / h2d_ms / 1e6,
                                     "d2h_GB_s": hout.size / d2h_ms / 1e6, "h2d_fraction_of_call": h2d_ms / (e2e_s * 1e3),
                                     "note": "the call overlaps its copies out with the copies in, so the texture's "
                                             "copy in alone bounds it"}
        del dtex, dblk, scratch_out
        if saved_cpus is not None:
            os.sched_setaffinity(0, saved_cpus)  # the CPU baseline below uses every host thread
        # reference CPU on the same texture; parity of the GPU output against it
        cpu = reference_cpu(hin, zap_b200.BC7, reps=2) if world == 1 else None
        if cpu is not None:
            line["cpu_baseline"] = {"value": mpix / cpu["seconds"], "unit": "Mpix/s", "cores": cpu["threads"], "kind": "reference",
                                    "sample": f"full {W}x{H} texture, best of 2, 8-block-row bands on all host threads"}
            one = reference_cpu_1core(hin, zap_b200.BC7)
            if one is not None:  # the reference self-test's own method (tex_bench.c:208-210): one call, best of 3
                line["cpu_baseline"]["one_core"] = {"value": mpix / one, "unit": "Mpix/s", "cores": 1,
                                                    "sample": f"full {W}x{H} texture, one zap_bc_encode call, best of 3"}
            same = np.mean(np.all(hout.reshape(-1, 16) == cpu["out"].reshape(-1, 16), axis=1))
            line["parity"] = {"identical_blocks": float(same)}
        if not args.no_extra:
            line["extra"] = extra_workloads(args, dev, mhz, sms)
            line["batched"] = batched_workload(args, dev)
            line["refine"] = refine_workload(args, dev)
            line["rdo"] = rdo_workload(dev)
            line["hbm_kernels"] = hbm_workloads(dev)
        fill_alu(line.get("extra"))
        line["alu_peak"] = ALU_PEAK
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def hbm_workloads(dev, side=4096, ring=4):
    """The HBM-bound kernels against the HBM roofline: one mip level of a side^2 RGBA8 texture (linear and sRGB
    averaging) and the BC1 / BC7 decoders of side^2 textures, over rings of `ring` distinct textures (256 MB of source
    texels, twice the L2). Algorithmic bytes: a mip level reads its source and writes a quarter of it; a decode reads
    the blocks and writes the texels. Timed like the secondary figures: one captured CUDA graph per segment of `ring`
    steps, queued behind a 3 ms spin kernel, median of five segments."""
    import torch

    import zap_b200
    import zap_b200.synth as S
    hbm, peak_kind = peaks()
    texs = [S.colour_texture(side, side, seed=60000 + k, alpha="noise", device=dev) for k in range(ring)]
    res = {"peak_GB_s": hbm, "peak_source": peak_kind, "texture": f"{side}x{side} RGBA8, ring of {ring}"}

    def measure(name, step, alg_bytes):
        for k in range(ring):  # every output allocated before the capture
            step(k)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for k in range(ring):
                step(k)
        per = sorted(time_device(lambda k: g.replay(), 1, 1, 1, lead_in_ms=3.0) / ring for _ in range(5))
        gbs = alg_bytes / (per[2] / 1e3) / 1e9
        res[name] = {"ms_per_step": per[2], "GB_s_algorithmic": gbs, "frac_of_peak": gbs / hbm, "alg_bytes_per_step": alg_bytes,
                     "segments_ms_per_step": per}
        del g

    half = side // 2
    for srgb in (0, 1):
        mips = [torch.empty((half, half, 4), dtype=torch.uint8, device=dev) for _ in range(ring)]
        measure("mip_next_srgb" if srgb else "mip_next_linear",
                lambda k, srgb=srgb, mips=mips: zap_b200.mip_next_dev(texs[k], srgb, out=mips[k]), side * side * 4 + half * half * 4)
        del mips
    for fmt, name, bs in ((zap_b200.BC1, "bc1_decode", 8), (zap_b200.BC7, "bc7_decode", 16)):
        blocks = [zap_b200.bc_encode_dev(t, fmt) for t in texs]
        outs = [None] * ring

        def dec(k, blocks=blocks, outs=outs, fmt=fmt):
            outs[k] = zap_b200.bc_decode_dev(blocks[k], side, side, fmt)
        measure(name, dec, (side // 4) * (side // 4) * bs + side * side * 4)
        del blocks, outs
    del texs
    torch.cuda.empty_cache()
    return res


def batched_workload(args, dev, n=4096):
    """Batched encode: n textures, power-of-two sides 64..2048 (log-uniform, aspect <= 4:1), full sRGB mip chains,
    40% BC1 / 20% BC3 / 40% BC7, opaque colour-texture content per texture seed. One autotuned graph launch per step against
    the same work as one plain launch per texture and per level (issued natively, no Python in the loop)."""
    import torch

    import zap_b200
    import zap_b200.synth as S
    sizes = S.batch_sizes(n, seed=0)
    fmts = S.batch_formats(n, seed=0)
    t0 = time.perf_counter()
    texs = [S.colour_texture(w, h, seed=10000 + k, device=dev) for k, (w, h) in enumerate(sizes)]
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b = zap_b200.Batch(texs, fmts, autotune=True)
    plan_s = time.perf_counter() - t0
    b.run()
    b.run()
    ms_graph = time_device(lambda k: b.run(), 3, 0, 1) / 3
    graph_out = [o.clone() for o in b.outputs]
    b.run_plain()
    ms_plain = time_device(lambda k: b.run_plain(), 2, 0, 1) / 2
    same = all(torch.equal(g, o) for g, o in zip(graph_out, b.outputs))
    mpix = b.pixels / 1e6
    res = {"textures": n, "pixels_incl_mips": b.pixels, "source_bytes": sum(t.numel() for t in texs),
           "mix": {"bc1": fmts.count(0), "bc3": fmts.count(1), "bc7": fmts.count(4)},
           "batched_graph": {"ms": ms_graph, "Mpix_s": mpix / (ms_graph / 1e3), "launches": 1},
           "plain_per_texture_per_level": {"ms": ms_plain, "Mpix_s": mpix / (ms_plain / 1e3),
                                           "launches": sum(2 * L - 1 for L in b.levels) + sum(1 for f in fmts if f == 4) *
                                           0},
           "speedup_batched_vs_plain": ms_plain / ms_graph, "identical_bytes": bool(same),
           "plan": b.info().strip().splitlines(), "generate_s": gen_s, "plan_s": plan_s}
    b.close()
    del texs, graph_out
    torch.cuda.empty_cache()
    return res


def rdo_workload(dev, lam=30.0):
    """Rate-distortion mode (rdo > 0): the reference's choice of each block depends on the 16 blocks chosen before
    it, so one call is one serial chain (one CTA on the device); callers that encode in 8-block-row bands get one
    chain per band. GPU: device API, CUDA events, inputs resident; the reference on one host core for the same call
    (its own code, oracle/_ref), and whether the bytes are identical."""
    import numpy as np
    import torch

    import zap_b200
    import zap_b200.synth as S
    import oracle_lib
    ref = oracle_lib.reference()
    res = {"lambda": lam}
    for name, side, fmt, band in (("bc1_512_one_call", 512, zap_b200.BC1, 0), ("bc7_512_one_call", 512, zap_b200.BC7, 0),
                                  ("bc1_2048_bands8", 2048, zap_b200.BC1, 8), ("bc7_2048_bands8", 2048, zap_b200.BC7, 8)):
        img = S.colour_texture(side, side, seed=300, alpha="noise").numpy()
        t = torch.from_numpy(img).to(dev)
        out = zap_b200.bc_encode_rdo_dev(t, fmt, lam, band_rows=band)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = zap_b200.bc_encode_rdo_dev(t, fmt, lam, band_rows=band, out=out)
        e1.record()
        torch.cuda.synchronize()
        r = {"gpu_ms": e0.elapsed_time(e1), "chains": 1 if not band else (side // 4 + band - 1) // band}
        if ref is not None and side <= 512:
            t0 = time.perf_counter()
            want = ref.bc_encode(img, fmt, rdo=lam)
            r["reference_1core_ms"] = (time.perf_counter() - t0) * 1e3
            r["identical"] = bool(np.array_equal(out.cpu().numpy(), want))
        res[name] = r
    return res


def bc7_modes(blocks):
    """Mode of every BC7 block (the lowest set bit of its first byte; 8 = reserved), as an int64 tensor."""
    import torch
    b0 = blocks.view(-1, 16)[:, 0].long()
    mode = torch.full_like(b0, 8)
    for m in range(7, -1, -1):
        mode = torch.where(((b0 >> m) & 1) == 1, torch.full_like(b0, m), mode)
    return mode


def refine_workload(args, dev, n=1024, side=256, steps=8, lr=1.0):
    """Refinement: n textures of side^2 (opaque colour-texture content, per-texture seed), BC1 and BC7; the encoder's blocks then
    `steps` Adam steps of gradient endpoint refinement through the palette-decode adjoint, accepted per block only
    if the error drops. Textures are stacked into one image: blocks are independent, so this is n encodes at once.
    BC7's gain is split by the blocks' mode (6, 5, 1); its cost is also timed on an atlas of 64x64 textures, where
    modes 5 and 1 are a third of the blocks instead of a few per cent."""
    import math

    import torch

    import zap_b200
    import zap_b200.synth as S
    tex = torch.cat([S.colour_texture(side, side, seed=20000 + k, device=dev) for k in range(n)], 0).contiguous()
    atlas = atlas_textures(2048, 64, 50000, dev, 1)[0]
    res = {"textures": n, "side": side, "adam_steps": steps, "lr": lr}
    psnr = lambda e, nval: 99.0 if e == 0 else 10 * math.log10(255.0 ** 2 * nval / e)  # noqa: E731
    for fmt, name, chans, img in ((zap_b200.BC1, "bc1", 3, tex), (zap_b200.BC7, "bc7", 4, tex),
                                  (zap_b200.BC7, "bc7_atlas_of_64x64", 4, atlas)):
        npix = img.shape[0] * img.shape[1]
        out = zap_b200.bc_encode_dev(img, fmt)
        base = out.clone()
        ms_enc = time_device(lambda k: zap_b200.bc_encode_dev(img, fmt, out=out), 5, 2, 1) / 5
        work = base.clone()

        def refine_step(k):
            work.copy_(base)
            zap_b200.refine_dev(img, fmt, work, steps=steps, lr=lr)
        ms_ref = time_device(refine_step, 5, 2, 1) / 5
        work.copy_(base)
        s0, s1 = zap_b200.refine_dev(img, fmt, work, steps=steps, lr=lr)
        torch.cuda.synchronize()
        e0, e1 = float(s0.double().sum()), float(s1.double().sum())
        nval = npix * chans
        r = {"pixels": npix, "encode_ms": ms_enc, "encode_Mpix_s": npix / 1e6 / (ms_enc / 1e3), "refine_ms": ms_ref,
             "refine_Mpix_s": npix / 1e6 / (ms_ref / 1e3), "psnr_db": psnr(e0, nval), "psnr_refined_db": psnr(e1, nval),
             "psnr_gain_db": psnr(e1, nval) - psnr(e0, nval), "blocks_improved": float((s1 < s0).float().mean()),
             "cost_vs_encode": ms_ref / ms_enc}
        if fmt == zap_b200.BC7:
            modes = bc7_modes(base)
            same_mode = bool(torch.equal(modes, bc7_modes(work)))
            by = {}
            for m in (6, 5, 1):
                sel = modes == m
                cnt = int(sel.sum())
                if not cnt:
                    continue
                a0, a1 = float(s0[sel].double().sum()), float(s1[sel].double().sum())
                by[f"mode{m}"] = {"blocks": cnt, "share": cnt / modes.numel(), "sse_before": a0, "sse_after": a1,
                                  "sse_reduction": (a0 - a1) / a0 if a0 else 0.0,
                                  "blocks_improved": float((s1[sel] < s0[sel]).float().mean()),
                                  "psnr_gain_db_over_these_blocks": psnr(a1, cnt * 16 * chans) - psnr(a0, cnt * 16 * chans)}
            r["by_mode"] = by
            r["modes_kept"] = same_mode
        res[name] = r
    del tex, atlas
    torch.cuda.empty_cache()
    return res


def atlas_textures(side, tile, seed, device, count):
    """`count` side x side texture atlases of the same (side / tile)^2 textures of the batch's recipe (colour_texture,
    one seed per tile), each in its own order (seeded 0 .. count - 1): small textures carry more detail per 4x4 block,
    so more BC7 blocks leave mode 6 than in one large texture of the same recipe."""
    import torch

    import zap_b200.synth as S
    n = side // tile
    tiles = torch.stack([S.colour_texture(tile, tile, seed=seed + k, device=device) for k in range(n * n)])
    out = []
    for k in range(count):
        perm = torch.randperm(n * n, generator=torch.Generator().manual_seed(k)).to(device)
        grid = tiles[perm].view(n, n, tile, tile, 4).permute(0, 2, 1, 3, 4).reshape(side, side, 4)
        out.append(grid.contiguous())
    return out


def log2_psnr(src, dec):
    """BC6H quality in log space: L(v) = log2(max(v, 2^-14)) per RGB channel, 10 log10(30^2 / mean squared
    difference); 99 when identical (the reference defines no HDR PSNR)."""
    import numpy as np
    a = np.log2(np.maximum(src[..., :3].astype(np.float64), 2.0 ** -14))
    b = np.log2(np.maximum(dec[..., :3].astype(np.float64), 2.0 ** -14))
    mse = float(np.mean((a - b) ** 2))
    return 99.0 if mse == 0 else 10 * np.log10(30.0 ** 2 / mse)


def extra_workloads(args, dev, sm_mhz=None, sms=148):
    """Secondary figures, one entry per format and input: BC1 (512^2 from seed 0, and 2048^2), BC4 R8 / BC5 RG8
    (2048^2), BC6H / ASTC (2048^2), and BC7 on content where many blocks go past mode 6 (opaque 2048^2, and an
    atlas of 64^2 textures). Each entry has, beside its device figure (CUDA events, inputs resident): the fraction of
    blocks identical to the reference encoder on the first ring texture, the PSNR of both outputs (as the reference's
    tex_bench.c:200-214 table prints it), and the reference's CPU figure on that texture, on all host threads
    (8-block-row bands) and on one core (one call, wall clock, tex_bench.c:205-208)."""
    import numpy as np
    import torch

    import oracle_lib
    import zap_b200
    import zap_b200.synth as S
    ref = oracle_lib.reference()
    threads = os.cpu_count() or 1
    res = {}
    steps = max(5, args.steps // 2)

    def widen(t, chans):  # narrow input -> the RGBA8 texels the reference reads (missing channels 0, alpha 255)
        host = t.cpu().numpy()
        if chans == 4:
            return host
        wide = np.zeros(host.shape[:2] + (4,), np.uint8)
        wide[..., :chans] = host
        wide[..., 3] = 255
        return wide

    def parity(t, got, fmt, chans):
        """identical blocks, PSNR of ours and of the reference, and the reference's CPU time on texture t"""
        if ref is None:
            return {"unavailable": "oracle/_ref/libzapref.so is not built"}
        h, w = t.shape[0], t.shape[1]
        if fmt == "bc6h":
            src = np.ones((h, w, 4), np.float32)
            src[..., :3] = t.cpu().numpy().astype(np.float32)
            run = lambda k: ref.bc6h_encode(src, threads=k)  # noqa: E731
            dec = lambda bc: ref.bc6h_decode(bc, w, h).view(np.float16).astype(np.float32)  # noqa: E731
            quality = lambda bc: log2_psnr(src, dec(bc))  # noqa: E731
        elif fmt == "astc":
            src = widen(t, chans)
            run = lambda k: ref.astc_encode(src, threads=k)  # noqa: E731
            quality = lambda bc: oracle_lib.psnr(src, ref.astc_decode(bc, w, h), 15)  # noqa: E731
        else:
            src = widen(t, chans)
            run = lambda k: ref.bc_encode(src, fmt, threads=k)  # noqa: E731
            quality = lambda bc: oracle_lib.psnr(src, ref.bc_decode(bc, w, h, fmt), oracle_lib.chmask(fmt))  # noqa: E731
        t0 = time.perf_counter()
        want = run(1)
        one = time.perf_counter() - t0
        best = float("inf")
        for _ in range(2):
            t0 = time.perf_counter()
            run(threads)
            best = min(best, time.perf_counter() - t0)
        mine = got.cpu().numpy()
        bs = 8 if fmt in (oracle_lib.BC1, oracle_lib.BC4) else 16
        same = float(np.mean(np.all(mine.reshape(-1, bs) == want.reshape(-1, bs), axis=1)))
        mpix = w * h / 1e6
        return {"identical_blocks": same, "psnr_db": quality(mine), "psnr_reference_db": quality(want),
                "psnr_kind": "log2 RGB, 30 dB span" if fmt == "bc6h" else "tex_bench.c:17-22",
                "cpu_baseline": {"value": mpix / best, "unit": "Mpix/s", "cores": threads, "kind": "reference",
                                 "sample": f"first ring texture ({w}x{h}), best of 2, 8-block-row bands on all host threads",
                                 "one_core": {"value": mpix / one, "unit": "Mpix/s", "cores": 1,
                                              "sample": "same texture, one call, wall clock (tex_bench.c:205-208)"}}}

    def bench(name, make, fmt, npix, ring, alg_bytes_per_px, chans=4, enc=None, counted=None):
        texs = [make(k) for k in range(ring)]
        outs = [None] * ring
        f = enc or (lambda t, o: zap_b200.bc_encode_dev(t, fmt, out=o))

        def step(k):
            outs[k % ring] = f(texs[k % ring], outs[k % ring])
        for k in range(ring):  # allocates every output before the timed region
            step(k)
        # A segment is `seg` consecutive encodes over the ring, captured once as a CUDA graph, so a timed segment is
        # one launch queued behind a 3 ms spin kernel and the events bracket device work: encodes issued one by one
        # left the GPU idle whenever the host stalled (one run's ASTC segments read 0.24 to 2.6 ms per encode). The
        # median of five segments, each after one untimed replay (a segment that starts on an idle GPU carries its
        # ramp-up).
        seg = max(20, steps // 5)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for k in range(seg):
                step(k)
        with ClockSampler(torch.cuda.current_device()) as clk:
            per = sorted(time_device(lambda k: graph.replay(), 1, 1, 1, lead_in_ms=3.0) / seg for _ in range(5))
        ms = per[2] * steps
        mps = steps * npix / 1e6 / (ms / 1e3)
        res[name] = {"Mpix_s": mps, "ms_per_encode": ms / steps, "GB_s_algorithmic": mps * 1e6 * alg_bytes_per_px / 1e9,
                     "timing": "median of 5 segments of %d encodes (one CUDA graph over the ring, replayed once untimed "
                               "before each timed replay; CUDA events, the replay queued behind a 3 ms spin kernel)" % seg,
                     "segments_ms_per_encode": per, "clocks": clk.summary()}
        del graph
        if counted:  # the whole encode against the ALU roofline, once the peak is measured (main's fill_alu)
            res[name]["_alu_in"] = (counted, ms / steps)
        torch.cuda.synchronize()
        res[name].update(parity(texs[0], outs[0], fmt, chans))
        cpu = res[name].get("cpu_baseline")
        if cpu:
            res[name]["speedup_vs_cpu_all_threads"] = mps / cpu["value"]
        del texs, outs

    bench("bc1_512x512_seed0", lambda k: S.colour_texture(512, 512, seed=k, device=dev), zap_b200.BC1, 512 * 512, 64, 4.5)
    bench("bc1_2048x2048", lambda k: S.colour_texture(2048, 2048, seed=k, device=dev), zap_b200.BC1, 2048 * 2048, 10, 4.5,
          counted="bc1_encode")
    bench("bc4_2048x2048_r8", lambda k: S.colour_texture(2048, 2048, seed=k, device=dev)[..., :1].contiguous(), zap_b200.BC4,
          2048 * 2048, 40, 1.5, chans=1, counted="bc4_encode")
    bench("bc5_2048x2048_rg8", lambda k: S.normal_map(2048, 2048, seed=k, device=dev), zap_b200.BC5, 2048 * 2048, 20, 3.0,
          chans=2, counted="bc5_encode")
    bench("astc4x4_2048x2048", lambda k: S.colour_texture(2048, 2048, seed=k, alpha="noise", device=dev), "astc",
          2048 * 2048, 10, 5.0, enc=lambda t, o: zap_b200.astc_encode_dev(t, out=o), counted="astc_encode")
    bench("bc6h_2048x2048_rgb16f", lambda k: S.hdr_texture(2048, 2048, seed=k, device=dev), "bc6h", 2048 * 2048, 6, 7.0,
          chans=3, enc=lambda t, o: zap_b200.bc6h_encode_dev(t, out=o), counted="bc6h_encode")
    bench("bc7_2048x2048_opaque", lambda k: S.colour_texture(2048, 2048, seed=k, device=dev), zap_b200.BC7, 2048 * 2048, 10, 5.0)
    atlases = atlas_textures(2048, 64, 40000, dev, 10)
    bench("bc7_2048x2048_atlas_of_64x64", lambda k: atlases[k], zap_b200.BC7, 2048 * 2048, 10, 5.0)
    del atlases
    torch.cuda.empty_cache()
    return res


if __name__ == "__main__":
    main()
