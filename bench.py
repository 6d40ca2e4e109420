#!/usr/bin/env python
"""Stroke-field benchmark: forward + backward stroke x sample evaluations per second.

One step = one forward + adjoint backward of the fused stroke field over every scene
of the workload (all rays, all strokes), captured once into a CUDA graph and
replayed; inputs are resident in HBM. Upstream gradients are N(0, 1) on rgb,
opacity and depth. An "eval" is one (stroke, sample) pair of the nominal dense
product S x P per scene, the same count whatever culling skips.

Default workload: 16 uneven scenes (strokes log-uniform in [50, 2000], rays
log-uniform in [4096, 65536], 64 samples each, six primitive types mixed) in one
batched launch per pass + CUDA graph. Other workloads: --config 0..4.

Second workload (--workload grid): the multi-resolution hash-grid encoder alone at
the MLP class defaults (10 levels x 4 channels, 2^21 rows per fine level, 240 MB of
float32 table) over 65,536 rays x 64 samples; one step = zero the table gradient,
forward, table backward; value in (point, level) lookups per second; the reference's
own kernels, built from its sources, are timed beside it when present.

Third (--workload prop): the proposal and error fields' density networks of one
training step (PropMLP at 512 and 2048, ErrorMLP at 256; 2^14 rays x 64 samples
each): warp, grid encoding, Linear-ReLU-Linear, softplus, hash decay statistics and
their backward, fused (tensor cores for the layers); value in points per second; the
reference's formulation (its grid kernels + torch layers + autograd) timed beside it.

Fourth (--workload ops): every other operator once at a stated size through its
public API (the drop-in _strokelib operators, the composition modes, a colour field,
the texture, proposal resampling, stroke insertion, the field at a tenth of config 3
and its Adam step), timed with CUDA events; it is the command the all-kernels ncu
summary runs.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--config C] [--impl reference]
  python bench.py --workload grid|prop [--steps K] [--warmup W] [--impl reference]
  python bench.py --workload ops [--steps K] [--warmup W]
Multi-GPU (torchrun): every rank runs the same workload on its own GPU (replicas, no
data-path collective); the value is the sum over ranks of evals divided by the
slowest rank's time.
"""
import argparse
import glob
import json
import math
import os
import statistics
import subprocess
import sys
import time

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd stroke×sample evals/s on 1 B200: batched+graph vs plain op @≤1e-4 rel"
UNIT = "evals/s"

# Algorithmic FP32 flops per evaluated (sample, stroke) pair, forward: inverse
# transform + SDF + 15 (soft step 4 + over-composite 11); transforms without rotation
# (sphere, aacube, aabb) are 6, the curves have none; a per-axis scale under
# inv_scale_radius adds 10 for the radius factor. Backward = 2.5 x forward per pair
# it evaluates (recompute, adjoint of each step, reduction share); it evaluates only
# the strokes the forward's block masks keep, counted on the device. Capped torus,
# line and triangular prism counted the same way from their SDFs (16, 17, 10).
FWD_FLOPS_BY_KIND = {
    "sphere": 6 + 6 + 15, "ellipsoid": 21 + 6 + 10 + 15, "aacube": 6 + 14 + 15, "cube": 21 + 14 + 15,
    "aabb": 6 + 14 + 10 + 15, "obb": 21 + 14 + 10 + 15, "roundcube": 21 + 16 + 15, "roundbox": 21 + 16 + 10 + 15,
    "cappedtorus": 21 + 16 + 15, "capsule": 21 + 9 + 15, "scapsule": 21 + 9 + 10 + 15, "line": 21 + 17 + 15,
    "triprism": 21 + 10 + 15, "octahedron": 21 + 6 + 15, "tetrahedron": 21 + 8 + 15,
    "quadratic_bezier": 75 + 15, "cubic_bezier": 190 + 15, "catmull_rom": 190 + 15,
}
BWD_FACTOR = 2.5
# DRAM bytes per step of the backward segment kernel on the batched uneven-scene
# workload (config 3), from one ncu capture at a quarter of its rays (all passes of
# one step, dram__bytes_read.sum + dram__bytes_write.sum; launch-list summary in
# profiles/launches_cfg3_quarter.md); traffic grows with the ray count.
SEG_BWD_TRAFFIC_CFG3_QUARTER = 576.0e6
KIND_BASE = {"sphere": 0, "ellipsoid": 0, "aacube": 1, "cube": 1, "aabb": 1, "obb": 1, "roundcube": 2,
             "roundbox": 2, "cappedtorus": 3, "capsule": 4, "scapsule": 4, "line": 5, "triprism": 6,
             "octahedron": 7, "tetrahedron": 8, "quadratic_bezier": 9, "cubic_bezier": 10, "catmull_rom": 11}
CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def base_flops(kinds):
    """Forward flops per evaluated pair for each base SDF index, weighted by the
    workload's stroke mix (sphere and ellipsoid share base 0)."""
    acc, cnt = {}, {}
    for k in kinds:
        b = KIND_BASE[k]
        acc[b] = acc.get(b, 0.0) + FWD_FLOPS_BY_KIND[k]
        cnt[b] = cnt.get(b, 0) + 1
    return {b: acc[b] / cnt[b] for b in acc}


class ClockSampler:
    """nvidia-smi sampling (every 50 ms) of SM clocks and throttle reasons. A reader
    thread stamps each line with the host clock; ``stop(lo, hi)`` keeps the samples
    stamped inside [lo, hi], the host times around the timed region (the GPU is busy
    from just after ``lo`` until the synchronisation that precedes ``hi``)."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={CLOCK_FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def read():
            for line in self.proc.stdout:
                self.lines.append((time.monotonic(), line))
        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()
        t_end = time.monotonic() + 3.0  # sampling is live before the timed region starts
        while not self.lines and time.monotonic() < t_end and self.proc.poll() is None:
            time.sleep(0.01)

    def stop(self, lo=None, hi=None):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        stamped = list(self.lines)
        inside = [l for t, l in stamped if (lo is None or t >= lo) and (hi is None or t <= hi)]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in inside:
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "note": "no nvidia-smi sample fell inside the timed region"}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(v, world, device):
    if world == 1:
        return v
    t = torch.tensor([float(v)], device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(local_step_s, pairs_per_rank, world, device):
    """Whole-job evals/s of N replicas: every rank processes pairs_per_rank per step;
    the job's step time is the slowest rank's. Returns (value, max step seconds)."""
    step = max_over_ranks(local_step_s, world, device)
    return pairs_per_rank * world / step, step


def workload_upstream(field, seed=7):
    g = torch.Generator().manual_seed(seed)
    R = field.rgb.shape[0]
    return (torch.randn(R, 3, generator=g), torch.randn(R, generator=g), torch.randn(R, generator=g))


def fp32_peak(device, repeats=8):
    """Measured FP32 FMA throughput (TFLOP/s) of this GPU with the library's probe."""
    from neural3dstrokes_b200 import _lib
    lib = _lib.load()
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    blocks, iters = sms * 8, 8192
    out = torch.empty(blocks * 256, device=device)
    best = 0.0
    for _ in range(repeats + 2):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        _lib.check(lib.n3ds_fp32_probe(_lib.ptr(out), blocks, iters, _lib.stream_ptr(device)))
        e.record()
        e.synchronize()
        best = max(best, blocks * 256.0 * iters * 32 / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


# The CPU legs (this arm's cpu_baseline and the reference arm) time the same fixed
# sample of each workload: these evenly spaced rays of every scene (first and last
# included), with every stroke of the scene, and fixed N(0,1) upstream gradients.
CPU_SAMPLE_RAYS = {0: 512, 1: 64, 2: 16, 3: 24, 4: 8}


def cpu_sample(workload, cfg):
    """The fixed CPU sample of a workload: per scene (scene, rays subset, upstream
    gradients), and its nominal pairs."""
    from oracle.accuracy import ray_subset, take_rays
    k = CPU_SAMPLE_RAYS.get(cfg, 16)
    g = torch.Generator().manual_seed(11)
    items, pairs = [], 0
    for sc, rays in zip(workload.scenes, workload.rays):
        idx = ray_subset(rays.n_rays, k)
        sub = take_rays(rays, idx)
        n = idx.numel()
        gr = (torch.randn(n, 3, generator=g), torch.randn(n, generator=g), torch.randn(n, generator=g))
        items.append((sc, sub, gr))
        pairs += sc.n_strokes * n * rays.n_samples
    desc = (f"{k} evenly spaced rays of each scene ({pairs} nominal pairs per pass, every stroke): float32 "
            f"torch restatement of the reference strokelib kernels + render.py, forward + backward")
    return items, pairs, desc


def cpu_pass(workload, items):
    from oracle import cpu_port
    for sc, sub, gr in items:
        cpu_port.port_step(sc, sub.x, sub.radius, sub.tdist, sub.dirs, *gr, delta=workload.sdf_delta,
                           laplace=workload.use_laplace, inv=workload.inv_scale_radius)


def cpu_baseline(workload, cfg, budget_s=15.0):
    """The labelled float32 CPU port of the reference step (oracle/cpu_port.py) on the
    fixed ray sample of the workload, all host threads, repeated for about budget_s."""
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    items, pairs, desc = cpu_sample(workload, cfg)
    cpu_pass(workload, items)  # warm-up
    reps, t0 = 0, time.perf_counter()
    while True:
        cpu_pass(workload, items)
        reps += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": pairs * reps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{desc}; {reps} passes in {dt:.1f} s"}


def run_reference(args, world, rank):
    """Reference arm: the reference implementation of the path timed on the host cores
    (its kernels are CUDA-only, so its CPU form is the labelled float32 port), plus,
    as an extra field, the unmodified reference CUDA op on this GPU."""
    if rank != 0:
        return
    from neural3dstrokes_b200 import scenes
    w = scenes.config(args.config)
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    # one step = one pass over the same fixed ray sample as this arm's cpu_baseline leg
    items, pairs, desc = cpu_sample(w, args.config)
    rates = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cpu_pass(w, items)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            rates.append(pairs / dt)
    value = statistics.mean(rates)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": w.name, "nominal_pairs_per_full_step": w.nominal_pairs},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"one step = one pass over {desc}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if torch.cuda.is_available() and not args.no_plain_op:
        try:
            line["plain_op_gpu"] = plain_op_gpu(w, args)
        except Exception as e:  # the extra field must not sink the arm
            line["plain_op_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    print(json.dumps(line), flush=True)


def plain_op_gpu(w, args, max_seconds=60.0):
    """The unmodified reference CUDA op (oracle/_ref) driven as models.py drives it,
    one scene at a time, over the whole workload; CUDA events."""
    from oracle import cpu_port
    ref = cpu_port.reference_extension()
    if ref is None:
        return {"unavailable": "reference extension not built (oracle/_ref)"}
    dev = torch.device("cuda")
    g = torch.Generator().manual_seed(7)
    data = []
    for sc, rays in zip(w.scenes, w.rays):
        R = rays.n_rays
        data.append((sc.to(dev), rays.to(dev), torch.randn(R, 3, generator=g).to(dev),
                     torch.randn(R, generator=g).to(dev), torch.randn(R, generator=g).to(dev)))

    def step():
        for sc, rays, a, b, c in data:
            cpu_port.plain_op_step(ref, sc, rays.x, rays.radius, rays.tdist, rays.dirs, a, b, c, w.sdf_delta,
                                   w.use_laplace, w.inv_scale_radius)
    step()  # warm-up
    torch.cuda.synchronize()
    times = []
    t_start = time.perf_counter()
    while len(times) < 3 and (time.perf_counter() - t_start) < max_seconds:
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        step()
        e.record()
        e.synchronize()
        times.append(s.elapsed_time(e) * 1e-3)
    t = statistics.median(times)
    return {"value": w.nominal_pairs / t, "unit": UNIT, "ms_per_step": t * 1e3, "steps": len(times),
            "note": "reference _strokelib built from its own sources for sm_100a, per scene, per primitive "
                    "group, ray-chunked (P_chunk*S < 2^29), torch autograd for render.py, grad_x requested"}


# evenly spaced rays per scene that the float64 oracle checks in the accuracy leg
ACCURACY_RAYS = {0: 128, 1: 64, 2: 16, 3: 16, 4: 6}


def accuracy_leg(field, w, args):
    """Every output and gradient of the benchmarked field against the float64 oracle
    and the reference op (oracle/accuracy.py), untimed; errors are normwise relative,
    worst scene."""
    from oracle import accuracy, cpu_port
    torch.set_num_threads(os.cpu_count() or 1)
    ref = cpu_port.reference_extension()
    t0 = time.perf_counter()
    w = accuracy.workload_from_field(field, w)  # the parameters as the timed (training) steps left them
    out = accuracy.subset_accuracy(field, w, ACCURACY_RAYS.get(args.config, 16), ref=ref)
    if args.config == 3 and ref is not None and args.scale == 1.0:
        out["vs_16_sequential_plain_op_calls"] = accuracy.plain_op_compare(field, w, ref)
    if args.config == 2:
        out["fd_slice"] = accuracy.fd_slice(w.scenes[0], w.rays[0], 32, 8, device=field.device)
    out["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def loss_curves(args):
    """Config 4's training comparison: the graphed step (forward, MSE, exact or compat
    adjoint, Adam + clamp in one CUDA graph) against the reference op trained as the
    reference trains (plain_op_train), K steps each from the same parameters."""
    from neural3dstrokes_b200 import scenes
    from neural3dstrokes_b200.field import FieldOptions
    from neural3dstrokes_b200.train import BatchedField, GraphedTrainer
    from oracle import cpu_port
    dev = torch.device("cuda", 0)
    exclude = tuple(k for k in args.exclude_kinds.split(",") if k)
    w = scenes.config(4, scale=args.scale, exclude=exclude)
    ref = cpu_port.reference_extension()
    grad_mode = "compat"
    tf = BatchedField(w.target_scenes, w.rays, w.sdf_delta, w.use_laplace, w.inv_scale_radius, device=dev,
                      need_grad_x=False)
    tf.forward()
    target = tf.rgb.clone()
    del tf
    field = BatchedField(w.scenes, w.rays, w.sdf_delta, w.use_laplace, w.inv_scale_radius,
                         options=FieldOptions(grad_mode=grad_mode, cull_alpha=args.cull_alpha), device=dev,
                         need_grad_x=False)
    trainer = GraphedTrainer(field, target, lr=1e-3)
    ours = []
    t0 = time.time()
    for _ in range(args.loss_curve):
        trainer.step()
        ours.append(float(trainer.loss))
    t_ours = time.time() - t0
    line = {"mode": "loss_curve", "config": w.name, "excluded_kinds": list(exclude), "scale": args.scale,
            "steps": args.loss_curve,
            "grad_mode": grad_mode, "cull_alpha": args.cull_alpha, "ours": ours, "ours_s": t_ours}
    if ref is None:
        line["plain_op"] = "unavailable: oracle/_ref holds no reference extension"
    else:
        n0 = 0
        targets = []
        for r in w.rays:
            targets.append(target[n0:n0 + r.n_rays])
            n0 += r.n_rays
        ranges = []
        for sc in w.scenes:
            lo, hi = zip(*[scenes.param_ranges(k) for k in sc.kinds])
            ranges.append((torch.tensor(lo, device=dev), torch.tensor(hi, device=dev)))
        t0 = time.time()
        theirs, _ = cpu_port.plain_op_train(ref, [s.to(dev) for s in w.scenes], [r.to(dev) for r in w.rays],
                                            targets, args.loss_curve, lr=1e-3, delta=w.sdf_delta,
                                            laplace=w.use_laplace, inv=w.inv_scale_radius, ranges=ranges)
        line["plain_op"] = theirs
        line["plain_op_s"] = time.time() - t0
        line["max_rel_diff"] = max(abs(a - b) / max(abs(b), 1e-30) for a, b in zip(ours, theirs))
        if args.ref_twice:
            # the reference op trained again from the same start: its own run-to-run
            # spread (its gradients are sums of float atomics in varying order, and
            # Adam with eps 1e-15 turns a gradient's sign into a full lr step)
            again, _ = cpu_port.plain_op_train(ref, [s.to(dev) for s in w.scenes], [r.to(dev) for r in w.rays],
                                               targets, args.loss_curve, lr=1e-3, delta=w.sdf_delta,
                                               laplace=w.use_laplace, inv=w.inv_scale_radius, ranges=ranges)
            line["plain_op_again"] = again
            line["plain_op_vs_itself_max_rel_diff"] = max(abs(a - b) / max(abs(b), 1e-30)
                                                          for a, b in zip(again, theirs))
    print(json.dumps(line), flush=True)
    if args.curve_out:
        with open(args.curve_out, "w") as f:
            json.dump(line, f)


GRID_METRIC = ("grid-encoder fwd+bwd (point, level) lookups/s on 1 B200: hash grid of the MLP class "
               "defaults (10 levels x 4 ch, 2^21 rows/level)")
GRID_UNIT = "lookups/s"


def grid_workload(dev, scale=1.0, seed=0):
    """The largest grid the reference defines, the MLP class defaults (models.py:305-333:
    10 levels, 4 channels, base 16, finest 8192, 2^21 rows; NerfMLP's; PropMLP and
    ErrorMLP narrow it, see --workload prop) and 65,536 x scale rays of 64 samples
    inside the unit cube, points ordered along each ray as the proposal sampler emits
    them."""
    from neural3dstrokes_b200 import gridencoder as ge
    enc = ge.GridEncoder(input_dim=3, num_levels=10, level_dim=4, base_resolution=16, desired_resolution=8192,
                         log2_hashmap_size=21).to(dev)
    g = torch.Generator(device=dev).manual_seed(seed)
    with torch.no_grad():
        enc.embeddings.uniform_(-1, 1, generator=g)
    R, N = max(1, int(65536 * scale)), 64
    o = torch.rand(R, 1, 3, device=dev, generator=g) * 0.5 + 0.25
    d = torch.nn.functional.normalize(torch.randn(R, 1, 3, device=dev, generator=g), dim=-1)
    t = torch.linspace(-0.25, 0.25, N, device=dev)[None, :, None]
    x = (o + d * t).clamp(0, 1).reshape(R * N, 3).contiguous()
    grad = torch.randn(enc.num_levels, R * N, 4, device=dev, generator=g)
    return enc, x, grad


def grid_reference_module():
    """The reference's grid encoder extension built from its sources (oracle/_ref/grid),
    or None."""
    import glob
    import importlib.machinery
    import importlib.util
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "grid", "_gridencoder*.so"))
    if not hits:
        return None
    loader = importlib.machinery.ExtensionFileLoader("_gridencoder", hits[0])
    spec = importlib.util.spec_from_file_location("_gridencoder", hits[0], loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def grid_step_fn(mod, enc, x, grad, out, gemb):
    import numpy as np
    B, L, C = x.shape[0], enc.num_levels, 4
    S, H = float(np.log2(enc.per_level_scale)), enc.base_resolution
    E, offs = enc.embeddings.data, enc.offsets

    def step():
        gemb.zero_()
        mod.grid_encode_forward(x, E, offs, out, B, 3, C, L, S, H, None, 0, False, 0)
        mod.grid_encode_backward(grad, x, E, offs, gemb, B, 3, C, L, S, H, None, None, 0, False, 0)
    return step


def grid_cpu_baseline(enc, x, grad, budget_s=15.0):
    """The oracle's forward + table backward (float64, torch on all host threads) on a
    bounded sample of the points, in lookups/s."""
    import numpy as np
    from oracle import gridencoder as og
    table = enc.embeddings.detach().double().cpu()
    offs = enc.offsets.cpu()
    S, H = float(np.log2(enc.per_level_scale)), enc.base_resolution
    n = 4096
    xs, gs = x[:n].cpu(), grad[:, :n].cpu()
    done, t0 = 0, time.perf_counter()
    while True:
        og.grid_encode_forward(xs, table, offs, S, H)
        og.grid_encode_backward(gs, xs, table, offs, S, H)
        done += n
        if time.perf_counter() - t0 > budget_s / 3:
            break
    dt = time.perf_counter() - t0
    return {"value": done * enc.num_levels / dt, "unit": GRID_UNIT, "cores": torch.get_num_threads(), "kind": "port",
            "sample": f"the first {n} points, repeated {done // n}x (oracle float64, torch on the host threads)"}


def run_grid(args, world, rank, local):
    from neural3dstrokes_b200.train import capture
    dev = torch.device("cuda", local)
    enc, x, grad = grid_workload(dev, args.scale)
    B, L, C = x.shape[0], enc.num_levels, 4
    lookups = B * L
    out = torch.empty(L, B, C, device=dev)
    gemb = torch.zeros_like(enc.embeddings.data)
    if args.impl == "reference":
        ref = grid_reference_module()
        if ref is None:
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "reference grid encoder not built "
                                  "(python oracle/build_ref.py --only grid)"}), flush=True)
            return
        step = grid_step_fn(ref, enc, x, grad, out, gemb)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lo = time.monotonic()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize(dev)
        clk = clocks.stop(lo, time.monotonic())
        t = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / args.steps, world, dev)
        if rank == 0:
            print(json.dumps({"impl": "reference", "metric": GRID_METRIC, "value": lookups * world / t,
                              "unit": GRID_UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
                              "dtype": "f32", "data": "synthetic", "clocks": clk,
                              "config": {"workload": "MLP-default hash grid", "points": B, "levels": L},
                              "note": "the reference's grid_encode_forward / grid_encode_backward kernels built "
                                      "from its sources for sm_100a, eager on the default stream"}), flush=True)
        return

    from neural3dstrokes_b200 import gridencoder as ge
    step = grid_step_fn(ge, enc, x, grad, out, gemb)
    step()  # offsets checked once (one host read) before capture
    graph = capture(step, dev, warmup=1)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lo = time.monotonic()
    e0.record()
    for _ in range(args.steps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize(dev)
    clk = clocks.stop(lo, time.monotonic())
    t_step = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / args.steps, world, dev)

    # per-kernel durations (events on the launching stream) for the roofline
    import numpy as np
    S, H = float(np.log2(enc.per_level_scale)), enc.base_resolution
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    tf, tb = [], []
    for _ in range(5):
        gemb.zero_()
        ev[0].record()
        ge.grid_encode_forward(x, enc.embeddings.data, enc.offsets, out, B, 3, C, L, S, H)
        ev[1].record()
        ge.grid_encode_backward(grad, x, enc.embeddings.data, enc.offsets, gemb, B, 3, C, L, S, H)
        ev[2].record()
        torch.cuda.synchronize(dev)
        tf.append(ev[0].elapsed_time(ev[1]) * 1e-3)
        tb.append(ev[1].elapsed_time(ev[2]) * 1e-3)
    t_fwd, t_bwd = statistics.mean(tf), statistics.mean(tb)
    table_bytes = enc.embeddings.numel() * 4
    # algorithmic bytes: points (12 B) and output rows (16 B per level) once, the
    # table once (forward); points, upstream rows and a read + write of the gradient
    # table (backward)
    fwd_bytes = B * 12 + L * B * C * 4 + table_bytes
    bwd_bytes = B * 12 + L * B * C * 4 + 2 * table_bytes
    peak, src = hbm_peak()
    roofline = {"bound": "hbm", "kernel": "grid_bwd_kernel (table scatter)", "achieved": bwd_bytes / t_bwd / 1e9,
                "peak": peak, "unit": "GB/s", "frac": bwd_bytes / t_bwd / 1e9 / peak, "traffic": None,
                "peak_source": src, "bytes_per_launch": bwd_bytes, "launch_ms": t_bwd * 1e3,
                "forward_kernel": {"name": "grid_fwd_kernel", "achieved": fwd_bytes / t_fwd / 1e9,
                                   "launch_ms": t_fwd * 1e3, "frac": fwd_bytes / t_fwd / 1e9 / peak}}

    # plain op: the reference's kernels on the same GPU, eager (they launch on the
    # legacy default stream, which a graph cannot capture)
    plain = None
    ref = grid_reference_module()
    if ref is not None:
        rstep = grid_step_fn(ref, enc, x, grad, out, gemb)
        for _ in range(2):
            rstep()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(args.steps):
            rstep()
        e1.record()
        torch.cuda.synchronize(dev)
        tr = e0.elapsed_time(e1) * 1e-3 / args.steps
        plain = {"value": lookups / tr, "unit": GRID_UNIT, "ms_per_step": tr * 1e3,
                 "speedup": tr / t_step, "what": "the reference's CUDA kernels built from its sources, eager"}

    # end to end: points uploaded from pinned host memory, the step, the table
    # gradient read back, every step
    e2e = None
    if not args.no_e2e:
        hx = x.cpu().pin_memory()
        hg = torch.empty(gemb.shape, dtype=gemb.dtype, pin_memory=True)
        n = max(3, min(args.steps, 10))
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(n):
            x.copy_(hx, non_blocking=True)
            graph.replay()
            hg.copy_(gemb, non_blocking=True)
        e1.record()
        torch.cuda.synchronize(dev)
        te = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / n, world, dev)
        e2e = {"value": lookups * world / te, "unit": GRID_UNIT, "ms_per_step": te * 1e3,
               "h2d_bytes_per_step": hx.numel() * 4, "d2h_bytes_per_step": hg.numel() * 4}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = grid_cpu_baseline(enc, x, grad, args.cpu_seconds)
    if rank == 0:
        print(json.dumps({
            "metric": GRID_METRIC, "value": lookups * world / t_step, "unit": GRID_UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded rays in the unit cube)",
            "config": {"workload": "MLP-default hash grid, 65,536 rays x 64 samples" if args.scale == 1.0 else
                       f"MLP-default hash grid, {B // 64} rays x 64 samples", "points": B, "levels": L, "channels": C,
                       "table_mb": table_bytes / 1e6, "l2": "inputs larger than L2 (outputs %.0f MB, table %.0f MB)"
                       % (L * B * C * 4 / 1e6, table_bytes / 1e6),
                       "graph": "zero + forward + backward captured in one CUDA graph"},
            "roofline": roofline, "plain_op": plain, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": 3 * args.steps, "gpu_launches_per_step": 3}), flush=True)


PROP_METRIC = ("proposal-side density networks fwd+bwd points/s on 1 B200: PropMLP (512) + PropMLP (2048) + "
               "ErrorMLP (256) of one training step, 2^14 rays x 64 samples each")
PROP_UNIT = "points/s"


def prop_workload(dev, scale=1.0, seed=0):
    """The networks one training step runs before the stroke level, at the reference's
    defaults: Model.num_prop_samples = 64 on two proposal levels whose grids reach
    desired resolutions 512 and 2048 (models.py:56-58, 73, 86-96; 6 and 8 levels x 1
    channel), and the error field (256: 5 levels x 2 channels) on the first level's
    samples (models.py:247-249), over Config.batch_size = 2^14 rays (configs.py:30),
    scaled by `scale`. The blender config's coordinate map (configs/blender.gin:44-45:
    warp_fn None, bbox_size 3). Synthetic rays from a sphere of radius 4 towards the
    origin, samples in t [2, 6] in ray order; reference initialisation; upstream
    density gradients N(0, 1)."""
    import torch.nn.functional as F
    from neural3dstrokes_b200 import mlp
    torch.manual_seed(seed)
    nets = [mlp.PropMLP(grid_disired_resolution=512, warp_fn=None, bbox_size=3.0),
            mlp.PropMLP(grid_disired_resolution=2048, warp_fn=None, bbox_size=3.0),
            mlp.ErrorMLP(grid_disired_resolution=256, disable_rgb=True, warp_fn=None, bbox_size=3.0)]
    nets = [n.to(dev).train() for n in nets]
    R, N = max(1, int(16384 * scale)), 64
    g = torch.Generator(device=dev).manual_seed(seed)
    xs = []
    for _ in range(2):
        o = F.normalize(torch.randn(R, 3, device=dev, generator=g), dim=-1) * 4.0
        d = F.normalize(-o + 0.5 * torch.randn(R, 3, device=dev, generator=g), dim=-1)
        t = torch.sort(torch.rand(R, N, device=dev, generator=g) * 4 + 2, dim=-1).values
        xs.append((o[:, None] + d[:, None] * t[..., None]).reshape(R * N, 3).contiguous())
    coords = [xs[0], xs[1], xs[0]]
    grads = [torch.randn(R * N, device=dev, generator=g) for _ in nets]
    return nets, coords, grads


class _RefGridFn(torch.autograd.Function):
    """The reference's grid kernels with the table as the differentiable input, as
    source/gridencoder/grid.py:24-88 calls them (no input gradient)."""

    @staticmethod
    def forward(ctx, inputs, embeddings, offsets, S, H, mod):
        B, L, C = inputs.shape[0], offsets.shape[0] - 1, embeddings.shape[1]
        out = torch.empty(L, B, C, device=inputs.device)
        mod.grid_encode_forward(inputs, embeddings, offsets, out, B, 3, C, L, S, H, None, 0, False, 0)
        ctx.save_for_backward(inputs, embeddings, offsets)
        ctx.dims = (S, H, mod)
        return out.permute(1, 0, 2).reshape(B, L * C)

    @staticmethod
    def backward(ctx, grad):
        inputs, embeddings, offsets = ctx.saved_tensors
        S, H, mod = ctx.dims
        B, L, C = inputs.shape[0], offsets.shape[0] - 1, embeddings.shape[1]
        gg = grad.reshape(B, L, C).permute(1, 0, 2).contiguous()
        gemb = torch.zeros_like(embeddings)
        mod.grid_encode_backward(gg, inputs, embeddings, offsets, gemb, B, 3, C, L, S, H, None, None, 0, False, 0)
        return None, gemb, None, None, None, None


def prop_reference_step_fn(nets, coords, grads, mod):
    """One step of the reference's formulation on the GPU: _warp_coords, GridEncoder
    (its own kernels), density_layer as torch layers, softplus, the hash decay
    statistics by scatter_reduce_ (models.py:19-33, 362-372, 430-431, 472-488), then
    autograd with the upstream density gradients and the hash-decay loss of the two
    proposal networks (loss.py:371-378, hash_decay_mult 0.1)."""
    import numpy as np
    import torch.nn.functional as F

    def step():
        outs, ups = [], []
        for i, (net, x, g) in enumerate(zip(nets, coords, grads)):
            for p in net.parameters():
                p.grad = None
            w = x / (net.bbox_size / 2)
            u = ((w + 1.0) / (2 * 1.0)).contiguous()
            enc = net.encoder
            feats = _RefGridFn.apply(u, enc.embeddings, enc.offsets, float(np.log2(enc.per_level_scale)),
                                     enc.base_resolution, mod)
            raw = net.density_layer(feats)[..., 0]
            dens = F.softplus(raw + net.density_bias)
            hlm = torch.zeros(enc.num_levels, enc.embeddings.shape[-1], device=x.device).scatter_reduce_(
                0, enc.idx.unsqueeze(1), torch.square(enc.embeddings), reduce="mean", include_self=False)
            outs.append(dens)
            ups.append(g)
            if i < 2:
                outs.append(0.1 * hlm.mean())
                ups.append(None)
        torch.autograd.backward([o for o in outs], [u if u is not None else torch.ones_like(o)
                                                    for o, u in zip(outs, ups)])
    return step


def prop_fused_step_fn(nets, coords, grads):
    """One step through the fused kernels (the C ABI, buffers allocated once): per
    network the forward (density, feature record, warped coordinates) and the hash
    decay statistics, then the backward into zeroed gradients and, for the two
    proposal networks, the hash-decay gradient (0.1 / (L C) per entry)."""
    import ctypes
    from neural3dstrokes_b200 import _lib, mlp
    lib = _lib.load()
    state = []
    for net, x, g in zip(nets, coords, grads):
        enc, lay = net.encoder, net.density_layer
        L, C = enc.num_levels, enc.level_dim
        n = x.shape[0]
        stride = lib.n3ds_density_net_feature_stride(L, C)
        st = dict(net=net, x=x, g=g, n=n, L=L, C=C,
                  desc=mlp._net_struct(enc, lay[0].weight, lay[0].bias, lay[2].weight, lay[2].bias,
                                       net.density_bias, mlp.WARP_SCALE, net.bbox_size, False),
                  density=torch.empty(n, device=x.device), feats=torch.empty(n, stride, device=x.device),
                  warped=torch.empty(n, 3, device=x.device), hlm=torch.empty(L, C, device=x.device),
                  hlm_grad=torch.full((L, C), 0.1 / (L * C), device=x.device),
                  grads=[torch.zeros_like(t) for t in (enc.embeddings, lay[0].weight, lay[0].bias, lay[2].weight,
                                                        lay[2].bias)])
        state.append(st)

    def step():
        sp = _lib.stream_ptr()
        for i, st in enumerate(state):
            enc = st["net"].encoder
            for t in st["grads"]:
                t.zero_()
            _lib.check(lib.n3ds_density_net_forward(ctypes.byref(st["desc"]), _lib.ptr(st["x"]), st["n"],
                                                    _lib.ptr(st["density"]), _lib.ptr(st["feats"]),
                                                    _lib.ptr(st["warped"]), sp))
            _lib.check(lib.n3ds_grid_level_mean_sq(_lib.ptr(enc.embeddings), _lib.ptr(enc.offsets), st["L"],
                                                   st["C"], 0, _lib.ptr(st["hlm"]), sp))
            _lib.check(lib.n3ds_density_net_backward(ctypes.byref(st["desc"]), _lib.ptr(st["x"]),
                                                     _lib.ptr(st["feats"]), _lib.ptr(st["g"]), st["n"],
                                                     *[_lib.ptr(t) for t in st["grads"]], sp))
            if i < 2:
                _lib.check(lib.n3ds_grid_level_mean_sq_backward(_lib.ptr(enc.embeddings), _lib.ptr(enc.offsets),
                                                                st["L"], st["C"], 0, _lib.ptr(st["hlm_grad"]),
                                                                _lib.ptr(st["grads"][0]), sp))
    return step, state


def prop_cpu_baseline(nets, coords, grads, budget_s=15.0):
    """The float64 oracle's forward + backward of the three networks on host threads,
    on the first `n` points of each network's samples, in points/s."""
    import numpy as np
    from oracle import density_net as odn
    n = 2048
    done, t0 = 0, time.perf_counter()
    while True:
        for net, x, g in zip(nets, coords, grads):
            enc, lay = net.encoder, net.density_layer
            args = (enc.embeddings, enc.offsets, float(np.log2(enc.per_level_scale)), enc.base_resolution,
                    lay[0].weight, lay[0].bias, lay[2].weight, lay[2].bias)
            kw = dict(density_bias=net.density_bias, warp=odn.WARP_SCALE, bbox_size=net.bbox_size)
            odn.forward(x[:n], *args, **kw)
            odn.backward(g[:n], x[:n], *args, **kw)
            done += n
        if time.perf_counter() - t0 > budget_s / 3:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": PROP_UNIT, "cores": torch.get_num_threads(), "kind": "port",
            "sample": f"the first {n} points of each network, repeated {done // (3 * n)}x (oracle float64, "
                      "torch on the host threads)"}


def run_prop(args, world, rank, local):
    from neural3dstrokes_b200.train import capture
    dev = torch.device("cuda", local)
    nets, coords, grads = prop_workload(dev, args.scale)
    points = sum(x.shape[0] for x in coords)
    R = coords[0].shape[0] // 64
    cfg = {"workload": f"proposal-side networks of one training step, {R} rays x 64 samples per network",
           "networks": "PropMLP(512): 6 x 1, PropMLP(2048): 8 x 1, ErrorMLP(256): 5 x 2; Linear(L*C, 64), ReLU, "
                       "Linear(64, 1), softplus; hash decay statistics", "points": points,
           "l2": "tables 2 x 43 MB + 21 MB; feature records and gradients stream from HBM"}
    ref = grid_reference_module()
    if args.impl == "reference":
        if ref is None:
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "reference grid encoder not built "
                                  "(python oracle/build_ref.py --only grid)"}), flush=True)
            return
        step = prop_reference_step_fn(nets, coords, grads, ref)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lo = time.monotonic()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize(dev)
        clk = clocks.stop(lo, time.monotonic())
        t = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / args.steps, world, dev)
        if rank == 0:
            v = points * world / t
            print(json.dumps({"impl": "reference", "metric": PROP_METRIC, "value": v, "unit": PROP_UNIT,
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
                              "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
                              "clocks": clk, "config": cfg,
                              "cpu_baseline": None,
                              "e2e": {"value": v, "unit": PROP_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                              "note": "the reference's formulation on the GPU: its grid kernels built from their "
                                      "sources, torch layers and autograd, eager"}), flush=True)
        return

    step, state = prop_fused_step_fn(nets, coords, grads)
    step()  # resolves occupancy and sets the kernels' shared-memory limits before capture
    graph = capture(step, dev, warmup=1)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lo = time.monotonic()
    e0.record()
    for _ in range(args.steps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize(dev)
    clk = clocks.stop(lo, time.monotonic())
    t_step = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / args.steps, world, dev)

    # per-kernel durations by events on the launching stream (the largest network)
    import ctypes
    from neural3dstrokes_b200 import _lib
    lib = _lib.load()
    st = state[1]
    enc = st["net"].encoder
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    tf, tb = [], []
    sp = _lib.stream_ptr()
    for _ in range(5):
        for t in st["grads"]:
            t.zero_()
        ev[0].record()
        _lib.check(lib.n3ds_density_net_forward(ctypes.byref(st["desc"]), _lib.ptr(st["x"]), st["n"],
                                                _lib.ptr(st["density"]), _lib.ptr(st["feats"]),
                                                _lib.ptr(st["warped"]), sp))
        ev[1].record()
        _lib.check(lib.n3ds_density_net_backward(ctypes.byref(st["desc"]), _lib.ptr(st["x"]), _lib.ptr(st["feats"]),
                                                 _lib.ptr(st["g"]), st["n"], *[_lib.ptr(t) for t in st["grads"]], sp))
        ev[2].record()
        torch.cuda.synchronize(dev)
        tf.append(ev[0].elapsed_time(ev[1]) * 1e-3)
        tb.append(ev[1].elapsed_time(ev[2]) * 1e-3)
    t_fwd, t_bwd = statistics.mean(tf), statistics.mean(tb)
    cfg["ctas"] = {"forward": lib.n3ds_density_net_resident_ctas(0), "backward": lib.n3ds_density_net_resident_ctas(1)}
    n, stride = st["n"], st["feats"].shape[1]
    table_bytes = enc.embeddings.numel() * 4
    # algorithmic bytes: coordinates, density, feature record and warped coordinates
    # once and the table once (forward); coordinates, record, upstream gradient once
    # and a read + write of the table gradient (backward)
    fwd_bytes = n * (12 + 4 + 4 * stride + 12) + table_bytes
    bwd_bytes = n * (12 + 4 * stride + 4) + 2 * table_bytes
    peak, src = hbm_peak()
    roofline = {"bound": "hbm", "kernel": "density_bwd_kernel (PropMLP 2048: tensor-core adjoint + table scatter)",
                "achieved": bwd_bytes / t_bwd / 1e9, "peak": peak, "unit": "GB/s",
                "frac": bwd_bytes / t_bwd / 1e9 / peak, "traffic": None, "peak_source": src,
                "bytes_per_launch": bwd_bytes, "launch_ms": t_bwd * 1e3,
                "forward_kernel": {"name": "density_fwd_kernel", "achieved": fwd_bytes / t_fwd / 1e9,
                                   "launch_ms": t_fwd * 1e3, "frac": fwd_bytes / t_fwd / 1e9 / peak}}

    plain = None
    if ref is not None and not args.no_plain_op:
        rstep = prop_reference_step_fn(nets, coords, grads, ref)
        for _ in range(2):
            rstep()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(args.steps):
            rstep()
        e1.record()
        torch.cuda.synchronize(dev)
        tr = e0.elapsed_time(e1) * 1e-3 / args.steps
        plain = {"value": points / tr, "unit": PROP_UNIT, "ms_per_step": tr * 1e3, "speedup": tr / t_step,
                 "what": "the reference's formulation on this GPU: its grid kernels built from their sources, "
                         "torch layers, autograd"}

    # end to end through the public API: coordinates and upstream gradients uploaded
    # from pinned host memory, module forward + autograd backward, densities read back
    e2e = None
    if not args.no_e2e:
        hx = [x.cpu().pin_memory() for x in coords]
        hg = [g.cpu().pin_memory() for g in grads]
        hd = [torch.empty(x.shape[0], pin_memory=True) for x in coords]
        dx = [torch.empty_like(x) for x in coords]
        dg = [torch.empty_like(g) for g in grads]

        def api_step():
            outs, ups = [], []
            for i, net in enumerate(nets):
                dx[i].copy_(hx[i], non_blocking=True)
                dg[i].copy_(hg[i], non_blocking=True)
                for p in net.parameters():
                    p.grad = None
                out = net(dx[i], None)
                outs.append(out["density"])
                ups.append(dg[i])
                if i < 2:
                    outs.append(0.1 * out["hash_levelwise_mean"].mean())
                    ups.append(torch.ones((), device=dev))
                hd[i].copy_(out["density"].detach(), non_blocking=True)
            torch.autograd.backward(outs, ups)
        for _ in range(2):
            api_step()
        k = max(3, min(args.steps, 10))
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(k):
            api_step()
        e1.record()
        torch.cuda.synchronize(dev)
        te = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / k, world, dev)
        e2e = {"value": points * world / te, "unit": PROP_UNIT, "ms_per_step": te * 1e3,
               "h2d_bytes_per_step": sum(x.numel() * 4 for x in hx) + sum(g.numel() * 4 for g in hg),
               "d2h_bytes_per_step": sum(d.numel() * 4 for d in hd)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = prop_cpu_baseline(nets, coords, grads, args.cpu_seconds)
    if rank == 0:
        print(json.dumps({
            "metric": PROP_METRIC, "value": points * world / t_step, "unit": PROP_UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (first layer tf32 x3 split, adjoint bf16 x3 split)",
            "data": "synthetic (seeded rays, reference initialisation)", "config": cfg,
            "graph": "three networks' forward, hash decay statistics and backward in one CUDA graph",
            "roofline": roofline, "plain_op": plain, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": 11 * args.steps, "gpu_launches_per_step": 11}), flush=True)


def _ref_softmax_density_weighted(alphas, colors, density_params):
    """compose_strokes(..., 'softmax_density_weighted') as the reference writes it in
    torch (source/strokelib/strokes.py:408-415): the comparison leg of the ops workload."""
    inv_temp = 1.0 / 0.05
    adw = alphas * torch.broadcast_to(density_params, alphas.shape)
    sm = torch.softmax(adw * inv_temp, dim=-1)
    density = torch.einsum('...s,...s->...', sm, adw)
    color = torch.einsum('...s,...sc->...c', sm, colors)
    return density, color


def _ref_image_texture(image, texcoords, colors, alphas, tint_ratio=1.0):
    """ImageTexture.forward as the reference writes it (source/textures.py: grid_sample
    with align_corners=True of the [1, C, H, W] image, tint by the colour)."""
    import torch.nn.functional as F
    pre = colors.shape[:-1]
    uvs = texcoords.reshape(1, 1, -1, 2) * 2 - 1
    tint = F.grid_sample(image, uvs, align_corners=True)[0, :, 0, :].permute(1, 0)
    c = colors.reshape(-1, 3) * tint_ratio + (1.0 - tint_ratio)
    return (c * tint).reshape(*pre, 3), alphas


def _ref_resample(sdist, weights, num_samples, dilation, padding, domain=(0.0, 1.0)):
    """One proposal level of the reference's sampling loop as torch ops
    (source/models.py:160-185 with source/utils/stepfun.py: max_dilate_weights
    renormalised, the end posts dropped, logits log(w + padding), sample_intervals with
    single jitter and the mask-based sorted_interp)."""
    eps = torch.finfo(torch.float32).eps

    def sorted_interp(x, xp, fp):
        mask = x[..., None, :] >= xp[..., :, None]

        def find_interval(v):
            v0 = torch.max(torch.where(mask, v[..., None], v[..., :1, None]), -2).values
            v1 = torch.min(torch.where(~mask, v[..., None], v[..., -1:, None]), -2).values
            return v0, v1
        fp0, fp1 = find_interval(fp)
        xp0, xp1 = find_interval(xp)
        off = torch.clip(torch.nan_to_num((x - xp0) / (xp1 - xp0), 0), 0, 1)
        return fp0 + off * (fp1 - fp0)

    t, w = sdist, weights
    p = w / (t[..., 1:] - t[..., :-1]).clamp_min(eps)
    t0, t1 = t[..., :-1] - dilation, t[..., 1:] + dilation
    td = torch.clip(torch.sort(torch.cat([t, t0, t1], dim=-1), dim=-1).values, *domain)
    pd = torch.max(torch.where((t0[..., None, :] <= td[..., None]) & (t1[..., None, :] > td[..., None]),
                               p[..., None, :], torch.zeros_like(p[..., None, :])), dim=-1).values[..., :-1]
    wd = pd * (td[..., 1:] - td[..., :-1])
    wd = wd / torch.sum(wd, dim=-1, keepdim=True).clamp_min(eps)
    t, w = td[..., 1:-1], wd[..., 1:-1]
    logits = torch.where(t[..., 1:] > t[..., :-1], torch.log(w + padding), -torch.inf)
    u_max = eps + (1 - eps) / num_samples
    max_jitter = (1 - u_max) / (num_samples - 1) - eps
    u = torch.linspace(0, 1 - u_max, num_samples, device=t.device) + \
        torch.rand(t.shape[:-1] + (1,), device=t.device) * max_jitter
    wsm = torch.softmax(logits, dim=-1)
    cw = torch.cumsum(wsm[..., :-1], dim=-1).clamp_max(1)
    shape = cw.shape[:-1] + (1,)
    cw = torch.cat([torch.zeros(shape, device=t.device), cw, torch.ones(shape, device=t.device)], dim=-1)
    centers = sorted_interp(u, cw, t)
    mid = (centers[..., 1:] + centers[..., :-1]) / 2
    first = (2 * centers[..., :1] - mid[..., :1]).clamp_min(domain[0])
    last = (2 * centers[..., -1:] - mid[..., -1:]).clamp_max(domain[1])
    return torch.cat([first, mid, last], dim=-1)


def run_ops(args, rank, local):
    """Each operator at a stated size, events around ``args.steps`` calls after
    ``args.warmup``; one JSON line with per-op ms and algorithmic GB/s."""
    from neural3dstrokes_b200 import scenes, stepfun, strokelib, strokes, textures
    from neural3dstrokes_b200.insertion import StrokeInserter
    from neural3dstrokes_b200.train import BatchedField, GraphedTrainer
    dev = torch.device("cuda", local)
    g = torch.Generator().manual_seed(0)
    res = []

    def time_of(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    jobs = []

    def timed(name, fn, nbytes, ref_fn=None):
        fn()  # every kernel launches once before the timed (and profiled) window
        if ref_fn is not None:
            ref_fn()
        jobs.append((name, fn, nbytes, ref_fn))

    ref = None
    hits = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "_strokelib*.so")))
    if hits:
        import importlib.machinery
        import importlib.util
        loader = importlib.machinery.ExtensionFileLoader("_strokelib", hits[0])
        ref = importlib.util.module_from_spec(importlib.util.spec_from_file_location("_strokelib", hits[0],
                                                                                    loader=loader))
        loader.exec_module(ref)

    # drop-in operators: 256 cubes x 65,536 samples ([P, S] tensors of 67 / 201 MB)
    P, S = 65536, 256
    sc = scenes.make_strokes(["cube"] * S, g)
    rays = scenes.make_rays(P // 64, 64, g)
    sid = scenes.SDF_ID["cube"]
    ps = sc.shape_params[:, :7].contiguous().to(dev)
    col = sc.color_params.to(dev)
    x = rays.x.reshape(-1, 3).contiguous().to(dev)
    r = rays.radius.reshape(-1).contiguous().to(dev)
    vd = rays.dirs.to(dev)
    a = torch.empty(P, S, device=dev)
    c = torch.empty(P, S, 3, device=dev)
    none = torch.empty(0, device=dev)
    R = (lambda f: f) if ref is not None else (lambda f: None)
    timed("stroke_forward (cube, 65536 x 256)", lambda: strokelib.stroke_forward(
        a, c, none, none, x, r, vd, ps, col, sid, 0, 0.02, True, True), P * S * 16,
        R(lambda: ref.stroke_forward(a, c, none, none, x, r, vd, ps, col, sid, 0, 0.02, True, True)))
    ga, gc = torch.randn(P, S, device=dev), torch.randn(P, S, 3, device=dev)
    gps, gcol, gx = torch.zeros_like(ps), torch.zeros_like(col), torch.zeros_like(x)
    timed("stroke_backward (cube, 65536 x 256)", lambda: strokelib.stroke_backward(
        gps, gcol, gx, ga, gc, none, x, r, vd, a, ps, col, sid, 0, 0.02, True, True), P * S * 20,
        R(lambda: ref.stroke_backward(gps, gcol, gx, ga, gc, none, x, r, vd, a, ps, col, sid, 0, 0.02, True, True)))
    dp = torch.rand(S, device=dev) * 10
    dens, ccol = torch.empty(P, device=dev), torch.empty(P, 3, device=dev)
    timed("compose_forward over (65536 x 256)", lambda: strokelib.compose_forward(dens, ccol, a, c, dp), P * S * 16,
          R(lambda: ref.compose_forward(dens, ccol, a, c, dp)))
    gda, gdc, gdp = torch.zeros_like(a), torch.zeros_like(c), torch.zeros_like(dp)
    gd, gcc = torch.randn(P, device=dev), torch.randn(P, 3, device=dev)
    # the backward reads alphas and colours and accumulates into both gradient tensors
    timed("compose_backward over (65536 x 256)", lambda: strokelib.compose_backward(
        gda, gdc, gdp, gd, gcc, a, c, dp), P * S * 48,
        R(lambda: ref.compose_backward(gda, gdc, gdp, gd, gcc, a, c, dp)))
    a_req = a.detach().requires_grad_(True)

    def softmax_fb():
        d_, c_ = strokes.compose_strokes(a_req, c, dp, "softmax_density_weighted")
        (d_.sum() + c_.sum()).backward()

    def softmax_ref():
        d_, c_ = _ref_softmax_density_weighted(a_req, c, dp)
        (d_.sum() + c_.sum()).backward()
    timed("compose softmax_density_weighted fwd+bwd (65536 x 256)", softmax_fb, P * S * 32, softmax_ref)
    # colour field: SH3 on 128 spheres
    sph = scenes.make_strokes(["sphere"] * 128, g)
    sh = torch.randn(128, 27, generator=g).to(dev)
    a2, c2 = torch.empty(P, 128, device=dev), torch.empty(P, 128, 3, device=dev)
    vdn = torch.nn.functional.normalize(vd, dim=-1)
    sph_ps = sph.shape_params[:, :4].contiguous().to(dev)
    timed("stroke_forward sphere + SH3 colour (65536 x 128)", lambda: strokelib.stroke_forward(
        a2, c2, none, none, x, r, vdn, sph_ps, sh, scenes.SDF_ID["sphere"], 3, 0.02, True, True), P * 128 * 16,
        R(lambda: ref.stroke_forward(a2, c2, none, none, x, r, vdn, sph_ps, sh, scenes.SDF_ID["sphere"], 3, 0.02,
                                     True, True)))
    # texture on the cube pairs
    tex = textures.ImageTexture(torch.rand(256, 256, 3, generator=g) * 255, (256, 256)).to(dev)
    tc = torch.rand(P, S, 2, device=dev)
    c_req = c.detach().requires_grad_(True)

    def tex_fb():
        co, al = tex(tc, c_req, a)
        co.sum().backward()
    image = tex.image_texture if hasattr(tex, "image_texture") else None

    def tex_ref():
        co, al = _ref_image_texture(image, tc, c_req, a)
        co.sum().backward()
    timed("ImageTexture fwd+bwd (65536 x 256)", tex_fb, P * S * (40 + 20), tex_ref if image is not None else None)
    # proposal resampling: 65,536 rays, 64 bins -> 32 samples, dilation
    sd = torch.sort(torch.rand(65536, 65, device=dev), -1).values
    sd[:, 0], sd[:, -1] = 0, 1
    wts = torch.rand(65536, 64, device=dev)
    timed("resample_intervals (65536 rays, 64 -> 32, dilation)", lambda: stepfun.resample_intervals(
        sd, wts, 32, rand=True, dilation=0.01, resample_padding=0.01), 65536 * (65 + 64 + 33) * 4,
        lambda: _ref_resample(sd, wts, 32, 0.01, 0.01))
    # stroke insertion: 2000 strokes, 30,000 error points
    ins = StrokeInserter("sphere", max_num_strokes=2000, init_num_strokes=10, device=dev)
    ec, _ = ins.sample_error_coords()
    err = torch.rand(ec.shape[0], device=dev)
    step = [100]

    def ins_step():
        ins.step_update(step[0], 200000, errors=err, error_coords=ec)
        step[0] += 7
    timed("insertion step_update (2000 strokes, 30000 error points)", ins_step, 0)
    # the field at a tenth of config 3, forward + MSE + backward + Adam (eager)
    w = scenes.config(3, scale=0.1)
    field = BatchedField(w.scenes, w.rays, device=dev)
    trainer = GraphedTrainer(field, torch.zeros_like(field.rgb), lr=1e-3)
    timed("field training step (config 3 at 0.1 of its rays, eager)", trainer._step, 0)
    torch.cuda.synchronize(dev)
    torch.cuda.profiler.start()  # the window an ncu --profile-from-start off capture sees
    for name, fn, nbytes, ref_fn in jobs:
        ms = time_of(fn)
        item = {"op": name, "ms": round(ms, 4), "bytes": int(nbytes),
                "gbs": round(nbytes / ms / 1e6, 1) if nbytes else None}
        if ref_fn is not None:  # the reference's operator (or torch formulation) on the same tensors
            item["reference_ms"] = round(time_of(ref_fn), 4)
            item["speedup"] = round(item["reference_ms"] / ms, 1)
        res.append(item)
    torch.cuda.profiler.stop()
    if rank == 0:
        print(json.dumps({"workload": "ops", "steps": args.steps, "warmup": args.warmup, "ops": res}), flush=True)


def hbm_peak():
    """Measured HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        for k in ("hbm_gbs", "hbm_GBs", "hbm"):
            if k in pk:
                return float(pk[k]), "measured (MEASURED_PEAKS.json hbm copy)"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback 6.65 TB/s"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--workload", default="field", choices=["field", "grid", "prop", "ops"],
                    help="field: the stroke field (default); grid: a hash-grid encoder alone; prop: the "
                         "proposal and error fields' density networks; ops: every other operator once (profiling)")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="ray-count scale (profiling small cases)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain-op", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the untimed accuracy leg")
    ap.add_argument("--schedule", default="auto", choices=["auto", "runs", "segments"],
                    help="field kernel work decomposition (auto: the autotuner picks)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (library defaults)")
    ap.add_argument("--loss-curve", type=int, default=0, metavar="K",
                    help="config 4 only: train K steps with the graphed step and with the plain reference op "
                         "from the same start, print both loss curves (not a throughput run)")
    ap.add_argument("--curve-out", default="", help="write the loss curves as JSON to this file")
    ap.add_argument("--exclude-kinds", default="",
                    help="loss-curve runs: comma-separated stroke kinds left out of config 4's draw")
    ap.add_argument("--ref-twice", action="store_true",
                    help="loss-curve runs: train the reference op a second time (its run-to-run spread)")
    ap.add_argument("--cull-alpha", type=float, default=1e-9,
                    help="loss-curve runs: the field's culling threshold (0: every pair evaluated)")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)
    if args.workload == "ops":
        run_ops(args, rank, local)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload in ("grid", "prop"):
        (run_grid if args.workload == "grid" else run_prop)(args, world, rank, local)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.loss_curve:
        if rank == 0:
            loss_curves(args)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    from neural3dstrokes_b200 import scenes
    from neural3dstrokes_b200.field import FieldOptions
    from neural3dstrokes_b200.train import BatchedField, GraphedTrainer, capture

    dev = torch.device("cuda", local)
    w = scenes.config(args.config, scale=args.scale)
    field = BatchedField(w.scenes, w.rays, w.sdf_delta, w.use_laplace, w.inv_scale_radius,
                         options=FieldOptions(schedule=args.schedule), device=dev)
    g_rgb, g_acc, g_depth = workload_upstream(field)
    trainer = None
    if args.config == 4:
        # target image: render of a separate seeded 2000-stroke scene per ray set
        tf = BatchedField(w.target_scenes, w.rays, w.sdf_delta, w.use_laplace, w.inv_scale_radius, device=dev,
                          need_grad_x=False)
        tf.forward()
        trainer = GraphedTrainer(field, tf.rgb.clone(), lr=1e-3)
        del tf
        step_fn = trainer._step
    else:
        field.g_rgb.copy_(g_rgb)
        field.g_acc.copy_(g_acc)
        field.g_depth.copy_(g_depth)
        step_fn = field.step
    pairs = field.nominal_pairs

    # launch configuration: the autotuner times the candidates on this workload (not timed)
    tuned = None
    tune_table = None
    if args.schedule == "auto" and not args.no_tune:
        from neural3dstrokes_b200 import autotune
        tuned = autotune.tune(field, reps=2, use_cache=False)
        tune_table = [[f"{o.schedule} w{o.warps}/{o.warps_bwd} c{o.chunk_fwd}/{o.chunk_bwd}"
                       + (f" rays/claim {o.rays_per_item}" if o.rays_per_item > 1 else ""), round(ms, 3)]
                      for ms, o in autotune.last_results]
    segments = field.options.schedule != "runs"

    # statistics pass (not timed; the only one with the pair counters on): evaluated
    # pairs per primitive type (forward) and in total (backward), status word
    import dataclasses
    field.c_opt = dataclasses.replace(field.options, count_pairs=True).c()
    field.forward()
    field.backward()
    torch.cuda.synchronize(dev)
    per_base = field.pair_counts()
    bwd_evaluated = field.backward_pairs()
    status, evaluated = field.status()
    field.c_opt = field.options.c()
    if status != 0:
        raise SystemExit(f"device status {status}")

    graph = capture(step_fn, dev, warmup=1) if trainer is None else trainer.capture()
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    barrier(world)
    clocks = ClockSampler(torch.cuda.current_device() if world == 1 else local)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    barrier(world)
    host_lo = time.monotonic()
    t0.record()
    for _ in range(args.steps):
        graph.replay()
    t1.record()
    torch.cuda.synchronize(dev)
    host_hi = time.monotonic()
    barrier(world)
    clk = clocks.stop(host_lo, host_hi)
    value, step_s = replica_throughput(t0.elapsed_time(t1) * 1e-3 / args.steps, pairs, world, dev)

    # dominant-kernel timing with CUDA events recorded on the launching stream
    from neural3dstrokes_b200 import _lib
    import ctypes
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    field.c_opt = field.options.c(ev)
    fwd_t, bwd_t = [], []
    for _ in range(max(3, min(10, args.steps))):
        field.forward()
        field.backward()
        ev[3].synchronize()
        fwd_t.append(ev[0].elapsed_time(ev[1]) * 1e-3)
        bwd_t.append(ev[2].elapsed_time(ev[3]) * 1e-3)
    field.c_opt = field.options.c()
    t_fwd, t_bwd = statistics.mean(fwd_t), statistics.mean(bwd_t)
    bf = base_flops(field.kinds)
    fwd_flops = sum(per_base[b] * bf.get(b, 0.0) for b in range(16))
    bwd_flops = BWD_FACTOR * fwd_flops * (bwd_evaluated / evaluated if (bwd_evaluated and evaluated) else 1.0)
    peak = fp32_peak(dev)
    kname = ("seg_bwd_kernel (segment adjoint)" if segments else "run_bwd_kernel (sample-run adjoint)")
    traffic = SEG_BWD_TRAFFIC_CFG3_QUARTER * args.scale / 0.25 if (args.config == 3 and segments) else None
    roofline = {"bound": "fp32", "kernel": kname, "achieved": bwd_flops / t_bwd / 1e12,
                "peak": peak, "unit": "TFLOP/s", "frac": bwd_flops / t_bwd / 1e12 / peak, "traffic": traffic,
                "traffic_note": "DRAM bytes per step over the backward launches, ncu at 1/4 of the rays, scaled"
                                if traffic else None,
                "peak_source": "measured: FP32 FMA probe kernel on this GPU (no FP32 figure in the peaks file)",
                "flops_per_launch": bwd_flops, "launch_ms": t_bwd * 1e3,
                "forward_kernel": {"name": "seg_fwd_kernel" if segments else "run_fwd_kernel",
                                   "achieved": fwd_flops / t_fwd / 1e12, "launch_ms": t_fwd * 1e3,
                            "frac": fwd_flops / t_fwd / 1e12 / peak}}

    # end to end through the public API with host buffers: H2D of the step's inputs,
    # the step, D2H of its results, every step; HostPipeline overlaps the copies of one
    # step with the compute of its neighbours (two staging sets, a copy stream)
    e2e = None
    if not args.no_e2e:
        ins = [field.x, field.radius, field.tdist, field.dirs, field.g_rgb, field.g_acc, field.g_depth, field.shape,
               field.color, field.density, field.delta, field.sdf_ids]
        # every result of the step comes back, the sample-position gradient included
        outs = [field.rgb, field.acc, field.depth, field.grad_shape, field.grad_color, field.grad_density,
                field.grad_delta] + ([field.grad_x] if field.grad_x is not None else [])
        h_in = [t.detach().cpu().pin_memory() for t in ins]
        h_out = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in outs]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_e2e = max(3, min(args.steps, 10))
        from neural3dstrokes_b200.train import HostPipeline
        pipe = HostPipeline(graph, ins, outs, dev)

        def e2e_run(n):
            pipe.upload(0, h_in)
            for i in range(n):
                if i + 1 < n:
                    pipe.upload(i + 1, h_in)
                pipe.run(i, h_out)
        e2e_run(2)
        pipe.synchronize()
        barrier(world)
        e0.record()
        pipe.copy.wait_event(e0)  # the first upload is inside the timed region
        e2e_run(n_e2e)
        pipe.compute.wait_stream(pipe.down)  # ... and so is the last download
        e1.record()
        torch.cuda.synchronize(dev)
        t_e2e = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / n_e2e, world, dev)
        e2e = {"value": pairs * world / t_e2e, "unit": UNIT, "ms_per_step": t_e2e * 1e3,
               "h2d_bytes_per_step": sum(t.numel() * t.element_size() for t in h_in),
               "d2h_bytes_per_step": sum(t.numel() * t.element_size() for t in h_out),
               "overlap": "uploads and downloads on two copy streams (both link directions at once), "
                          "double-buffered, overlapping compute"}

    # accuracy at the workload's own shape (untimed; the float64 oracle and the
    # reference op are the checkers): the whole workload with upstream gradients on a
    # fixed ray subset, plus the 16 sequential plain-op calls (config 3) and the FP64
    # finite-difference slice (config 2)
    accuracy = None
    if rank == 0 and not args.no_accuracy:
        accuracy = accuracy_leg(field, w, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, args.config, args.cpu_seconds)

    lf, lb = field.launch_count()
    launches_per_step = lf + lb + (3 if trainer is not None else 0)  # + 3 Adam launches when training
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators, no dataset)",
            "config": {"workload": w.name, "scenes": len(w.scenes), "nominal_pairs_per_step": pairs,
                       "evaluated_pairs_per_step": int(evaluated),
                       "backward_evaluated_pairs_per_step": int(bwd_evaluated), "rays": int(field.rgb.shape[0]),
                       "samples_per_ray": field.n_samples, "strokes": int(field.shape.shape[0]),
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (x alone %.0f MB)" % (field.x.numel() * 4 / 1e6),
                       "graph": "forward+backward captured in one CUDA graph" if trainer is None
                       else "forward+MSE+backward+Adam captured in one CUDA graph",
                       "launch": {"schedule": "segments" if segments else "runs", "warps": field.options.warps,
                                  "warps_bwd": field.options.warps_bwd, "chunk_fwd": field.options.chunk_fwd,
                                  "chunk_bwd": field.options.chunk_bwd,
                                  "rays_per_claim": max(1, field.options.rays_per_item),
                                  "picked_by": "autotuner" if tuned is not None else "flags",
                                  "tried_ms": tune_table}},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "accuracy": accuracy,
            "gpu_launches": launches_per_step * args.steps,
            "gpu_launches_per_step": launches_per_step,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        del graph
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
