#!/usr/bin/env python
"""Benchmark: ms2dirty + dirty2ms round trip on synthetic MeerKAT-shaped data.

Workload (default): 64 antennas (2016 baselines) x 512 integrations of 8 s x
1024 channels over 856-1712 MHz = 1,056,964,608 complex64 visibilities, the
sum of 50 seeded point sources plus complex Gaussian noise (sigma 0.1), 20 %
seeded random flags, unit weights; image 4096 x 4096 at 1.0 arcsec;
epsilon 1e-5, single-precision working type (the kernel table's
single-precision rows).

One step = vis2dirty (scan, plan, binning, gridding, FFT, projection) then
dirty2vis (scan, plan, binning, w-screens, FFT, degridding) of the same
visibilities and mask: the reference's two stateless calls.

* `value`: Mvis/s of the step with inputs resident in HBM (device API,
  CUDA events on torch's current stream, max over ranks).
* `e2e`: the same through the reference-facing C ABI (`rang._core`) with
  pinned host arrays: host-to-device copies of the inputs and the
  device-to-host copies of the image and the visibilities are inside the
  timed region (host clock around the synchronous calls).
* `roofline`: the dominant kernel's algorithmic HBM bytes per launch over its
  event-timed average launch, against the measured copy bandwidth.
* `cpu_baseline`: the CPU oracle (a C++/OpenMP restatement of the
  reference's Rust wgridder; the reference itself cannot be built here) on
  every 64th integration of the workload (the same uv extent, w range and
  plan, one sixty-fourth of the visibilities), all host threads.
* `accuracy`: every gridding method's dirty image and visibilities on that
  sample against the oracle's FP64 run at epsilon 1e-7, L-inf and RMS over
  the peak with the image border (outer two pixels) apart from the interior
  (eight pixels in), and each method's time at the full size.
* `config1`: the 16.5 M-visibility, 1024^2 configuration on the GPU (f32 and
  f64 at epsilon 1e-5) beside the CPU oracle run as the reference's own
  harness runs it (a fresh process per repeat, three repeats, the median, all
  threads and one, peak RSS and output SHA256).

`--impl reference` times the CPU oracle alone, on the same workload sample.
Multi-GPU (`--gpus N` under torchrun): independent replicas, one per GPU.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "rang-core_b200"))

from rang import synth  # noqa: E402

WORKLOAD = "ms2dirty+dirty2ms 1.06G vis 4096^2"
CONFIG1 = "ms2dirty 16.5M vis 1024^2"
PROFILE_CASE = "ms2dirty+dirty2ms 132M vis 2048^2"
# DRAM bytes (read + written) per launch of the dominant kernels, from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) of each on the
# 132 M-visibility profiling case, as (bytes, active visibilities of that
# launch): a launch of another workload is scaled by its active visibilities.
# A profiler figure, not something this script can time.
DRAM_CAPTURE = {
    "k_grid_i8": (7.865198e9 + 0.640229e9, 105697663),
    "k_degrid_h": (6.992914e9 + 1.269871e9, 105697663),
}
METRIC = "Mvis/s ms2dirty+dirty2ms @eps=1e-5 vs FP64"
UNIT = "Mvis/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD, choices=sorted(synth.WORKLOADS))
    ap.add_argument("--epsilon", type=float, default=1e-5)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"],
                    help="working precision of the timed step (f64: complex128 visibilities)")
    ap.add_argument("--cpu-stride", type=int, default=None,
                    help="the CPU sample: every n-th integration of the workload (default: 64 for the CPU "
                         "baseline leg; for --impl reference, 16, 32 or 64 as the step count allows)")
    ap.add_argument("--cpu-worker", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--no-config1", action="store_true")
    ap.add_argument("--fista-cap", type=int, default=3000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fista", action="store_true")
    ap.add_argument("--no-weights", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-msv4", action="store_true")
    ap.add_argument("--learned-patches", type=int, default=20000)
    ap.add_argument("--learned-steps", type=int, default=2500)
    ap.add_argument("--trace-e2e", default=None, metavar="PATH",
                    help="after the e2e leg, one more e2e step under the PyTorch profiler (CUDA activity), "
                         "its trace written to PATH (Chrome trace JSON)")
    return ap.parse_args()


def _plain(o):
    """JSON for numpy scalars."""
    if hasattr(o, "item"):
        return o.item()
    raise TypeError(f"{type(o).__name__} is not JSON serialisable")


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of this GPU during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) > 8 for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_observation(wl, seed=0):
    uvw = synth.uvw_tracks(nant=64, ntime=wl["ntime"], tint=8.0, dec_deg=-30.0)
    freq = synth.channels(wl["nchan"])
    sky = synth.point_sky(wl["npix"], nsrc=50, seed=11 + seed)
    return uvw, freq, sky


# ------------------------------------------------------------------ CPU (oracle)

NBL = 2016  # baselines of the 64-antenna array
# The reference's published CPU figures for this path (dirty + PSF per image,
# f64, epsilon 1e-6, 23.8 M gridded visibilities at 1024^2, Ryzen 7 7700X):
# ns per visibility per image at 1, 4 and 16 threads.
PUBLISHED_NS_PER_VIS = {"1": 477, "4": 149, "16": 81}


def _oracle():
    if str(REPO / "oracle") not in sys.path:
        sys.path.insert(0, str(REPO / "oracle"))
    import oracle

    return oracle


def sample_rows(ntime, stride):
    """The rows of every `stride`-th integration, starting in the middle of
    the first stride: the sample keeps the observation's uv extent and w
    range, so its plan (kernel, grid, planes) is the full workload's."""
    t = np.arange(stride // 2, ntime, stride)
    return (t[:, None] * NBL + np.arange(NBL)[None, :]).ravel(), len(t)


def cpu_round_trip(oracle, uvw, freq, vis, mask, npix, cell, eps):
    kw = dict(uvw=uvw, freq=freq, mask=mask, pixsize_x=cell, pixsize_y=cell, epsilon=eps)
    t0 = time.perf_counter()
    dirty = oracle.vis2dirty(vis=vis, npix_x=npix, npix_y=npix, **kw)
    oracle.dirty2vis(dirty=dirty, **kw)
    return time.perf_counter() - t0


def cpu_model():
    """The host CPU's model name and logical core count."""
    name = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                name = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{name}, {os.cpu_count()} logical cores"


def cpu_sample(wl, stride, seed=0):
    """Host data of every `stride`-th integration: visibilities predicted
    from the point sky by the oracle's degridder (float32, epsilon 1e-5)
    plus seeded noise (sigma 0.1) and flags."""
    oracle = _oracle()
    uvw, freq, sky = make_observation(wl, seed)
    rows, nt = sample_rows(wl["ntime"], stride)
    uvw = np.ascontiguousarray(uvw[rows])
    cell = wl["cell_arcsec"] * synth.ARCSEC
    model = oracle.dirty2vis(uvw=uvw, freq=freq, dirty=sky.astype(np.float32), pixsize_x=cell, pixsize_y=cell,
                             epsilon=1e-5)
    rng = np.random.default_rng(1000 + seed)
    shape = model.shape
    vis = (model + 0.1 * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))).astype(np.complex64)
    mask = (rng.uniform(size=shape) >= wl["flag"]).astype(np.uint8)
    return oracle, uvw, freq, vis, mask, nt


def sample_text(wl, stride, nt, nvis):
    full = NBL * wl["ntime"] * wl["nchan"]
    return (f"every {stride}th integration: {nt} of {wl['ntime']} integrations ({nvis} visibilities, "
            f"{100.0 * nvis / full:.2f} % of the workload, the same uv extent, w range and plan), "
            f"full {wl['npix']}^2 image and grid")


def workload_config(wl, name, eps, world, precision="f32"):
    """The `config` of both arms' lines: the workload, by what it is."""
    nvis = NBL * wl["ntime"] * wl["nchan"]
    return {"workload": name, "visibilities": nvis, "image": [wl["npix"], wl["npix"]],
            "cell_arcsec": wl["cell_arcsec"], "epsilon": eps, "precision": precision, "flags": wl["flag"],
            "parallelism": f"replicas{world}",
            "l2": f"inputs larger than L2 ({nvis * 8 / 1e9:.2f} GB of visibilities)"}


def maxrss_mb():
    import resource

    return resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 1024.0


def sha256(a):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def strided(a, ntime, stride):
    """Rows of every `stride`-th integration of a (ntime * NBL, ...) array."""
    if stride <= 1:
        return a
    rows, _ = sample_rows(ntime, stride)
    return np.ascontiguousarray(a[rows])


def cpu_worker(spec_json):
    """One timed oracle vis2dirty in this fresh process, as the reference's
    harness times one image (`examples/bench_df2.py:568-615`): the inputs
    from an .npz, the threads, precision, epsilon and sample from the spec;
    prints wall and CPU time, peak RSS (after loading and at the end), the
    load average before and after, and the image's SHA256."""
    spec = json.loads(spec_json)
    load0 = os.getloadavg()
    oracle = _oracle()
    d = np.load(spec["inputs"])
    ntime = int(d["ntime"])
    uvw = strided(d["uvw"], ntime, spec["stride"])
    vis = strided(d["vis"], ntime, spec["stride"]).astype(np.complex64 if spec["single"] else np.complex128)
    freq = d["freq"]
    threads = oracle.set_threads(spec["threads"])
    loaded = maxrss_mb()
    cell = float(d["cell"])
    w0, c0 = time.perf_counter(), time.process_time()
    dirty = oracle.vis2dirty(uvw=uvw, freq=freq, vis=vis, npix_x=int(d["npix"]), npix_y=int(d["npix"]),
                             pixsize_x=cell, pixsize_y=cell, epsilon=spec["epsilon"])
    wall = time.perf_counter() - w0
    print(json.dumps({"wall": wall, "cpu": time.process_time() - c0, "threads": threads, "visibilities": vis.size,
                      "dirty_sha256": sha256(dirty), "max_rss_mb": maxrss_mb(), "rss_mb_after_loading": loaded,
                      "loadavg_before_after": [load0, os.getloadavg()], "simd": oracle.simd_level()}), flush=True)


def cpu_protocol(inputs, repeats=3, stride1=8):
    """The CPU baseline as the reference's harness measures it
    (`examples/bench_df2.py:618-673`): a fresh process per (threads,
    precision, repeat), repeats interleaved, the median wall reported with
    peak RSS, load average and output hashes. All host threads run the whole
    configuration; one thread runs every `stride1`-th integration (a bounded
    sample), and the same sample on all threads shows whether the bits depend
    on the thread count."""
    allth = os.cpu_count() or 1
    cases = [(allth, True, 1), (allth, False, 1), (1, True, stride1), (1, False, stride1)]
    runs = {c: [] for c in cases}
    for _ in range(repeats):
        for c in cases:
            threads, single, stride = c
            spec = json.dumps({"inputs": str(inputs), "threads": threads, "single": single, "stride": stride,
                               "epsilon": 1e-5})
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            out = subprocess.run([sys.executable, str(Path(__file__).resolve()), "--cpu-worker", spec], env=env,
                                 capture_output=True, text=True, check=True)
            runs[c].append(json.loads(out.stdout.strip().splitlines()[-1]))
    same = {}
    for single in (True, False):
        spec = json.dumps({"inputs": str(inputs), "threads": allth, "single": single, "stride": stride1,
                           "epsilon": 1e-5})
        out = subprocess.run([sys.executable, str(Path(__file__).resolve()), "--cpu-worker", spec],
                             env=dict(os.environ, OMP_NUM_THREADS=str(allth)), capture_output=True, text=True,
                             check=True)
        rec = json.loads(out.stdout.strip().splitlines()[-1])
        same["f32" if single else "f64"] = rec["dirty_sha256"] == runs[(1, single, stride1)][0]["dirty_sha256"]
    rows = []
    for (threads, single, stride), recs in runs.items():
        walls = [r["wall"] for r in recs]
        med = statistics.median(walls)
        n = recs[0]["visibilities"]
        rows.append({"threads": recs[0]["threads"], "precision": "f32" if single else "f64", "epsilon": 1e-5,
                     "sample": "the whole configuration" if stride == 1 else
                               f"every {stride}th integration ({n} visibilities)",
                     "visibilities": n, "wall_median_s": med, "walls_s": [round(w, 4) for w in walls],
                     "cpu_median_s": statistics.median(r["cpu"] for r in recs),
                     "mvis_per_s": n / med / 1e6, "ns_per_vis": 1e9 * med / n,
                     "max_rss_mb": max(r["max_rss_mb"] for r in recs),
                     "rss_mb_after_loading": max(r["rss_mb_after_loading"] for r in recs),
                     "loadavg_before_after": recs[0]["loadavg_before_after"],
                     "hashes_identical_over_repeats": len({r["dirty_sha256"] for r in recs}) == 1,
                     "dirty_sha256": recs[0]["dirty_sha256"]})
    return {"harness": f"fresh process per (threads, precision, repeat), {repeats} interleaved repeats, median; "
                       "oracle vis2dirty (the C++/OpenMP restatement of the reference's Rust wgridder)",
            "cpu_model": cpu_model(), "simd": runs[cases[0]][0]["simd"], "runs": rows,
            "bits_independent_of_threads": same,
            "published_reference_ns_per_vis_per_image": {
                "values": PUBLISHED_NS_PER_VIS,
                "setting": "dirty + PSF, f64, epsilon 1e-6, 23.8 M visibilities at 1024^2, Ryzen 7 7700X "
                           "(other hardware and data)"}}


def replica_env():
    """(world size, rank, local rank) of this process under torchrun; one
    process per GPU, each an independent replica of the workload."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value, dist, device):
    """The largest of every rank's `value` (a time): the job is as slow as its
    slowest replica. `dist` None means one process."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_ranks(flag, dist, device):
    """Whether `flag` holds on every rank (a collective: every rank calls it)."""
    if dist is None:
        return bool(flag)
    import torch

    t = torch.tensor([1 if flag else 0], device=device, dtype=torch.int32)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return bool(t.item())


def job_rate(world, units_per_rank, steps, seconds):
    """Whole-job throughput in millions of units per second: every replica
    processes `units_per_rank` per step, timed as the slowest rank."""
    return world * units_per_rank * steps / seconds / 1e6


def reference_stride(steps, warmup):
    """The reference arm's sample: as large as the run's length allows. A
    sample pays the full grid's plan and FFTs (about 3.4 s on the 16 threads
    of the GPU box) however few visibilities it has, so a small one
    understates the CPU's rate on the whole workload; every 16th integration
    (66 M visibilities, about 10 s a round trip) when the run has at most 24
    steps, else every 32nd or 64th, keeps the run within a few minutes."""
    n = steps + warmup
    return 16 if n <= 24 else 32 if n <= 48 else 64


def run_reference(args):
    world, rank, _ = replica_env()
    if rank != 0:
        return  # the CPU reference runs once, on rank 0; the other ranks exit without work
    if args.cpu_stride is None:
        args.cpu_stride = reference_stride(args.steps, args.warmup)
    wl = synth.WORKLOADS[args.workload]
    oracle, uvw, freq, vis, mask, nt = cpu_sample(wl, args.cpu_stride)
    if args.precision == "f64":
        vis = vis.astype(np.complex128)
    threads = oracle.set_threads(os.cpu_count() or 1)
    cell = wl["cell_arcsec"] * synth.ARCSEC
    for _ in range(args.warmup):
        cpu_round_trip(oracle, uvw, freq, vis, mask, wl["npix"], cell, args.epsilon)
    load = os.getloadavg()
    times = [cpu_round_trip(oracle, uvw, freq, vis, mask, wl["npix"], cell, args.epsilon) for _ in range(args.steps)]
    t = sum(times)
    value = vis.size * args.steps / t / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
        "data": "synthetic", "config": workload_config(wl, args.workload, args.epsilon, world, args.precision),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample_text(wl, args.cpu_stride, nt, vis.size) + ", one round trip per step",
                         "cpu_model": cpu_model(), "simd": oracle.simd_level(),
                         "median_step_s": statistics.median(times), "step_s": [round(x, 4) for x in times],
                         "load_avg_before": list(load)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line, default=_plain), flush=True)


# ------------------------------------------------------------------ FISTA


def run_fista(dev, max_iterations=200, sigma=0.05, learn=None, cap=3000):
    """Plain FISTA (L1 with positivity, step 1 / ||A^H A|| from 30 power
    iterations) on 2048^2 at 1.5 arcsec: 300 point sources and 40 elliptical
    Gaussians predicted by the degridder onto the 64-antenna coverage of 128
    integrations at 256 channels (66 M visibilities), noise sigma 0.05 per
    component. Runs until the visibility residual RMS (per real component)
    first reaches 1.2 sigma, or `cap` iterations; reports the GPU time to
    that point (plan and power iteration included), the RMS after the
    configuration's `max_iterations` iterations and every 20 iterations;
    with `learn`, learned-preconditioned FISTA on the same measurement
    (`run_learned`)."""
    import torch

    from rang import fista, wgrid_torch

    npix, cell = 2048, 1.5 * synth.ARCSEC
    uvw = torch.from_numpy(synth.uvw_tracks(nant=64, ntime=128, tint=8.0, dec_deg=-30.0)).to(dev)
    freq = synth.channels(256)
    common = dict(npix_x=npix, npix_y=npix, pixsize_x=cell, pixsize_y=cell)
    sky = torch.from_numpy(synth.extended_sky(npix)).to(dev)
    gen = wgrid_torch.DevicePlan(uvw, freq, epsilon=1e-6, single=True, **common)
    vis = gen.degrid(sky)
    gen.close()
    g = torch.Generator(device=dev)
    g.manual_seed(77)
    vis += sigma * float(np.sqrt(2.0)) * torch.randn(vis.shape, dtype=torch.complex64, device=dev, generator=g)
    nvis = vis.numel()
    target = 1.2 * sigma
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    plan = wgrid_torch.DevicePlan(uvw, freq, epsilon=1e-5, single=True, **common)
    dirty, q = plan.residual(vis, None)
    ev[1].record()
    lmax, _ = fista.power_iteration(plan.gram, plan.shape, dev, max_iterations=30)
    ev[2].record()
    lam = 1e-4 * float(dirty.max())
    # rms = sqrt(2 misfit / (2 nvis)) per real component: the target's misfit.
    res = fista.solve(plan.gram, dirty, lam, 1.0 / lmax, cap, q0=0.5 * q, target_misfit=target * target * nvis,
                      events=True, check_every=10)
    ev[3].record()
    torch.cuda.synchronize()
    x, restarts = res.x, res.restarts
    rms = np.sqrt(np.maximum(2.0 * res.misfits.cpu().numpy(), 0.0) / (2 * nvis))
    trajectory = [[k, float(rms[k])] for k in range(0, len(rms), 20)]
    t_setup = ev[0].elapsed_time(ev[1]) / 1e3
    t_power = ev[1].elapsed_time(ev[2]) / 1e3
    t_iter = ev[2].elapsed_time(ev[3]) / 1e3
    t_target = ev[0].elapsed_time(res.events[res.first]) / 1e3 if res.first is not None else None
    err = float((x - sky).norm() / sky.norm())
    # The learned solver's first comparison level: plain FISTA's RMS after the
    # configuration's iterations, and plain FISTA's time to first reach it.
    final_rms = float(rms[min(max_iterations, len(rms) - 1)])
    t_final = ev[0].elapsed_time(res.events[int(np.argmax(rms <= final_rms))]) / 1e3
    reached = {"rms_at_config_iterations": final_rms if len(rms) > max_iterations else None, "k": res.k,
               "rms": float(rms[-1])}
    t_first = {"k": res.first}
    learned_report = None
    if learn is not None:
        learned_report = run_learned(dev, plan, dirty, q, lmax, lam, sky, nvis, target, final_rms, t_final,
                                     t_setup + t_power, max_iterations, learn)
    # The visibility-free Gram operator on the same measurement: setup, one
    # apply, and its distance from the exact A^H A on the dirty image.
    from rang import gram

    ones = torch.ones((uvw.shape[0], freq.size), dtype=torch.float64, device=dev)
    probe = dirty.double()
    exact = plan.gram(probe.float()).double()
    gram_report = {}
    for single in (True, False):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        op = gram.GramOperator(uvw, freq, ones, npix=npix, pixsize_x=cell, pixsize_y=cell,
                               expansion=gram.WExpansion(10, 1.0, 1e-13), epsilon=1e-5 if single else 1e-7,
                               single=single)
        e[1].record()
        got = op.apply(probe)  # the first apply sets up the FFT plan's work area
        torch.cuda.synchronize()
        e[1].record()
        got = op.apply(probe)
        e[2].record()
        torch.cuda.synchronize()
        gram_report["float32" if single else "float64"] = {
            "planes": op.planes(), "setup_s": op.stats["setup_grid_seconds"] + op.stats["setup_fft_seconds"],
            "apply_ms": e[1].elapsed_time(e[2]),
            "rel_diff_to_exact": float((got - exact).abs().max() / exact.abs().max())}
        op.close()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    plan.gram(probe.float())
    torch.cuda.synchronize()
    t0.record()
    plan.gram(probe.float())
    t1.record()
    torch.cuda.synchronize()
    gram_report["exact_apply_ms"] = t0.elapsed_time(t1)
    del ones
    plan.close()
    headline = None
    if learned_report is not None:
        lt = learned_report.get("time_to_target_s")
        headline = {"plain_time_to_target_s": t_target, "learned_time_to_target_s": lt,
                    "learned_over_plain": lt / t_target if lt and t_target else None,
                    "target": f"residual RMS 1.2 sigma ({target})",
                    "plain_cap_iterations": cap}
    return {"config": "2048^2 at 1.5 arcsec, 300 points + 40 Gaussians, 66 M visibilities, sigma 0.05, "
                      "L1 with positivity, lambda 1e-4 max(dirty), step 1/||A^H A|| from 30 power iterations",
            "target_rms": target, "time_to_target_s": t_target, "iterations_to_target": t_first.get("k"),
            "cap_iterations": cap, "config_iterations": max_iterations,
            "rms_at_config_iterations": reached.get("rms_at_config_iterations"),
            "iterations_run": reached.get("k"), "final_rms": reached.get("rms"), "rms_trajectory": trajectory,
            "restarts": int(restarts), "plan_and_dirty_s": t_setup, "power_iteration_s": t_power,
            "fista_s": t_iter, "ms_per_iteration": 1e3 * t_iter / (reached.get("k", 0) + 1),
            "time_to_target_learned_vs_plain": headline,
            "model_rel_error": err, "time_to_final_rms_s": t_final, "gram_operator": gram_report,
            "learned": learned_report}


def conv3_kernels(dev, batch=16):
    """The U-Net's 3x3 convolutions at the training batch on both kernels
    (rang_b200_nn_set_conv_path: 0 tcgen05 with TMA operands and a TMEM
    accumulator, 1 mma.sync): forward with bias and ReLU, then weight
    gradients with the bias gradient; CUDA events over 20 launches after 3;
    seeded random bf16 inputs and weights."""
    import torch

    from rang import learned

    lib = learned._library()
    s = torch.cuda.current_stream(dev).cuda_stream
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    rows = []
    for name, hw, cin, cout in (("enc1b", 256, 32, 32), ("enc2a", 128, 32, 64), ("enc2b", 128, 64, 64),
                                ("enc3b", 64, 128, 128), ("enc4b", 32, 256, 256), ("dec3a", 64, 384, 128),
                                ("dec3a input gradient", 64, 128, 384), ("dec1a", 256, 96, 32)):
        x = torch.randn(batch * hw * hw, cin, device=dev, generator=g).to(torch.bfloat16)
        w = (torch.randn(cout * 9 * cin, device=dev, generator=g) / np.sqrt(9 * cin)).to(torch.bfloat16)
        b = torch.randn(cout, device=dev, generator=g)
        o = torch.empty(batch * hw * hw, cout, device=dev, dtype=torch.bfloat16)
        flops = 2.0 * 9 * cin * cout * batch * hw * hw
        row = {"layer": name, "size": hw, "cin": cin, "cout": cout}
        for path, key in ((0, "tcgen05"), (1, "mma_sync")):
            old = lib.rang_b200_nn_set_conv_path(path)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            for i in range(23):
                if i == 3:
                    ev[0].record()
                learned._call("conv3", x.data_ptr(), cin, w.data_ptr(), b.data_ptr(), o.data_ptr(), cout, None, 0,
                              batch, hw, hw, cin, cout, 1, 0, s)
            ev[1].record()
            torch.cuda.synchronize()
            lib.rang_b200_nn_set_conv_path(old)
            assert lib.rang_b200_nn_device_status(s) == 0
            ms = ev[0].elapsed_time(ev[1]) / 20
            row[key + "_ms"] = ms
            row[key + "_tflops"] = flops / ms / 1e9
        rows.append(row)
        del x, w, b, o
    # weight gradients (dw and the bias gradient) where both kernels apply: 64-channel multiples
    for name, hw, cin, cout in (("enc2b weight gradient", 128, 64, 64), ("enc3b weight gradient", 64, 128, 128),
                                ("enc4b weight gradient", 32, 256, 256), ("dec3a weight gradient", 64, 384, 128)):
        x = torch.randn(batch * hw * hw, cin, device=dev, generator=g).to(torch.bfloat16)
        dz = torch.randn(batch * hw * hw, cout, device=dev, generator=g).to(torch.bfloat16)
        dw = torch.zeros(cout * 9 * cin, device=dev)
        db = torch.zeros(cout, device=dev)
        flops = 2.0 * 9 * cin * cout * batch * hw * hw
        row = {"layer": name, "size": hw, "cin": cin, "cout": cout}
        for path, key in ((0, "tcgen05"), (1, "mma_sync")):
            old = lib.rang_b200_nn_set_conv_path(path)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            for i in range(23):
                if i == 3:
                    ev[0].record()
                learned._call("conv3_weight_grad", x.data_ptr(), cin, dz.data_ptr(), cout, dw.data_ptr(),
                              db.data_ptr(), batch, hw, hw, cin, cout, s)
            ev[1].record()
            torch.cuda.synchronize()
            lib.rang_b200_nn_set_conv_path(old)
            assert lib.rang_b200_nn_device_status(s) == 0
            ms = ev[0].elapsed_time(ev[1]) / 20
            row[key + "_ms"] = ms
            row[key + "_tflops"] = flops / ms / 1e9
        rows.append(row)
        del x, dz, dw, db
    return rows


def run_learned(dev, plan, dirty, q, lmax, lam, sky, nvis, target, plain_rms, plain_time, t_shared, max_iterations,
                learn):
    """Learned-preconditioned FISTA (rang.learned) on the FISTA measurement.
    The U-Net is first trained by the library's own kernels on patches the
    gridder generates from other seeds (random skies of the same
    distribution over 8 random subsets of 32-64 antennas at 64 channels);
    that one-off cost is reported apart. The solve shares the plain run's
    plan, dirty image and power iteration (their time is added to its own)
    and adds the PSF and the network; it reports the GPU time until the
    residual RMS first reaches plain FISTA's final RMS and 1.2 sigma."""
    import torch

    from rang import learned

    npix = dirty.shape[0]
    t0 = time.perf_counter()
    data = learned.make_training_set(dev, n_patches=learn["patches"])
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = learned.UNet(dev, seed=0)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e[0].record()
    losses = learned.train(net, data, steps=learn["steps"], batch=learn["batch"], lr=1e-3, warmup=100,
                           log_every=max(1, learn["steps"] // 10))
    e[1].record()
    torch.cuda.synchronize()
    t_train = e[0].elapsed_time(e[1]) / 1e3
    training = {"patches": len(data), "coverages": data.info["coverages"], "skies": data.info["skies"],
                "data_s": t_data, "steps": learn["steps"], "batch": learn["batch"], "train_s": t_train,
                "train_tflops": learn["steps"] * learn["batch"] * learned.flops(training=True) / t_train / 1e12,
                "loss": losses}
    del data
    torch.cuda.empty_cache()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record()
    psf, peak = learned.psf_patch(plan.grid(None))
    prop = learned.Proposer(net, npix)
    res = learned.solve(plan.gram, dirty, lam, 1.0 / lmax, prop, psf, peak, max_iterations + 1, q0=0.5 * q,
                        events=True)
    ev[1].record()
    torch.cuda.synchronize()
    x, gx, applies, st = res
    mis = res.misfits.cpu().numpy()
    first = {}
    trajectory = []
    for k, e in res.events:
        r = float(np.sqrt(max(2.0 * mis[k], 0.0) / (2 * nvis)))
        if k % 20 == 0:
            trajectory.append([k, r])
        for name, level in (("plain", plain_rms), ("target", target)):
            if r <= level and name not in first:
                first[name] = (k, e)
    rms = float(np.sqrt(max(2.0 * mis[applies], 0.0) / (2 * nvis)))
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    prop(dirty, psf, 1.0 / peak)
    p1.record()
    torch.cuda.synchronize()
    t_plain = t_shared + ev[0].elapsed_time(first["plain"][1]) / 1e3 if "plain" in first else None
    t_target = t_shared + ev[0].elapsed_time(first["target"][1]) / 1e3 if "target" in first else None
    return {"network": "U-Net 32/64/128/256 channels, bf16 weights, f32 accumulation, 256^2 residual + PSF patches",
            "training": training, "proposal_ms": p0.elapsed_time(p1), "proposal_patches": prop.batch,
            "proposal_tflops": prop.batch * learned.flops() / p0.elapsed_time(p1) / 1e9,
            "solve": "FISTA with a proposal every 40 iterations from the first, split into a 4-pixel Gaussian "
                     "low-pass part and the rest, each scaled by the exact minimiser of the misfit (exact gridder)",
            "time_to_plain_final_rms_s": t_plain, "iterations_to_plain_final_rms": first.get("plain", (None,))[0],
            "plain_time_to_final_rms_s": plain_time,
            "speedup_vs_plain": plain_time / t_plain if t_plain else None,
            "time_to_target_s": t_target, "iterations_to_target": first.get("target", (None,))[0],
            "applies": applies, "final_rms": rms, "rms_trajectory": trajectory,
            "model_rel_error": float((x - sky).norm() / sky.norm()), "proposals": st["proposals"],
            "accepted": st["accepted"], "first_step": st["steps"][0] if st["steps"] else None,
            "solve_s": ev[0].elapsed_time(ev[1]) / 1e3, "conv3_kernels": conv3_kernels(dev)}


# ------------------------------------------------------------------ MSv4 ingest


def run_msv4(threads=None):
    """The MSv4 reader feeding the gridder (rang.msv4): a processing set of
    the 16.5 M-visibility workload's shape (64 antennas, 128 integrations,
    64 channels, 4 linear correlations; noise visibilities, 5 % flags,
    random weights) written to local disk as xradio stores it (Blosc/LZ4
    byte-shuffled data in chunks of 8 integrations and 1 MiB blocks, zstd
    coordinates), then read back: the chunks decoded on all host threads,
    the rows in the reference's layout, Stokes I on the GPU and vis2dirty
    (1024^2 at 1.5 arcsec, epsilon 1e-5) through the C ABI, each timed."""
    from rang import gridder, msv4

    wl = synth.WORKLOADS["ms2dirty 16.5M vis 1024^2"]
    ntime, nchan, nant = wl["ntime"], wl["nchan"], 64
    a1, a2 = np.triu_indices(nant, 1)
    nbl = len(a1)
    rng = np.random.default_rng(5)
    shape = (ntime, nbl, nchan, 4)
    vis = np.empty(shape, np.complex64)
    vis.real = rng.standard_normal(shape, np.float32)
    vis.imag = rng.standard_normal(shape, np.float32)
    part = {"time": 1.6e9 + 8.0 * np.arange(ntime), "frequency": synth.channels(nchan),
            "polarization": ["XX", "XY", "YX", "YY"], "antenna_name": [f"m{i:03d}" for i in range(nant)],
            "antenna1": a1, "antenna2": a2, "VISIBILITY": vis, "FLAG": rng.random(shape, np.float32) < 0.05,
            "WEIGHT": rng.uniform(0.5, 1.5, shape).astype(np.float32),
            "UVW": synth.uvw_tracks(nant=nant, ntime=ntime).reshape(ntime, nbl, 3)}
    raw = sum(part[k].nbytes for k in ("VISIBILITY", "FLAG", "WEIGHT", "UVW"))
    with tempfile.TemporaryDirectory() as tmp:
        t0 = time.perf_counter()
        root = msv4.write_processing_set(Path(tmp) / "ps.zarr", {"obs_0": part}, time_chunk=8, blocksize=1 << 20)
        t_write = time.perf_counter() - t0
        stored = sum(f.stat().st_size for f in root.rglob("*") if f.is_file())
        del part, vis
        t0 = time.perf_counter()
        p = msv4.open_processing_set(root).partition("obs_0")
        for var in ("VISIBILITY", "FLAG", "WEIGHT", "UVW"):
            p._read(var)
        t_decode = time.perf_counter() - t0
        t0 = time.perf_counter()
        rows = p.rows()
        t_rows = time.perf_counter() - t0
        t0 = time.perf_counter()
        g = msv4.gridder_inputs(p, rows)
        t_stokes = time.perf_counter() - t0
        cell = wl["cell_arcsec"] * synth.ARCSEC
        t0 = time.perf_counter()
        dirty = gridder.vis2dirty(uvw=g["uvw"], freq=g["freq"], vis=g["vis"], wgt=g["wgt"], mask=g["mask"],
                                        npix_x=wl["npix"], npix_y=wl["npix"], pixsize_x=cell, pixsize_y=cell,
                                        epsilon=1e-5)
        t_grid = time.perf_counter() - t0
    nvis = g["vis"].size
    total = t_decode + t_rows + t_stokes + t_grid
    return {"store": f"{ntime} integrations x {nbl} baselines x {nchan} channels x 4 correlations, "
                     "Blosc/LZ4 byte shuffle, chunks of 8 integrations, 1 MiB blocks",
            "raw_bytes": int(raw), "stored_bytes": int(stored), "write_s": t_write,
            "decode_s": t_decode, "decode_gb_per_s": raw / t_decode / 1e9, "threads": os.cpu_count(),
            "rows_s": t_rows, "stokes_i_s": t_stokes, "vis2dirty_s": t_grid, "stokes_i_visibilities": int(nvis),
            "store_to_dirty_s": total, "store_to_dirty_mvis_per_s": nvis / total / 1e6,
            "dirty_finite": bool(np.isfinite(dirty).all())}


# ------------------------------------------------------------------ imaging weights


def run_imaging_weights(wl, uvw_np, freq, mask, args):
    """WSClean Briggs weights (robust 0.5, rank filter 3 over 16 cells) of
    every sample of the workload, the image's padded size and pixel scale,
    with the flags as zero weights: through the C ABI binding with pinned,
    caller-owned host arrays (copies included, as for the gridder's e2e),
    against the oracle on the CPU sample's integrations."""
    import torch

    from rang import core, weighting

    nrow, nchan = uvw_np.shape[0], freq.size
    wave = weighting.wavelengths(freq)
    size = weighting.padded_size(wl["npix"])
    scale = wl["cell_arcsec"] * synth.ARCSEC
    w_h = torch.empty((nrow, nchan), dtype=torch.float32, pin_memory=True)
    w_h.copy_(mask.to(torch.float32))
    w_np = w_h.numpy()
    sel = np.ones(nrow, np.uint8)
    kw = dict(mode="briggs", robust=0.5, width=size, height=size, pixel_scale=scale, rank_filter=(3.0, 16))
    out_h = torch.empty((nrow, nchan), dtype=torch.float32, pin_memory=True)
    out_np, sums = out_h.numpy(), np.zeros(4)
    ext = core.extension()

    def call():
        st = ext.imaging_weights(nrow, nchan, uvw_np, wave, w_np, sel, 2, 0.5, size, size, scale, scale, 1.0, 3.0, 16,
                                 out_np, None, sums)
        assert st == 0, ext.wgridder_last_error()

    for _ in range(2):
        call()
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        call()
        times.append(time.perf_counter() - t0)
    t = min(times)
    out = {"samples": nrow * nchan, "gpu_e2e_ms": 1e3 * t, "gpu_e2e_msamples_per_s": nrow * nchan / t / 1e6,
           "h2d_bytes": int(w_np.nbytes + uvw_np.nbytes), "d2h_bytes": int(w_np.nbytes)}
    if not args.no_cpu:
        oracle = _oracle()
        rows, nt = sample_rows(wl["ntime"], args.cpu_stride)
        t0 = time.perf_counter()
        oracle.imaging_weights(uvw_np[rows], wave, w_np[rows], sel[rows], **kw)
        tc = time.perf_counter() - t0
        out["cpu_oracle"] = {"samples": rows.size * nchan, "ms": 1e3 * tc,
                             "msamples_per_s": rows.size * nchan / tc / 1e6, "cores": 1, "kind": "port",
                             "sample": f"every {args.cpu_stride}th integration ({nt} of {wl['ntime']})"}
    return out


# ------------------------------------------------------------------ accuracy and configuration 1


def border_interior(x, ref):
    """(border, interior, rms) of x - ref over max |ref|: L-inf over the
    outer two pixels of the image, L-inf over the pixels eight or more in
    from the edge, and the RMS over the whole image (the reference's edge
    protocol, research/df2-wgridder-speed.md:446-487)."""
    err = np.abs(np.asarray(x, np.float64) - ref)
    peak = float(np.abs(ref).max())
    inner = np.zeros(err.shape, bool)
    inner[8:-8, 8:-8] = True
    outer = np.ones(err.shape, bool)
    outer[2:-2, 2:-2] = False
    return (float(err[outer].max() / peak), float(err[inner].max() / peak),
            float(np.sqrt(np.mean(err * err)) / peak))


def vis_errors(v, ref):
    """(L-inf, RMS) of the visibilities v - ref over max |ref|."""
    err = np.abs(np.asarray(v, np.complex128) - ref)
    peak = float(np.abs(ref).max())
    return float(err.max() / peak), float(np.sqrt(np.mean(err * err)) / peak)


# The gridding methods of the single-precision path (rang_b200_wgridder_set_method).
METHODS = (("int8", 3), ("tf32x3", 1), ("bf16x3", 2), ("fp32", 0))


def run_accuracy(dev, ext, wl, uvw, uvw_np, freq, vis, mask, common, args):
    """Every gridding method against the oracle's FP64 run, and its time at
    the full size.

    Errors, on every `cpu_stride`-th integration of the workload's own data
    (the same uv extent, w range and plan): the dirty image of the data, and
    the visibilities of one fixed image (the oracle's FP64 dirty image,
    rounded to float32), each against the oracle in float64 at epsilon 1e-7,
    with the border apart from the interior. Times: one plan + grid and one
    plan + degrid of the whole workload per method, after a warm-up, the
    best of two. The single-precision kernels stop at epsilon 8.1e-7, so
    1e-7 runs in double precision. Degridding has one single-precision
    kernel for every method."""
    import torch

    from rang import gridder, wgrid_torch

    oracle = _oracle()
    oracle.set_threads(os.cpu_count() or 1)
    rows, nt = sample_rows(wl["ntime"], args.cpu_stride)
    ridx = torch.from_numpy(rows).to(dev)
    s_vis = vis.index_select(0, ridx).cpu().numpy()
    s_mask = mask.index_select(0, ridx).cpu().numpy()
    npix, cell = common["npix_x"], common["pixsize_x"]
    kw = dict(uvw=np.ascontiguousarray(uvw_np[rows]), freq=freq, mask=s_mask, pixsize_x=cell, pixsize_y=cell)
    t0 = time.perf_counter()
    d_ref = oracle.vis2dirty(vis=s_vis.astype(np.complex128), npix_x=npix, npix_y=npix, epsilon=1e-7, **kw)
    img = d_ref.astype(np.float32)
    v_ref = oracle.dirty2vis(dirty=img.astype(np.float64), epsilon=1e-7, **kw)
    t_oracle = time.perf_counter() - t0
    cases = [(e, name, code, True) for e in (1e-5, 1e-6) for name, code in METHODS]
    cases += [(1e-5, "fp64", 3, False), (1e-7, "fp64", 3, False)]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    methods = []
    for eps_m, name, code, single in cases:
        ext.wgridder_set_method(code)
        d = gridder.vis2dirty(vis=s_vis if single else s_vis.astype(np.complex128), npix_x=npix, npix_y=npix,
                              epsilon=eps_m, **kw)
        v = gridder.dirty2vis(dirty=img if single else img.astype(np.float64), epsilon=eps_m, **kw)
        b, i, r = border_interior(d, d_ref)
        vl, vr = vis_errors(v, v_ref)
        entry = {"method": name, "precision": "f32" if single else "f64", "epsilon": eps_m,
                 "dirty_border_linf": b, "dirty_interior_linf": i, "dirty_rms": r, "vis_linf": vl, "vis_rms": vr}
        del d, v
        vin = vis if single else vis.to(torch.complex128)
        iin = torch.from_numpy(img).to(dev) if single else torch.from_numpy(img).to(dev, torch.float64)
        best = [float("inf"), float("inf")]
        for rep in range(3):  # the first is a warm-up; the best of the other two is kept
            torch.cuda.synchronize()
            if rep == 1:
                ext.wgridder_profile_read()
                ext.wgridder_profile(1)
            ev[0].record()
            pa = wgrid_torch.DevicePlan(uvw, freq, vis=vin, mask=mask, epsilon=eps_m, single=single, **common)
            dm = pa.grid(vin, scanned=True)
            ev[1].record()
            pb = wgrid_torch.DevicePlan(uvw, freq, mask=mask, epsilon=eps_m, single=single, **common)
            vm = pb.degrid(iin)
            ev[2].record()
            torch.cuda.synchronize()
            supp = pa.info["supp"]
            pa.close()
            pb.close()
            if rep > 0:
                best = [min(best[0], ev[0].elapsed_time(ev[1])), min(best[1], ev[1].elapsed_time(ev[2]))]
            del dm, vm
        ext.wgridder_profile(0)
        prof = ext.wgridder_profile_read()
        entry.update({"supp": int(supp), "vis2dirty_ms": best[0], "dirty2vis_ms": best[1],
                      "stages_per_round_trip": {k: [v[0] / 2, round(v[1] / 2, 3)] for k, v in prof.items() if v[0]},
                      "stages_note": "[launches, ms] per plan + grid + plan + degrid"})
        methods.append(entry)
        del vin, iin
    ext.wgridder_set_method(3)
    # The methods on sparse data, where the split error of a single footprint
    # does not average away: the dirty image of one and of eight visibilities
    # (seeded baselines up to 2 km, 1 GHz, 256^2 at 4 arcsec) against the FP64
    # direct Fourier transform.
    srng = np.random.default_rng(11)
    sparse = []
    for nsparse in (1, 8):
        suvw = srng.uniform(-2000.0, 2000.0, size=(nsparse, 3)) * np.array([1.0, 1.0, 0.2])
        svis = srng.standard_normal((nsparse, 1)) + 1j * srng.standard_normal((nsparse, 1))
        px = 4.0 * np.pi / 648000.0
        skw = dict(uvw=suvw, freq=np.array([1.0e9]), npix_x=256, npix_y=256, pixsize_x=px, pixsize_y=px)
        ref = oracle.dft_dirty(suvw, np.array([1.0e9]), svis, 256, 256, px, px)
        for eps_m in (1e-5, 1e-6):
            entry = {"visibilities": nsparse, "epsilon": eps_m}
            for name, code in METHODS:
                ext.wgridder_set_method(code)
                dm = gridder.vis2dirty(vis=svis.astype(np.complex64), epsilon=eps_m, **skw)
                entry[name + "_dirty_linf"] = float(np.abs(dm - ref).max() / np.abs(ref).max())
            sparse.append(entry)
    ext.wgridder_set_method(3)
    return {"reference": "the oracle's FP64 run at epsilon 1e-7 on the sample; errors over the reference's peak",
            "sample": sample_text(wl, args.cpu_stride, nt, s_vis.size), "oracle_s": t_oracle,
            "methods": methods, "methods_sparse": sparse,
            "methods_sparse_reference": "FP64 direct Fourier transform"}


def run_config1(dev, args):
    """The 16.5 M-visibility configuration: 64 antennas x 128 integrations x 64
    channels, 50 point sources plus noise (sigma 0.1), unit weights, no flags,
    1024^2 at 1.5 arcsec, epsilon 1e-5, f32 and f64. The GPU's vis2dirty
    through the host-array API (copies included) and on device-resident
    inputs, each the median of five after two warm-ups, with the output's
    SHA256 over the repeats; the errors against the oracle's FP64 run at
    epsilon 1e-7 (border apart); and the CPU oracle as the reference's
    harness runs it, beside it."""
    import torch

    from rang import gridder, wgrid_torch

    wl = synth.WORKLOADS[CONFIG1]
    npix, cell = wl["npix"], wl["cell_arcsec"] * synth.ARCSEC
    uvw_np = synth.uvw_tracks(nant=64, ntime=wl["ntime"], tint=8.0, dec_deg=-30.0, seed=7)
    freq = synth.channels(wl["nchan"])
    sky = synth.point_sky(npix, nsrc=50, seed=11)
    kw = dict(uvw=uvw_np, freq=freq, pixsize_x=cell, pixsize_y=cell)
    model = gridder.dirty2vis(dirty=sky, epsilon=1e-9, **kw)
    rng = np.random.default_rng(101)
    vis = (model + 0.1 * (rng.standard_normal(model.shape) + 1j * rng.standard_normal(model.shape))).astype(
        np.complex64)
    del model
    nvis = vis.size
    uvw = torch.from_numpy(uvw_np).to(dev)
    common = dict(npix_x=npix, npix_y=npix, pixsize_x=cell, pixsize_y=cell)
    out = {"configuration": "64 antennas x 128 integrations x 64 channels (16,515,072 visibilities), 50 point "
                            "sources + noise sigma 0.1, unit weights, no flags, 1024^2 at 1.5 arcsec",
           "gpu": []}
    images = {}
    for single, eps in ((True, 1e-5), (False, 1e-5), (False, 1e-7)):
        hv = vis if single else vis.astype(np.complex128)
        walls, hashes = [], set()
        for rep in range(7):
            t0 = time.perf_counter()
            d = gridder.vis2dirty(vis=hv, npix_x=npix, npix_y=npix, epsilon=eps, **kw)
            if rep >= 2:
                walls.append(time.perf_counter() - t0)
                hashes.add(sha256(d))
        images[(single, eps)] = d
        dv = torch.from_numpy(hv).to(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        times = []
        for rep in range(7):
            ev[0].record()
            p = wgrid_torch.DevicePlan(uvw, freq, vis=dv, epsilon=eps, single=single, **common)
            p.grid(dv, scanned=True)
            ev[1].record()
            torch.cuda.synchronize()
            p.close()
            if rep >= 2:
                times.append(ev[0].elapsed_time(ev[1]) / 1e3)
        del dv
        w, t = statistics.median(walls), statistics.median(times)
        out["gpu"].append({"precision": "f32" if single else "f64", "epsilon": eps,
                           "e2e_s": w, "e2e_mvis_per_s": nvis / w / 1e6,
                           "h2d_bytes": int(hv.nbytes + uvw_np.nbytes + freq.nbytes), "d2h_bytes": int(d.nbytes),
                           "device_s": t, "device_mvis_per_s": nvis / t / 1e6,
                           "dirty_sha256": sorted(hashes)[0], "identical_over_repeats": len(hashes) == 1})
    if not args.no_cpu:
        oracle = _oracle()
        oracle.set_threads(os.cpu_count() or 1)
        t0 = time.perf_counter()
        ref = oracle.vis2dirty(vis=vis.astype(np.complex128), npix_x=npix, npix_y=npix, epsilon=1e-7, **kw)
        out["oracle_fp64_s"] = time.perf_counter() - t0
        for g in out["gpu"]:
            b, i, r = border_interior(images[(g["precision"] == "f32", g["epsilon"])], ref)
            g.update({"vs_oracle_fp64_1e-7": {"border_linf": b, "interior_linf": i, "rms": r}})
        with tempfile.TemporaryDirectory() as tmp:
            path = Path(tmp) / "config1.npz"
            np.savez(path, uvw=uvw_np, freq=freq, vis=vis, ntime=wl["ntime"], npix=npix, cell=cell)
            cpu = cpu_protocol(path)
        out["cpu"] = cpu
        allth = {r["precision"]: r for r in cpu["runs"] if r["sample"] == "the whole configuration"}
        for g in out["gpu"]:
            c = allth.get(g["precision"]) if g["epsilon"] == 1e-5 else None
            if c:
                g["e2e_vs_cpu_all_threads"] = g["e2e_mvis_per_s"] / c["mvis_per_s"]
    return out


# ------------------------------------------------------------------ GPU


def run_b200(args):
    import torch

    from rang import core, wgrid_torch

    world, rank, local = replica_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    ext = core.extension()
    wl = synth.WORKLOADS[args.workload]
    npix, cell, eps = wl["npix"], wl["cell_arcsec"] * synth.ARCSEC, args.epsilon

    uvw_np, freq, sky = make_observation(wl)
    nrow, nchan = uvw_np.shape[0], freq.size
    nvis = nrow * nchan
    uvw = torch.from_numpy(uvw_np).to(dev)
    common = dict(npix_x=npix, npix_y=npix, pixsize_x=cell, pixsize_y=cell)

    # Synthetic data on the device: the point sky predicted by the degridder
    # (float32, epsilon 1e-6), seeded noise and flags.
    gen = wgrid_torch.DevicePlan(uvw, freq, epsilon=1e-6, single=True, **common)
    vis = gen.degrid(torch.from_numpy(sky).to(dev, torch.float32))
    gen.close()
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    for a in range(0, nrow, 65536):
        b = min(nrow, a + 65536)
        vis[a:b] += 0.1 * torch.randn((b - a, nchan), dtype=torch.complex64, device=dev, generator=g) * np.sqrt(2.0)
    mask = (torch.rand((nrow, nchan), device=dev, generator=g) >= wl["flag"]).to(torch.uint8)
    single = args.precision == "f32"
    svis = vis if single else vis.to(torch.complex128)
    torch.cuda.synchronize()

    # Between phases and legs (outside every timed region) the library's
    # cached device buffers of the previous phase go back to the device: the
    # next is a workload of other shapes (here the data's making at epsilon
    # 1e-6), partly on PyTorch's allocator, which cannot use memory the
    # library holds.
    def release_cached():
        torch.cuda.synchronize()
        assert ext.wgridder_release_cached() == 0, ext.wgridder_last_error()
        torch.cuda.empty_cache()

    release_cached()

    def step():
        p1 = wgrid_torch.DevicePlan(uvw, freq, vis=svis, mask=mask, epsilon=eps, single=single, **common)
        dirty = p1.grid(svis, scanned=True)
        p2 = wgrid_torch.DevicePlan(uvw, freq, mask=mask, epsilon=eps, single=single, **common)
        out = p2.degrid(dirty)
        return p1, p2, dirty, out

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        keep = step()
        keep[0].status()
        del keep
    barrier()
    stream = torch.cuda.current_stream(dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local)
    clocks.start()
    n0 = ext.wgridder_launch_count()
    ext.wgridder_profile_read()
    ext.wgridder_profile(1)
    last = None
    torch.cuda.nvtx.range_push("timed")
    start.record(stream)
    for _ in range(args.steps):
        last = None  # releases the previous step's plans and outputs
        last = step()
    end.record(stream)
    torch.cuda.nvtx.range_pop()
    barrier()
    ext.wgridder_profile(0)
    prof = ext.wgridder_profile_read()
    launches = ext.wgridder_launch_count() - n0
    clk = clocks.stop()
    plan_info = last[0].info
    dirty32, vis32 = last[2], last[3]
    last[0].status()
    last[1].status()
    last = None
    ms = max_over_ranks(start.elapsed_time(end), dist, dev)
    value = job_rate(world, nvis, args.steps, ms / 1e3)

    # Dominant kernel and its roofline (algorithmic bytes per launch).
    hbm, peak_kind = peaks()
    nact = int(plan_info["nvis"])
    nplanes = max(int(plan_info["nplanes"]), 1)
    supp = int(plan_info["supp"])
    # The algorithmic bytes of one direction, per unit as the hot-path survey
    # counts them: every visibility's value (8 B; 16 in double), weight (4 B)
    # and flag (1 B) read (or the value written, degridding), 24 B of uvw per
    # row, each plane's grid written and read once (2 x 8 B per cell; 16 in
    # double) and the image (4 B per pixel; 8 in double).
    vb = 8 if single else 16
    per_direction = (nvis * (vb + 4 + 1) + nrow * 24 + nplanes * plan_info["nu"] * plan_info["nv"] * vb * 2
                     + npix * npix * vb // 2)
    alg = {"grid": per_direction, "degrid": per_direction}
    dom = max(("grid", "degrid"), key=lambda k: prof[k][1])
    kernel = ({"grid": "k_grid_i8", "degrid": "k_degrid_h"} if single else {"grid": "k_grid_f64", "degrid": "k_degrid"})[dom]
    dom_launches, dom_ms = prof[dom]
    per_launch_s = dom_ms / max(dom_launches, 1) / 1e3
    achieved = alg[dom] / per_launch_s / 1e9
    total_prof = sum(v[1] for v in prof.values())
    # Useful arithmetic: S^3 complex-by-real multiply-adds per visibility
    # (4 flops each), against the FP32 CUDA-core FMA peak at the maximum SM
    # clock; the HBM bound and this bound together are the kernel's roofline.
    flops = 4.0 * supp**3 * nact
    fp32_peak = 148 * 128 * 2 * 1965e6 / 1e12
    cap = DRAM_CAPTURE.get(kernel)
    traffic = cap[0] * nact / cap[1] if cap and args.epsilon == 1e-5 else None
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": peak_kind,
                "traffic": traffic,
                "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on the "
                                   f"{PROFILE_CASE} case ({cap[0] / 1e9:.2f} GB for {cap[1]} active visibilities), "
                                   f"scaled by the active visibilities") if traffic else None,
                "algorithmic_bytes_per_launch": alg[dom], "avg_launch_ms": per_launch_s * 1e3,
                "share_of_step": dom_ms / max(total_prof, 1e-9),
                "compute": {"useful_tflop_per_launch": flops / 1e12, "achieved_tflops": flops / per_launch_s / 1e12,
                            "fp32_fma_peak_tflops": fp32_peak, "peak_kind": "nominal (148 SMs x 128 FMA x 1965 MHz)",
                            "frac": flops / per_launch_s / 1e12 / fp32_peak}}

    # End to end through the C ABI with pinned host arrays.
    release_cached()
    e2e = None
    pinned = None
    reason = "pinned host memory refused on another rank"
    if not args.no_e2e:
        # Each rank pins about 18 GB of host memory; if any rank cannot, every
        # rank skips this leg together (its timing is a collective).
        try:
            cdt, rdt = (torch.complex64, torch.float32) if single else (torch.complex128, torch.float64)
            pinned = [torch.empty((nrow, nchan), dtype=cdt, pin_memory=True),
                      torch.empty((nrow, nchan), dtype=torch.uint8, pin_memory=True),
                      torch.empty((nrow, nchan), dtype=cdt, pin_memory=True),
                      torch.empty((npix, npix), dtype=rdt, pin_memory=True)]
        except RuntimeError as exc:
            pinned = None
            reason = f"pinned host memory: {exc}".splitlines()[0][:200]
        if not all_ranks(pinned is not None, dist, dev):
            pinned = None
            e2e = {"unavailable": reason}
    if pinned is not None:
        from rang.gridder import options_list

        vis_h, mask_h, out_h, dirty_h = pinned
        pinned = None
        vis_h.copy_(svis)
        mask_h.copy_(mask)
        vis_np, mask_np, out_np, dirty_np = vis_h.numpy(), mask_h.numpy(), out_h.numpy(), dirty_h.numpy()
        opts = options_list(npix, npix, cell, cell, eps, {})
        info = np.empty(14)

        v2d = ext.wgridder_vis2dirty_f32 if single else ext.wgridder_vis2dirty_f64
        d2v = ext.wgridder_dirty2vis_f32 if single else ext.wgridder_dirty2vis_f64
        real = np.float32 if single else np.float64

        def e2e_step():
            st = v2d(opts, uvw_np, freq, vis_np, None, None, mask_np, dirty_np, None, info)
            assert st == 0, ext.wgridder_last_error()
            st = d2v(opts, uvw_np, freq, dirty_np, None, mask_np, out_np.view(real), info)
            assert st == 0, ext.wgridder_last_error()

        for _ in range(args.warmup):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        te = max_over_ranks(time.perf_counter() - t0, dist, dev)
        h2d = 2 * (uvw_np.nbytes + freq.nbytes + mask_np.nbytes) + vis_np.nbytes + dirty_np.nbytes
        d2h = dirty_np.nbytes + out_np.nbytes
        e2e = {"value": job_rate(world, nvis, args.steps, te), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * te / args.steps}
        if args.trace_e2e and rank == 0:  # untimed: the copies' and kernels' timeline of one step
            from torch.profiler import ProfilerActivity, profile

            with profile(activities=[ProfilerActivity.CUDA]) as tprof:
                e2e_step()
            tprof.export_chrome_trace(args.trace_e2e)
        del vis_h, mask_h, out_h, dirty_h

    release_cached()
    accuracy = None
    if world == 1 and not args.no_accuracy:
        accuracy = run_accuracy(dev, ext, wl, uvw, uvw_np, freq, vis, mask, common, args)

    release_cached()
    fst = None
    if world == 1 and not args.no_fista:
        learn = None if args.no_learned else {"patches": args.learned_patches, "steps": args.learned_steps, "batch": 16}
        fst = run_fista(dev, learn=learn, cap=args.fista_cap)

    # The CPU oracle on a bounded sample of the same workload (one process,
    # all host threads: one warm-up and three timed round trips).
    cpu = None
    if world == 1 and not args.no_cpu:
        oracle, suvw, sfreq, svis, smask, nt = cpu_sample(wl, args.cpu_stride)
        threads = oracle.set_threads(os.cpu_count() or 1)
        cpu_round_trip(oracle, suvw, sfreq, svis, smask, npix, cell, eps)
        load = os.getloadavg()
        times = [cpu_round_trip(oracle, suvw, sfreq, svis, smask, npix, cell, eps) for _ in range(3)]
        t = statistics.median(times)
        cpu = {"value": svis.size / t / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": sample_text(wl, args.cpu_stride, nt, svis.size) + ", median of three round trips",
               "cpu_model": cpu_model(), "simd": oracle.simd_level(), "load_avg_before": list(load),
               "step_s": [round(x, 4) for x in times], "ns_per_vis": 1e9 * t / svis.size}
        del svis, smask
        # The sample pays the full grid's FFTs, a fixed cost, for a fraction of
        # the visibilities. A second sample of twice the integrations separates
        # the two: t = a + b n, and the whole workload would take a + b N.
        if args.cpu_stride >= 2:
            _, uv2, fr2, vis2, mask2, nt2 = cpu_sample(wl, args.cpu_stride // 2)
            t2 = cpu_round_trip(oracle, uv2, fr2, vis2, mask2, npix, cell, eps)
            n1, n2 = NBL * nt * wl["nchan"], vis2.size
            b = (t2 - t) / (n2 - n1) if n2 > n1 else float("nan")
            a = t - b * n1
            cpu["two_sample_model"] = {
                "samples": [[n1, t], [n2, t2]], "fixed_s": a, "ns_per_vis": 1e9 * b,
                "whole_workload_mvis_per_s": nvis / (a + b * nvis) / 1e6 if a + b * nvis > 0 else None,
                "note": "fixed cost (plan, FFTs of the full grid) and per-visibility cost fitted to two samples"}
            del vis2, mask2

    release_cached()
    config1 = None
    if world == 1 and not args.no_config1:
        config1 = run_config1(dev, args)

    release_cached()
    weights_leg = None
    if world == 1 and not args.no_weights:
        weights_leg = run_imaging_weights(wl, uvw_np, freq, mask, args)

    msv4_leg = None
    if world == 1 and not args.no_msv4:
        msv4_leg = run_msv4()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "config": workload_config(wl, args.workload, eps, world, args.precision),
            "plan": dict({k: plan_info[k] for k in ("kernel_index", "supp", "nu", "nv", "nplanes")}, active=nact),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk, "accuracy": accuracy, "config1": config1, "fista": fst, "imaging_weights": weights_leg,
            "msv4_ingest": msv4_leg,
            "stages_ms": {k: round(v[1], 3) for k, v in prof.items() if v[0]},
        }
        print(json.dumps(line, default=_plain), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl != "reference" and args.cpu_stride is None:
        args.cpu_stride = 64
    if args.cpu_worker:
        cpu_worker(args.cpu_worker)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
