"""Benchmark: Mvoxels/s of voronoi_otsu_labeling + statistics_of_labelled_pixels.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload lightsheet|nuclei|lightsheet_dense|blobs2d|batch|served|published]

Default workload (N=1): the light-sheet volume, uint16 512x1024x1024 (30000
ellipsoidal cells, slow sinusoidal background, Poisson noise, seed 2), the
largest single-GPU configuration; one step = voronoi_otsu_labeling
(spot_sigma=2, outline_sigma=2) followed by statistics_of_labelled_pixels on
the same intensity volume.  Data are synthetic (seeded generator with the
workload's shapes and value distributions).

  value   device-resident throughput: the input already in HBM, every step's
          device time measured with CUDA events on the launching stream; the
          1 GiB input and 2 GiB of labels exceed the 126 MB L2.
  e2e     the same step end to end through the public serving API
          (SegmentationServer): every step uploads the uint16 volume from
          pinned host memory and returns its label image (into a pinned host
          buffer) and its statistics table; steps overlap (upload, compute and
          download on their own streams), the time runs from the first upload
          to the last result on the host.  e2e_per_call is the same with one
          synchronous call after another (push, the two ops, pull).
  roofline   the dominant kernel stage, timed live with the library's stage
          events inside the timed steps; achieved = algorithmic bytes / time.
  pipeline_roofline   the whole step against 36 B/voxel (read the source and
          write the blur, read the blur for the histogram, read source + blur
          and write mask and seeds, read them and write uint32 labels, two
          statistics reads of labels + intensity).
  served_vs_per_call   the serving form against the plain per-call loop on a
          Poisson trace of mixed request sizes (p50/p95/p99 latency,
          Mvoxels/s), and both at saturation (all requests waiting at once).
  cpu_baseline   the CPU oracle (C/OpenMP restatement of the reference's
          algorithm, all host threads) on a bounded sample of the same workload.

--impl reference times the reference's algorithm on the host cores on the
same workload (the whole volume every step): the reference itself cannot run
here (pyopencl, a CPU OpenCL runtime and its clij-opencl-kernels sources are
absent), so its C restatement (oracle/) runs instead, with every host thread.
Both arms print the same `config`.

Multi-GPU: replicas (one process per GPU, each runs the full workload; no
collective on the data path; timing = max over ranks).
"""
import argparse
import ctypes
import json
import os
import statistics as st
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mvoxels/s voronoi_otsu_labeling; p50/p99 latency served vs per-call"
UNIT = "Mvoxels/s"
DEFAULT_WORKLOAD = "lightsheet"

WORKLOADS = {
    "nuclei": dict(desc="nuclei volume uint16 128x512x512 (2000 ellipsoids, PSF (1.5,1,1), Poisson, seed 1): "
                        "voronoi_otsu_labeling(spot_sigma=2, outline_sigma=1) + statistics_of_labelled_pixels",
                   shape=(128, 512, 512), spot=2.0, outline=1.0),
    "lightsheet": dict(desc="light-sheet volume uint16 512x1024x1024 (30000 ellipsoids, sinusoidal background, "
                            "Poisson, seed 2): voronoi_otsu_labeling(spot_sigma=2, outline_sigma=2) + "
                            "statistics_of_labelled_pixels", shape=(512, 1024, 1024), spot=2.0, outline=2.0),
    "lightsheet_slab": dict(desc="light-sheet slab uint16 128x1024x1024 (7500 ellipsoids, sinusoidal background, "
                                 "Poisson, seed 2): voronoi_otsu_labeling(spot_sigma=2, outline_sigma=2) + "
                                 "statistics_of_labelled_pixels (the light-sheet recipe at a quarter of the depth, "
                                 "for profiler captures)", shape=(128, 1024, 1024), spot=2.0, outline=2.0, cells=7500),
    "lightsheet_dense": dict(desc="light-sheet volume uint16 512x1024x1024 (as above): gauss_otsu_labeling("
                                  "outline_sigma=2) (blur, Otsu, connected components of the dense mask) + "
                                  "statistics_of_labelled_pixels", shape=(512, 1024, 1024), spot=None,
                             outline=2.0, op="gauss_otsu"),
    "published": dict(desc="the reference's own published benchmark cases (benchmarks/*.ipynb): "
                           "seeded inputs of the notebooks' shapes and distributions", shape=None,
                      spot=None, outline=None),
    "batch": dict(desc="512 tiles, voxel counts log-uniform between 2D 64x64 and 3D 96x512x512 (2D and 3D "
                       "mixed), Gaussian-blob tiles with U(0.5,5)e-4 blobs/voxel and per-tile seeds (4+i); "
                       "voronoi_otsu_labeling(spot_sigma=3.5, outline_sigma=1) on float32 tiles, uint32 labels",
                  shape=None, spot=3.5, outline=1.0),
    "served": dict(desc="Poisson arrivals at 200 req/s; request volumes uint16 from {512x512, 64x256x256, "
                        "128x512x512, 256x1024x1024} with p {0.4,0.3,0.2,0.1}, blob tiles with per-request "
                        "seeds; 60 GB HBM budget; voronoi_otsu_labeling(spot_sigma=2, outline_sigma=2) + "
                        "statistics_of_labelled_pixels", shape=None, spot=2.0, outline=2.0),
    "blobs2d": dict(desc="2D float32 256x256 blobs (seed 0): voronoi_otsu_labeling(spot_sigma=3.5, "
                         "outline_sigma=1) + statistics_of_labelled_pixels", shape=(256, 256), spot=3.5,
                    outline=1.0),
}


def config_of(name, nvox):
    """The `config` object both arms print for a workload (identical keys)."""
    return {"workload": WORKLOADS[name]["desc"], "voxels_per_step": int(nvox)}


# Algorithmic bytes per voxel of each stage (each input read once, each
# output written once; uint16 source).  Index = stage event interval.
STAGES = ["blur_spot", "detect_maxima", "blur_outline", "minmax_hist_otsu", "threshold_seeds",
          "seed_ccl", "voronoi_growth", None, "stats_pass1", "stats_final1", "stats_pass2",
          "stats_final2"]
ALGO_BYTES = {"blur_spot": 2 + 4, "detect_maxima": 4 + 1, "blur_outline": 2 + 4,
              "minmax_hist_otsu": 4 + 4, "threshold_seeds": 4 + 1 + 1 + 4,
              "voronoi_growth": 1 + 1 + 4, "stats_pass1": 4 + 2, "stats_pass2": 4 + 2}


def algo_bytes(w, labelled_fraction=None):
    """ALGO_BYTES for a workload: with equal spot and outline sigmas the blur
    runs once (its stage carries the min / max) and the maxima are found in
    the seed pass (read T, write the mask and the labels; no spots image, no
    second blur).  The second statistics pass reads the label and intensity
    of labelled voxels only."""
    b = dict(ALGO_BYTES)
    if w.get("spot") is not None and w.get("spot") == w.get("outline"):
        b["threshold_seeds"] = 4 + 1 + 4
        del b["detect_maxima"], b["blur_outline"]
    if labelled_fraction is not None:
        b["stats_pass2"] = (4 + 2) * labelled_fraction
    return b
# The pipeline's compulsory traffic per voxel (the minimal pass structure the
# two global reductions force): read src + write blur 8, read blur for the
# histogram 4, read src + blur and write mask + seeds 10, read mask + seeds
# and write uint32 labels 6, statistics 2 x (labels 4 + intensity 4).
PIPELINE_BYTES_PER_VOXEL = 8 + 4 + 10 + 6 + 8


# DRAM bytes per launch from one ncu capture per kernel (dram__bytes_read.sum +
# dram__bytes_write.sum, or the DRAM bandwidth x the duration of the same
# launch); the captures are summarised in profiles/<kernel>_<workload>.md.
MEASURED_TRAFFIC = {
    "nuclei": {"voronoi_growth": (0.347e9, "voronoi_keys_kernel_nuclei_128x512x512.md"),
               "blur_spot": (67.164e6 + 81.208e6, "blur_fused_kernel_nuclei_128x512x512.md"),
               "blur_outline": (67.155e6 + 81.081e6, "blur_fused_kernel_nuclei_128x512x512.md"),
               "detect_maxima": (135.090e6 + 19.932e6, "maxima_kernel_nuclei_128x512x512.md"),
               },
    # slab captures (128x1024x1024) scaled by 4 to the 512x1024x1024 volume:
    # the same recipe and cell density, traffic in proportion to the voxels
    "lightsheet": {"voronoi_growth": (4 * 1.494e9, "voronoi_keys_kernel_lightsheet_slab_128x1024x1024.md"),
                   "blur_spot": (4 * 0.792e9, "blur_fused_kernel_lightsheet_slab_128x1024x1024.md"),
                   "threshold_seeds": (4 * 1.165e9, "maxima_seeds_kernel_lightsheet_slab_128x1024x1024.md")},
    "lightsheet_slab": {"voronoi_growth": (1.494e9, "voronoi_keys_kernel_lightsheet_slab_128x1024x1024.md"),
                        "blur_spot": (0.792e9, "blur_fused_kernel_lightsheet_slab_128x1024x1024.md"),
                        "threshold_seeds": (1.165e9, "maxima_seeds_kernel_lightsheet_slab_128x1024x1024.md")},
}

# Algorithmic bytes per voxel of a whole gauss_otsu_labeling + statistics step
# (u16 source): blur 2+4, min/max 4, histogram 4, threshold 4+1, CCL of the
# dense mask 1+4, two statistics passes 2 x (4+2).
DENSE_BYTES_PER_VOXEL = 6 + 4 + 4 + 5 + 5 + 12


def cpu_step(f, w):
    """One step of the workload on the oracle (f: float32 host volume)."""
    import oracle
    if w.get("op") == "gauss_otsu":
        lab = oracle.gauss_otsu_labeling(f, w["outline"])
    else:
        lab = oracle.voronoi_otsu_labeling(f, w["spot"], w["outline"])
    oracle.statistics_of_labelled_pixels(f, lab)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_input(name, device=None):
    """The workload's input volume: numpy (nuclei, blobs2d) or a torch uint16
    tensor (light-sheet: generated with torch on the GPU when one is visible,
    so both arms of the benchmark see the same volume)."""
    from pyclesperanto_prototype_b200 import synthetic
    w = WORKLOADS[name]
    if name == "nuclei":
        return synthetic.cached("c2_nuclei_128x512x512_s1", synthetic.nuclei_volume)
    if name == "blobs2d":
        return synthetic.blobs_2d((256, 256), 60, seed=0)
    import torch
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
    vol = synthetic.lightsheet_volume(w["shape"], w.get("cells", 30000), seed=2, device=dev)
    return vol


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of one GPU, sampled every
    `period` seconds through NVML (the fields nvidia-smi reports as
    clocks.sm, clocks.max.sm and clocks_event_reasons.*) from start() to
    stop(); nvidia-smi at 200 ms when NVML is not available."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device_index, period=0.01):
        self.dev = int(device_index)
        self.period = float(period)
        self.samples = []          # (t, sm_mhz, max_mhz, reasons bitmask)
        self.windows = []
        self._stop = threading.Event()
        self.t = None
        self.source = None
        self.proc = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            import pynvml
            h = self._nvml_handle()
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def loop():
                while not self._stop.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((time.perf_counter(), float(sm), float(mx), int(rs)))
                    except Exception:
                        pass
                    self._stop.wait(self.period)
            self.t = threading.Thread(target=loop, daemon=True)
            self.t.start()
            self.source = "nvml every %d ms" % int(self.period * 1e3)
        except Exception:
            self._start_smi()

    def _start_smi(self):
        self.source = "nvidia-smi -lms 200"
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)

            def read():
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for line in self.proc.stdout:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < len(self.FIELDS):
                        continue
                    try:
                        rs = 0
                        for nm, v in zip(names, parts[5:9]):
                            if v.lower() == "active":
                                rs |= self.REASONS[nm]
                        self.samples.append((time.perf_counter(), float(parts[1]), float(parts[2]), rs))
                    except ValueError:
                        continue
            self.t = threading.Thread(target=read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def mark(self, t0, t1):
        """Records a timed window [t0, t1] (perf_counter seconds)."""
        self.windows.append((t0, t1))

    def stop(self):
        self._stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t is not None:
            self.t.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"],
                    "samples": 0}
        inside = [s for s in self.samples if any(a <= s[0] <= b for a, b in self.windows)]
        use = inside if len(inside) >= 5 else self.samples
        reasons = sorted(nm for nm, bit in self.REASONS.items() if any(s[3] & bit for s in use))
        return {"sm_mhz": float(np.median([s[1] for s in use])), "sm_max_mhz": max(s[2] for s in use),
                "reasons": reasons, "samples": len(use), "samples_in_timed_region": len(inside),
                "source": self.source}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(x, world):
    """Max of a host scalar over the ranks (NCCL: through the GPU; gloo: CPU)."""
    import torch
    if world == 1:
        return x
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline_sample(vol, w, reps=2, max_voxels=48 * 1024 * 1024):
    """Oracle on the host cores (all threads); returns (Mvox/s, cores, voxels,
    seconds).  Volumes above max_voxels are sampled as their first z planes."""
    import oracle
    oracle.build()
    cores = oracle.num_threads()
    if vol.ndim == 3 and vol.size > max_voxels:
        vol = vol[:max(1, max_voxels // (vol.shape[1] * vol.shape[2]))]
    f = vol.astype(np.float32)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        cpu_step(f, w)
        ts.append(time.perf_counter() - t0)
    t = min(ts)
    return f.size / t / 1e6, cores, f.shape, t


def e2e_served(pinned_in, w, steps, world, ref_labels=None, slots=3):
    """Throughput through the public serving API: `steps` requests of the
    workload's volume, all waiting at t=0; each uploads the pinned uint16
    volume and returns its label image into a pinned host buffer plus its
    statistics table.  Returns the e2e dict (max over ranks)."""
    import torch
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer
    server = SegmentationServer(budget_bytes=60e9, slots=slots, spot_sigma=w["spot"],
                                outline_sigma=w["outline"])
    outs = [torch.empty(tuple(pinned_in.shape), dtype=torch.uint32).pin_memory() for _ in range(slots)]
    # warm-up: every slot's device buffers allocated before the timed requests
    server.run([Request(-1 - k, pinned_in, 0.0, labels_out=outs[k]) for k in range(slots)], realtime=False)
    torch.cuda.synchronize()
    reqs = [Request(i, pinned_in, 0.0, labels_out=outs[i % slots]) for i in range(steps)]
    barrier(world)
    t0 = time.perf_counter()
    server.run(reqs, realtime=False)
    t = max_over_ranks(time.perf_counter() - t0, world)
    bad = [r.error for r in reqs if not r.ok]
    if bad:
        raise RuntimeError("e2e request failed: " + bad[0])
    nvox = pinned_in.numel()
    L = reqs[-1].num_labels
    out = {"value": round(nvox * world * steps / t / 1e6, 2), "unit": UNIT,
           "h2d_bytes_per_step": int(pinned_in.numel() * pinned_in.element_size()),
           "d2h_bytes_per_step": int(nvox * 4 + 35 * L * 4 + 8), "ms_per_step": round(t / steps * 1e3, 3),
           "steps": steps, "api": "pyclesperanto_prototype_b200.serving.SegmentationServer, %d slots: "
                                  "upload / compute / download of consecutive steps overlap" % slots}
    if ref_labels is not None:
        out["labels_equal_device_run"] = bool(torch.equal(outs[(steps - 1) % slots], ref_labels))
    del server, outs
    torch.cuda.empty_cache()
    return out


def e2e_per_call(pinned_in, w, reps, world, flush):
    """One synchronous public-API call after another: push, the two ops,
    labels to pinned host memory, statistics dict."""
    import torch
    import pyclesperanto_prototype_b200 as cle
    dense = w.get("op") == "gauss_otsu"
    pinned_lab = torch.empty(tuple(pinned_in.shape), dtype=torch.uint32).pin_memory()
    ts = []
    for i in range(reps + 1):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img = cle.push_native(pinned_in)
        if dense:
            lab = cle.gauss_otsu_labeling(img, outline_sigma=w["outline"])
        else:
            lab = cle.voronoi_otsu_labeling(img, spot_sigma=w["spot"], outline_sigma=w["outline"])
        stats = cle.statistics_of_labelled_pixels(img, lab)
        pinned_lab.copy_(lab.tensor, non_blocking=True)
        torch.cuda.synchronize()
        if i:
            ts.append(time.perf_counter() - t0)
        del img, lab
    te = max_over_ranks(st.mean(ts), world)
    nvox = pinned_in.numel()
    return {"value": round(nvox * world / te / 1e6, 2), "unit": UNIT,
            "h2d_bytes_per_step": int(pinned_in.numel() * pinned_in.element_size()),
            "d2h_bytes_per_step": int(nvox * 4 + 35 * len(stats["label"]) * 4 + 8),
            "ms_per_step": round(te * 1e3, 3), "steps": reps}


SERVED_CLASSES = [(512, 512), (64, 256, 256), (128, 512, 512), (256, 1024, 1024)]
SERVED_PROBS = [0.4, 0.3, 0.2, 0.1]


def served_pools(pool_per_class):
    """Pinned uint16 request volumes per size class (blob tiles, per-volume seeds)."""
    import torch
    from pyclesperanto_prototype_b200 import synthetic
    dev = "cuda:%d" % torch.cuda.current_device()
    return {c: [synthetic.blob_tile(c, 2e-4 if len(c) == 3 else 1e-3, seed=5000 + 10 * k + j, device=dev)
                .clamp_(0, 65535).to(torch.int32).to(torch.uint16).cpu().pin_memory()
                for j in range(pool_per_class)] for k, c in enumerate(SERVED_CLASSES)}


def served_trace(rate, duration, pool_per_class, seed=5):
    rng = np.random.default_rng(seed)
    t, trace = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        c = SERVED_CLASSES[rng.choice(len(SERVED_CLASSES), p=SERVED_PROBS)]
        trace.append((t, c, int(rng.integers(pool_per_class))))
    return trace


def _summarize(reqs, vox_of):
    lat = np.array([r.done - r.arrival for r in reqs]) * 1e3
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    vox = sum(vox_of[r.rid] for r in reqs)
    return {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p95_ms": round(float(np.percentile(lat, 95)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3), "mvoxels_per_s": round(vox / span / 1e6, 2),
            "requests": len(reqs), "span_s": round(span, 3)}


def _tables_close(a, b, rtol=1e-5):
    """Statistics tables equal within the parity tolerance (same NaN positions)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if a.shape != b.shape or not np.array_equal(np.isnan(a), np.isnan(b)):
        return False
    m = ~np.isnan(a)
    return bool(np.allclose(a[m], b[m], rtol=rtol, atol=0))


def served_vs_per_call(rate, duration, lanes, pool_per_class=3, closed_requests=120, spot=2.0, outline=2.0,
                       compute_streams=1, express_voxels=8 << 20):
    """The served form against the per-call loop: (1) on a Poisson trace at
    `rate` req/s for `duration` s, (2) at saturation (closed_requests
    requests all waiting at t=0).  Single GPU."""
    import torch
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer, per_call_loop
    pool = served_pools(pool_per_class)
    trace = served_trace(rate, duration, pool_per_class)
    rng = np.random.default_rng(55)
    closed = [(0.0, SERVED_CLASSES[rng.choice(len(SERVED_CLASSES), p=SERVED_PROBS)],
               int(rng.integers(pool_per_class))) for _ in range(closed_requests)]

    def make(tr):
        return [Request(i, pool[c][j], arrival=a) for i, (a, c, j) in enumerate(tr)]

    server = SegmentationServer(budget_bytes=60e9, slots=lanes, compute_streams=compute_streams,
                                express_voxels=express_voxels, spot_sigma=spot, outline_sigma=outline)
    # warm-up: one untimed saturating burst, so the buffer pool holds what the
    # busiest moments need (a device allocation inside a timed run synchronises
    # the GPU)
    server.run(make(closed), realtime=False)
    per_call_loop([Request(i, pool[c][0], arrival=0.0) for i, c in enumerate(SERVED_CLASSES)], spot, outline,
                  realtime=False)
    torch.cuda.synchronize()
    out = {}
    for name, tr, realtime in (("trace", trace, True), ("saturation", closed, False)):
        vox_of = {i: pool[c][j].numel() for i, (a, c, j) in enumerate(tr)}
        served = server.run(make(tr), realtime=realtime)
        plain = per_call_loop(make(tr), spot, outline, realtime=realtime)
        s, p = _summarize(served, vox_of), _summarize(plain, vox_of)
        same = all(a.ok and b.ok and a.num_labels == b.num_labels and _tables_close(a.table, b.table)
                   for a, b in zip(served, plain))
        out[name] = {"served": s, "per_call": p, "results_equal": bool(same),
                     "throughput_ratio": round(s["mvoxels_per_s"] / p["mvoxels_per_s"], 3)}
    out["trace"]["desc"] = ("Poisson arrivals at %g req/s for %g s; request sizes {512x512, 64x256x256, "
                            "128x512x512, 256x1024x1024} with p {0.4,0.3,0.2,0.1}; %d volumes per size class"
                            % (rate, duration, pool_per_class))
    out["saturation"]["desc"] = "%d requests of the same size mix, all waiting at t=0" % closed_requests
    out["served_p99_below_per_call_p50"] = bool(out["trace"]["served"]["p99_ms"] <
                                                out["trace"]["per_call"]["p50_ms"])
    out["form"] = ("served: %d requests in flight, uploads and downloads on copy streams, %d compute "
                   "stream(s), express lane for requests of <= %d voxels, 60 GB budget"
                   % (lanes, compute_streams, express_voxels))
    del server, pool
    torch.cuda.empty_cache()
    return out


def run_b200(args):
    import torch
    import pyclesperanto_prototype_b200 as cle
    from pyclesperanto_prototype_b200 import _lib

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _lib.load()
    w = WORKLOADS[args.workload]
    host = make_input(args.workload, device=dev)
    if isinstance(host, torch.Tensor):
        # generated on the device; a host copy feeds the end-to-end legs
        src = cle.B200Array(host.contiguous())
        host_np = host.cpu().numpy()
    else:
        host_np = host
        src = cle.push_native(host_np)
    nvox = int(np.prod(src.shape))
    stream = torch.cuda.current_stream()
    # between steps a 256 MiB write evicts the 126 MB L2 (the light-sheet
    # inputs exceed it anyway)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    labels = cle.create_labels_like(src)

    dense = w.get("op") == "gauss_otsu"

    # the statistics read the label count the pipeline leaves on the device
    # (cle_statistics_of_labelled_pixels_device_count, as the served form
    # does): no label-maximum pass over the image and no host round trip
    # inside a step; the table is sized for one label per 64 voxels
    stream_ptr = stream.cuda_stream
    if not dense:
        ws_vol = cle._ops.workspaces.get(src)
        count_ptr = lib.cle_workspace_label_count(ws_vol.data_ptr())
        cap = max(1024, nvox // 64)
        table_dev = torch.empty((35, cap), dtype=torch.float32, device=dev)
        sdesc, ldesc = _lib.tensor_desc(src.tensor), _lib.tensor_desc(labels.tensor)
        stats_ws = torch.empty(int(lib.cle_statistics_workspace_bytes(_lib.ref(ldesc), cap)), dtype=torch.uint8,
                               device=dev)

    def step():
        if dense:
            cle.gauss_otsu_labeling(src, labels, outline_sigma=w["outline"])
            L = cle._ops._label_max(labels)
            return cle.statistics_table(src, labels, L), L
        cle._ops._vol(src, labels, w["spot"], w["outline"], check=False)
        _lib.check(lib.cle_statistics_of_labelled_pixels_device_count(
            _lib.ref(sdesc), _lib.ref(ldesc), count_ptr, cap, table_dev.data_ptr(), stats_ws.data_ptr(),
            stats_ws.numel(), stream_ptr), "statistics_of_labelled_pixels")
        return table_dev, None

    # correctness of the loop status once (not timed)
    if not dense:
        cle._ops._vol(src, labels, w["spot"], w["outline"], check=True)
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    lib.cle_profile_enable(3 if args.trace else 1)
    stage_buf = (ctypes.c_float * 16)()
    barrier(world)
    n0 = lib.cle_kernel_launches()
    times, stage_ms = [], []
    t_timed0 = time.perf_counter()
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        table, L = step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        k = lib.cle_profile_stage_ms(stage_buf, 16)
        stage_ms.append([stage_buf[i] for i in range(k)])
    clocks.mark(t_timed0, time.perf_counter())
    launches = lib.cle_kernel_launches() - n0
    trace = (ctypes.c_uint64 * (4 * 256))()
    lib.cle_profile_trace(trace, ctypes.sizeof(trace))
    vor_trace = [tuple(int(v) for v in trace[4 * i:4 * i + 4]) for i in range(256)
                 if trace[4 * i] or trace[4 * i + 1]]
    barrier(world)
    clk = clocks.stop()
    lib.cle_profile_enable(0)
    if L is None:
        L = cle._ops._label_max(labels)
    total_ms = max_over_ranks(sum(times), world)
    ms_per_step = total_ms / args.steps
    value = nvox * world * args.steps / (total_ms / 1e3) / 1e6
    labels_dev = labels.tensor.cpu() if not dense else None

    # end to end through the public API with pinned host buffers
    e2e = e2e_serial = None
    if not args.no_e2e:
        pinned_in = torch.from_numpy(host_np).pin_memory()
        e2e = None if dense else e2e_served(pinned_in, w, args.steps, world, ref_labels=labels_dev)
        e2e_serial = e2e_per_call(pinned_in, w, max(2, min(5, args.steps // 4)), world, flush)
        if e2e is None:
            e2e = e2e_serial
    del labels_dev

    # roofline: the dominant kernel stage
    sm = np.array([s + [0.0] * (12 - len(s)) for s in stage_ms])[:, :12]
    mean_stage = sm.mean(axis=0)
    frac_lab = None
    if not dense and L:
        from pyclesperanto_prototype_b200._ops import STAT_KEYS
        frac_lab = float(table[STAT_KEYS.index("area")][:int(L)].double().sum()) / nvox
    abytes = algo_bytes(w, frac_lab)
    cands = [(mean_stage[i], STAGES[i]) for i in range(12) if STAGES[i] in abytes]
    peak, peak_kind = load_peaks()
    if dense:
        # no stage events on this composition: the whole step against the peak
        dom, t_dom, bpv = "gauss_otsu_labeling + statistics (whole step)", ms_per_step, DENSE_BYTES_PER_VOXEL
    else:
        t_dom, dom = max(cands)
        bpv = abytes[dom]
    achieved = bpv * nvox / (t_dom / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": None, "algorithmic_bytes_per_voxel": bpv, "ms": round(float(t_dom), 4)}
    tr = MEASURED_TRAFFIC.get(args.workload, {}).get(dom)
    if tr:
        roofline["traffic"] = tr[0]
        roofline["traffic_source"] = ("ncu DRAM bytes of one launch, profiles/" + tr[1]
                                      + (" (128x1024x1024 capture x 4)" if args.workload == "lightsheet" else ""))
    stages = {STAGES[i]: round(float(mean_stage[i]), 4) for i in range(12) if STAGES[i]}
    stage_roofline = {name: round(abytes[name] * nvox / (stages[name] / 1e3) / 1e9 / peak, 4)
                      for name in abytes if stages.get(name)}
    # the whole pipeline against the same peak at the compulsory bytes per voxel
    bpv_pipe = DENSE_BYTES_PER_VOXEL if dense else PIPELINE_BYTES_PER_VOXEL
    pipe_bytes = bpv_pipe * nvox
    pipeline_roofline = {"bytes_per_voxel": bpv_pipe,
                         "achieved": round(pipe_bytes / (ms_per_step / 1e3) / 1e9, 1),
                         "frac": round(pipe_bytes / (ms_per_step / 1e3) / 1e9 / peak, 4)}
    lat = np.array(times)

    served = None
    if world == 1 and args.served_duration > 0 and not dense:
        del src, labels, host
        torch.cuda.empty_cache()
        served = served_vs_per_call(args.rate, args.served_duration, args.lanes,
                                    closed_requests=args.closed_requests,
                                    compute_streams=args.compute_streams, express_voxels=args.express_voxels)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and host_np is not None:
        v, cores, shp, t = cpu_baseline_sample(host_np, w)
        what = "full workload" if int(np.prod(shp)) == nvox else "first %d z planes of the workload" % shp[0]
        cpu = {"value": round(v, 3), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{what} ({'x'.join(map(str, shp))} voxels) per repetition, best of 2, {t:.2f} s"}
    if rank == 0:
        out = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic", "impl": "b200",
               "config": config_of(args.workload, nvox),
               "run": {"labels": int(L), "input_dtype": str(host_np.dtype), "parallelism": "replicas",
                       "l2": "a 256 MiB write between steps evicts the 126 MB L2 (input %d MiB, labels %d MiB)"
                             % (host_np.nbytes >> 20, (nvox * 4) >> 20)},
               "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 4),
                              "p99": round(float(np.percentile(lat, 99)), 4)},
               "stages_ms": stages, "stage_roofline_frac": stage_roofline,
               "voronoi_trace": vor_trace if args.trace else None,
               "e2e": e2e, "e2e_per_call": e2e_serial, "gpu_launches": int(launches),
               "roofline": roofline, "pipeline_roofline": pipeline_roofline,
               "served_vs_per_call": served, "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def batch_shapes(n, seed=4):
    """Tile shapes: voxel counts log-uniform in [64*64, 96*512*512]; below
    512*512 voxels half the tiles are 2D; 3D tiles keep the 96:512:512 aspect."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(64 * 64), np.log(96 * 512 * 512)
    shapes = []
    for i in range(n):
        v = float(np.exp(rng.uniform(lo, hi)))
        if v < 512 * 512 and rng.uniform() < 0.5:
            a = max(8, int(round(np.sqrt(v) / 8)) * 8)
            shapes.append((a, a))
        else:
            x = max(16, int(round((v / 0.1875) ** (1 / 3) / 8)) * 8)
            z = max(4, int(round(v / (x * x))))
            shapes.append((z, x, x))
    return shapes


def run_batch(args):
    import torch
    import pyclesperanto_prototype_b200 as cle
    from pyclesperanto_prototype_b200 import _lib, synthetic
    from pyclesperanto_prototype_b200.batch import VolBatch
    torch.cuda.set_device(0)
    w = WORKLOADS["batch"]
    shapes = batch_shapes(args.tiles)
    rng = np.random.default_rng(44)
    tiles = [synthetic.blob_tile(sh, float(rng.uniform(0.5e-4, 5e-4)), seed=4 + i) for i, sh in enumerate(shapes)]
    nvox = sum(t.numel() for t in tiles)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    # per-call: the public API, one tile after another, inputs resident
    ref_out = [cle.create_labels_like(cle.B200Array(t)) for t in tiles]

    def per_call():
        for t, o in zip(tiles, ref_out):
            cle.voronoi_otsu_labeling(cle.B200Array(t), o, w["spot"], w["outline"])

    batch = VolBatch(tiles, w["spot"], w["outline"], lanes=args.batch_lanes).capture()

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ts.append((e0.elapsed_time(e1) / 1e3, time.perf_counter() - t0))
        return ts

    for _ in range(args.warmup):
        per_call()
        batch.run()
    torch.cuda.synchronize()
    tb = timed(batch.run, args.steps)
    # graph replays launch the captured kernels without host calls
    launches = batch.launches_per_run * args.steps
    tp = timed(per_call, max(1, args.steps // 2))
    batch.check()
    exact = all(torch.equal(a, b.tensor) for a, b in zip(batch.outputs, ref_out))
    dev_b = st.mean(t[0] for t in tb)
    wall_b = st.mean(t[1] for t in tb)
    dev_p = st.mean(t[0] for t in tp)
    wall_p = st.mean(t[1] for t in tp)
    out = {"metric": METRIC, "value": round(nvox / dev_b / 1e6, 2), "unit": UNIT, "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dev_b * 1e3, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "impl": "b200", "form": "batched (one CUDA graph, %d lanes)" % batch.lanes,
           "config": {"workload": w["desc"], "tiles": len(tiles), "voxels_per_step": int(nvox),
                      "l2": "flushed between steps (256 MiB write)"},
           "per_call": {"value": round(nvox / dev_p / 1e6, 2), "ms_per_step": round(dev_p * 1e3, 3),
                        "wall_ms_per_step": round(wall_p * 1e3, 3)},
           "batched_wall_ms_per_step": round(wall_b * 1e3, 3),
           "speedup_vs_per_call": round(dev_p / dev_b, 3),
           "tile_by_tile_bit_exact": bool(exact), "gpu_launches": int(launches)}
    print(json.dumps(out), flush=True)


def run_served(args):
    """The served form alone: the Poisson trace (default 200 req/s for 60 s)
    and saturation, served against the per-call loop; under torchrun the
    trace is routed over replicas."""
    import torch
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer, per_call_loop, request_bytes
    rank, world, local = dist_setup(args.gpus)
    w = WORKLOADS["served"]
    if world == 1:
        res = served_vs_per_call(args.rate, args.duration, args.lanes, pool_per_class=args.pool,
                                 closed_requests=args.closed_requests, spot=w["spot"], outline=w["outline"],
                                 compute_streams=args.compute_streams, express_voxels=args.express_voxels)
        s = res["trace"]["served"]
        out = {"metric": METRIC, "value": s["mvoxels_per_s"], "unit": UNIT, "n_gpus": 1,
               "steps": s["requests"], "warmup": len(SERVED_CLASSES), "ms_per_step": None,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic", "impl": "b200", "form": res["form"],
               "config": {"workload": w["desc"], "rate_per_s": args.rate, "duration_s": args.duration,
                          "volumes": "%d pre-generated per size class, reused" % args.pool},
               "served_vs_per_call": res}
        print(json.dumps(out), flush=True)
        return
    # replicas: every rank routes the same trace and serves its share
    from pyclesperanto_prototype_b200.replicas import serve_replicated
    pool = served_pools(args.pool)
    trace = served_trace(args.rate, args.duration, args.pool)

    def make():
        return [Request(i, pool[c][j], arrival=a) for i, (a, c, j) in enumerate(trace)]
    server = SegmentationServer(budget_bytes=60e9, slots=args.lanes, compute_streams=args.compute_streams,
                                express_voxels=args.express_voxels, spot_sigma=w["spot"],
                                outline_sigma=w["outline"])
    server.run([Request(i, pool[c][0], arrival=0.0) for i, c in enumerate(SERVED_CLASSES)], realtime=False)

    class _PerCall:
        def run(self, reqs, realtime=True):
            return per_call_loop(reqs, w["spot"], w["outline"], realtime=realtime)

    nbytes = lambda r: request_bytes(tuple(r.volume.shape), r.volume.dtype)
    barrier(world)
    served = serve_replicated(make(), lambda _: server, nbytes, 60e9)
    barrier(world)
    plain = serve_replicated(make(), lambda _: _PerCall(), nbytes, 60e9)
    barrier(world)
    import torch.distributed as dist
    if rank == 0:
        vox_of = {i: pool[c][j].numel() for i, (a, c, j) in enumerate(trace)}
        s, p = _summarize(served, vox_of), _summarize(plain, vox_of)
        out = {"metric": METRIC, "value": s["mvoxels_per_s"], "unit": UNIT, "n_gpus": world,
               "steps": len(trace), "warmup": len(SERVED_CLASSES), "ms_per_step": None,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic", "impl": "b200",
               "form": "served, %d replicas, requests routed by device memory (no data-path collective)" % world,
               "config": {"workload": w["desc"], "rate_per_s": args.rate, "duration_s": args.duration},
               "served": s, "per_call_loop": p}
        print(json.dumps(out), flush=True)
    dist.destroy_process_group()


def _tissue_2d(width, height, dx, dy, seed):
    """Label image of a jittered-grid Voronoi tessellation (the shape of
    artificial_tissue_2d: one cell per dx x dy grid cell)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    gy, gx = np.mgrid[dy / 2:height:dy, dx / 2:width:dx]
    pts = np.stack([gy.ravel(), gx.ravel()], 1) + rng.uniform(-0.3, 0.3, (gy.size, 2)) * [dy, dx]
    yy, xx = np.mgrid[0:height, 0:width]
    _, idx = cKDTree(pts).query(np.stack([yy.ravel(), xx.ravel()], 1))
    return (idx.reshape(height, width) + 1).astype(np.float32)


def _spheres(n, size, radius, seed):
    rng = np.random.default_rng(seed)
    img = np.zeros((size, size, size), np.uint8)
    r = int(radius)
    zz, yy, xx = np.mgrid[-r:r + 1, -r:r + 1, -r:r + 1]
    ball = zz * zz + yy * yy + xx * xx <= radius * radius
    for c in (rng.random((n, 3)) * size).astype(int):
        lo, hi = np.maximum(c - r, 0), np.minimum(c + r + 1, size)
        b = ball[lo[0] - c[0] + r:hi[0] - c[0] + r, lo[1] - c[1] + r:hi[1] - c[1] + r,
                 lo[2] - c[2] + r:hi[2] - c[2] + r]
        img[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= b
    return img.astype(np.float32)


def run_published(args):
    """Times the cases the reference's notebooks publish timings for, on seeded
    inputs of the same shape and distribution, inputs resident on the device:
    CUDA-event time per call and wall time with a synchronize."""
    import torch
    import pyclesperanto_prototype_b200 as cle
    torch.cuda.set_device(0)
    rng = np.random.default_rng(7)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    tissue = _tissue_2d(2048, 1024, 128, 96, 8)
    cases = [
        ("voronoi_otsu_labeling 2048x2048 uniform random, spot_sigma=outline_sigma=1",
         lambda: cle.push(rng.random((2048, 2048))), lambda a, o: cle.voronoi_otsu_labeling(a, o, 1, 1),
         cle.create_labels_like, 530.0, "Apple M1 Max CPU, OpenCL (benchmarks/apple_m1_voronoi_otsu_labeling.ipynb)"),
        ("gaussian_blur sigma=2, 64x1024x1024 uniform random",
         lambda: cle.push(rng.random((64, 1024, 1024))), lambda a, o: cle.gaussian_blur(a, o, 2, 2, 2),
         cle.create_like, 49.8, "RTX 2070 (benchmarks/benchmarking_some_operations.ipynb)"),
        ("gaussian_blur sigma=10, 64x1024x1024 uniform random",
         lambda: cle.push(rng.random((64, 1024, 1024))), lambda a, o: cle.gaussian_blur(a, o, 10, 10, 10),
         cle.create_like, 134.1, "RTX 2070 (benchmarks/benchmarking_some_operations.ipynb)"),
        ("gaussian_blur sigma=10, 100x512x512 uniform random",
         lambda: cle.push(rng.random((100, 512, 512))), lambda a, o: cle.gaussian_blur(a, o, 10, 10, 10),
         cle.create_like, 214.0, "RTX 3050 Ti Laptop (benchmarks/gaussian_blur.ipynb)"),
        ("histogram 256 bins with min/max, 100x1024x1024 normal",
         lambda: cle.push(rng.normal(size=(100, 1024, 1024))), lambda a, o: cle.histogram(a, num_bins=256),
         None, 140.0, "RTX 3050 Ti Laptop (benchmarks/histograms.ipynb)"),
        ("threshold_otsu 100x512x512 uniform random",
         lambda: cle.push(rng.random((100, 512, 512))), lambda a, o: cle.threshold_otsu(a, o),
         cle.create_binary_like, 38.0, "RTX 2070 (benchmarks/threshold_otsu.ipynb, best of 38-50 ms)"),
        ("connected_components_labeling_box 400^3, 200 balls of radius 10",
         lambda: cle.push(_spheres(200, 400, 10, 9)), lambda a, o: cle.connected_components_labeling_box(a, o),
         cle.create_labels_like, 98.0, "RTX 2080 Ti (benchmarks/connected_component_labeling.ipynb, best of 98-156 ms)"),
        ("statistics_of_labelled_pixels 2048x1024 tissue labels (intensity None)",
         lambda: cle.push(tissue), lambda a, o: cle.statistics_of_labelled_pixels(None, a),
         None, 39.0, "RTX 2070 (benchmarks/statistics_of_labeled_pixels.ipynb)"),
        ("statistics_of_labelled_pixels 128x1024x1024 (the tissue stacked, intensity None)",
         lambda: cle.push(np.broadcast_to(tissue[:, :1024], (128, 1024, 1024)).copy()),
         lambda a, o: cle.statistics_of_labelled_pixels(None, a),
         None, 765.0, "RTX 2070 (benchmarks/statistics_of_labeled_pixels.ipynb)"),
    ]
    out_cases = []
    for name, make, call, creator, pub_ms, pub_hw in cases:
        a = make()
        o = creator(a) if creator else None
        for _ in range(args.warmup):
            call(a, o)
        torch.cuda.synchronize()
        dev, wall = [], []
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            call(a, o)
            e1.record(stream)
            e1.synchronize()
            wall.append((time.perf_counter() - t0) * 1e3)
            dev.append(e0.elapsed_time(e1))
        d, w = float(np.median(dev)), float(np.median(wall))
        out_cases.append({"case": name, "ms_device": round(d, 3), "ms_wall": round(w, 3),
                          "published_ms": pub_ms, "published_hardware": pub_hw,
                          "wall_speedup_vs_published": round(pub_ms / w, 1)})
        del a, o
        torch.cuda.empty_cache()
    print(json.dumps({"metric": "ms per call on the reference's published benchmark cases", "impl": "b200",
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
                      "config": {"workload": WORKLOADS["published"]["desc"],
                                 "timing": "median over steps; L2 flushed between calls; inputs resident"},
                      "cases": out_cases}), flush=True)


def run_reference(args):
    """The reference arm: the oracle (the reference's algorithm restated in C,
    OpenMP on every host thread) on the same workload and volume, the whole
    volume every timed step; warm-up steps run on a slab of it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    oracle.build()
    w = WORKLOADS[args.workload]
    if args.workload in ("batch", "served", "published"):
        print(json.dumps({"impl": "reference", "workload": args.workload,
                          "note": "the CPU arm times the single-volume workloads (lightsheet, nuclei, "
                                  "lightsheet_dense, blobs2d); run it with one of those"}), flush=True)
        return
    host = make_input(args.workload)
    if hasattr(host, "cpu"):
        host = host.cpu().numpy()
    f = host.astype(np.float32)
    del host
    cores = oracle.num_threads()
    warm = f if f.ndim == 2 or f.shape[0] <= 32 else np.ascontiguousarray(f[:32])
    for _ in range(args.warmup):
        cpu_step(warm, w)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cpu_step(f, w)
        ts.append(time.perf_counter() - t0)
    total = sum(ts)
    v = f.size * args.steps / total / 1e6
    print(json.dumps({
        "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference", "config": config_of(args.workload, f.size),
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "the whole volume (%s voxels) every timed step; warm-up steps on %s "
                                   "voxels" % ("x".join(map(str, f.shape)), "x".join(map(str, warm.shape)))},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU OpenCL path unavailable (no pyopencl / CPU OpenCL runtime / kernel sources); "
                "its C restatement runs on all host threads"}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="leave out the end-to-end legs (profiler runs)")
    ap.add_argument("--trace", action="store_true", help="include the Voronoi per-step trace")
    ap.add_argument("--tiles", type=int, default=512, help="batch workload: number of tiles")
    ap.add_argument("--lanes", type=int, default=8, help="served: requests in flight (slots)")
    ap.add_argument("--batch-lanes", type=int, default=0,
                    help="batch: lanes (CUDA streams) of the batched form; 0 = the library's tuned table")
    ap.add_argument("--duration", type=float, default=60.0, help="served workload: trace length in s")
    ap.add_argument("--served-duration", type=float, default=10.0,
                    help="single-volume workloads: length (s) of the served-vs-per-call trace in the "
                         "line (0: leave it out)")
    ap.add_argument("--closed-requests", type=int, default=120,
                    help="served comparison at saturation: requests waiting at t=0")
    ap.add_argument("--pool", type=int, default=6, help="served workload: volumes per size class")
    ap.add_argument("--rate", type=float, default=200.0, help="served workload: arrivals per s")
    ap.add_argument("--compute-streams", type=int, default=1, help="served workload: compute streams")
    ap.add_argument("--express-voxels", type=int, default=8 << 20,
                    help="served workload: requests up to this size take the express lane (0: off)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "published":
        run_published(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
