"""Benchmark: STEM probe*slices/s of the fused multislice engine on one or more B200s.

Workload (``--workload stem-adf``, the default): SrTiO3 [001], 8x8x50 unit cells, 2 slices per
cell (100 slices), Peng parameters, 300 kV, 25 mrad probe with C3 = -5 um, 64x64 raster at
0.5 Angstrom (8 px at 0.0625 Angstrom/px), 512^2 window, 1024^2 potential grid, ADF 60-200 mrad and
BF 0-10 mrad detectors.  Synthetic (seeded) structure; no dataset.

One "step" is one complete STEM request on the device: transmission build (potential, FFT,
exp) + slice loop for all 4096 probes + detector reduction, inputs already resident in HBM.
``value`` = probe*slices per second over all ranks: with ``--scaling weak`` (default) every rank
runs its own request; with ``--scaling strong`` the request's scan rows are split over the ranks
(the sharded path of ``totem_b200.shard``).  ``e2e`` = the same metric through ``totem_stem_run``
with host buffers (upload, run, download every step).

``--impl reference`` times the FP64 CPU oracle (the NumPy restatement of the reference's CPU
path; MATLAB is not available) on a bounded sample of the same workload with all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_ELEM = 8  # complex64


def build_workload(name: str, seed: int | None = None, raster: int = 64):
    from totem_b200 import request
    if name == "stem-adf":
        # a smaller raster keeps every per-probe cost identical (same window, potential, slices);
        # it is used to time slow comparators on a subset of the 64 x 64 probes
        return request.build_srtio3_stem(phonon_seed=seed, raster=(raster, raster), p=1024)
    if name == "stem-adf-small":
        return request.build_srtio3_stem(cells=(4, 4, 10), n=256, raster=(32, 32), sampling=0.0625, step=8)
    raise SystemExit(f"unknown workload {name}")


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [ln.strip().split(", ") for ln in self.f.read().splitlines() if ln.strip()]
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
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------------------
# CPU sample (oracle) -- used for cpu_baseline and for --impl reference
# ----------------------------------------------------------------------------------------------

def _potential_chunk(args):
    req, lo, hi = args
    from oracle import stem_oracle as so
    import copy
    r = copy.copy(req)
    r.ele_n = req.ele_n[lo:hi]
    r.series_n = np.array([hi - lo], dtype=float)
    r.ele_n_i = req.ele_n_i[:0]
    r.series_n_i = np.array([0.0])
    return so.potential_fourier(r)[0]


def _loop_sample(args):
    psi, T, r0, c0, prop = args
    import scipy.fft as sfft
    for k in range(T.shape[0]):
        psi = psi * T[k, r0:r0 + psi.shape[0], c0:c0 + psi.shape[1]]
        psi = sfft.ifft2(sfft.fft2(psi) * prop)
    return float(np.abs(psi).sum())


def cpu_sample(req, workers: int, sample_slices: int = 2):
    """Time the oracle on a bounded sample and extrapolate to the full request.

    (a) the potential + transmission of one slice (its atoms split over ``workers`` processes);
    (b) ``workers`` probes through ``sample_slices`` slices each, in parallel.
    Full-request CPU time = slices * t(a) + probe_slices / rate(b).
    """
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    from oracle import stem_oracle as so
    import copy
    ctx = mp.get_context("spawn")
    n0 = int(req.padded_series()[0][0])
    bounds = np.linspace(0, n0, workers + 1).astype(int)
    one = copy.copy(req)
    one.ele_n = req.ele_n[:n0]
    with ProcessPoolExecutor(workers, mp_context=ctx) as ex:
        list(ex.map(_potential_chunk, [(one, 0, 1)] * workers))  # warm the workers up
        t0 = time.perf_counter()
        parts = list(ex.map(_potential_chunk, [(one, int(bounds[i]), int(bounds[i + 1])) for i in range(workers)]))
        vg = np.sum(parts, axis=0)[None]
        one.series_n = np.array([n0], dtype=float)
        one.series_n_i = np.array([0.0])
        T1 = so.transmission(one, vg)
        t_pot = time.perf_counter() - t0
        T = np.repeat(T1, sample_slices, axis=0)
        rows = req.beginrow + (np.arange(workers) // req.width_red) * req.step
        cols = req.begincol + (np.arange(workers) % req.width_red) * req.step
        jobs = [(req.probe[0], T, int(rows[i]), int(cols[i]), req.prop) for i in range(workers)]
        t0 = time.perf_counter()
        list(ex.map(_loop_sample, jobs))
        t_loop = time.perf_counter() - t0
    rate = workers * sample_slices / t_loop
    total = req.slices * t_pot + req.probe_slices / rate
    value = req.probe_slices / total
    sample = (f"oracle (FP64 NumPy/SciPy) on {workers} processes: potential+transmission of 1 of "
              f"{req.slices} slices ({n0} atoms, {req.p_height}^2 grid) in {t_pot:.2f} s; {workers} probes x "
              f"{sample_slices} slices ({req.height}^2 window) in {t_loop:.2f} s; extrapolated to "
              f"{req.probe_slices} probe*slices")
    return value, sample, t_pot + t_loop


# ----------------------------------------------------------------------------------------------

def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(ns):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import stem_oracle as so
    req = build_workload(ns.workload, raster=ns.raster)
    workers = so.cpu_count()
    for _ in range(ns.warmup):
        cpu_sample(req, workers, sample_slices=1)
    vals, samples, secs = [], None, 0.0
    for _ in range(ns.steps):
        v, samples, s = cpu_sample(req, workers)
        vals.append(v)
        secs += s
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": "STEM probe*slices/s", "value": value, "unit": "probe*slices/s",
        "n_gpus": ns.gpus, "steps": ns.steps, "warmup": ns.warmup,
        "ms_per_step": 1000.0 * secs / max(ns.steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SrTiO3 supercell)",
        "config": workload_config(ns, req),
        "cpu_baseline": {"value": value, "unit": "probe*slices/s", "cores": workers, "kind": "port",
                         "sample": samples},
        "e2e": {"value": value, "unit": "probe*slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _event_seconds(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1000.0


def plain_comparators(ns, req, local, stream, fused_value):
    """The metric's comparator: the plain cuFFT path (cuFFT plus one element-wise kernel per step)
    on the same GPU, (a) batched over the whole request (1 GiB of waves per batch) and (b) one
    probe at a time, the reference's loop structure (cuda_source_lobato.cu:1313-1398 runs one
    cuFFT plan over the probes of a batch; ToTem's CPU path and small batches go probe by probe),
    on a sample of 8x8 probes of the same workload (same window, potential and slices: the
    per-probe cost does not depend on the raster)."""
    from totem_b200 import capi
    s = capi.Session(device=local, stream=stream.cuda_stream)
    s.upload(req)
    s.run(path=capi.PATH_PLAIN)  # cuFFT plans, transmission
    t_batched = _event_seconds(stream, lambda: s.run(path=capi.PATH_PLAIN))
    batch_plain = s.timing().batch
    s.close()
    sub = build_workload(ns.workload, raster=8)
    s = capi.Session(device=local, stream=stream.cuda_stream)
    s.upload(sub)
    s.run(path=capi.PATH_PLAIN, batch=1)
    t_probe = _event_seconds(stream, lambda: s.run(path=capi.PATH_PLAIN, batch=1, skip_transmission=True))
    s.close()
    batched = req.probe_slices / t_batched
    per_probe = sub.probe_slices / t_probe
    return {
        "batched": {"value": batched, "unit": "probe*slices/s", "batch": batch_plain,
                    "what": "whole request (transmission + slice loop), same workload, CUDA events"},
        "per_probe": {"value": per_probe, "unit": "probe*slices/s", "batch": 1,
                      "what": f"slice loop of {sub.depth} probes of the same workload, one probe per cuFFT plan "
                              "execution, transmission built beforehand"},
        "fused_vs_batched": fused_value / batched, "fused_vs_per_probe": fused_value / per_probe,
    }


def serving_leg(local):
    """Latency under load: a seeded mix of STEM requests (windows 256^2 / 512^2, probes
    log-uniform 1-256, 20-100 slices, Peng / Lobato) through the continuous-batching server,
    first all at once (capacity), then with seeded Poisson arrivals at 85 % of that capacity."""
    from totem_b200 import serving
    reqs = serving.make_workload(count=32, seed=0, sizes=(256, 512), max_probes=256, slices=(20, 100))
    serving.serve(reqs[:4], np.zeros(4), device=local)  # kernels, pools
    _, lat_b, mk_b = serving.serve(reqs, np.zeros(len(reqs)), device=local)
    rate = 0.85 * len(reqs) / mk_b
    _, lat_p, mk_p = serving.serve(reqs, serving.poisson_arrivals(len(reqs), rate, 0), device=local)
    ps = sum(r.probe_slices for r in reqs)
    return {"workload": "32 seeded requests, windows 256^2/512^2, probes log-uniform 1-256, slices 20-100, "
                        "Peng/Lobato, SrTiO3 filling the potential grid",
            "burst": {"probe_slices_per_s": ps / mk_b, "p50_ms": float(np.percentile(lat_b, 50)),
                      "p99_ms": float(np.percentile(lat_b, 99))},
            "poisson": {"rate_hz": rate, "probe_slices_per_s": ps / mk_p, "p50_ms": float(np.percentile(lat_p, 50)),
                        "p99_ms": float(np.percentile(lat_p, 99))}}


def workload_config(ns, req):
    return {"workload": f"{ns.workload}: SrTiO3 [001] STEM-ADF, {req.depth} probes x {req.slices} slices, "
                        f"window {req.height}^2, potential {req.p_height}^2, Peng, 300 kV",
            "probes": req.depth, "slices": req.slices, "window": req.height, "potential_grid": req.p_height,
            "detectors": req.aper_num, "path": ns.path, "l2": "inputs larger than L2 (transmission stack "
            f"{req.slices * req.p_height * req.p_width * 8 / 2**20:.0f} MiB)",
            "parallelism": (f"scan rows split over {ns.gpus} GPUs" if ns.scaling == "strong" and ns.gpus > 1 else
                            f"one request per GPU, {ns.gpus} GPU(s)") + ", no collective in the data path"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="stem-adf")
    ap.add_argument("--path", default="fused", choices=["fused", "plain"])
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--raster", type=int, default=64,
                    help="scan positions per side (64 = the full workload; smaller only to time slow comparators)")
    ap.add_argument("--col-variant", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-comparators", action="store_true", help="skip the plain cuFFT and serving legs")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="weak: every rank runs the whole request; strong: the request's scan rows are split "
                         "over the ranks (shard.band_request), each rank building its own transmission")
    ap.add_argument("--no-band-skip", action="store_true",
                    help="compute the wave columns the propagator zeroes too (totem_set_band_skip(0))")
    ns = ap.parse_args()
    if ns.impl == "reference":
        run_reference(ns)
        return

    import torch
    ws, rank, local = dist_env()
    # the one-shot C ABI (the e2e leg) picks its device by free memory unless TOTEM_DEVICE is set:
    # pin it to this rank's GPU
    os.environ["TOTEM_DEVICE"] = str(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    from totem_b200 import capi
    if ns.no_band_skip:
        capi.set_band_skip(False)
    path = capi.PATH_FUSED if ns.path == "fused" else capi.PATH_PLAIN
    req = build_workload(ns.workload, raster=ns.raster)
    # a dedicated stream: the engine launches on it and the CUDA events below are recorded on it
    # (the legacy default stream has handle 0, which the C ABI reads as "make your own stream")
    stream = torch.cuda.Stream()
    sess = capi.Session(device=local, stream=stream.cuda_stream)
    strong = ns.scaling == "strong" and ws > 1
    if strong:
        # the product's sharded path: contiguous bands of scan rows, one per rank, no collective
        # in the data path (the A x depth detector images are gathered once, after the timing)
        from totem_b200 import shard
        r0, r1 = shard.row_bands(req.hight_red, ws)[rank]
        sess.upload(shard.band_request(req, r0, r1))
    else:
        sess.upload(req)

    def step():
        sess.run(path=path, batch=ns.batch, col_variant=ns.col_variant)

    for _ in range(max(ns.warmup, 0)):
        step()
    torch.cuda.synchronize()
    launches = sess.timing().kernel_launches
    batch_used = sess.timing().batch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(ns.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms_total = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms_total], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / ns.steps
    units = req.probe_slices
    # weak: every rank did the whole request; strong: the ranks did one request together
    value = (1 if strong else ws) * units * ns.steps / (ms_total / 1000.0)

    # per-kernel device times (events around every pass) for the roofline
    sess.run(path=path, batch=ns.batch, profile=True, col_variant=ns.col_variant)
    tm = sess.timing()
    peak, peak_kind = measured_peaks()
    n2 = req.height * req.width
    roofline = None
    if path == capi.PATH_FUSED and tm.row_pass_launches:
        # this rank's units: the whole request (weak) or its band (strong)
        alg_bytes = sess.req.probe_slices * 3 * n2 * BYTES_PER_ELEM  # read psi, write psi, read T window
        step_ms = tm.row_pass_ms + tm.col_pass_ms
        achieved = alg_bytes / (step_ms / 1000.0) / 1e9
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "slice_step_traffic.json")
        if os.path.exists(tpath):
            tr = json.load(open(tpath))
            if tr.get("window") == req.height:
                traffic = tr["dram_bytes_per_probe_slice"] * units / tm.col_pass_launches
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_source": f"{peak_kind} hbm_gbs", "traffic": traffic,
                    "kernel": "slice step = k_row_pass + k_col_pass (one launch of each per slice)",
                    "algorithmic_bytes_per_probe_slice": 3 * n2 * BYTES_PER_ELEM,
                    "row_pass_ms_avg": tm.row_pass_ms / tm.row_pass_launches,
                    "col_pass_ms_avg": tm.col_pass_ms / tm.col_pass_launches,
                    "probes_per_launch": tm.batch,
                    "transmission_ms": tm.transmission_ms, "slice_loop_ms": tm.slice_loop_ms}

    # the compute-side ceiling: algorithmic FFT flops (two 2-D transforms, 5 N^2 log2 N^2 each, and
    # 14 N^2 for the multiplies) over the same pass time, against the measured FP32 FMA throughput
    compute = None
    if roofline is not None and rank == 0:
        ffma, ffma2 = capi.fp32_peak(local)
        flops_ps = 2 * 5 * n2 * math.log2(n2) + 14 * n2
        achieved_tf = flops_ps * sess.req.probe_slices / (step_ms / 1000.0) / 1e12
        peak_tf = max(ffma, ffma2)
        compute = {"bound": "fp32", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                   "frac": achieved_tf / peak_tf, "peak_source": "measured FFMA / FFMA2 chains (totem_fp32_peak)",
                   "ffma_tflops": ffma, "ffma2_tflops": ffma2, "algorithmic_flops_per_probe_slice": flops_ps}

    # end to end through the C ABI with host buffers
    e2e = None
    if not ns.no_e2e:
        e2e_req = sess.req  # the whole request, or this rank's band of it
        capi.stem_run(e2e_req, path=path, batch=ns.batch)  # warm the default session
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ns.steps):
            capi.stem_run(e2e_req, path=path, batch=ns.batch)
        dt = time.perf_counter() - t0
        if dist:
            t = torch.tensor([dt], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        h2d = tm.h2d_bytes
        d2h = 8 * e2e_req.aper_num * e2e_req.depth * (1 + len(e2e_req.mid_layer))
        e2e = {"value": (1 if strong else ws) * units * ns.steps / dt, "unit": "probe*slices/s",
               "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "api": "totem_stem_run (host buffers)"}

    plain = serve = None
    if rank == 0 and ws == 1 and not ns.no_comparators and path == capi.PATH_FUSED:
        plain = plain_comparators(ns, req, local, stream, value)
        serve = serving_leg(local)

    cpu = None
    if rank == 0 and ws == 1 and not ns.no_cpu_baseline:
        from oracle import stem_oracle as so
        cores = so.cpu_count()
        v, sample, _ = cpu_sample(req, cores)
        cpu = {"value": v, "unit": "probe*slices/s", "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": "STEM probe*slices/s", "value": value, "unit": "probe*slices/s", "n_gpus": ws,
            "steps": ns.steps, "warmup": ns.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong" if strong else "weak", "vs_baseline": None,
            "dtype": "f32 (complex64; FP64 detector sums)",
            "data": "synthetic (seeded SrTiO3 supercell, random-free probe)",
            "config": workload_config(ns, req), "batch": batch_used,
            "gpu_launches": launches * ns.steps, "clocks": clk.summary(), "roofline": roofline, "compute": compute,
            "e2e": e2e, "cpu_baseline": cpu, "plain_cufft": plain, "serving": serve,
        }
        if serve:
            line["latency"] = {"p50_ms": serve["poisson"]["p50_ms"], "p99_ms": serve["poisson"]["p99_ms"],
                               "what": "serving leg, Poisson arrivals at 85 % of capacity"}
        print(json.dumps(line), flush=True)
    sess.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
