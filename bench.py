#!/usr/bin/env python3
"""Benchmark of the per-gulp search path at the 4096-channel, DM 0-2000
workload: beam-seconds searched per second (whole job) of several beams
served together on one GPU with FP16 plane storage, their p50/p99 gulp
latency, the plain single-beam FP32 and FP16 paths beside them, the same
served run fed from pinned host memory (e2e; --staging N keeps N gulps in
flight per beam, each uploaded into a staging block at submit), the FDMT
level kernel's HBM
roofline, and the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl frost|reference]
                    [--beams B] [--served-tile T] [--workload config2|config1]

A beam-gulp is one 262144-sample gulp of one beam through RFI excision
(moments, IQRM, Kadane along time and frequency, zero-DM subtract,
narrow/broad-band neighbour fills) -> normalisation -> streaming FDMT ->
boxcar search of 11 sub-band planes (widths 1-256). A step is one gulp of
each served beam (B beams, admitted by device memory; each has one gulp in
flight). Each rank serves its own beams (replicas, weak scaling; beams are
independent, so no collective is needed). Inputs are seeded synthetic
filterbanks with the workload's noise, RFI and pulse recipe; every
beam-gulp reads a 1 GiB raw gulp and writes/reads multi-GiB planes, so
inputs exceed the 126 MB L2 without a flush.
"""

from __future__ import annotations

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

METRIC = "beam-s searched/s @4096ch DM2000"
UNIT = "beam-s/s"
# The headline workload (4096 channels, DM 0-2000, 11 planes) and the small
# 1024-channel DM 0-500 full-band workload used for profiling captures.
WORKLOADS = {
    "config2": dict(nchans=4096, gulp=262144, fch1=1535.958984375, foff=-0.08203125,
                    dm_max=2000.0, max_boxcar=256, depth=2, full_rfi=True,
                    text=("4096ch 1200-1536MHz 64us uint8, 262144-sample gulps, DM 0-2000 "
                          "(3625 trials), boxcar 1-256, 11 sub-band planes, "
                          "moments+IQRM+Kadane(time,freq)+zero-DM RFI")),
    "config1": dict(nchans=1024, gulp=65536, fch1=1500.0, foff=-0.29296875, dm_max=500.0,
                    max_boxcar=64, depth=0, full_rfi=False,
                    text=("1024ch 1200-1500MHz 64us uint8, 65536-sample gulps, DM 0-500 "
                          "(886 trials), boxcar 1-64, full band, default RFI")),
}
TSAMP = 64e-6
W = dict(WORKLOADS["config2"])
NCHANS, GULP, FCH1, FOFF = W["nchans"], W["gulp"], W["fch1"], W["foff"]
DM_MAX, MAX_BOXCAR, DEPTH, WORKLOAD = W["dm_max"], W["max_boxcar"], W["depth"], W["text"]


def select_workload(name):
    global W, NCHANS, GULP, FCH1, FOFF, DM_MAX, MAX_BOXCAR, DEPTH, WORKLOAD
    W = dict(WORKLOADS[name])
    NCHANS, GULP, FCH1, FOFF = W["nchans"], W["gulp"], W["fch1"], W["foff"]
    DM_MAX, MAX_BOXCAR, DEPTH, WORKLOAD = W["dm_max"], W["max_boxcar"], W["depth"], W["text"]


def rfi_config():
    from frost_b200.config import RfiConfig, ZeroDMMode
    cfg = RfiConfig()
    if W["full_rfi"]:
        cfg.moments.enabled = True
        cfg.iqrm.enabled = True
        cfg.kadane_channel.enabled = True
        cfg.kadane_spectrum.enabled = True
        cfg.zero_dm = ZeroDMMode.SUBTRACT
    return cfg


def layout(nsamps=None):
    from frost_b200.config import BlockLayout, DataType
    return BlockLayout(NCHANS, nsamps or GULP, DataType.UINT8, TSAMP, FCH1, FOFF)


def search_config(storage):
    """frost's search defaults (threshold 6, one peak per run per width) with
    room for every candidate of the 20 injected pulses in 11 planes."""
    from frost_b200.config import BoxcarConfig
    return BoxcarConfig(max_boxcar=MAX_BOXCAR, wtsp=2.0, detect_thresh=6.0, storage=storage,
                        max_candidates=1 << 20, max_cands_per_dm=4096)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def ranks_barrier(world):
    """All ranks of the job meet here (one process per GPU; gloo)."""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def ranks_max(x, world):
    """The largest of every rank's `x` (timings are the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.lines, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic_per_launch(algorithmic_per_launch):
    """Level-kernel DRAM bytes per launch at full size, scaled from the
    committed small-case ncu capture (profiles/fdmt_level_config1.json: the
    1024-channel gulp's measured DRAM bytes over its algorithmic bytes, the
    level kernels' traffic growing in proportion to the rows and samples
    they stream), or None."""
    path = os.path.join(ROOT, "profiles", "fdmt_level_config1.json")
    try:
        with open(path) as f:
            ratio = float(json.load(f)["traffic_over_algorithmic"])
    except (OSError, ValueError, KeyError):
        return None
    return int(ratio * algorithmic_per_launch)


def beam_seed(rank, beam):
    """Seed of one beam's synthetic gulp (beam 0 of rank 0: 0x46524F5354)."""
    return 0x46524F5354 ^ (rank << 20) ^ (beam << 8)


def make_gulp(seed):
    from frost_b200.synth import config1_gulp, config2_gulp
    if NCHANS == 1024:
        return config1_gulp(seed=seed, nsamps=GULP).data
    return config2_gulp(seed=seed).data  # [T][C] uint8


def run_gpu(args):
    import numpy as np
    import torch

    from frost_b200.config import Storage
    from frost_b200.pipeline import GulpPipeline, plan_for

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=600))

    # Every served beam has its own seeded gulp; beam 0's is the one the
    # plain single-beam paths run, so their candidate lists can be compared.
    gulps_dev, gulps_pin = [], []
    for b in range(max(args.beams, 1)):
        raw_host = make_gulp(beam_seed(rank, b))
        nbytes = raw_host.size
        gulps_dev.append(torch.from_numpy(raw_host.reshape(-1)).to(dev))
        pin = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        pin.copy_(torch.from_numpy(raw_host.reshape(-1)))
        gulps_pin.append(pin)
        del raw_host
    raw_dev, pinned = gulps_dev[0], gulps_pin[0]
    lay = layout()
    plan = plan_for(lay, 0.0, DM_MAX, DEPTH)

    barrier = lambda: ranks_barrier(world)
    max_over_ranks = lambda x: ranks_max(x, world)

    def measure(storage, e2e=False, sample_clocks=False):
        pipe = GulpPipeline(rfi_config(), lay, 2.0, plan, search_config(storage), device=local)
        tuned = pipe.search.autotune()  # the same launch-shape choice the server makes per beam
        step = (lambda: pipe.execute_device(pinned.data_ptr(), GULP, on_device=False)) if e2e else \
               (lambda: pipe.execute_device(raw_dev.data_ptr(), GULP, on_device=True))
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        barrier()
        pipe.search.enable_timing(True)
        l0 = pipe.rfi.launches()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ncands, d2h = 0, 0
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.__enter__()
        torch.cuda.synchronize()
        starts[0].record()
        for i in range(args.steps):
            res = step()
            ncands += res.candidates.size
            d2h += res.candidates.nbytes
            starts[i + 1].record()
        last = res.candidates.copy()
        torch.cuda.synchronize()
        if sampler:
            sampler.__exit__(None, None, None)
        barrier()
        lat = [starts[i].elapsed_time(starts[i + 1]) for i in range(args.steps)]
        total_ms = starts[0].elapsed_time(starts[-1])
        timing = pipe.search.timing()
        launches = timing["total_launches"] + (pipe.rfi.launches() - l0)
        rep = pipe.rfi.report()
        out = {"total_ms": max_over_ranks(total_ms), "lat": lat, "timing": timing, "tuned": tuned, "last": last,
               "launches": launches, "ncands": ncands, "d2h": d2h,
               "dropped": [res.dropped_global, res.dropped_per_dm],
               "clocks": sampler.summary() if sampler else None,
               "rfi_ms": {k: round(rep[k] * 1e3, 2) for k in
                          ("t_bandpass", "t_moments", "t_scan", "t_flags", "t_apply")},
               "rfi_counts": {k: rep[k] for k in ("chans_masked", "samps_flagged", "cells_narrow",
                                                  "cells_kadane_channel", "cells_kadane_spectrum")},
               "device_bytes": pipe.search.info()["device_bytes"]}
        del pipe
        torch.cuda.empty_cache()
        return out

    def measure_served(nbeams, on_device, sample_clocks=False, postprocess=False):
        """Beams of the workload on one GPU through the server: each beam has
        one gulp in flight (the next is submitted when the previous one's
        candidates are ready), so every beam is busy and its latency is
        service time under contention. Beams are admitted by device memory;
        the admitted count is reported."""
        from frost_b200._lib import FrostError
        from frost_b200.serve import BeamServer
        srv = BeamServer(device=local, slots=nbeams)
        bc = search_config(Storage.FP16)
        bc.tile_nsamps = args.served_tile
        beams = []
        for _ in range(nbeams):
            try:
                beams.append(srv.add_beam(rfi_config(), lay, 2.0, plan, bc))
            except FrostError as e:
                if e.code != -2:  # ERR_OUT_OF_MEMORY: admission refused
                    raise
                break
        if postprocess:
            # frost's per-gulp publish: clustering, DM wings, carry and
            # sub-band dedup of every gulp's detections, on the device
            for b in beams:
                srv.set_postprocess(b, postprocess_config(int(bc.max_candidates)))
        src = {b: (gulps_dev[i] if on_device else gulps_pin[i]).data_ptr() for i, b in enumerate(beams)}
        counts = {b: [0, 0] for b in beams}  # candidates (or giants), bytes
        last = {}
        # Host gulps with --staging N: N in flight per beam, the next ones
        # uploaded into staging blocks while the beam works on the one before.
        depth = 1 if on_device else max(1, args.staging)
        if not on_device and args.staging > 0:
            for b in beams:
                srv.set_staging(b, depth)

        def run_beam(b, n, keep):
            def collect(t):
                cands, _ = srv.wait_giants(t) if postprocess else srv.wait(t)
                if keep:
                    counts[b][0] += cands.size
                    counts[b][1] += cands.nbytes
                    last[b] = cands
            pending = []
            for _ in range(n):
                pending.append(srv.submit_ptr(b, src[b], nbytes, GULP, on_device))
                if len(pending) == depth:
                    collect(pending.pop(0))
            for t in pending:
                collect(t)

        def run_all(n, keep):
            ths = [threading.Thread(target=run_beam, args=(b, n, keep)) for b in beams]
            for t in ths:
                t.start()
            for t in ths:
                t.join()

        run_all(args.warmup, False)
        torch.cuda.synchronize()
        barrier()
        srv.reset_stats()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.__enter__()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record()
        run_all(args.steps, True)
        torch.cuda.synchronize()
        ev[1].record()
        torch.cuda.synchronize()
        if sampler:
            sampler.__exit__(None, None, None)
        barrier()
        st = srv.stats()
        out = {"total_ms": max_over_ranks(ev[0].elapsed_time(ev[1])), "beams": len(beams),
               "last0": last.get(beams[0]) if beams else None,
               "stats": st, "ncands": sum(c[0] for c in counts.values()),
               "d2h": sum(c[1] for c in counts.values()),
               "clocks": sampler.summary() if sampler else None}
        srv.close()
        torch.cuda.empty_cache()
        return out

    def measure_prefetch(storage):
        """The plain single-beam path fed by the library's input staging: a
        reader thread copies each gulp from host memory into pinned slots and
        on to the device, depth 3, while the previous gulp is searched."""
        import numpy as np
        from frost_b200.pipeline import GulpPipeline
        from frost_b200.staging import GulpPrefetch
        rows = np.tile(pinned.numpy().reshape(GULP, NCHANS), (args.warmup + args.steps, 1))
        pipe = GulpPipeline(rfi_config(), lay, 2.0, plan, search_config(storage), device=local)
        pipe.search.autotune()
        pf = GulpPrefetch.from_memory(rows, GULP, depth=3, device=local)
        for _ in range(args.warmup):
            ptr, n = pf.next()
            pipe.execute_device(ptr, n, on_device=True)
        torch.cuda.synchronize()
        barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        st0 = pf.stats()
        ev[0].record()
        for _ in range(args.steps):
            ptr, n = pf.next()
            pipe.execute_device(ptr, n, on_device=True)
        ev[1].record()
        torch.cuda.synchronize()
        st1 = pf.stats()
        barrier()
        out = {"total_ms": max_over_ranks(ev[0].elapsed_time(ev[1])),
               "read_ms_per_gulp": round(1e3 * (st1.read_s - st0.read_s) / args.steps, 2),
               "wait_ms_per_gulp": round(1e3 * (st1.wait_s - st0.wait_s) / args.steps, 2)}
        pf.close()
        del pipe, rows
        torch.cuda.empty_cache()
        return out

    single16 = measure(Storage.FP16)
    single16_host = measure(Storage.FP16, e2e=True)
    single16_pf = measure_prefetch(Storage.FP16)
    single32 = measure(Storage.FP32)
    served = measure_served(args.beams, on_device=True, sample_clocks=True)
    e2e = measure_served(args.beams, on_device=False)
    served_pp = measure_served(args.beams, on_device=True, postprocess=True)

    gulp_s = GULP * TSAMP
    per_beam_steps = args.steps * world
    value = served["beams"] * per_beam_steps * gulp_s / (served["total_ms"] / 1e3)
    plain32 = per_beam_steps * gulp_s / (single32["total_ms"] / 1e3)
    plain16 = per_beam_steps * gulp_s / (single16["total_ms"] / 1e3)
    e2e_value = e2e["beams"] * per_beam_steps * gulp_s / (e2e["total_ms"] / 1e3)
    t = single16["timing"]
    peak, peak_kind = measured_peaks()
    level_gbs = t["algorithmic_level_bytes"] / (t["level_ms"] / 1e3) / 1e9 if t["level_ms"] else 0.0
    traffic = ncu_traffic_per_launch(t["algorithmic_level_bytes"] / max(t["level_launches"], 1))
    roofline = {
        "bound": "hbm",
        "kernel": ("FDMT level phase: k_level2_pipe<__half> (two levels per pass) + k_level_pipe<__half> "
                   "(the rows no plane searches of single steps into searched levels; their searched rows are "
                   "computed inside the search kernel), plain FP16 single-beam run"),
        "achieved": round(level_gbs, 1),
        "peak": peak,
        "unit": "GB/s",
        "frac": round(level_gbs / peak, 4),
        "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else "fallback",
        "traffic": traffic,
        "algorithmic_bytes_per_launch": int(t["algorithmic_level_bytes"] / max(t["level_launches"], 1)),
        "launches": int(t["level_launches"]),
        "phase_ms_per_step": {k: round(t[k] / args.steps, 3) for k in
                              ("level1_ms", "level_ms", "search_ms", "history_ms", "variance_ms")},
    }
    # the unfused per-beam-gulp model: two raw passes and the normalised
    # waterfall's write and read, plus every FDMT level read and written once
    # with its history and every searched plane read once
    rfi_model = 2 * NCHANS * GULP * 1 + 2 * NCHANS * GULP * 4  # uint8 samples
    fdmt_model = t["unfused_model_bytes"] / max(t["executes"], 1)
    model = rfi_model + fdmt_model
    step_s = single16["total_ms"] / args.steps / 1e3
    roofline["unfused_model"] = {
        "bytes_per_beam_gulp": int(model), "rfi_bytes": int(rfi_model), "fdmt_search_bytes": int(fdmt_model),
        "achieved_gbs": round(model / step_s / 1e9, 1), "frac": round(model / step_s / 1e9 / peak, 4),
        "what": "unfused model bytes of one beam-gulp over the plain FP16 step time (fusion moves fewer bytes)"}
    from frost_b200.search import candidate_list_diff
    fp16_vs_fp32 = candidate_list_diff(single32["last"], served["last0"], 7.0)
    fp16_vs_fp32["what"] = ("served FP16 beam 0 against the plain FP32 path on the same gulp after the same "
                            "number of gulps, detections above S/N 7 (same plane, DM, width and peak sample)")
    st = served["stats"]
    lat1 = sorted(single16["lat"])
    p = lambda q: lat1[min(len(lat1) - 1, int(round(q * (len(lat1) - 1))))]
    n_gulps = served["beams"] * args.steps
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(served["total_ms"] / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (fp16 plane storage)",
        "data": ("synthetic (seeded filterbank, 4096-channel noise/RFI/pulse recipe); each served beam has its "
                 "own seeded gulp, replayed every step (beam 0's is the plain paths' gulp)"),
        "config": {"workload": WORKLOAD, "storage": "fp16", "served_beams_per_gpu": served["beams"],
                   "step": f"one gulp of each of the {served['beams']} served beams",
                   "served_tile_nsamps": args.served_tile or GULP,
                   "l2": "inputs larger than L2 (1 GiB raw gulp per beam-gulp)",
                   "timing": "CUDA events bracketing device-wide synchronisations (beams run on their own streams)",
                   "parallelism": f"replicas x{world}"},
        "latency_ms": {"p50": round(st.p50_latency_s * 1e3, 2), "p99": round(st.p99_latency_s * 1e3, 2),
                       "max": round(st.max_latency_s * 1e3, 2), "realtime_gulp_ms": gulp_s * 1e3,
                       "what": "served gulp, submit to candidates ready, one gulp in flight per beam"},
        "plain_fp32": {"value": round(plain32, 3), "ms_per_step": round(single32["total_ms"] / args.steps, 3),
                       "what": "single beam, FP32 planes, no server", "launch_shape": single32["tuned"]},
        "plain_fp16": {"value": round(plain16, 3), "ms_per_step": round(single16["total_ms"] / args.steps, 3),
                       "p50_ms": round(p(0.5), 2), "p99_ms": round(p(0.99), 2),
                       "launch_shape": single16["tuned"]},
        "plain_fp16_host_input": {
            "value": round(per_beam_steps * gulp_s / (single16_host["total_ms"] / 1e3), 3),
            "what": "plain FP16 from pinned host gulps, copied inside each gulp's call (no overlap)"},
        "plain_fp16_prefetch": {
            "value": round(per_beam_steps * gulp_s / (single16_pf["total_ms"] / 1e3), 3),
            "read_ms_per_gulp": single16_pf["read_ms_per_gulp"],
            "caller_wait_ms_per_gulp": single16_pf["wait_ms_per_gulp"],
            "what": "plain FP16 fed by GulpPrefetch (reader thread: host memory -> pinned slots -> device, "
                    "depth 3), overlapping the next gulp's read and copy with the current search"},
        "served_with_postprocess": {
            "value": round(served_pp["beams"] * per_beam_steps * gulp_s / (served_pp["total_ms"] / 1e3), 3),
            "p99_ms": round(served_pp["stats"].p99_latency_s * 1e3, 2),
            "giants_per_beam_gulp": round(served_pp["ncands"] / max(served_pp["beams"] * args.steps, 1), 1),
            "what": "the same served beams with frost's per-gulp post-processing (clustering, DM wings, carry, "
                    "sub-band dedup) on the device after each search"},
        "served_vs_plain_fp32": round(value / plain32, 3),
        "fp16_vs_fp32": fp16_vs_fp32,
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                "h2d_bytes_per_step": nbytes * e2e["beams"],
                "d2h_bytes_per_step": int(e2e["d2h"] / args.steps),
                "what": "served beams fed from pinned host gulps through frost_server_submit",
                "gulps_in_flight_per_beam": max(1, args.staging), "staging_blocks_per_beam": max(0, args.staging)},
        "gpu_launches": int(st.launches),
        "roofline": roofline,
        "clocks": served["clocks"],
        "candidates_per_beam_gulp": round(served["ncands"] / max(n_gulps, 1), 1),
        "dropped_last_step": single16["dropped"],
        "rfi_stage_ms_last_step": single16["rfi_ms"],
        "rfi_counts_last_step": single16["rfi_counts"],
        "device_bytes_served": int(st.device_bytes),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


CPU_SAMPLE = 16384  # rows of the gulp timed on the host cores


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline(sample=CPU_SAMPLE, steps=1):
    """The reference's CPU RFI cleaner (oracle/_ref, shipped -O3 -ffast-math
    build) plus this project's CPU port of the FDMT + boxcar search
    (oracle/cpu_fdmt.c; the reference's own engine, dmt, is not available)
    on a `sample`-row block of the same recipe; beam-s/s of that work."""
    from frost_b200.config import DedispPlanConfig
    from frost_b200.synth import config2_gulp
    from oracle import ref
    from oracle.fdmt import cpu_search, widths

    raw = config2_gulp(seed=0x46524F5354, nsamps=sample, n_pulses=2).data
    lay = layout(sample)
    full = layout()
    # frost's plan arguments (make_dedisp_plan_config, lib/pipeline/pipeline.cpp:290-304);
    # the DM list and band edges come from the reference's own lib/dedisp
    # compiled into oracle/_ref, so this leg maps none of this repo's libraries
    plan = DedispPlanConfig(nchans=full.nchans, dt=float(full.tsamp), f0=float(full.f0), df=float(full.df),
                            dm_min=0.0, dm_max=DM_MAX, dm_pulse_width=40.0, dm_tol=1.25,
                            block_nsamps=full.max_nsamps, subband_depth=DEPTH)
    f_min, f_max = ref.fdmt_band_edges(plan)
    dms = ref.generate_dm_list(plan)
    ws = widths(MAX_BOXCAR, 2.0)
    fast = ref.available(fast=True)
    cleaner = ref.RefRFICleaner(rfi_config(), lay, 2.0, fast=fast)
    t_rfi = t_fdmt = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        wf = cleaner.execute_normalized(raw.reshape(-1))
        t1 = time.perf_counter()
        cpu_search(wf, f_min, f_max, TSAMP, dms, DEPTH, ws, 6.0)
        t2 = time.perf_counter()
        t_rfi += t1 - t0
        t_fdmt += t2 - t1
    beam_s = steps * sample * TSAMP
    return {"value": round(beam_s / (t_rfi + t_fdmt), 4), "unit": UNIT,
            "cores": os.cpu_count(), "cpu_model": cpu_model(), "kind": "port",
            "sample": (f"{steps} x {sample} rows x 4096 ch: reference RFICleaner "
                       f"({'shipped -ffast-math' if fast else 'strict'} build of its own sources) "
                       f"{t_rfi:.2f} s + CPU port of FDMT+boxcar (11 planes, widths 1-256, zero "
                       f"history) {t_fdmt:.2f} s; OpenMP threads={os.cpu_count()}")}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    if args.warmup > 0:
        cpu_baseline(steps=1)
    cb = cpu_baseline(steps=args.steps)
    value = cb["value"]
    total = args.steps * CPU_SAMPLE * TSAMP / value
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD + f"; each step a {CPU_SAMPLE}-row sample",
                       "parallelism": "host cores"},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": os.cpu_count(),
                             "cpu_model": cb["cpu_model"], "kind": "port", "sample": cb["sample"] if cb else ""},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


SERVING = dict(beams=64, gulp=65536, gulps=4, tile=16384, slots=8, jitter_s=0.05)


def serving_gulp(beam, C, is_float, dm_max):
    """One beam's seeded 65536-sample gulp of the 4096-channel recipe scaled
    to its band: 4 dispersed pulses (DM 100 to dm_max - 100, widths 1-128,
    S/N 7-50), 5 % noisy channels, 5 zero-DM bursts and a dropout."""
    from frost_b200.synth import make_filterbank
    foff = -336.0 / C
    return make_filterbank(C, SERVING["gulp"], 1536.0 + foff / 2, foff, TSAMP, beam_seed(0, 1000 + beam),
                           dtype="float32" if is_float else "uint8", n_pulses=4,
                           dm_range=(100.0, dm_max - 100.0), width_range=(1.0, 128.0), snr_range=(7.0, 50.0),
                           rfi_channel_fraction=0.05, n_bursts=5, n_dropouts=1).data


def run_serving(args):
    """Beams at real-time cadence: 64 simulated beams (1024 or 4096 channels,
    uint8 or float32, DM max 1000-3000, 4 sub-band planes) each emit their
    own seeded 65536-sample gulps (the noise, RFI and pulse recipe) every
    65536 x 64 us = 4.19 s with exponential arrival jitter; the server
    admits beams by device memory and reports the gulp latency (arrival to
    candidates ready) of every gulp after each beam's first."""
    import numpy as np
    import torch

    from frost_b200._lib import FrostError
    from frost_b200.config import BlockLayout, DataType
    from frost_b200.pipeline import plan_for
    from frost_b200.serve import BeamServer

    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    S = SERVING
    gulp, cadence = S["gulp"], S["gulp"] * TSAMP
    rng = np.random.default_rng(0x46524F5354)
    classes = [(1024, DataType.UINT8), (1024, DataType.FLOAT32), (4096, DataType.UINT8),
               (4096, DataType.FLOAT32)]
    srv = BeamServer(device=local, slots=S["slots"])
    from frost_b200.config import BoxcarConfig, Storage as St
    bc = BoxcarConfig(max_boxcar=256, wtsp=2.0, detect_thresh=6.0, storage=St.FP16,
                      max_candidates=1 << 18, max_cands_per_dm=4096, tile_nsamps=S["tile"])
    admitted, refused = [], 0
    t_gen = time.perf_counter()
    for b in range(S["beams"]):
        C, dt = classes[b % 4]
        foff = -336.0 / C
        dm_max = float(rng.uniform(1000.0, 3000.0))
        lay = BlockLayout(C, gulp, dt, TSAMP, 1536.0 + foff / 2, foff)
        plan = plan_for(lay, 0.0, dm_max, 1)
        try:
            bid = srv.add_beam(rfi_config(), lay, 2.0, plan, bc)
        except FrostError as e:
            if e.code != -2:
                raise
            refused += 1
            continue
        data = serving_gulp(b, C, dt == DataType.FLOAT32, dm_max)
        buf = torch.empty(data.nbytes, dtype=torch.uint8, pin_memory=True)
        buf.copy_(torch.from_numpy(np.ascontiguousarray(data).reshape(-1).view(np.uint8)))
        admitted.append((bid, buf, (C, dt)))
        del data
    t_gen = time.perf_counter() - t_gen
    events = []
    for bid, _, _ in admitted:
        off = float(rng.uniform(0.0, cadence))
        for g in range(S["gulps"]):
            events.append((off + g * cadence + float(rng.exponential(S["jitter_s"])), bid, g))
    events.sort()
    bufs = {bid: buf for bid, buf, _ in admitted}
    lat, lock = [], threading.Lock()
    pending, ncands = [], [0]

    def waiter(ticket, g):
        cands, l = srv.wait(ticket)
        with lock:
            ncands[0] += cands.size
            if g > 0:
                lat.append(l)

    sampler = ClockSampler(local)
    sampler.__enter__()
    t0 = time.perf_counter()
    for at, bid, g in events:
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        buf = bufs[bid]
        t = srv.submit_ptr(bid, buf.data_ptr(), buf.numel(), gulp, on_device=False)
        th = threading.Thread(target=waiter, args=(t, g))
        th.start()
        pending.append(th)
    for th in pending:
        th.join()
    wall = time.perf_counter() - t0
    sampler.__exit__(None, None, None)
    st = srv.stats()
    lat.sort()
    q = lambda f: lat[min(len(lat) - 1, int(round(f * (len(lat) - 1))))] if lat else None
    beam_s = len(admitted) * S["gulps"] * cadence
    mix = {}
    for _, _, (C, dt) in admitted:
        k = f"{C}ch_{'f32' if dt == DataType.FLOAT32 else 'u8'}"
        mix[k] = mix.get(k, 0) + 1
    line = {
        "metric": "served beams at real-time cadence; p50/p99 gulp latency",
        "value": round(beam_s / wall, 3), "unit": UNIT, "n_gpus": 1, "steps": S["gulps"], "warmup": 1,
        "ms_per_step": round(wall * 1e3 / S["gulps"], 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (fp16 plane storage)",
        "data": ("synthetic: every admitted beam its own seeded gulp (noise, 5 % noisy channels, bursts, a "
                 "dropout, 4 dispersed pulses), replayed at each of its arrivals"),
        "config": {"workload": "64 beams: 1024/4096 ch, uint8/float32, DM max U[1000,3000], 4 planes, "
                               "65536-sample gulps at 64 us cadence with exponential jitter "
                               f"(mean {S['jitter_s']} s)",
                   "beams_offered": S["beams"], "beams_admitted": len(admitted), "beams_refused": refused,
                   "admitted_mix": mix, "device_bytes_admitted": int(st.device_bytes), "slots": S["slots"],
                   "tile_nsamps": S["tile"], "gulp_generation_s": round(t_gen, 1)},
        "latency_ms": {"p50": round(q(0.5) * 1e3, 1), "p99": round(q(0.99) * 1e3, 1),
                       "max": round(lat[-1] * 1e3, 1), "realtime_gulp_ms": round(cadence * 1e3, 1),
                       "gulps_timed": len(lat)},
        "p99_below_realtime": bool(lat and q(0.99) < cadence),
        "candidates_per_gulp": round(ncands[0] / max(len(events), 1), 1),
        "clocks": sampler.summary(),
    }
    srv.close()
    print(json.dumps(line), flush=True)


def postprocess_config(nrows):
    from frost_b200.postprocess import SearchConfig
    return SearchConfig(boxcar_max=MAX_BOXCAR, detect_thresh=6.0, max_candidates=max(nrows, 1))


def run_postprocess(args):
    """Candidate post-processing of the headline workload's own detections:
    one FP16 gulp of the config-2 beam is searched, and its raw candidates
    (every plane, DM trial and width above S/N 6) are replayed gulp after
    gulp with their samples advanced by a gulp each step, so clusters carry
    across gulps as in a stream. A step is CandidatePostprocessPlan::execute
    over one gulp's rows (chain clustering per plane, DM wings, carry,
    sub-band dedup), input resident on the device. The reference arm's CPU
    plan (its own lib/search sources) runs on the same rows."""
    import numpy as np
    import torch

    from frost_b200.config import Storage
    from frost_b200.pipeline import GulpPipeline, plan_for
    from frost_b200.postprocess import CandidatePostprocessLayout, CandidatePostprocessPlan

    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    raw_host = make_gulp(0x46524F5354)
    raw_dev = torch.from_numpy(raw_host.reshape(-1)).to(dev)
    del raw_host
    lay = layout()
    plan = plan_for(lay, 0.0, DM_MAX, DEPTH)
    pipe = GulpPipeline(rfi_config(), lay, 2.0, plan, search_config(Storage.FP16), device=local)
    pipe.execute_device(raw_dev.data_ptr(), GULP, on_device=True)
    cands = pipe.execute_device(raw_dev.data_ptr(), GULP, on_device=True).candidates.copy()
    del pipe, raw_dev
    torch.cuda.empty_cache()
    n = cands.size
    nsteps = args.warmup + args.steps

    def shifted(i):
        c = cands.copy()
        for f in ("peak_sample", "begin_sample", "end_sample"):
            c[f] = c[f] + np.uint64(i * GULP)
        return c

    gulps = [shifted(i) for i in range(nsteps)]
    dev_rows = [torch.from_numpy(g.view(np.uint8)).to(dev) for g in gulps]
    cfg = postprocess_config(n)
    ppl = CandidatePostprocessLayout(NCHANS, TSAMP, FOFF)
    pp = CandidatePostprocessPlan(cfg, ppl, device=local)
    frontier_lag = MAX_BOXCAR

    def step(i, rows_ptr=None):
        sr = (i + 2) * GULP
        if rows_ptr is None:
            return pp.execute(gulps[i], sr, GULP, False, sr - frontier_lag)
        return pp.execute_device(rows_ptr, n, sr, GULP, False, sr - frontier_lag)

    for i in range(args.warmup):
        step(i, dev_rows[i].data_ptr())
    torch.cuda.synchronize()
    times, out_rows, pend, launches, phases = [], 0, 0, 0, [0.0, 0.0]
    for i in range(args.warmup, nsteps):
        t0 = time.perf_counter()
        r = step(i, dev_rows[i].data_ptr())
        times.append(time.perf_counter() - t0)
        out_rows += r.candidates.size
        pend = r.pending_candidates
        launches += r.launches
        phases[0] += r.cluster_s
        phases[1] += r.dedup_s
    ms = 1e3 * sum(times) / len(times)
    # end to end: host rows in, giants out (the C ABI's host path)
    pp_e2e = CandidatePostprocessPlan(cfg, ppl, device=local)
    e2e_t = []
    for i in range(nsteps):
        sr = (i + 2) * GULP
        t0 = time.perf_counter()
        pp_e2e.execute(gulps[i], sr, GULP, False, sr - frontier_lag)
        if i >= args.warmup:
            e2e_t.append(time.perf_counter() - t0)
    e2e_ms = 1e3 * sum(e2e_t) / len(e2e_t)
    line = {"metric": "candidate rows post-processed/s @4096ch DM2000", "value": round(n / (ms / 1e3), 1),
            "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64/u64 (coincidence arithmetic)", "data": "the search's own detections of a synthetic "
            "config-2 gulp, replayed with samples advanced a gulp per step",
            "config": {"workload": f"CandidatePostprocessPlan over {n} raw rows per gulp (11 planes, "
                                   "chain + DM wings + carry + transitive sub-band dedup, frost defaults)",
                       "rows_per_gulp": n, "giants_out_per_gulp": round(out_rows / args.steps, 1),
                       "pending_after_last": pend},
            "phase_ms_per_step": {"cluster": round(1e3 * phases[0] / args.steps, 3),
                                  "dedup": round(1e3 * phases[1] / args.steps, 3)},
            "e2e": {"value": round(n / (e2e_ms / 1e3), 1), "unit": "rows/s",
                    "h2d_bytes_per_step": int(gulps[0].nbytes), "d2h_bytes_per_step": None,
                    "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": launches}
    if not args.no_cpu_baseline:
        from oracle import postprocess as op
        if op.ref_available():
            rp = op.backend("reference").plan(cfg, ppl)
            t = []
            for i in range(min(nsteps, 2)):
                sr = (i + 2) * GULP
                t0 = time.perf_counter()
                rp.execute(gulps[i], sr, GULP, False, sr - frontier_lag)
                t.append(time.perf_counter() - t0)
            line["cpu_baseline"] = {"value": round(n / t[-1], 1), "unit": "rows/s", "cores": 1,
                                    "kind": "reference", "ms_per_gulp": round(1e3 * t[-1], 1),
                                    "sample": "the reference's own CandidatePostprocessPlan (lib/search "
                                              "sources, strict build) on the second replayed gulp"}
    print(json.dumps(line), flush=True)


BATCH = dict(beams=32, tile=32768)


def batch_beams(n):
    """The multi-beam workload's beams, seeded: channels 1024 / 2048 / 4096,
    uint8 or float32, gulps of 2^15 - 2^18 samples, DM max 500 - 3000, 1, 4
    or 11 sub-band planes. A gulp must exceed the beam's largest dispersion
    delay plus the widest boxcar (frost's rule), so a drawn length is doubled
    until it does (1200-1536 MHz at 64 us: 17.54 samples per unit DM)."""
    import numpy as np
    rng = np.random.default_rng(0x46524F5354 ^ 3)
    out = []
    for b in range(n):
        C = int(rng.choice([1024, 2048, 4096]))
        f32 = bool(rng.integers(0, 2))
        T = int(2 ** rng.integers(15, 19))
        dm_max = float(round(rng.uniform(500.0, 3000.0), 1))
        depth = int(rng.choice([0, 1, 2]))
        while T <= 17.6 * dm_max + 2 * MAX_BOXCAR:
            T *= 2
        out.append(dict(C=C, f32=f32, T=T, dm_max=dm_max, depth=depth))
    return out


def batch_gulp(b, spec):
    """A beam's seeded gulp of the 4096-channel recipe scaled to its shape:
    pulses at DM 100 to dm_max - 100 (one per 2^15 samples), 5 % noisy
    channels, bursts and a dropout."""
    from frost_b200.synth import make_filterbank
    C, T = spec["C"], spec["T"]
    foff = -336.0 / C
    return make_filterbank(C, T, 1536.0 + foff / 2, foff, TSAMP, beam_seed(0, 2000 + b),
                           dtype="float32" if spec["f32"] else "uint8", n_pulses=max(1, T // 32768),
                           dm_range=(100.0, spec["dm_max"] - 100.0), width_range=(1.0, 128.0),
                           snr_range=(7.0, 50.0), rfi_channel_fraction=0.05, n_bursts=max(1, T // 16384),
                           n_dropouts=1).data


def run_config3(args):
    """Batched multi-beam search: 32 seeded beams of uneven shapes (channels,
    sample type, gulp length, DM range, plane count) searched together, one
    gulp of every beam per step, their level steps and searches run as
    single launches over all beams and replayed from a CUDA graph; beside it
    the same beams served concurrently by the server (one stream and worker
    per beam). Gulps resident on the device; beams admitted by memory."""
    import numpy as np
    import torch

    from frost_b200._lib import FrostError
    from frost_b200.batch import BeamBatch
    from frost_b200.config import BlockLayout, DataType, Storage
    from frost_b200.pipeline import plan_for
    from frost_b200.serve import BeamServer

    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    specs = batch_beams(BATCH["beams"])
    bc = search_config(Storage.FP16)
    bc.tile_nsamps = BATCH["tile"]

    def layout_of(sp):
        foff = -336.0 / sp["C"]
        return BlockLayout(sp["C"], sp["T"], DataType.FLOAT32 if sp["f32"] else DataType.UINT8, TSAMP,
                           1536.0 + foff / 2, foff)

    def admit(add):
        ids = []
        for sp in specs:
            lay = layout_of(sp)
            try:
                ids.append(add(rfi_config(), lay, 2.0, plan_for(lay, 0.0, sp["dm_max"], sp["depth"]), bc))
            except FrostError as e:
                if e.code != -2:
                    raise
                ids.append(None)
        return ids

    # the beams' device-resident gulps are allocated after admission: keep
    # their bytes (and 2 GiB) out of the batch's and the server's budgets
    gulp_bytes = sum(sp["T"] * sp["C"] * (4 if sp["f32"] else 1) for sp in specs)
    free, _ = torch.cuda.mem_get_info(local)
    budget = max(int(0.9 * (free - gulp_bytes - (2 << 30))), 1)
    batch = BeamBatch(device=local, memory_budget=budget)
    ids = admit(batch.add_beam)
    keep = [i for i, b in enumerate(ids) if b is not None]
    dev = {}
    t_gen = time.perf_counter()
    for i in keep:
        data = batch_gulp(i, specs[i])
        dev[i] = torch.from_numpy(np.ascontiguousarray(data).reshape(-1).view(np.uint8)).to("cuda")
        del data
    t_gen = time.perf_counter() - t_gen
    ptrs = [dev[i].data_ptr() for i in keep]
    nread = [specs[i]["T"] for i in keep]
    beam_s = sum(specs[i]["T"] for i in keep) * TSAMP

    def timed(step):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(args.steps):
            step()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / args.steps

    ms_batch = timed(lambda: batch.execute_ptrs(ptrs, nread, on_device=True))
    st = batch.stats()
    batch.close()
    torch.cuda.empty_cache()
    srv = BeamServer(device=local, memory_budget=budget, slots=len(keep))
    sid = admit(srv.add_beam)
    served = [i for i in keep if sid[i] is not None]

    def serve_step():
        tickets = [srv.submit_ptr(sid[i], dev[i].data_ptr(), dev[i].numel(), specs[i]["T"], True) for i in served]
        for t in tickets:
            srv.wait(t)
    ms_served = timed(serve_step)
    srv.close()
    mix = {}
    for i in keep:
        sp = specs[i]
        k = f"{sp['C']}ch_{'f32' if sp['f32'] else 'u8'}_{ {0: 1, 1: 4, 2: 11}[sp['depth']]}p"
        mix[k] = mix.get(k, 0) + 1
    line = {
        "metric": "beam-s searched/s, batched uneven beams", "value": round(beam_s / (ms_batch / 1e3), 3),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_batch, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (fp16 plane storage)",
        "data": "synthetic: every beam its own seeded gulp (noise, RFI, pulses), resident on the device",
        "config": {"workload": f"{BATCH['beams']} beams: 1024/2048/4096 ch, uint8/float32, gulps 2^15-2^18, "
                               "DM max U[500,3000], 1/4/11 planes, boxcar 1-256; one gulp of every beam a step",
                   "beams_offered": len(specs), "beams_admitted": len(keep), "mix": mix,
                   "fdmt_tile_nsamps": BATCH["tile"], "gulp_generation_s": round(t_gen, 1)},
        "batch_stats": st,
        "served": {"value": round(sum(specs[i]["T"] for i in served) * TSAMP / (ms_served / 1e3), 3),
                   "ms_per_step": round(ms_served, 3), "beams": len(served),
                   "what": "the same beams through the server, one worker and stream per beam"},
    }
    print(json.dumps(line), flush=True)


def run_pipeline(args):
    """One plain FP16 pipeline (RFI, FDMT, search) over the seeded gulp of
    `--pipeline-config` (config1: 1024 channels, 65536 samples; config2: the
    headline gulp), W warm-up gulps then K timed ones, with the engine's
    per-phase CUDA-event times. The small case for multi-pass ncu captures
    of the FDMT and search kernels; not the headline metric."""
    import numpy as np
    import torch

    from frost_b200.config import Storage
    from frost_b200.pipeline import GulpPipeline, plan_for

    select_workload(args.pipeline_config)
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    lay = layout()
    raw = torch.from_numpy(np.ascontiguousarray(make_gulp(0x46524F5354)).reshape(-1)).to("cuda")
    pipe = GulpPipeline(rfi_config(), lay, 2.0, plan_for(lay, 0.0, DM_MAX, DEPTH), search_config(Storage.FP16),
                        device=local)
    for _ in range(args.warmup):
        pipe.execute_device(raw.data_ptr(), GULP, on_device=True)
    torch.cuda.synchronize()
    pipe.search.enable_timing(True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(args.steps):
        res = pipe.execute_device(raw.data_ptr(), GULP, on_device=True)
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    t = pipe.search.timing()
    print(json.dumps({"metric": "plain FP16 pipeline, beam-s searched per second",
                      "value": round(GULP * TSAMP / (ms / 1e3), 3), "unit": UNIT, "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f32 (fp16 plane storage)", "data": "synthetic",
                      "config": {"workload": WORKLOAD}, "candidates": int(res.candidates.size),
                      "phase_ms_per_step": {k: round(t[k] / args.steps, 3) for k in
                                            ("level1_ms", "level_ms", "search_ms", "history_ms")},
                      "algorithmic_level_bytes_per_launch":
                          int(t["algorithmic_level_bytes"] / max(t["level_launches"], 1))}), flush=True)


def run_rfi(args):
    """The RFI stage of the headline gulp alone (4096 channels, uint8, the
    config-2 RFI recipe and strategies: bandpass, moments, IQRM, Kadane in
    time and frequency, zero-DM) on its first `--rfi-nsamps` samples: one
    step cleans and normalises one block on the device. A profiling case for
    the order-exact statistics kernels, small enough for multi-pass ncu
    captures; not the headline metric."""
    import numpy as np
    import torch

    from frost_b200.rfi import RFICleaner

    select_workload("config2")
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    n = int(args.rfi_nsamps)
    raw = np.ascontiguousarray(make_gulp(0x46524F5354)[:n])
    dev = torch.from_numpy(raw.reshape(-1)).to("cuda")
    cl = RFICleaner(rfi_config(), layout(n), 2.0, device=local)
    for _ in range(args.warmup):
        cl.execute_normalized_device(dev.data_ptr(), raw.size, n, on_device=True)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(args.steps):
        cl.execute_normalized_device(dev.data_ptr(), raw.size, n, on_device=True)
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    rep = cl.report()
    print(json.dumps({"metric": "RFI stage, samples cleaned per second", "value": round(n / (ms / 1e3), 1),
                      "unit": "samples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f64 statistics, f32 output", "data": "synthetic",
                      "config": {"workload": f"4096ch uint8, config-2 RFI recipe, first {n} samples of the gulp"},
                      "rfi_stage_ms": {k: round(rep[k] * 1e3, 2) for k in
                                       ("t_bandpass", "t_moments", "t_scan", "t_flags", "t_apply")}}),
          flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["frost", "reference"], default="frost")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["serving", "postprocess", "rfi", "config3",
                                                              "pipeline"],
                    default="config2",
                    help="config2 (headline), config1 (1024-channel profiling case), serving "
                         "(64 beams at real-time cadence), postprocess (candidate clustering and "
                         "dedup of the headline gulp's detections), rfi (the RFI stage alone, a "
                         "profiling case), pipeline (one plain FP16 pipeline, a profiling case) or "
                         "config3 (32 uneven beams searched as one batch)")
    ap.add_argument("--beams", type=int, default=3, help="served beams per GPU (admitted by memory)")
    ap.add_argument("--staging", type=int, default=0,
                    help="e2e leg: staging blocks (and gulps in flight) per beam; 0 = one gulp in flight, "
                         "uploaded when it is processed")
    ap.add_argument("--served-tile", type=int, default=0,
                    help="FDMT tile of the served beams in samples (0 = the whole gulp)")
    ap.add_argument("--pipeline-config", choices=sorted(WORKLOADS), default="config1",
                    help="the pipeline workload's gulp geometry")
    ap.add_argument("--rfi-nsamps", type=int, default=131072,
                    help="samples of the headline gulp the rfi workload cleans per step")
    args = ap.parse_args()
    if args.workload == "config3":
        run_config3(args)
        return
    if args.workload == "rfi":
        run_rfi(args)
        return
    if args.workload == "pipeline":
        run_pipeline(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "postprocess":
        run_postprocess(args)
        return
    select_workload(args.workload)
    if args.warmup < 3 and args.impl == "frost":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
