"""Benchmark: binary-pursuit throughput (Msample*ch/s) on B200.

Workload (default): the 16-channel linear-probe recording, 40 kHz, 10 min
float32 (N = 24e6 samples per channel), 40 templates of 101 samples/channel on
4-6 channel neighbourhoods, lognormal rates (median 10 Hz, cap 80 Hz), 20% of
spikes forced to overlap, overlap recheck on with n_max_shift_inds = W - 1.
Synthetic, seeded (spikesorting_fullpursuit_b200.synth); no dataset.

A step is one full binary pursuit of the recording (all passes, overlap
recheck included) -- the unit the metric is quoted on.
* value: device-resident throughput of the chosen ("fast") path: the chunk's
  voltage is already in HBM; per step the pristine voltage is restored into
  the working buffer outside the timed interval; each step is timed with CUDA
  events on the launching stream; inputs (1.5 GB voltage, 3.8 GB likelihood)
  are far larger than L2.
* e2e: the public API binary_pursuit() with host numpy voltage in and host
  numpy spikes out (host<->device copies inside the timed region).
* plain_fp32: the plain FP32 path on the same data, and the fraction of spikes
  (index, label) the chosen path shares with it.

Multi-GPU (torchrun): the path shards by recording (each rank pursues its own
recording, no data-path collective): weak scaling, max time over ranks.

--impl reference: the reference's OpenCL kernels compiled for the host CPU
(oracle/_ref) on a bounded leading slice of the same workload.
"""
from __future__ import annotations

import argparse
import copy
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "binary-pursuit Msample·ch/s, chosen vs plain FP32 on B200, ≥99.9% spike match"


# DRAM bytes per unit measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of one
# launch of the 60 s slice of the linear16 workload, divided by the windows it processed)
DRAM_PER_UNIT = {
    "lik_tc_kernel": (17.0e3, "listed", "profiles/lik_tc_persist_kernel_linear16_60s.md: 105.9 MB / 6,240 windows"),
    "partial_corr_kernel": (35.8e3, "flagged", "profiles/partial_corr_kernel_linear16_60s.md: 107.3 MB / 3,001 windows"),
    "screen_kernel": (39.1e3, "flagged", "profiles/screen_kernel_linear16_60s.md: 117.3 MB / 3,001 windows"),
    "argmax_kernel": (18.8, "listed", "profiles/residual_accept_compact_linear16_60s.md: argmax_lazy_kernel, "
                      "0.45 MB / 23,808 windows"),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="linear16", choices=["linear16", "tetrode", "dense64", "batched"])
    p.add_argument("--batch-streams", type=int, default=8,
                   help="batched: segments pursued at once (one CUDA stream and host thread each)")
    p.add_argument("--batch-scale", type=float, default=1.0,
                   help="batched: segment durations times this factor (1.0: uniform 5-60 s)")
    p.add_argument("--autotune", action="store_true",
                   help="batched: launch shapes measured per segment shape (spikesorting_fullpursuit_b200.autotune)")
    p.add_argument("--duration", type=float, default=None, help="seconds of recording (default: config's)")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--gpu-synth", action="store_true",
                   help="generate the recording's noise on the GPU (for the full-length dense 64-channel recording)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample-s", type=float, default=1.0)
    p.add_argument("--adjoint", action="store_true",
                   help="time the residual-energy gradient (template refinement) on the 16-ch, 2 min, "
                        "40-template workload instead of the pursuit")
    p.add_argument("--only-device", action="store_true",
                   help="time the device-resident steps only (no e2e, plain, stage or CPU legs); for profiling")
    return p.parse_args()


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


def leading_slice(V, si, seconds):
    """The first `seconds` of a recording (same templates and thresholds)."""
    n = min(V.shape[1], max(si["n_samples_per_chan"] + 1, int(round(seconds * si["sampling_rate"]))))
    return np.ascontiguousarray(V[:, :n]), dict(si, n_samples=n)


def run_reference(args, rank):
    """The reference kernels on the host cores, on a bounded leading slice of
    the same recording the other arm pursues (same seed, templates, thresholds)."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    from spikesorting_fullpursuit_b200 import synth
    import ref_host
    Vfull, sifull, sm, _ = synth.config_recording(args.config, seed=1, duration_s=args.duration)
    # warm-up steps load the library and touch the code path on a 0.1 s slice; the timed
    # slice is sized from the warm-up rate so that the K timed steps take about 150 s
    Vw, siw = leading_slice(Vfull, sifull, 0.1)
    Ww = siw["n_samples_per_chan"]
    rate = None
    for _ in range(args.warmup):
        t0 = time.perf_counter()
        ref_host.binary_pursuit(Vw, siw, copy.deepcopy(sm), n_max_shift_inds=Ww - 1)
        rate = Vw.shape[1] / (time.perf_counter() - t0)   # samples per second
    sample_s = args.cpu_sample_s
    if rate:
        sample_s = float(np.clip(150.0 / max(1, args.steps) * rate / siw["sampling_rate"], 0.25, args.cpu_sample_s))
    V, si = leading_slice(Vfull, sifull, sample_s)
    W = si["n_samples_per_chan"]
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref_host.binary_pursuit(V, si, copy.deepcopy(sm), n_max_shift_inds=W - 1)
        times.append(time.perf_counter() - t0)
    tot = float(np.sum(times))
    value = V.shape[0] * V.shape[1] * len(times) / tot / 1e6
    cores = ref_host.threads()
    line = {
        "metric": METRIC, "value": value, "unit": "Msample*ch/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": "%s (leading %.2f s slice of the seed-1 recording)" % (args.config, sample_s)},
        "cpu_baseline": {"value": value, "unit": "Msample*ch/s", "cores": cores, "kind": "reference",
                         "sample": "leading %.2f s of the %s recording (seed 1), %d channels, reference OpenCL "
                                   "kernels compiled for the CPU, host loop restated" %
                                   (sample_s, args.config, V.shape[0])},
        "e2e": {"value": value, "unit": "Msample*ch/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.adjoint:
        run_adjoint(args)
        return
    if args.config == "batched":
        run_batched(args)
        return
    import torch
    import torch.distributed as dist
    from spikesorting_fullpursuit_b200 import _native, binary_pursuit, synth
    from spikesorting_fullpursuit_b200.overlap.binary_pursuit_parallel import plan_chunks

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=dev)
    assert args.warmup >= 3, "at least 3 warm-up steps"
    if args.gpu_synth:
        # recordings too long to band-pass on the host: noise drawn and filtered on the device
        Vg, si, sm = synth.config_recording_gpu(args.config, seed=1 + rank, device=dev, duration_s=args.duration)
        V = Vg.cpu().numpy()
        del Vg
        torch.cuda.empty_cache()
    else:
        V, si, sm, _ = synth.config_recording(args.config, seed=1 + rank, duration_s=args.duration)
    C, N = V.shape
    W = si["n_samples_per_chan"]
    S = W - 1
    T = np.float32(sm["templates"])
    M = T.shape[0]
    bias = np.float32(-0.5 * sm["template_SS"])
    theta = np.float32(sm["neuron_lower_thresholds"])
    total_mem = torch.cuda.get_device_properties(dev).total_memory
    onsets, chunk = plan_chunks(N, C, M, W, si["sampling_rate"], S, total_mem)
    assert len(onsets) == 1 and chunk >= N, "workload must fit one chunk"
    lib = _native.lib()
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    Vd0 = torch.from_numpy(V).to(dev)
    Vw = torch.empty_like(Vd0)
    Td = torch.from_numpy(T).to(dev)
    bd = torch.from_numpy(bias).to(dev)
    thd = torch.from_numpy(theta).to(dev)
    d = _native.dims(C, N, M, W, S)
    cap = 16 * (N // W + 1) + 1024   # every pass adds at most one spike per window; dense probes need several passes
    idx = torch.empty(cap, dtype=torch.int32, device=dev)
    lab = torch.empty(cap, dtype=torch.int32, device=dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def run_mode(mode_flags, steps, warmup, timing=False):
        flags = mode_flags | _native.FBP_OVERLAP_RECHECK | (_native.FBP_TIMING if timing else 0)
        ws = torch.empty(_native.workspace_bytes(d, flags), dtype=torch.uint8, device=dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms, stats, result = [], None, None
        for i in range(warmup + steps):
            Vw.copy_(Vd0)
            n = ctypes.c_uint32(0)
            st = _native.FbpChunkStats()
            if i == warmup:
                if world > 1:
                    dist.barrier()
                torch.cuda.synchronize()
            ev0.record(stream)
            _native.check(lib.fbp_pursue_chunk(ctypes.byref(d), flags, P(Vw), P(Td), P(bd), P(thd), P(ws),
                                               ws.numel(), P(idx), P(lab), cap, ctypes.byref(n),
                                               ctypes.byref(st), _native.MAX_PASSES, sptr))
            ev1.record(stream)
            torch.cuda.synchronize()
            if i >= warmup:
                ms.append(ev0.elapsed_time(ev1))
            stats = st.as_dict()
            k = n.value
            result = (idx[:k].cpu().numpy(), lab[:k].cpu().numpy())
        del ws
        return ms, stats, result

    # chosen path, device-resident
    with Clocks(local) as clk:
        ms_fast, st_fast, res_fast = run_mode(0, args.steps, args.warmup)
    clocks = clk.summary()
    t_fast = sum(ms_fast)
    if world > 1:
        t = torch.tensor([t_fast], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_fast = float(t.item())
    units = C * N * args.steps * world
    value = units / (t_fast * 1e-3) / 1e6
    if args.only_device:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "Msample*ch/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_fast / args.steps,
                              "config": {"workload": args.config, "samples": N, "channels": C},
                              "stats": st_fast, "clocks": clocks}), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    # per-stage breakdown (separate untimed run with stage events)
    _, st_stage, _ = run_mode(0, 1, 0, timing=True)

    # e2e through the public API (host in, host out)
    sm_e2e = copy.deepcopy(sm)
    binary_pursuit(V, np.float32, si, sm_e2e, n_max_shift_inds=S, verbose=False)  # warm
    e2e_ms = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=S, verbose=False)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_t = float(np.sum(e2e_ms))
    if world > 1:
        t = torch.tensor([e2e_t], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
    e2e_value = C * N * len(e2e_ms) * world / (e2e_t * 1e-3) / 1e6
    n_sp = len(out[0])

    plain = None
    # the plain path's brute-force recheck costs (2S+1)^2 * M * C * W multiply-adds per flagged
    # window; above ~1e10 (e.g. 64 ch, 200 templates) one pursuit would take hours
    plain_work = (2 * S + 1) ** 2 * M * C * W
    if not args.no_plain and plain_work > 1e10:
        plain = {"skipped": "brute-force recheck of %.1e multiply-adds per flagged window" % plain_work}
    elif not args.no_plain:
        ms_plain, _, res_plain = run_mode(_native.FBP_PLAIN_FP32, 1, 1)
        _, st_plain, _ = run_mode(_native.FBP_PLAIN_FP32, 1, 0, timing=True)   # stage times (serialised)
        a = set(zip(res_fast[0].tolist(), res_fast[1].tolist()))
        b = set(zip(res_plain[0].tolist(), res_plain[1].tolist()))
        match = len(a & b) / max(1, len(a | b))
        plain = {"value": C * N / (ms_plain[0] * 1e-3) / 1e6, "unit": "Msample*ch/s",
                 "ms_per_step": ms_plain[0], "spike_match": match,
                 "identical_order": bool(np.array_equal(res_fast[0], res_plain[0])
                                         and np.array_equal(res_fast[1], res_plain[1])),
                 "stages_ms": {k: v for k, v in st_plain.items() if k.startswith("ms_")}}

    hbm, tflops, peak_kind = load_peaks()
    # per-kernel device time of one step (separate run with FBP_TIMING) and the
    # algorithmic work each kernel family does in that step
    S2 = 2 * S + 1
    listed, flagged = st_stage["listed"], st_stage["flagged"]
    # FP32 FMA issue peak of the SIMT pipes (148 SMs x 128 lanes x 2 flop) at the
    # median SM clock of the timed region (nominal max clock if no sample)
    fma_peak = 148 * 128 * 2 * (clocks.get("sm_mhz") or 1965.0) * 1e6 / 1e12
    fam = {
        "lik_tc_kernel": (st_stage["ms_lik_tc"], "tensor", 2.0 * M * C * W * W * listed,
                          "2*M*C*W*W flop per listed window (nominal dense product); launched as "
                          "lik_tc_persist_kernel up to 128 template columns, lik_tc_kernel above"),
        "fixup_kernel": (st_stage["ms_fixup"], "fp32", 2.0 * C * W * 4 * st_stage["fixup_runs_queued"],
                         "2*C*W flop per sample recomputed"),
        "partial_corr_kernel": (st_stage["ms_partial_corr"], "fp32", 2.0 * st_stage["pc_macs"],
                                "2 flop per multiply-add done (device counter)"),
        "screen_kernel": (st_stage["ms_screen"], "latency", None, "L2-latency-bound table scan"),
        "score_kernel": (st_stage["ms_score"], "latency", None, "one sequential C*W chain per candidate"),
        "argmax_kernel": (st_stage["ms_argmax"], "hbm", 24.0 * listed,
                          "3 window keys (8 B) per listed window (argmax_lazy_kernel)"),
    }
    kernels = {}
    for name, (ms, bound, work, what) in fam.items():
        if ms <= 0:
            continue
        if bound == "latency":
            kernels[name] = {"ms": ms, "bound": "latency", "note": what}
        elif bound == "hbm":
            ach = work / (ms * 1e-3) / 1e9
            kernels[name] = {"ms": ms, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                             "frac": ach / hbm, "work": what}
        elif bound == "tensor":
            ach = work / (ms * 1e-3) / 1e12
            kernels[name] = {"ms": ms, "bound": "tensor", "achieved": ach, "peak": tflops, "unit": "TFLOP/s",
                             "frac": ach / tflops, "work": what}
        else:
            ach = work / (ms * 1e-3) / 1e12
            kernels[name] = {"ms": ms, "bound": "fp32-simt", "achieved": ach, "peak": fma_peak,
                             "unit": "TFLOP/s", "frac": ach / fma_peak, "work": what,
                             "peak_kind": "nominal FP32 FMA issue rate at the sampled clock"}
    # the roofline line reports the dominant kernel among those bound by the tensor pipe
    # or by HBM; the FP32-pipe and latency-bound kernels are in `kernels`
    dom = max((k for k in kernels if kernels[k]["bound"] in ("tensor", "hbm")), key=lambda k: kernels[k]["ms"])
    roof = dict(kernels[dom])
    # DRAM bytes (read + write) per launch: ncu's per-unit figure from the captures in
    # profiles/ (60 s slice of this workload) times the units of an average launch here
    per_unit = DRAM_PER_UNIT.get(dom)
    traffic, traffic_detail = None, None
    if per_unit is not None:
        units = {"listed": listed, "flagged": flagged}[per_unit[1]]
        traffic = per_unit[0] * units / max(1, st_stage["passes"])   # bytes per launch
        traffic_detail = {"bytes_per_unit": per_unit[0], "unit": per_unit[1] + " window",
                          "launches_per_step": st_stage["passes"], "source": per_unit[2]}
    slowest = max(kernels, key=lambda k: kernels[k]["ms"])
    roof.update({"kernel": dom, "traffic": traffic, "traffic_detail": traffic_detail, "peak_kind": peak_kind,
                 "note": ("peak = measured dense bf16 burst (the kernel computes in TF32, whose nominal rate is half)"
                          if roof["bound"] == "tensor" else "peak = measured HBM copy bandwidth"),
                 "slowest_kernel": slowest})
    launches = int(st_fast["launches"]) * args.steps

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, V, si, sm)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Msample*ch/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_fast / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "%s: %d ch x %d samples (%.0f s at %d Hz), %d templates x %d samples, "
                                   "S=%d, overlap recheck on" % (args.config, C, N, N / si["sampling_rate"],
                                                                si["sampling_rate"], M, W, S),
                       "l2": "inputs larger than L2 (voltage %.2f GB, likelihood %.2f GB)" % (
                           4 * C * N / 1e9, 4 * M * N / 1e9),
                       "spikes": n_sp, "passes": st_fast["passes"], "mode": "fast"},
            "e2e": {"value": e2e_value, "unit": "Msample*ch/s", "h2d_bytes_per_step": int(4 * C * N + T.nbytes + 8 * M),
                    "d2h_bytes_per_step": int(8 * n_sp), "ms_per_step": e2e_t / len(e2e_ms)},
            "gpu_launches": launches,
            "stages_ms": {k[3:]: v for k, v in st_stage.items() if k.startswith("ms_") and v > 0},
            "kernels": kernels,
            "stats": {k: st_stage[k] for k in ("passes", "n_spikes", "listed", "flagged", "fixups", "fixup_runs_queued",
                                               "pair_exact", "pc_macs", "pass_spikes")},
            "roofline": roof,
            "plain_fp32": plain,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_adjoint(args):
    """Residual energy + hand-written adjoint at fixed assignments (template refinement):
    16-ch linear probe, 2 min at 40 kHz, 40 templates; assignments from one pursuit of the
    recording, amplitudes ~ N(1, 0.1), shifts ~ U(-0.5, 0.5) samples.  A step is one
    forward (energy) and one backward (gradients w.r.t. templates, amplitudes, shifts)."""
    import torch
    from spikesorting_fullpursuit_b200 import binary_pursuit, synth
    from spikesorting_fullpursuit_b200.adjoint import residual_energy

    dur = 120.0 if args.duration is None else args.duration
    V, si, sm, _ = synth.config_recording("linear16", seed=3, duration_s=dur)
    C, N = V.shape
    W = si["n_samples_per_chan"]
    M = sm["templates"].shape[0]
    si = dict(si, get_adjusted_clips=False)
    ev, lab, _, _ = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=W - 1, verbose=False)
    pre = -int(round(-1.0e-3 * si["sampling_rate"]))
    idx = np.asarray(ev, dtype=np.int64) - pre
    rng = np.random.default_rng(3)
    n = len(idx)
    dev = torch.device("cuda", 0)
    Vd = torch.from_numpy(V).to(dev)
    Td = torch.from_numpy(np.float32(sm["templates"]).reshape(M, C, W)).to(dev).requires_grad_(True)
    ad = torch.from_numpy(rng.normal(1.0, 0.1, n).astype(np.float32)).to(dev).requires_grad_(True)
    sd = torch.from_numpy(rng.uniform(-0.5, 0.5, n).astype(np.float32)).to(dev).requires_grad_(True)
    idd = torch.from_numpy(idx).to(dev)
    ld = torch.from_numpy(np.asarray(lab, dtype=np.int64)).to(dev)

    def step():
        Td.grad = ad.grad = sd.grad = None
        e = residual_energy(Vd, Td, idd, ld, ad, sd)
        e.backward()
        return e

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
        step()
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    print(json.dumps({
        "metric": "residual-energy gradient (templates, amplitudes, shifts) Msample*ch/s", "value": C * N / (ms * 1e-3) / 1e6,
        "unit": "Msample*ch/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "f64 sums of f32 inputs", "data": "synthetic",
        "config": {"workload": "adjoint: %d ch x %d samples (%.0f s at %d Hz), %d templates x %d samples, %d spikes "
                               "(from one pursuit), linear-interpolation shifts" % (C, N, N / si["sampling_rate"],
                                                                                   si["sampling_rate"], M, W, n)}}))


def run_batched(args):
    """Many independent segments (64, uniform 5-60 s at 40 kHz, 4-12 channels,
    5-30 templates each): one after another on one stream, against
    --batch-streams of them at once, each on a CUDA stream of its own issued by
    its own host thread (longest segments first).  A step is one pursuit of all
    segments; both schedules must give identical spikes per segment."""
    import queue
    import threading

    import torch
    from spikesorting_fullpursuit_b200 import _native, synth

    dev = torch.device("cuda", 0)
    segs = synth.batched_segments(2, scale=args.batch_scale)
    lib = _native.lib()
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    flags = _native.FBP_OVERLAP_RECHECK
    jobs = []
    for V, si, sm in segs:
        C, N = V.shape
        W = si["n_samples_per_chan"]
        T = np.float32(sm["templates"])
        M = T.shape[0]
        d = _native.dims(C, N, M, W, W - 1)
        cap = 8 * (N // W + 1) + 1024
        jobs.append({
            "d": d, "V0": torch.from_numpy(V).to(dev), "V": torch.empty((C, N), device=dev),
            "T": torch.from_numpy(T).to(dev), "b": torch.from_numpy(np.float32(-0.5 * sm["template_SS"])).to(dev),
            "th": torch.from_numpy(np.float32(sm["neuron_lower_thresholds"])).to(dev),
            "ws": torch.empty(_native.workspace_bytes(d, flags), dtype=torch.uint8, device=dev),
            "idx": torch.empty(cap, dtype=torch.int32, device=dev), "lab": torch.empty(cap, dtype=torch.int32, device=dev),
            "cap": cap, "units": C * N, "seconds": N / si["sampling_rate"]})
    order = sorted(range(len(jobs)), key=lambda k: -jobs[k]["units"])
    tune_s = 0.0
    if args.autotune:
        from spikesorting_fullpursuit_b200 import autotune
        t0 = time.perf_counter()
        for j, (V, si, sm) in zip(jobs, segs):
            j["tuning"] = autotune.tune(j["V0"], np.float32(sm["templates"]), np.float32(-0.5 * sm["template_SS"]),
                                        np.float32(sm["neuron_lower_thresholds"]), si["n_samples_per_chan"],
                                        si["n_samples_per_chan"] - 1, device=dev)
        tune_s = time.perf_counter() - t0

    def pursue(j, stream):
        if args.autotune:
            autotune.apply(j["tuning"])
        n = ctypes.c_uint32(0)
        _native.check(lib.fbp_pursue_chunk(ctypes.byref(j["d"]), flags, P(j["V"]), P(j["T"]), P(j["b"]), P(j["th"]),
                                           P(j["ws"]), j["ws"].numel(), P(j["idx"]), P(j["lab"]), j["cap"],
                                           ctypes.byref(n), None, _native.MAX_PASSES, ctypes.c_void_p(stream.cuda_stream)))
        j["n"] = n.value

    def step(nstreams):
        for j in jobs:
            j["V"].copy_(j["V0"])
        torch.cuda.synchronize()
        main = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        if nstreams <= 1:
            for k in order:
                pursue(jobs[k], main)
        else:
            streams = [torch.cuda.Stream(dev) for _ in range(nstreams)]
            todo = queue.Queue()
            for k in order:
                todo.put(k)
            errors = []

            def worker(st):
                st.wait_event(e0)
                while True:
                    try:
                        k = todo.get_nowait()
                    except queue.Empty:
                        return
                    try:
                        pursue(jobs[k], st)
                    except BaseException as exc:  # re-raised below
                        errors.append(exc)
            threads = [threading.Thread(target=worker, args=(st,)) for st in streams]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            if errors:
                raise errors[0]
            for st in streams:
                main.wait_stream(st)
        e1.record(main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), [(j["idx"][:j["n"]].cpu().numpy().copy(), j["lab"][:j["n"]].cpu().numpy().copy())
                                     for j in jobs]

    res = {}
    for mode, ns in (("sequential", 1), ("concurrent", args.batch_streams)):
        for _ in range(args.warmup):
            step(ns)
        ms, out = [], None
        for _ in range(args.steps):
            t, out = step(ns)
            ms.append(t)
        res[mode] = (float(np.sum(ms)), out)
    same = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
               for a, b in zip(res["sequential"][1], res["concurrent"][1]))
    units = sum(j["units"] for j in jobs) * args.steps
    v_seq = units / (res["sequential"][0] * 1e-3) / 1e6
    v_con = units / (res["concurrent"][0] * 1e-3) / 1e6
    print(json.dumps({
        "metric": METRIC + " (batched segments)", "value": v_con, "unit": "Msample*ch/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["concurrent"][0] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched: %d segments, %.0f s in total (uniform %.1f-%.1f s), 4-12 channels, 5-30 "
                               "templates, 40 kHz" % (len(jobs), sum(j["seconds"] for j in jobs),
                                                     5 * args.batch_scale, 60 * args.batch_scale),
                   "streams": args.batch_streams,
                   "autotune": {"on": bool(args.autotune), "tuning_s": tune_s,
                                "shapes": len({json.dumps(j.get("tuning"), sort_keys=True) for j in jobs})}},
        "sequential": {"value": v_seq, "ms_per_step": res["sequential"][0] / args.steps},
        "speedup_vs_sequential": v_con / v_seq, "identical_spikes": bool(same),
        "spikes": int(sum(o[0].size for o in res["concurrent"][1]))}), flush=True)


def cpu_baseline(args, Vfull, sifull, sm):
    """The reference kernels on the host cores over the leading slice of the
    benchmark's own recording (the --impl reference arm times the same code on
    the same slice)."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    sample_s = args.cpu_sample_s
    V, si = leading_slice(Vfull, sifull, sample_s)
    W = si["n_samples_per_chan"]
    try:
        import ref_host
        kind = "reference"
        t0 = time.perf_counter()
        ref_host.binary_pursuit(V, si, copy.deepcopy(sm), n_max_shift_inds=W - 1)
        dt = time.perf_counter() - t0
        cores = ref_host.threads()
        what = "reference OpenCL kernels compiled for the CPU (oracle/_ref), host loop restated"
    except Exception:  # reference library not built: the oracle port
        import oracle as _oracle
        kind = "port"
        t0 = time.perf_counter()
        _oracle.binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=W - 1)
        dt = time.perf_counter() - t0
        cores = os.cpu_count()
        what = "C restatement (oracle) with OpenMP"
    return {"value": V.shape[0] * V.shape[1] / dt / 1e6, "unit": "Msample*ch/s", "cores": cores,
            "kind": kind, "sample": "leading %.2f s of the benchmark's %s recording (seed 1, %d ch); %s" % (
                sample_s, args.config, V.shape[0], what)}


if __name__ == "__main__":
    main()
