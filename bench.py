#!/usr/bin/env python
"""Throughput of the B200 template-matching path on the Neuropixels-scale workload.

Workload: C=384 channels (Neuropixels-1.0-like geometry), K=600 templates,
20 batches of 60000 samples (+2*61 padding), nt=61, n_pcs=6, Th_learned=8,
seeded synthetic data (kilosort_b200.synth, seed 1002).  A step is one pass
over all 20 batches with X resident in HBM (1.85 GB per step, larger than L2).
Three forms are timed: `run_matching` per batch with the plain-FP32 and with
the split-BF16 projection, and the batched split form (every batch in one
captured graph: grouped tensor-core contraction, one cooperative peel launch
split into autotuned teams, one residual launch).  `value` is channel-samples/s
of the batched split form.  `e2e` runs that form from pinned host memory, with
the host->device copy of X and the device->host copy of the spikes inside the
timed region, through the pipelined front end (batched.HostPipeline: groups
of KS_BENCH_E2E_GROUP = 5 batches, copies and read-back beside the matching).

The default line also carries shortened runs of the other workloads
(`extract_sharded`, `uneven`, `stream`; `--no-extra` skips them).

    python bench.py --workload uneven     # three recordings, 200 uneven batches
    python bench.py --workload adjoint    # reconstruction loss + adjoint
    python bench.py --workload extract    # drop-in extract over an int16 filtered file
    python bench.py --workload filter     # the batch filter alone, one int16 batch

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --impl reference rank 0 times the CPU oracle of the reference's
run_matching (torch on all host threads) on a bounded sample of the same
workload (one batch per step).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

NT_BATCH = 60000
E2E_GROUP = int(os.environ.get("KS_BENCH_E2E_GROUP", "5"))   # batches per pipelined group
NT = 61
N_PCS = 6
TH = 8.0
CFG = 2
# ncu summaries of the peel launches on this workload; each holds a line
# "dram_bytes_per_batch: <bytes>" (dram__bytes_read.sum + dram__bytes_write.sum
# of the captured launch divided by the batches it covers), read at run time so
# the roofline's traffic comes from the capture committed beside the code
PEEL_PROFILE = "peel_kernel_c384_k600.txt"
PEEL_MULTI_PROFILE = "peel_multi_kernel_c384_k600_20batches.txt"
WORKLOAD = ("Neuropixels-scale matching: C=384 (NP1-like), K=600 templates, 20 batches x "
            "60000 samples (+2*61 pad), nt=61, n_pcs=6, Th_learned=8, max_peels=100")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batches", type=int, default=20)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extra", action="store_true",
                   help="np1 workload: skip the extra workloads carried in its line "
                        "(sharded extract, uneven batches, K=2000 stream)")
    p.add_argument("--workload", default="np1",
                   choices=["np1", "uneven", "adjoint", "stream", "detect", "extract", "filter"],
                   help="np1: C=384/K=600, 20 equal batches (default); uneven: three "
                        "recordings, 200 batches of uneven length, batched launches; "
                        "adjoint: reconstruction loss + hand-written adjoint on one "
                        "C=384/K=600 batch with the matcher's spikes; stream: int16 host "
                        "stream -> whitening -> batched matcher, C=384/K=2000, with "
                        "periodic template refinement; extract: the drop-in extract over "
                        "an int16 BinaryFiltered-style file, device batch filter; filter: "
                        "the batch filter alone on one 385-channel int16 batch")
    p.add_argument("--group", type=int, default=50,
                   help="uneven workload: batches per batched call (one graph each)")
    p.add_argument("--group-stream", type=int, default=4,
                   help="stream workload: batches per batched call")
    p.add_argument("--schedule", default=None,
                   help="np1 workload: 'TEAMS,GROUPS' of the batched form instead of the "
                        "autotuned schedule (for profiling a fixed launch)")
    return p.parse_args()


def profile_traffic(name):
    """DRAM bytes per batch from profiles/<name> (its dram_bytes_per_batch
    line) and the file it came from, or (None, None) without such a line."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_batch:"):
                    return float(line.split(":", 1)[1].split()[0]), "profiles/" + name
    except OSError:
        pass
    return None, None


def reference_gpu_batch(rec, b, dev, reps=3):
    """The reference's run_matching op sequence on the GPU: the oracle, which
    restates kilosort/template_matching.py:170-244 with the same torch ops, run
    on CUDA tensors with TF32 off (cudnn and matmul), on batch b of rec: one
    warm-up call, then the median of `reps` calls, each bracketed by CUDA
    events with the device synchronised on both sides (the loop syncs the
    host every iteration, as the reference does).  Returns ms per batch."""
    from oracle import matching as om
    flags = (torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32)
    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        U = torch.from_numpy(rec.U).to(dev)
        W = torch.from_numpy(rec.wPCA).to(dev)
        X = torch.from_numpy(np.ascontiguousarray(rec.batch(b))).to(dev)
        ops = dict(Th_learned=TH, nt=NT, max_peels=100, wPCA=W)
        ctc = om.prepare_matching(ops, U)
        times = []
        for i in range(1 + reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record()
            om.run_matching(ops, X, U, ctc)
            e1.record()
            torch.cuda.synchronize(dev)
            if i:
                times.append(e0.elapsed_time(e1))
        return statistics.median(times)
    finally:
        torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32 = flags


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        # raw samples go to KS_CLOCKS_DIR (default: the system temp directory);
        # the JSON line carries their summary
        import tempfile
        self.path = os.path.join(os.environ.get("KS_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"clocks_bench_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_batch(rec, b, threads):
    from oracle import matching as om
    torch.set_num_threads(threads)
    U = torch.from_numpy(rec.U)
    W = torch.from_numpy(rec.wPCA)
    ops = dict(Th_learned=TH, nt=NT, max_peels=100, wPCA=W)
    ctc = om.prepare_matching(ops, U)
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(b)))
    t0 = time.perf_counter()
    st, amps, th, _ = om.run_matching(ops, X, U, ctc)
    dt = time.perf_counter() - t0
    return st.numpy(), amps.numpy(), dt


def reference_arm(args, rank):
    """CPU oracle of the reference's run_matching, one cfg-2 batch per step."""
    if rank != 0:
        return
    from kilosort_b200 import synth
    threads = os.cpu_count() or 1
    rec = synth.config_recording(CFG, n_batches=1)
    times = []
    for i in range(args.warmup + args.steps):
        _, _, dt = cpu_oracle_batch(rec, 0, threads)
        if i >= args.warmup:
            times.append(dt)
    t = statistics.median(times)
    v = rec.n_chan * NT_BATCH / t
    line = {
        "impl": "reference", "metric": "channel-samples/s", "value": v,
        "unit": "channel-samples/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": "batch 0 of the 20 per step"},
        "cpu_baseline": {"value": v, "unit": "channel-samples/s", "cores": threads,
                         "kind": "port", "sample": "1 batch (C=384, 60000 samples) per step"},
        "e2e": {"value": v, "unit": "channel-samples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if torch.cuda.is_available():
        ms = reference_gpu_batch(rec, 0, torch.device("cuda", 0))
        line["reference_gpu"] = {"value": rec.n_chan * NT_BATCH / (ms * 1e-3),
                                 "unit": "channel-samples/s", "ms_per_batch": ms,
                                 "kind": "port on CUDA, TF32 off",
                                 "sample": "batch 0, median of 3 after 1 warm-up"}
    print(json.dumps(line), flush=True)

UNEVEN = ("three recordings (C/K = 96/150, 384/600, 384/1000), 200 padded batches with "
          "NT_b ~ U[8000, 60000] and a short tail batch each, nt=61, n_pcs=6, Th_learned=8, "
          "max_peels=100, split-BF16 projection")


def uneven_main(args, dev, rank, world, emit=True):
    """Batched form: every batch of three recordings through ks_match_batches.

    A step is one pass over all batches: groups of --group batches (grouped
    projection, one cooperative peel launch split into autotuned teams, one
    residual launch each), all captured in one CUDA graph, so a step is one
    graph launch.  The same batches through one run_matching call each are
    timed beside it.  X resident in HBM.
    """
    import kilosort_b200 as kb
    from kilosort_b200 import synth
    from kilosort_b200.batched import (BatchedMatcher, MatcherSequence, Recording,
                                       autotune_teams, workspace_size)
    recs = synth.uneven_recordings(seed=1003, n_batches_total=200)
    mrecs, items, ops_l = [], [], []
    for i, r in enumerate(recs):
        U = torch.from_numpy(r.U).to(dev)
        W = torch.from_numpy(r.wPCA).to(dev)
        ops = dict(Th_learned=TH, nt=r.nt, max_peels=100, wPCA=W)
        ctc = kb.prepare_matching(ops, U)
        mrecs.append(Recording.from_ops(ops, U, ctc))
        ops_l.append((ops, U, ctc))
        for b in range(r.n_batches):
            items.append((torch.from_numpy(np.ascontiguousarray(r.batch(b))).to(dev), i))
    # interleave recordings: groups mix template sets and lengths
    order = sorted(range(len(items)), key=lambda i: (i * 7919) % len(items))
    items = [items[i] for i in order]
    groups = [items[g:g + args.group] for g in range(0, len(items), args.group)]
    samples = sum(recs[r].n_chan * (X.shape[1] - 2 * recs[r].nt) for X, r in items)
    teams = autotune_teams(mrecs, groups[0], "bf16x3", candidates=(2, 4, 8, 12, 16, 24))
    # the groups run one after the other on one stream: one shared workspace
    ws = torch.empty(max(workspace_size(mrecs, g, "bf16x3", teams) for g in groups),
                     dtype=torch.uint8, device=dev)
    matchers = [BatchedMatcher(mrecs, [(X.shape[1], r) for X, r in g], "bf16x3", teams=teams,
                               graph=False, workspace=ws) for g in groups]
    for m, g in zip(matchers, groups):
        for dst, (X, _) in zip(m.X, g):
            dst.copy_(X)
    # every group of the step in one captured graph (one launch per step)
    seq = MatcherSequence(matchers)

    def batched_step():
        seq.launch()

    def loop_step():
        for X, r in items:
            ops, U, ctc = ops_l[r]
            kb.run_matching(dict(ops, projection="bf16x3"), X, U, ctc, device=dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    sampler = ClockSampler(dev.index or 0)
    for _ in range(args.warmup):
        batched_step()
    torch.cuda.synchronize()
    nsp = sum(len(r[0]) for m in matchers for r in m.results())
    sampler.__enter__()
    ms = timed(batched_step)
    sampler.__exit__()
    ms_loop = timed(loop_step)
    value = samples * world / (ms * 1e-3)
    line = {
        "metric": "channel-samples/s", "value": value, "unit": "channel-samples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (split-bf16 projection)", "data": "synthetic",
        "config": {"workload": UNEVEN, "batches": len(items), "group": args.group,
                   "teams": teams, "groups": len(matchers), "graphs": 1,
                   "l2": f"inputs larger than L2 ({sum(X.numel() for X, _ in items) * 4 / 1e9:.1f}"
                         " GB of X per step)", "parallelism": f"replicas x{world}"},
        "spikes_per_step": nsp,
        "per_batch_run_matching": {"ms_per_step": ms_loop,
                                   "channel_samples_per_s": samples * world / (ms_loop * 1e-3)},
        "speedup_batched_vs_per_batch": ms_loop / ms,
        "clocks": sampler.summary(),
        # per group: energy, {nm, 1/nm}, reorder per recording; temporal per
        # batch; grouped contraction, peel, residual
        "gpu_launches": sum(3 * len(mrecs) + len(m.items) + 3 for m in matchers),
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line

ADJOINT = ("fixed-assignment reconstruction loss ||X - R||^2 and its adjoint (dU, dwPCA, "
           "damps): C=384, K=600, one 60000-sample batch (+2*61 pad), spikes of the FP32 "
           "matcher (synthetic seed 1004, 2-37 Hz)")


def adjoint_main(args, dev, rank, world):
    """Forward (ks_recon_loss) and backward (ks_recon_adjoint) per step."""
    import kilosort_b200 as kb
    from kilosort_b200 import synth
    from kilosort_b200.adjoint import reconstruction_loss
    rec = synth.config_recording(4)
    U = torch.from_numpy(rec.U).to(dev)
    W = torch.from_numpy(rec.wPCA).to(dev)
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(0))).to(dev)
    ops = dict(Th_learned=TH, nt=NT, max_peels=100, wPCA=W)
    ctc = kb.prepare_matching(ops, U)
    st, amps, _, _ = kb.run_matching(dict(ops, projection="fp32"), X, U, ctc, device=dev)
    amps = amps.reshape(-1)
    C, L = X.shape
    K = U.shape[0]
    N = len(st)
    Uq, Wq, aq = (t.clone().requires_grad_(True) for t in (U, W, amps))

    def step():
        for t in (Uq, Wq, aq):
            t.grad = None
        reconstruction_loss(X, st, aq, Uq, Wq).backward()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index or 0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler.__enter__()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    sampler.__exit__()
    ms = e0.elapsed_time(e1) / args.steps
    # window bytes the adjoint reads per spike (C x nt residual floats) and
    # the flops of its per-spike work (H update, waveform dot product)
    win_bytes = 4.0 * C * NT * N
    samples = C * (L - 2 * NT)
    line = {
        "metric": "channel-samples/s", "value": samples * world / (ms * 1e-3),
        "unit": "channel-samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": ADJOINT, "spikes": N, "templates": K,
                   "l2": "X, Xres 92 MB each: the residual windows are L2 reads",
                   "parallelism": f"replicas x{world}"},
        "spikes_per_s": N * world / (ms * 1e-3),
        "window_gbs": win_bytes / (ms * 1e-3) / 1e9,
        "clocks": sampler.summary(),
        # forward: count, scan, fill, reconstruct, sum; backward: count, scan,
        # group, adjoint, dW, damps
        "gpu_launches": 11,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)

DETECT = ("universal-template detection (spikedetect.template_match + run's y and features): "
          "C=384 (NP1-like, 1532 template positions x 5 sizes x 6 waveforms, 10 nearest "
          "channels, 100 nearest positions), batches of 60000 samples (+2*61 pad) of the "
          "C=384/K=600 synthetic recording, Th_universal=9, nt0min=20")


def detect_main(args, dev, rank, world):
    """Universal-template detection per batch, X resident; CPU oracle beside it."""
    from kilosort_b200 import spikedetect, synth
    rec = synth.config_recording(2, n_batches=3)
    rng = np.random.default_rng(1006)
    wave = synth._waveforms(rng, 6, NT, 20)
    wTEMP = torch.from_numpy((wave / np.linalg.norm(wave, axis=1, keepdims=True)).astype(np.float32))
    settings = dict(nearest_chans=10, nearest_templates=100, min_template_size=10,
                    template_sizes=5, dmin=None, dminx=32, n_templates=6, n_pcs=6, nt0min=20)
    ops = dict(settings=settings, xc=rec.xc.astype(np.float32), yc=rec.yc.astype(np.float32),
               kcoords=np.zeros(rec.n_chan, np.float32), nt=NT, batch_size=NT_BATCH, fs=30000.0,
               Th_universal=9.0, max_channel_distance=32.0, wTEMP=wTEMP,
               wPCA=torch.from_numpy(rec.wPCA))
    iC, iC2, weigh = spikedetect.geometry(ops, device=dev)
    det = spikedetect.Detector(ops, iC, iC2, weigh, dev)
    Xs = [torch.from_numpy(np.ascontiguousarray(rec.batch(b))).to(dev) for b in range(3)]
    C, L = Xs[0].shape
    for i in range(max(3, args.warmup)):
        det(Xs[i % 3])
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index or 0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nsp = 0
    sampler.__enter__()
    e0.record()
    for i in range(args.steps):
        nsp += len(det(Xs[i % 3])[0])      # each call reads its count back (a sync)
    e1.record()
    torch.cuda.synchronize()
    sampler.__exit__()
    ms = e0.elapsed_time(e1) / args.steps
    samples = C * (L - 2 * NT)
    Nfilt = iC.shape[1]
    line = {
        "metric": "channel-samples/s", "value": samples * world / (ms * 1e-3),
        "unit": "channel-samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": DETECT, "positions": Nfilt,
                   "l2": "3 batches of 92 MB rotated; the 554 MB convolution does not fit L2",
                   "parallelism": f"replicas x{world}"},
        "spikes_per_step": nsp / args.steps,
        # FP32 work: the convolution 2*C*nk*nt*L, the sums 2*Nfilt*L*sizes*nk*nC
        "gflop_per_step": (2 * C * 6 * NT * L + 2 * Nfilt * L * 5 * 6 * 10) / 1e9,
        "clocks": sampler.summary(),
        # memset, conv, scores, peaks, count, scan, emit, gather, features, finish
        "gpu_launches": 9,
    }
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import detect as od
        Xc = Xs[0][:, :15000 + 2 * NT].cpu()
        t0 = time.perf_counter()
        od.template_match(Xc, wTEMP, iC.cpu(), iC2.cpu(), weigh.cpu(), NT, 20, 9.0)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": C * 15000 / dt, "unit": "channel-samples/s",
                                "cores": torch.get_num_threads(), "kind": "port",
                                "sample": "template_match on one 15000-sample stretch (C=384)"}
    if rank == 0:
        print(json.dumps(line), flush=True)

STREAM = ("long dense recording, shortened: C=384 (NP1-like), K=2000 templates (amplitudes "
          "5-40 sd, 1-30 Hz), {nb} batches of 60000 samples streamed from page-locked host "
          "int16 (channel-mixed, scale 200) through the GPU batch filter (mean, CAR median, "
          "300 Hz high-pass, whitening) into the batched split-BF16 matcher, one adjoint "
          "template-refinement step per group")


def stream_main(args, dev, rank, world, emit=True):
    """Config 5 on a shortened recording: host int16 -> results on the host."""
    import kilosort_b200 as kb  # noqa: F401
    from kilosort_b200 import synth
    from kilosort_b200.preprocess import highpass_filter
    from kilosort_b200.stream import StreamMatcher
    nb = args.batches if args.batches != 20 else 8
    rec = synth.make_recording(1005, n_chan=384, probe="np1", n_templates=2000,
                               batch_lengths=[NT_BATCH] * nb, rate_hz=(1.0, 30.0),
                               amp_sd=(5.0, 40.0))
    C = rec.n_chan
    rng = np.random.default_rng(1005)
    M = np.eye(C)
    for d in (1, 2):
        v = 0.25 / d * (1 + 0.2 * rng.standard_normal(C - d))
        M += np.diag(v, d) + np.diag(v, -d)
    # nb whole batches of the recording (the synthetic signal carries a margin)
    sig = rec.signal[:, :nb * NT_BATCH].astype(np.float64)
    raw = np.clip(np.round(200.0 * (M @ sig)).T, -32768, 32767)
    raw = np.ascontiguousarray(raw.astype(np.int16))
    Wrot = torch.from_numpy(np.linalg.inv(M)).float()
    U0 = torch.from_numpy(rec.U).to(dev)
    W = torch.from_numpy(rec.wPCA).to(dev)
    ops = dict(Th_learned=TH, nt=NT, max_peels=100, wPCA=W)
    U = U0.clone()
    # the whole batch filter of the reference (mean, CAR, high-pass, whitening)
    pre = dict(hp_filter=highpass_filter(), do_CAR=True)
    sm = StreamMatcher(raw, Wrot, 1.0 / 200.0, ops, U, NT=NT_BATCH, group=args.group_stream,
                       teams=None, refine_every=1, refine_lr=1e-7, preprocess=pre)
    for _ in range(max(1, args.warmup)):
        sm.run()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index or 0)
    sampler.__enter__()
    t0 = time.perf_counter()
    nsp = 0
    for _ in range(args.steps):
        times, templ, amps, _ = sm.run()
        nsp = len(times)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / args.steps
    sampler.__exit__()
    sm.close()
    samples = C * raw.shape[0]
    value = samples * world / dt
    h2d = sum((stop - start) for start, stop, _ in sm.windows) * C * 2
    line = {
        "metric": "channel-samples/s", "value": value, "unit": "channel-samples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int16 in, f32 (f32 filter, split-bf16 whitening and projection)",
        "data": "synthetic",
        "config": {"workload": STREAM.format(nb=nb), "batches": sm.n_batches,
                   "group": sm.group, "teams": sm.matchers[0].teams,
                   "refinements_per_step": sm.refinements // (args.steps + max(1, args.warmup)),
                   "timing": "host wall clock around the whole stream (host int16 in, "
                             "spike arrays on the host out)",
                   "parallelism": f"replicas x{world}"},
        "spikes_per_step": nsp,
        "spikes_per_s": nsp * world / dt,
        # per batch: filter (sums, CAR, high-pass, matrix split, whitening
        # contraction, artifact zeroing), temporal projection; per group:
        # energy, {nm, 1/nm}, reorder, contraction, peel; per refinement: loss
        # (5), adjoint (6), ctc (3), transpose (1)
        "gpu_launches": (7 * sm.n_batches + 5 * -(-sm.n_batches // sm.group)
                         + 15 * (sm.refinements // (args.steps + max(1, args.warmup)))),
        "e2e": {"value": value, "unit": "channel-samples/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": nsp * 20},
        "clocks": sampler.summary(),
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


FILTER = ("batch filter of one raw int16 batch on the device: 385 file channels (384 mapped), "
          "60122 samples, mean, CAR median, 300 Hz high-pass (1023 taps, split-BF16 tcgen05 "
          "Toeplitz product), whitening (split-BF16 tcgen05)")


def filter_main(args, dev, rank, world):
    """ks_preprocess_int16 on one resident raw batch (the kernel case of the
    FIR profile)."""
    from kilosort_b200 import synth
    from kilosort_b200.preprocess import Preprocessor, highpass_filter
    n_bin, L, C = 385, NT_BATCH + 2 * NT, 384
    raw = synth.raw_batch(7101, n_bin, L, n_spikes=3000)
    p = Preprocessor(n_bin, L, whiten=torch.eye(C) / 200.0, chan_map=np.arange(C),
                     hp_filter=highpass_filter(), device=dev)
    r = torch.from_numpy(raw).to(dev)
    X = torch.empty((C, L), device=dev)
    for _ in range(max(3, args.warmup)):
        p(r, X)
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index or 0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler.__enter__()
    e0.record()
    for _ in range(args.steps):
        p(r, X)
    e1.record()
    torch.cuda.synchronize()
    sampler.__exit__()
    status = p.status()
    if status[0] != 0:
        raise RuntimeError(f"batch filter failed: {status}")
    ms = e0.elapsed_time(e1) / args.steps
    line = {
        "metric": "channel-samples/s", "value": C * L * world / (ms * 1e-3),
        "unit": "channel-samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "int16 in, f32 out (split-bf16 FIR and whitening)", "data": "synthetic",
        "config": {"workload": FILTER, "l2": "one 46 MB batch resident; the 92 MB padded "
                   "operand and the 92 MB output exceed neither L2 nor its reuse",
                   "parallelism": f"replicas x{world}"},
        # FIR: 3 products x 2 flops x 128 x 192 x 1152 per tile, 940 tiles
        "fir_gflop_per_step": 3 * 2 * 128 * 192 * 1152 * 940 / 1e9,
        # sums, CAR, Toeplitz, FIR, matrix split, whitening, zeroing
        "gpu_launches": 7 * args.steps,
        "clocks": sampler.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


EXTRACT = ("drop-in extract over a BinaryFiltered-style int16 file in host memory: 385 file "
           "channels (384 mapped, NP1-like), K=600 templates, {nb} batches of 60000 samples, "
           "the reference's batch filter on the device (mean, CAR median, 300 Hz high-pass, "
           "whitening with one-block drift correction), split-BF16 projection, PC features")


def _extract_file(nb, reps, dev):
    """The extract workload's file: nb batches of the NP1 recording (int16,
    385 channels), repeated ``reps`` times along time for a sharded run, with
    its ops (split projection, one-block drift) and templates."""
    from kilosort_b200 import synth
    from kilosort_b200.preprocess import highpass_filter
    rec = synth.config_recording(CFG, n_batches=nb)
    C, n_bin = rec.n_chan, rec.n_chan + 1
    # raw = round(200 * whitened signal) + offsets, drifts, common mode and
    # noise of sd 20 on every file channel; whitening eye / 200 undoes the gain
    raw = synth.raw_recording(rec, n_bin, np.arange(C), seed=1102, gain=200.0)[:nb * NT_BATCH]
    data = raw if reps == 1 else synth.TiledSamples(raw, reps)
    rng = np.random.default_rng(1103)
    W = torch.eye(C) / 200.0
    xc, yc = rec.xc.astype(np.float32), rec.yc.astype(np.float32)
    pos = np.vstack((xc, yc)).T
    d2 = ((pos[:, None, :] - pos[None, :, :]) ** 2).sum(-1)
    Kxx = torch.from_numpy(np.exp(-d2 / (2 * 20.0 ** 2)))
    iKxx = torch.linalg.inv(Kxx + 0.01 * torch.eye(C)).to(dev)
    ops = dict(Th_learned=TH, nt=NT, max_peels=100, wPCA=torch.from_numpy(rec.wPCA).to(dev),
               projection="bf16x3", nt0min=20, batch_size=NT_BATCH, xc=xc, yc=yc, nblocks=1,
               yblk=np.array([yc.mean()]), probe=dict(xc=xc, yc=yc), iKxx=iKxx,
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=N_PCS, sig_interp=20.0))
    src = synth.FilteredBinary(data, NT=NT_BATCH, nt=NT, chan_map=np.arange(C),
                               hp_filter=highpass_filter(), whiten_mat=W,
                               dshift=rng.uniform(-5.0, 5.0, (nb * reps, 1)), device=dev)
    assert src.n_batches == nb * reps
    return rec, raw, src, ops, torch.from_numpy(rec.U).to(dev)


def extract_sharded_block(args, dev, rank, world, nb=8):
    """sharding.extract_sharded over nb batches per rank (weak scaling): the
    file repeats the nb-batch recording once per rank, rank r matches batches
    [r nb, (r+1) nb), rows and features gather on rank 0, which sorts them.
    Host wall clock per rank between barriers, max over ranks."""
    import torch.distributed as dist
    from kilosort_b200 import sharding
    _, _, src, ops, U = _extract_file(nb, world, dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(1, args.warmup)):
        sharding.extract_sharded(dict(ops), src, U, device=dev)
    barrier()
    t0 = time.perf_counter()
    n = 0
    for _ in range(args.steps):
        st, _, _ = sharding.extract_sharded(dict(ops), src, U, device=dev)
        n = len(st) if st is not None else n
    torch.cuda.synchronize()
    dt = torch.tensor([(time.perf_counter() - t0) / args.steps], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(dt, op=dist.ReduceOp.MAX)
        dist.barrier()
    dt = float(dt.item())
    C = len(src.chan_map)
    return {"value": C * nb * world * NT_BATCH / dt, "unit": "channel-samples/s",
            "ms_per_step": dt * 1e3, "batches_per_rank": nb, "spikes_per_step": n,
            "scaling": "weak",
            "timing": "host wall clock per rank (int16 file in, sorted st/tF on rank 0 out), "
                      "max over ranks"}


def extract_main(args, dev, rank, world):
    """kb.extract over a synth.FilteredBinary: host int16 file -> sorted host
    arrays; with several ranks, sharding.extract_sharded over nb batches per
    rank."""
    import kilosort_b200 as kb
    from kilosort_b200 import filtered, synth
    nb = args.batches if args.batches != 20 else 8
    if world > 1:
        blk = extract_sharded_block(args, dev, rank, world, nb)
        line = {"metric": "channel-samples/s", "value": blk["value"],
                "unit": "channel-samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": blk["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int16 in, f32 (f32 filter, split-bf16 whitening and projection)",
                "data": "synthetic",
                "config": {"workload": EXTRACT.format(nb=nb) + ", per rank",
                           "parallelism": f"batch shards x{world} (sharding.extract_sharded)"},
                "extract_sharded": blk,
                "e2e": {"value": blk["value"], "unit": "channel-samples/s",
                        "h2d_bytes_per_step": nb * (NT_BATCH + 2 * NT) * 385 * 2 * world,
                        "d2h_bytes_per_step": None}}
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    rec, raw, src, ops, U = _extract_file(nb, 1, dev)
    C, n_bin = rec.n_chan, rec.n_chan + 1
    W = src.whiten_mat
    assert filtered.supports(src)
    U = torch.from_numpy(rec.U).to(dev)
    for _ in range(max(1, args.warmup)):
        kb.extract(dict(ops), src, U, device=dev)
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index or 0)
    sampler.__enter__()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st, tF, _ = kb.extract(dict(ops), src, U, device=dev)
    dt = (time.perf_counter() - t0) / args.steps
    sampler.__exit__()
    # the same extract with the plain-FP32 projection (the default of ops)
    ops32 = dict(ops, projection="fp32")
    kb.extract(dict(ops32), src, U, device=dev)
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    for _ in range(args.steps):
        kb.extract(dict(ops32), src, U, device=dev)
    dt32 = (time.perf_counter() - t4) / args.steps
    # the stages alone, one after the other: the batch source, then matching
    # (the file's device source, as extract left it: pinned windows in place)
    fb = filtered.batches_for(src, dev)
    fb.batch(0, ops)                      # this thread's first use (library handles)
    fb.check()
    t1 = time.perf_counter()
    Xs = [fb.batch(b, ops) for b in range(nb)]
    fb.check()                            # synchronises with the last filter
    t_src = time.perf_counter() - t1
    ctc = kb.prepare_matching(ops, U)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    for X in Xs:
        kb.run_matching(ops, X, U, ctc, device=dev)
    torch.cuda.synchronize()
    t_match = time.perf_counter() - t2
    value = C * nb * NT_BATCH * world / dt
    L = NT_BATCH + 2 * NT
    line = {
        "metric": "channel-samples/s", "value": value, "unit": "channel-samples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int16 in, f32 (f32 filter, split-bf16 whitening and projection)",
        "data": "synthetic",
        "config": {"workload": EXTRACT.format(nb=nb), "batches": nb,
                   "timing": "host wall clock around extract (host int16 file in, sorted "
                             "st and tF on the host out)",
                   "parallelism": f"replicas x{world}"},
        "spikes_per_step": len(st),
        "stages_ms": {"batch_source_alone": t_src * 1e3, "matching_alone": t_match * 1e3},
        "fp32_projection": {"value": C * nb * NT_BATCH * world / dt32, "ms_per_step": dt32 * 1e3},
        # per batch: filter 6, matching 7, features 1; per call: template
        # channels, ctc (2), transpose
        "gpu_launches": 14 * nb + 4,
        "e2e": {"value": value, "unit": "channel-samples/s",
                "h2d_bytes_per_step": nb * L * n_bin * 2,
                "d2h_bytes_per_step": int(st.nbytes + tF.numel() * 4)},
        "clocks": sampler.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same extract fed the reference's way: the file slice transposed,
        # a pageable copy, float32, and the torch filter (FFT high-pass) on the
        # device -- the oracle's restatement of io.py:789-831 and :990-1026
        from oracle import preprocess as op

        class ReferenceRead(synth.FilteredBinary):
            def padded_batch_to_torch(self, ibatch, ops=None):
                return op.filtered_batch(self, ibatch, ops, self.device)

        ref = ReferenceRead(raw, NT=NT_BATCH, nt=NT, chan_map=np.arange(C),
                            hp_filter=src.hp_filter, whiten_mat=W, dshift=src.dshift, device=dev)
        ops_r = dict(ops, device_filter=False)
        kb.extract(dict(ops_r), ref, U, device=dev)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        reps = max(1, min(3, args.steps))
        for _ in range(reps):
            st_r, _, _ = kb.extract(dict(ops_r), ref, U, device=dev)
        dt_r = (time.perf_counter() - t3) / reps
        line["reference_batch_source"] = {
            "value": C * nb * NT_BATCH / dt_r, "unit": "channel-samples/s",
            "ms_per_step": dt_r * 1e3, "spikes_per_step": len(st_r),
            "kind": "port on CUDA (pageable float32 copy, torch FFT filter)",
            "speedup_device_source": dt_r / dt}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    import datetime
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    if args.workload in ("uneven", "adjoint", "stream", "detect", "extract", "filter"):
        {"uneven": uneven_main, "adjoint": adjoint_main, "stream": stream_main,
         "detect": detect_main, "extract": extract_main,
         "filter": filter_main}[args.workload](args, dev, rank, world)
        if world > 1:
            dist.destroy_process_group()
        return
    import kilosort_b200 as kb
    from kilosort_b200 import _lib, synth
    from tests.parity_util import agreement

    rec = synth.config_recording(CFG, n_batches=args.batches)
    C, K = rec.n_chan, rec.n_templates
    L = NT_BATCH + 2 * NT
    U = torch.from_numpy(rec.U).to(dev)
    W = torch.from_numpy(rec.wPCA).to(dev)
    Xs = [torch.from_numpy(np.ascontiguousarray(rec.batch(b))).to(dev) for b in range(args.batches)]
    Xh = [torch.from_numpy(np.ascontiguousarray(rec.batch(b))).pin_memory() for b in range(args.batches)]
    ops = dict(Th_learned=TH, nt=NT, max_peels=100, wPCA=W)
    ctc = kb.prepare_matching(ops, U)
    torch.cuda.synchronize()

    # projection forms the built library offers
    forms = ["fp32"]
    try:
        kb.run_matching(dict(ops, projection="bf16x3"), Xs[0], U, ctc, device=dev)
        forms.append("bf16x3")
    except _lib.KilosortB200Error as e:
        if e.status != _lib.KS_ERR_UNSUPPORTED:
            raise
    head = forms[-1]

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world > 1:
            t = torch.tensor([x], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    def device_step(form, spikes):
        o = dict(ops, projection=form)
        n = 0
        for X in Xs:
            st, _, _, _ = kb.run_matching(o, X, U, ctc, device=dev)
            n += len(st)
        spikes.append(n)

    def timed(fn, form, sampler=None):
        for _ in range(args.warmup):
            fn(form, [])
        barrier()
        spikes = []
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.__enter__()
        s0.record()
        for _ in range(args.steps):
            fn(form, spikes)
        s1.record()
        barrier()
        if sampler:
            sampler.__exit__()
        ms = max_over_ranks(s0.elapsed_time(s1)) / args.steps
        return ms, spikes[-1]

    sampler = ClockSampler(local)
    results = {}
    batched = "bf16x3" in forms
    for form in forms:
        ms, nsp = timed(device_step, form,
                        sampler if (form == head and not batched) else None)
        results[form] = dict(ms=ms, spikes=nsp)

    # the batched split form: all batches in one captured graph (grouped
    # tensor-core contraction, one cooperative peel launch split into teams,
    # one residual launch), teams autotuned; inputs resident as above
    matcher, teams, groups = None, None, None
    if batched:
        from kilosort_b200.batched import BatchedMatcher, Recording, autotune_schedule
        mrec = Recording.from_ops(ops, U, ctc)
        items = [(X, 0) for X in Xs]
        if args.schedule:
            teams, groups = (int(v) for v in args.schedule.split(","))
        else:
            teams, groups = autotune_schedule([mrec], items, "bf16x3", teams=(5, 10, 20),
                                              groups=(1, 2, 4, 5))
        matcher = BatchedMatcher([mrec], [(L, 0)] * len(Xs), "bf16x3", teams=teams,
                                 graph=True, groups=groups)
        for dst, X in zip(matcher.X, Xs):
            dst.copy_(X)

        def batched_step(form, spikes):
            matcher.launch()
            spikes.append(0)      # counted once after timing (reading them syncs)

        ms_b, _ = timed(batched_step, "bf16x3_batched", sampler)
        results["bf16x3_batched"] = dict(ms=ms_b,
                                         spikes=sum(len(r[0]) for r in matcher.results()))
        # the same batched form with the plain-FP32 projection (same schedule),
        # so the split/FP32 ratio is also stated at equal execution shape
        matcher32 = BatchedMatcher([mrec], [(L, 0)] * len(Xs), "fp32", teams=teams, graph=True,
                                   groups=groups)
        for dst, X in zip(matcher32.X, Xs):
            dst.copy_(X)

        def batched32_step(form, spikes):
            matcher32.launch()
            spikes.append(0)

        ms_b32, _ = timed(batched32_step, "fp32_batched")
        results["fp32_batched"] = dict(ms=ms_b32,
                                       spikes=sum(len(r[0]) for r in matcher32.results()))
        del matcher32
        forms.append("fp32_batched")
        forms.append("bf16x3_batched")
        head = "bf16x3_batched"

    # end to end from pinned host memory through the public API
    h2d = C * L * 4 * args.batches
    d2h = [0]

    def e2e_step(form, spikes):
        o = dict(ops, projection=form)
        n = 0
        d2h[0] = 0
        for Xhost in Xh:
            X = Xhost.to(dev, non_blocking=True)
            st, amps, th, _ = kb.run_matching(o, X, U, ctc, device=dev)
            st_h, a_h, t_h = st.cpu(), amps.cpu(), th.cpu()
            n += len(st_h)
            d2h[0] += st_h.numel() * 8 + a_h.numel() * 4 + t_h.numel() * 4
        spikes.append(n)

    pipe = None
    if matcher is not None:
        from kilosort_b200.batched import HostPipeline
        # groups of E2E_GROUP batches: the copies of one group and the read-back
        # of the previous run beside the matching of the current one
        pipe = HostPipeline([mrec], [(L, 0)] * len(Xh), "bf16x3",
                            teams=min(teams, E2E_GROUP), group=E2E_GROUP)

    def e2e_batched(form, spikes):
        n = 0
        d2h[0] = 0
        for st_h, a_h, t_h in pipe.run(Xh):
            n += len(st_h)
            d2h[0] += st_h.numel() * 8 + a_h.numel() * 4 + t_h.numel() * 4
        spikes.append(n)

    e2e_ms, _ = timed(e2e_batched if matcher is not None else e2e_step, head)

    # per-kernel breakdown of one pass through the public run_matching, timed
    # by events the library records inside the call (ks_trace_stages): energy
    # + copy, projection, peel kernel, residual kernel; one warm-up pass first
    lib = _lib.load()
    _lib.check(lib.ks_trace_stages(1), "ks_trace_stages")
    import ctypes
    ms4 = (ctypes.c_float * 4)()
    stage = {"energy": 0.0, "project": 0.0, "peel": 0.0, "residual": 0.0}
    stage_batches = {k: [] for k in stage}
    kused, nsp_total = 0, 0
    proj_head = "bf16x3" if "bf16x3" in results else "fp32"
    o_head = dict(ops, projection=proj_head)
    for pass_ in range(2):
        for X in Xs:
            st, amps, th, _ = kb.run_matching(o_head, X, U, ctc, device=dev)
            _lib.check(lib.ks_trace_read(ms4, 4), "ks_trace_read")
            if pass_ == 0:
                continue
            for key, v in zip(stage, ms4):
                stage[key] += v
                stage_batches[key].append(round(v, 3))
            kused += len(torch.unique(st[:, 1]))
            nsp_total += len(st)
    batched_stage = None
    if matcher is not None:
        matcher.launch_eager()
        _lib.check(lib.ks_trace_read(ms4, 4), "ks_trace_read")
        batched_stage = dict(zip(("setup", "project", "peel", "residual"),
                                 (round(v, 3) for v in ms4)))
    _lib.check(lib.ks_trace_stages(0), "ks_trace_stages")
    nb = args.batches
    hbm, bf16, peak_kind = peaks()
    flop_proj = 2.0 * L * C * N_PCS * (NT + K) * nb
    # compulsory bytes of the peel (B read once, X/Xres, ctc columns and
    # loadings of the templates used, outputs) and the no-reuse bound (every
    # spike's K x (2nt+1) read-modify-write of B plus its ctc column, and its
    # C x nt residual update)
    bytes_peel = 4.0 * K * L * nb + 4.0 * K * (2 * NT + 1) * kused \
        + 4.0 * N_PCS * C * kused + 24.0 * nsp_total
    bytes_res = 8.0 * C * L * nb
    bytes_noreuse = 4.0 * K * L * nb + nsp_total * (12.0 * K * (2 * NT + 1) + 8.0 * C * NT)
    proj_tflops = flop_proj / (stage["project"] * 1e-3) / 1e12
    peel_gbs = bytes_peel / (stage["peel"] * 1e-3) / 1e9
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
    same_sizes = (C, K, NT_BATCH) == (384, 600, 60000)
    tb_single, src_single = profile_traffic(PEEL_PROFILE) if same_sizes else (None, None)
    tb_multi, src_multi = profile_traffic(PEEL_MULTI_PROFILE) if same_sizes else (None, None)
    traffic = tb_single
    if batched_stage is not None and head == "bf16x3_batched":
        # one peel_multi_kernel launch covers all batches of the step and
        # applies their residuals too, so its algorithmic bytes add the 8*C*L
        # of X/Xres per batch; its traffic is the ncu figure per batch of the
        # committed capture times the batches of this step (same sizes)
        t_b = batched_stage["peel"] * 1e-3
        bytes_multi = bytes_peel + bytes_res
        traffic_m = tb_multi * nb if tb_multi else None
        roof = {"kernel": "peel_multi_kernel", "bound": "hbm",
                "achieved": bytes_multi / t_b / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": bytes_multi / t_b / 1e9 / hbm,
                "traffic": traffic_m, "traffic_source": src_multi, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": bytes_multi,
                "no_reuse_bytes_per_launch": bytes_noreuse,
                "traffic_gbs": (traffic_m / t_b / 1e9 if traffic_m else None),
                "ms_per_launch": batched_stage["peel"], "batches_per_launch": nb}
    elif stage["peel"] >= stage["project"]:
        roof = {"kernel": "peel_kernel", "bound": "hbm", "achieved": peel_gbs, "peak": hbm,
                "unit": "GB/s", "frac": peel_gbs / hbm, "traffic": traffic,
                "traffic_source": src_single, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": bytes_peel / nb,
                "no_reuse_bytes_per_launch": bytes_noreuse / nb,
                "traffic_gbs": (traffic / (stage["peel"] / nb * 1e-3) / 1e9
                                if traffic else None),
                "ms_per_launch": stage["peel"] / nb}
    elif proj_head == "bf16x3":
        roof = {"kernel": "project_bf16x3", "bound": "tensor", "achieved": proj_tflops,
                "peak": bf16, "unit": "TFLOP/s", "frac": proj_tflops / bf16, "traffic": None,
                "peak_source": peak_kind}
    else:
        roof = {"kernel": "project_fp32", "bound": "fp32-simt", "achieved": proj_tflops,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": proj_tflops / fp32_peak,
                "traffic": None, "peak_source": "nominal FP32 FMA"}

    cpu = None
    ref_gpu = None
    agr = {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        st_r, amps_r, dt = cpu_oracle_batch(rec, 0, threads)
        cpu = {"value": C * NT_BATCH / dt, "unit": "channel-samples/s", "cores": threads,
               "kind": "port", "sample": "batch 0 (C=384, 60000 samples), oracle run_matching"}
        ms_ref = reference_gpu_batch(rec, 0, dev)
        ref_gpu = {"value": C * NT_BATCH / (ms_ref * 1e-3), "unit": "channel-samples/s",
                   "ms_per_batch": ms_ref, "kind": "port on CUDA, TF32 off",
                   "sample": "batch 0, median of 3 after 1 warm-up",
                   "speedup_batched_split": (ms_ref * nb) / results[head]["ms"]}
        for form in forms:
            if form == "fp32_batched":
                continue          # bit-identical to one fp32 run_matching per batch (tests)
            if form == "bf16x3_batched":
                matcher.launch()
                st, amps, _, _ = matcher.results()[0]
            else:
                st, amps, _, _ = kb.run_matching(dict(ops, projection=form), Xs[0], U, ctc,
                                                 device=dev)
            a = agreement(st.cpu().numpy(), st_r, amps.cpu().numpy(), amps_r)
            agr[form] = {k: a[k] for k in ("agreement", "amp_rel_max", "matched", "n_a", "n_r")}

    # energy, reorder, temporal, contraction, {nm, 1/nm}, peel, residual
    launches_per_batch = 7
    per_step_samples = C * NT_BATCH * nb
    head_ms = results[head]["ms"]
    value = per_step_samples * world / (head_ms * 1e-3)
    line = {
        "metric": "channel-samples/s", "value": value, "unit": "channel-samples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": head_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if head == "fp32" else "f32 (split-bf16 projection)",
        # value/ms_per_step/e2e: the head form (the batched split form when
        # the tensor-core build is present); forms lists every form timed
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "projection": head, "batches": nb,
                   "l2": "inputs larger than L2 (1.85 GB of X per step)",
                   "parallelism": f"replicas x{world}"},
        "spikes_per_s": results[head]["spikes"] * world / (head_ms * 1e-3),
        "forms": {f: {"ms_per_step": r["ms"],
                      "channel_samples_per_s": per_step_samples * world / (r["ms"] * 1e-3),
                      "spikes_per_step": r["spikes"]} for f, r in results.items()},
        "speedup_split_vs_fp32": (results["fp32"]["ms"] / results["bf16x3"]["ms"]
                                  if "bf16x3" in results else None),
        "speedup_batched_split_vs_fp32": (results["fp32"]["ms"] / results[head]["ms"]
                                          if head == "bf16x3_batched" else None),
        "speedup_batched_split_vs_batched_fp32": (
            results["fp32_batched"]["ms"] / results[head]["ms"]
            if "fp32_batched" in results else None),
        "batched_teams": teams,
        "batched_groups": groups if matcher is not None else None,
        "stages_ms_per_step": stage,
        "stages_ms_per_batch": stage_batches,
        "batched_stages_ms_per_step": batched_stage,
        "agreement_vs_oracle_batch0": agr,
        "e2e": {"value": per_step_samples * world / (e2e_ms * 1e-3), "unit": "channel-samples/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h[0],
                "ms_per_step": e2e_ms},
        "roofline": roof,
        "roofline_all": {"project": {"achieved_tflops": proj_tflops,
                                     "flop_per_batch": flop_proj / nb},
                         "peel": {"achieved_gbs": peel_gbs, "algorithmic_bytes": bytes_peel},
                         "residual": {"achieved_gbs": bytes_res / (stage["residual"] * 1e-3) / 1e9,
                                      "algorithmic_bytes": bytes_res}},
        "cpu_baseline": cpu,
        "reference_gpu": ref_gpu,
        "clocks": sampler.summary(),
        # batched head: energy, {nm, 1/nm}, reorder, a temporal projection per
        # batch, grouped contraction, peel, residual
        "gpu_launches": (3 + nb + 3) if head == "bf16x3_batched" else launches_per_batch * nb,
    }
    # the other workloads, shortened (every rank takes part): the drop-in
    # extract sharded over the ranks, the uneven multi-recording batches, the
    # K=2000 stream
    del Xs, Xh
    if not args.no_extra:
        line["extract_sharded"] = extract_sharded_block(args, dev, rank, world)
        short = argparse.Namespace(**dict(vars(args), steps=2, warmup=2, batches=20))
        keep = ("value", "unit", "ms_per_step", "per_batch_run_matching",
                "speedup_batched_vs_per_batch", "spikes_per_step", "refinements_per_step",
                "clocks")
        for name, fn in (("uneven", uneven_main), ("stream", stream_main)):
            sub = fn(short, dev, rank, world, emit=False)
            line[name] = {k: sub[k] for k in keep if k in sub}
            line[name]["workload"] = sub["config"]["workload"]
            line[name]["steps"] = short.steps
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
