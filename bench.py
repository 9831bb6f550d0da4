#!/usr/bin/env python
"""Benchmark of the batched complex FFT path on B200.

Workload (one step): C2C FFT of N=4096 x 16384 complex64 lines, re and im
i.i.d. N(0,1) from a fixed seed, interleaved layout, forward, FP32 storage --
the tensor-core comparison workload (512 MiB read + 512 MiB written per step,
larger than the 126 MB L2, so no flush is needed between steps).  The
FP32 Stockham kernel and the tcgen05 split-FP16 kernel are both timed; the
headline `value` is the faster of those whose relative RMS error against an
FP64 FFT of sampled lines is <= 3e-6.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tc4096 | c2c4096x256 | mixed | conv | fconv | sar | sarfocus | stft | psd | xspec]

--workload selects another configuration (one JSON line each):
  c2c4096x256  N=4096 x 256 lines U[-1,1), forward then inverse per step, over a
               rotating pool of buffer sets larger than L2
  mixed        sizes 64..16384 plus 2^20, seeded counts U{1..512} up to 2^26
               points, one CUDA graph per step: ONE launch of the persistent
               queue kernel, which draws every 4096-point work item (four-step
               columns, whole lines, four-step rows) from a device-side
               descriptor array by atomic ticket
  conv         overlap-add convolution of 2^24 samples with 4095 taps
               (fftSize 8192): forward, then dx and dh, per step
  fconv        FusedConvolver (fftSize 4096) of 2^24 U[-1,1) samples with 512
               U[-1,1) taps, in each Precision mode (float32, float16Storage,
               float16Mixed, float16Pure); value = the fastest mode within the
               reference's error bound for it (1e-3 storage, 2e-2 mixed and
               pure, FusedConvolverTests.swift:40-50) against FP64
  sar          FP16 SAR chain 4096 pulses x 8192 range (64 targets, 10 dB):
               range matched filter, corner turn, azimuth FFT and the phase
               adjoint of sum |I|^4, one CUDA graph per step
  sarfocus     the same scene through the whole range-Doppler algorithm:
               range compression, azimuth FFT, RCMC + azimuth matched filter,
               inverse azimuth FFT (focused FP16 image), four launches per step
  stft         STFT of 2^24 N(0,1) samples, fftSize 1024, hop 512, Hann:
               every frame's complex spectrum and |X|^2, one launch per step
  psd          Welch PSD of 2^26 N(0,1) samples, fftSize 4096, hop 2048,
               Hann, one launch (+ a fixed-order reduction) per step
  r2c          real-input FFT, N=4096: R2C of 2^15 real N(0,1) lines (2049 bins
               each), then C2R of those bins back, per step
  xspec        cross-spectral density matrix of 8 channels x 2^23 samples
               (a shared N(0,1) component plus N(0,1) noise per channel),
               fftSize 1024, hop 512, Hann: powers, 28 cross-spectra and the
               reference's per-frame coherence; two launches per L2-sized
               chunk of frames, the Nyquist-bin sums and one reduction per step

Under torchrun each rank transforms its own 16384 lines (weak scaling, no
collective on the data path); rank 0 prints one JSON line.
`--impl reference` times the reference's algorithm on the host cores instead
(the FP32 radix-4 Stockham restatement in oracle/, OpenMP over lines; the
reference's own CPU path is Apple vDSP, which does not exist on Linux).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 4096
BATCH = 16384
SEED = 20261203
ERR_BAR = 3e-6
METRIC = "FP32 vs split-FP16 tensor-core FFT: transforms/s, % HBM peak at <=3e-6 rel err"
BYTES_PER_TRANSFORM = N * 8 * 2  # read + write, complex64
NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e, nominal (the roofline's `peak` is the measured copy bandwidth)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batch", type=int, default=BATCH)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--fs-log2", default="15-20",
                   help="fourstep workload: log2 sizes to sweep, a range lo-hi or one value")
    p.add_argument("--workload", default="tc4096", choices=["tc4096", "c2c4096x256", "mixed", "conv", "fconv", "sar", "sarfocus", "stft",
                                                        "psd", "xspec", "fourstep", "c2c4096sweep", "r2c"])
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch(kernel):
    """DRAM bytes per launch from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    v = d.get(kernel)
    return v.get("bytes_per_launch") if isinstance(v, dict) else None


class NvmlSampler:
    """SM clock and clock-event reasons read through NVML every ~0.5 ms by a
    host thread, started right before the timed region's first launch and
    stopped after its final synchronize, so that a timed region of a few
    milliseconds still gets samples taken while it runs (nvidia-smi samples
    every 200 ms at best)."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, uuid):
        self.samples = []
        self.handle = None
        self._stop = False
        self._thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            u = str(uuid) if uuid else None
            if u:
                self.handle = pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM) if self.handle else None
        except Exception:
            self.handle = None
            self.max_mhz = None

    def _run(self):
        nv = self._nv
        while not self._stop:
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                self.samples.append((mhz, rs))
            except Exception:
                return
            time.sleep(0.0005)

    def __enter__(self):
        import threading
        if self.handle is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop = True
        if self._thread:
            self._thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return None
        mhz = [m for m, _ in self.samples]
        reasons = sorted({name for _, r in self.samples for bit, name in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(mhz), "sm_mhz_min": min(mhz), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(mhz), "source": "NVML, every ~0.5 ms inside the timed region"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms, plus the
    NVML sampler over the timed region itself (summary() prefers it)."""
    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = None
        self.fast = NvmlSampler(uuid)

    def region(self):
        """Context manager around the timed region itself."""
        return self.fast

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [s.strip() for s in line.split(",")]
                if len(parts) < 10:
                    continue
                if self.uuid and self.uuid not in parts[1]:
                    continue
                rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        fast = self.fast.summary()
        smi = None
        if rows:
            sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
            mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i] == "Active"})
            smi = {"sm_mhz": statistics.median(sm) if sm else None,
                   "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}
        if fast:
            if smi:
                fast["nvidia_smi"] = smi
                fast["reasons"] = sorted(set(fast["reasons"]) | set(smi["reasons"]))
                if fast["sm_max_mhz"] is None:
                    fast["sm_max_mhz"] = smi["sm_max_mhz"]
            return fast
        return smi or {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}


def make_input(batch, rank):
    import numpy as np

    from metalfft_b200 import dist as D
    rng = np.random.default_rng(D.replica_seed(SEED, rank))
    z = rng.standard_normal(size=(batch, N, 2), dtype=np.float32)
    return z.view(np.complex64)[..., 0]


def fp64_check(x_rows, y_rows):
    """rel RMS of y against an FP64 FFT (numpy pocketfft) of x."""
    import numpy as np
    ref = np.fft.fft(x_rows.astype(np.complex128), axis=-1)
    return float(np.linalg.norm(y_rows - ref) / np.linalg.norm(ref))


def fft_flops(n):
    """The conventional FFT operation count of one complex n-point transform, 5 n log2 n."""
    return 5.0 * n * (n.bit_length() - 1)


def link_ceiling(hin, hout, din, dout, transforms, reps=3):
    """The host link's ceiling for the e2e call: the same bytes copied both ways at once
    (pinned host -> device on one stream, device -> host on another, no transform),
    timed with CUDA events. e2e value / link_transforms_per_s is the share of the link
    the C-ABI call reaches."""
    import torch
    cur = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()

    def both():
        up.wait_stream(cur)
        down.wait_stream(cur)
        with torch.cuda.stream(up):
            din.copy_(hin, non_blocking=True)
        with torch.cuda.stream(down):
            hout.copy_(dout, non_blocking=True)
        cur.wait_stream(up)
        cur.wait_stream(down)

    both()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(cur)
    for _ in range(reps):
        both()
    e1.record(cur)
    torch.cuda.synchronize()
    s = e0.elapsed_time(e1) / reps / 1e3
    nbytes = hin.numel() * hin.element_size()
    return {"link_gbs_per_direction": nbytes / s / 1e9,
            "link_transforms_per_s": transforms / s,
            "link_note": "plain pinned copies of the same bytes, both directions at once"}


def tc4096_config(batch):
    """The config of the default workload, the same in both arms."""
    return {"workload": "batched C2C FFT N=4096 x %d lines per GPU, complex64, re/im N(0,1) seeded, forward"
                        % batch,
            "n": N, "batch_per_gpu": batch, "parallelism": "replicas",
            "l2": "inputs larger than L2 (%d MiB read + %d MiB written per step)" % (batch // 32, batch // 32)}


def cpu_baseline(batch, seconds=10.0):
    """The reference algorithm (FP32 radix-4 Stockham, oracle/) on all host
    cores over whole steps of the same workload (the full batch per step),
    repeated for about `seconds`."""
    from oracle import oracle as O
    x = make_input(batch, 0)
    O.ref_fft(x[:64])  # warm
    reps, t0 = 0, time.perf_counter()
    while True:
        O.ref_fft(x)
        reps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": reps * batch / dt, "unit": "transforms/s", "cores": O.max_threads(),
            "kind": "port",
            "sample": "%d whole steps of %d lines of N=%d in %.1f s, FP32 radix-4 Stockham restatement of the "
                      "reference, OpenMP over lines" % (reps, batch, N, dt)}


def cpu_scipy(batch, seconds=5.0):
    """A second, third-party CPU point (not the reference's path, not an
    oracle): scipy.fft (pocketfft) over the same steps, complex64, all host
    threads."""
    try:
        import scipy.fft as sf
    except Exception as e:  # pragma: no cover
        return {"unavailable": str(e)}
    x = make_input(batch, 0)
    workers = os.cpu_count() or 1
    sf.fft(x[:64], axis=-1, workers=workers)
    reps, t0 = 0, time.perf_counter()
    while True:
        sf.fft(x, axis=-1, workers=workers)
        reps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": reps * batch / dt, "unit": "transforms/s", "cores": workers, "kind": "scipy.fft",
            "sample": "%d whole steps of %d lines in %.1f s, scipy.fft.fft complex64, workers=%d (a labelled "
                      "comparator: the reference's own CPU path is vDSP)" % (reps, batch, dt, workers)}


def cpu_baseline_other(workload, seconds=8.0):
    """The reference's CPU path for a non-default workload: the oracle's
    restatement (FP32 Stockham / four-step / overlap-add where the reference
    has them, the FP64 chain for SAR and the spectral estimators) on all host
    cores over a bounded sample of the same workload, in the workload's unit."""
    import numpy as np
    from oracle import oracle as O
    from metalfft_b200 import workloads
    rng = np.random.default_rng(SEED)
    if workload in ("c2c4096x256", "c2c4096sweep"):
        x = O.uniform_c64((256, 4096), SEED)

        def fn():
            O.ref_fft(O.ref_fft(x), inverse=True)
        units, unit = 512, "transforms/s"
        what = "256 lines of N=4096, forward then inverse, FP32 radix-4 Stockham restatement"
    elif workload == "fourstep":
        sample = [(1 << l, max(1, (1 << 19) >> l)) for l in range(15, 21)]
        xs = [O.normal_c64((c, n), SEED + i) for i, (n, c) in enumerate(sample)]

        def fn():
            for x in xs:
                O.ref_fft(x)
        units, unit = sum(n * c for n, c in sample), "points/s"
        what = "2^19 points of each size 2^15..2^20, FP32 four-step restatement"
    elif workload == "mixed":
        # every size class, lines capped at 2^18 points per class
        sample = [(n, max(1, min(c, (1 << 18) // n))) for n, c in workloads.mixed_size_classes()]
        xs = [O.normal_c64((c, n), SEED + i) for i, (n, c) in enumerate(sample)]

        def fn():
            for x in xs:
                O.ref_fft(x)
        units, unit = sum(n * c for n, c in sample), "points/s"
        what = "every size class of the batch, <= 2^18 points each (%d points), FP32 Stockham / four-step " \
               "restatement" % units
    elif workload in ("conv", "fconv"):
        fft, K = (8192, 4095) if workload == "conv" else (4096, 512)
        nx = 1 << 20
        x = rng.standard_normal(nx).astype(np.float32)
        h = rng.standard_normal(K).astype(np.float32)

        def fn():
            O.ref_conv(x, h, fft)
        units, unit = nx, "samples/s"
        what = "2^20 samples, %d taps, fftSize %d: the reference's overlap-add (FP32 forward FFT, complex " \
               "multiply, inverse, overlap-add) restated; forward only (the reference has no adjoint)" % (K, fft)
    elif workload in ("sar", "sarfocus"):
        import metalfft_b200 as M
        prm = M.SARParameters.default(256, 8192, 1024, 512.0)
        raw = O.sar_simulate(prm, workloads.sar_targets(prm, 8, seed=SEED), 10.0, SEED)
        ch = prm.chirp_reference()
        phi = np.zeros(prm.pulses)
        if workload == "sar":
            def fn():
                O.sar_loss_grad(prm, raw, ch, phi)
            what = "256 pulses x 8192 range: FP64 range matched filter, corner turn, azimuth FFT and the " \
                   "phase adjoint (oracle chain)"
        else:
            rd = O.sar_image(prm, raw, ch, phi)

            def fn():
                O.sar_focus(prm, O.sar_image(prm, raw, ch, phi))
            del rd
            what = "256 pulses x 8192 range: FP64 range compression, azimuth FFT, RCMC + azimuth matched " \
                   "filter, inverse azimuth FFT (oracle chain)"
        units, unit = prm.pulses * prm.range_n, "samples/s"
    elif workload in ("stft", "psd"):
        fft, hop = (1024, 512) if workload == "stft" else (4096, 2048)
        n = 1 << 20
        x = rng.standard_normal(n)
        w = O.window(0, fft)
        fn = (lambda: O.stft64(x, fft, hop, w)) if workload == "stft" else (lambda: O.welch64(x, fft, hop, w, 48000.0))
        units, unit = n, "samples/s"
        what = "2^20 samples, fftSize %d, hop %d, Hann: FP64 per-frame restatement" % (fft, hop)
    elif workload == "r2c":
        # the reference's real-input path: the samples packed as complex with a
        # zero imaginary part (Convolve.swift:47-53, FFTAnalyzer.swift:98-100),
        # a complex forward transform, and a complex inverse of the bins back
        x = (rng.standard_normal((256, 4096)).astype(np.float32) + 0j).astype(np.complex64)

        def fn():
            O.ref_fft(O.ref_fft(x), inverse=True)
        units, unit = 512, "transforms/s"
        what = "256 real lines of N=4096 packed as complex (zero imaginary), forward then inverse, FP32 radix-4 " \
               "Stockham restatement"
    elif workload == "xspec":
        n = 1 << 17
        x = rng.standard_normal((8, n))
        w = O.window(0, 1024)

        def fn():
            O.cross_spectral64(x, 1024, 512, w)
        units, unit = 8 * n, "samples/s"
        what = "8 channels x 2^17 samples, fftSize 1024, hop 512: FP64 per-frame restatement"
    else:
        return None
    fn()
    reps, t0 = 0, time.perf_counter()
    while True:
        fn()
        reps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": reps * units / dt, "unit": unit, "cores": O.max_threads(), "kind": "port",
            "sample": "%d x (%s)" % (reps, what)}


def run_reference(args, rank, world):
    """The reference's CPU path for this workload (its FP32 radix-4 Stockham
    restated in oracle/, all host cores): every step transforms the whole
    16384-line batch of the GPU arm's config, so both arms time the same work."""
    if rank != 0:
        return
    if args.workload != "tc4096":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the default workload only; "
                                                              "every other workload's line carries its own "
                                                              "cpu_baseline"}), flush=True)
        return
    from oracle import oracle as O
    B = args.batch
    x = make_input(B, 0)
    # every host core this process may run on: under torchrun OMP_NUM_THREADS is
    # 1, but the other ranks exit without work
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    for _ in range(args.warmup):
        O.ref_fft(x, threads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.ref_fft(x, threads=cores)
    dt = time.perf_counter() - t0
    v = args.steps * B / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "transforms/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "gflop_per_s": v * fft_flops(N) / 1e9, "gflop_note": "5 N log2 N per transform",
        "config": tc4096_config(B),
        "variant": "FP32 radix-4 Stockham (the reference's algorithm, host cores)",
        "cpu_baseline": {"value": v, "unit": "transforms/s", "cores": cores, "kind": "port",
                         "sample": "%d whole steps of %d lines of N=%d in %.2f s, FP32 radix-4 Stockham "
                                   "restatement of the reference, OpenMP over lines" % (args.steps, B, N, dt)},
        "e2e": {"value": v, "unit": "transforms/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed(fn, steps, warmup, barrier, dist, uuid):
    """Device time of `steps` calls of fn (one step each), max over ranks."""
    import torch
    for _ in range(max(3, warmup)):
        fn(0)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()
    with ClockSampler(uuid) as clk:
        with clk.region():
            e0.record(stream)
            for i in range(steps):
                fn(i)
            e1.record(stream)
            torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    from metalfft_b200 import dist as D
    return D.max_over_ranks(ms, device="cuda"), ms, clk.summary()


def run_other(args, M, rank, world, dist, barrier, uuid):
    """Every workload but the default one (configs 1, 2, 4, 5 and the
    spectral, SAR-focusing and FusedConvolver-precision workloads)."""
    import ctypes

    import numpy as np
    import torch
    from metalfft_b200 import workloads
    peak, peak_src = peaks()
    line = {"n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic"}
    if args.workload == "c2c4096x256":
        n, b = 4096, 256
        sets = 64  # 64 x 16 MiB = 1 GiB of rotating inputs and outputs, > L2
        rng = np.random.default_rng(SEED + rank)
        host = rng.uniform(-1, 1, size=(b, n, 2)).astype(np.float32).view(np.complex64)[..., 0]
        xs = torch.from_numpy(host).cuda().unsqueeze(0).repeat(sets, 1, 1).contiguous()
        ys = torch.empty_like(xs)
        f = M.MetalFFT(n)
        # one CUDA graph per buffer set: forward into ys[k], inverse back into xs[k]
        graphs = [f.capture([(xs[k], ys[k], b, M.FORWARD), (ys[k], xs[k], b, M.INVERSE)])
                  for k in range(sets)]

        def step(i):
            graphs[i % sets].replay()
        ms_max, ms, clk = timed(step, args.steps, args.warmup, barrier, dist, uuid)
        per_launch = ms / args.steps / 2 / 1e3
        gbs = b * n * 16 / per_launch / 1e9
        X = ys[0].cpu().numpy()
        err = fp64_check(host[:8], X[:8])
        line.update({"metric": "batched C2C FFT N=4096 x 256: transforms/s (forward + inverse)",
                     "value": 2 * b * world * args.steps / (ms_max / 1e3), "unit": "transforms/s",
                     "ms_per_step": ms_max / args.steps, "rel_rms": err,
                     "gflop_per_s": 2 * b * world * args.steps / (ms_max / 1e3) * fft_flops(n) / 1e9,
                     "gflop_note": "5 N log2 N per transform",
                     "config": {"workload": "C2C FFT N=4096 x 256 lines, U[-1,1) seeded, forward then inverse",
                                "l2": "64 rotating buffer sets (1 GiB) > L2",
                                "graph": "one CUDA graph per step (forward + inverse launch)"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src},
                     "gpu_launches": 2 * args.steps, "clocks": clk})
    elif args.workload == "mixed":
        classes = workloads.mixed_size_classes()
        mb = M.MixedBatch(classes)
        x = torch.from_numpy(workloads.normal_c64(mb.points, SEED + rank)).cuda()
        y = torch.empty_like(x)
        graph = mb.capture(x, y)  # the step's launches as one CUDA graph
        ms_max, ms, clk = timed(lambda i: graph.replay(), args.steps, args.warmup, barrier, dist, uuid)
        assert M.lib.mfft_context_check(M.shared_context()) == 0
        ntr = sum(c for _, c in classes)
        gbs = mb.points * 16 / (ms / args.steps / 1e3) / 1e9
        line.update({"metric": "mixed-size FFT batch on the persistent item kernel: points/s",
                     "value": mb.points * world * args.steps / (ms_max / 1e3), "unit": "points/s",
                     "ms_per_step": ms_max / args.steps, "transforms_per_step": ntr,
                     "gflop_per_s": sum(c * fft_flops(n) for n, c in classes) * world * args.steps
                     / (ms_max / 1e3) / 1e9,
                     "gflop_note": "5 N log2 N per transform, summed over the classes",
                     "config": {"workload": "sizes 2^6..2^14 + 2^20, counts U{1..512} seeded, <= 2^26 points",
                                "classes": classes, "points": mb.points,
                                "graph": "one CUDA graph per step: a memset of the queue counters and ONE launch of "
                                         "the queue kernel (k_fsq_queue) that draws every work item by atomic ticket"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "16 B per point algorithmic; four-step lines move 32 B"},
                     "gpu_launches": args.steps, "clocks": clk})
    elif args.workload == "c2c4096sweep":
        # config 1's step (one CUDA graph: forward, then inverse) over a range
        # of batches; a least-squares line through the per-launch times splits
        # them into a fixed cost per launch and a cost per line
        n = 4096
        f = M.MetalFFT(n)
        sweep, clk = {}, None
        for b in (32, 64, 128, 256, 512, 1024, 2048, 4096):
            sets = max(2, (1 << 30) // (b * n * 8))  # >= 1 GiB of rotating buffers, > L2
            xs = torch.randn(sets, b, n, dtype=torch.complex64, device="cuda")
            ys = torch.empty_like(xs)
            graphs = [f.capture([(xs[k], ys[k], b, M.FORWARD), (ys[k], xs[k], b, M.INVERSE)])
                      for k in range(sets)]
            ms_max, ms, c = timed(lambda i: graphs[i % sets].replay(), args.steps, args.warmup, barrier,
                                  dist, uuid)
            clk = clk or c
            us = ms_max / args.steps / 2 * 1e3
            sweep[b] = {"us_per_launch": us, "frac": b * n * 16 / (us / 1e6) / 1e9 / peak}
            del graphs, xs, ys
        bs = np.array(sorted(sweep), np.float64)
        ts = np.array([sweep[b]["us_per_launch"] for b in sorted(sweep)])
        slope, icpt = np.polyfit(bs, ts, 1)
        us256 = sweep[256]["us_per_launch"]
        gbs = 256 * n * 16 / (us256 / 1e6) / 1e9
        line.update({"metric": "batched C2C FFT N=4096 x 256: transforms/s (forward + inverse), batch sweep",
                     "value": 2 * 256 * world / (2 * us256 / 1e6), "unit": "transforms/s",
                     "ms_per_step": 2 * us256 / 1e3, "sweep": sweep,
                     "fit": {"fixed_us_per_launch": icpt, "ns_per_line": slope * 1e3,
                             "lines_per_s_marginal": 1e6 / slope,
                             "note": "least squares over the batches: per-launch time = fixed + lines x per-line"},
                     "config": {"workload": "C2C FFT N=4096, batches 32..4096, N(0,1), forward then inverse "
                                            "in one CUDA graph", "l2": ">= 1 GiB of rotating buffer sets"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src},
                     "gpu_launches": 16 * args.steps, "clocks": clk})
    elif args.workload == "fourstep":
        # every admissible split n = n1 x n2 of each four-step size, 2^25
        # points (256 MiB in, 256 MiB out) per launch, then the autotuner
        pts = 1 << 25
        x = torch.from_numpy(workloads.normal_c64(pts, SEED + rank)).cuda()
        y = torch.empty_like(x)
        table, best_ms, default_ms, auto = {}, 0.0, 0.0, {}
        clk, launches = None, 0
        lo, _, hi = args.fs_log2.partition("-")
        sizes = range(int(lo), int(hi or lo) + 1)
        for l in sizes:
            n = 1 << l
            b = pts // n
            f = M.MetalFFT(n)
            n1_default = f.split[0]
            row = {}
            for n1 in M.MetalFFT.splits(n):
                f.set_split(n1)
                ms_max, ms, c = timed(lambda i: f.exec(x, y, b, M.FORWARD), args.steps, args.warmup, barrier,
                                      dist, uuid)
                row[n1] = ms_max / args.steps
                clk = clk or c
                launches += 2 * args.steps  # column pass + row pass per call
            f.set_split(min(row, key=row.get))
            f.exec(x, y, b, M.FORWARD)
            torch.cuda.synchronize()
            err = fp64_check(x[:2 * n].view(2, n).cpu().numpy(), y[:2 * n].view(2, n).cpu().numpy())
            g = M.MetalFFT(n)
            auto[n] = g.autotune_split(batch=b)
            table[n] = {"ms_per_launch": row, "default_n1": n1_default, "autotuned_n1": auto[n],
                        "rel_rms": err}
            best_ms += min(row.values())
            default_ms += row[n1_default]
        assert M.lib.mfft_context_check(M.shared_context()) == 0
        ns = len(sizes)
        gbs = ns * pts * 16 / (best_ms / 1e3) / 1e9
        line.update({"metric": "four-step FFT, sizes 2^%d..2^%d, 2^25 points each: points/s (fastest split)" % (sizes[0], sizes[-1]),
                     "value": ns * pts * world / (best_ms / 1e3), "unit": "points/s",
                     "ms_per_step": best_ms,
                     "default_split_points_per_s": ns * pts * world / (default_ms / 1e3),
                     "splits": table,
                     "config": {"workload": "one forward launch of 2^25 complex64 N(0,1) points per size, "
                                            "every admissible split n1 (64..1024, n/n1 in 128..1024)",
                                "l2": "256 MiB in + 256 MiB out per launch > L2"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "16 B per point algorithmic; the intermediate adds 16 B"},
                     "gpu_launches": launches, "clocks": clk})
    elif args.workload in ("stft", "psd"):
        if args.workload == "stft":
            n, fft, hop = 1 << 24, 1024, 512
        else:
            n, fft, hop = 1 << 26, 4096, 2048
        rng = np.random.default_rng(SEED + rank)
        x = torch.from_numpy(rng.standard_normal(n, dtype=np.float32)).cuda()
        est = M.STFT(fft, hop, None, 48000.0)
        frames = est.frame_count(n)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731
        if args.workload == "stft":
            spec = torch.empty((frames, fft), dtype=torch.complex64, device="cuda")
            power = torch.empty((frames, fft), dtype=torch.float32, device="cuda")

            def step(i):
                M._check(M.lib.mfft_stft_analyze(est._h, P(x), n, P(spec), P(power), M.DEVICE, st))
            algo = 4 * n + frames * fft * 12  # signal in; spectra (8 B) and |X|^2 (4 B) out per bin
            metric = "STFT (complex spectra + |X|^2 of every frame): input samples/s"
            launches = 1
        else:
            out = torch.empty(fft, dtype=torch.float32, device="cuda")

            def step(i):
                M._check(M.lib.mfft_psd_welch(est._h, P(x), n, 48000.0, P(out), M.DEVICE, st))
            algo = 4 * n  # the signal once; the partial sums stay in L2
            metric = "Welch PSD: input samples/s"
            launches = 2
        ms_max, ms, clk = timed(step, args.steps, args.warmup, barrier, dist, uuid)
        gbs = algo / (ms / args.steps / 1e3) / 1e9
        line.update({"metric": metric, "value": n * world * args.steps / (ms_max / 1e3), "unit": "samples/s",
                     "ms_per_step": ms_max / args.steps,
                     "config": {"workload": "%d N(0,1) samples seeded, fftSize %d, hop %d, Hann window, %d frames"
                                            % (n, fft, hop, frames),
                                "l2": "input %d MiB%s" % (n * 4 >> 20, ", output %d MiB" % (frames * fft * 12 >> 20)
                                                           if args.workload == "stft" else "")},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "algorithmic bytes: the signal once (frames overlap: re-reads hit L2)"
                                          + (" plus the spectra and powers written" if args.workload == "stft" else "")},
                     "gpu_launches": launches * args.steps, "clocks": clk})
    elif args.workload == "fconv":
        nx, K = 1 << 24, 512
        rng = np.random.default_rng(SEED + rank)
        xh = rng.uniform(-1, 1, nx).astype(np.float32)
        hh = rng.uniform(-1, 1, K).astype(np.float32)
        x = torch.from_numpy(xh).cuda()
        y = torch.empty(nx + K - 1, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731
        # FP64 linear convolution (numpy) of a prefix: the first 2^18 outputs
        # depend on x[:2^18] only
        pre = 1 << 18
        L = 1 << 19
        ref = np.fft.irfft(np.fft.rfft(xh[:pre].astype(np.float64), L) * np.fft.rfft(hh.astype(np.float64), L),
                           L)[:pre]
        bounds = {"float32": 2e-6, "float16Storage": 1e-3, "float16Mixed": 2e-2, "float16Pure": 2e-2}
        modes = {}
        ms_max = ms = clk = None
        best = None
        for name in ("float32", "float16Storage", "float16Mixed", "float16Pure"):
            conv = M.FusedConvolver(hh, 4096, precision=name)

            def step(i, conv=conv):
                M._check(M.lib.mfft_conv_apply(conv._h, P(x), nx, P(y), M.DEVICE, st))
            mmax, mms, mclk = timed(step, args.steps, args.warmup, barrier, dist, uuid)
            yp = y[:pre].double().cpu().numpy()
            err = float(np.linalg.norm(yp - ref) / np.linalg.norm(ref))
            modes[name] = {"samples_per_s": nx * world * args.steps / (mmax / 1e3), "ms_per_step": mmax / args.steps,
                           "rel_err_vs_fp64": err, "bound": bounds[name]}
            if err <= bounds[name] and (best is None or mmax < ms_max):
                best, ms_max, ms, clk = name, mmax, mms, mclk
        algo = 4 * nx + 4 * (nx + K - 1)
        gbs = algo / (ms / args.steps / 1e3) / 1e9
        line.update({"metric": "FusedConvolver fftSize 4096, fastest Precision mode within its error bound: "
                               "samples/s",
                     "value": nx * world * args.steps / (ms_max / 1e3), "unit": "samples/s",
                     "ms_per_step": ms_max / args.steps, "dtype": best, "modes": modes,
                     "config": {"workload": "x 2^24 U[-1,1), h 512 taps U[-1,1), fftSize 4096, overlap-add; "
                                            "error on the first 2^18 outputs vs FP64"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "x read and y written once; the FFT arithmetic bounds it"},
                     "gpu_launches": args.steps, "clocks": clk})
    elif args.workload == "r2c":
        n, lines = 4096, 1 << 15
        h = n // 2 + 1
        rng = np.random.default_rng(SEED + rank)
        x = torch.from_numpy(rng.standard_normal((lines, n), dtype=np.float32)).cuda()
        X = torch.empty((lines, h), dtype=torch.complex64, device="cuda")
        y = torch.empty_like(x)
        f = M.MetalFFT(n)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731

        def step(i):
            M._check(M.lib.mfft_exec_r2c(f._plan, P(x), P(X), lines, M.DEVICE, st))
            M._check(M.lib.mfft_exec_c2r(f._plan, P(X), P(y), lines, M.DEVICE, st))
        ms_max, ms, clk = timed(step, args.steps, args.warmup, barrier, dist, uuid)
        assert M.lib.mfft_context_check(M.shared_context()) == 0
        # bins of sampled lines against an FP64 rfft, and the round trip
        rows = np.linspace(0, lines - 1, 16).astype(np.int64)
        xs = x[rows].double().cpu().numpy()
        Xs = X[rows].cpu().numpy().astype(np.complex128)
        ref = np.fft.rfft(xs, axis=1)
        err = float(np.linalg.norm(Xs - ref) / np.linalg.norm(ref))
        err_rt = float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x))
        per_line = 4 * n + 8 * h  # real samples one way, bins the other
        algo = 2 * lines * per_line
        gbs = algo / (ms / args.steps / 1e3) / 1e9
        line.update({"metric": "real-input FFT N=4096: transforms/s (R2C forward + C2R inverse, each counted)",
                     "value": 2 * lines * world * args.steps / (ms_max / 1e3), "unit": "transforms/s",
                     "ms_per_step": ms_max / args.steps, "rel_rms": err, "round_trip_rel": err_rt,
                     "config": {"workload": "2^15 real lines of N=4096, N(0,1) seeded: R2C (2049 bins per line), "
                                            "then C2R of the bins back",
                                "l2": "512 MiB of real samples and 537 MB of bins per direction > L2"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "4 B per real sample + 8 B per bin, each way"},
                     "gpu_launches": 2 * args.steps, "clocks": clk})
    elif args.workload == "xspec":
        C, n, fft, hop = 8, 1 << 23, 1024, 512
        rng = np.random.default_rng(SEED + rank)
        common = rng.standard_normal(n, dtype=np.float32)
        xh = np.stack([common + rng.standard_normal(n, dtype=np.float32) for _ in range(C)])
        x = torch.from_numpy(xh).cuda()
        del xh, common
        est = M.SpectralEstimator(fft, hop)
        frames = est.frame_count(n)
        pairs = C * (C - 1) // 2
        power = torch.empty((C, fft), dtype=torch.float32, device="cuda")
        cross = torch.empty((pairs, fft), dtype=torch.complex64, device="cuda")
        coh = torch.empty((pairs, fft), dtype=torch.float32, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731

        def step(i):
            M._check(M.lib.mfft_psd_cross_spectral(est._h, P(x), C, n, P(power), P(cross), P(coh), 0, M.DEVICE, st))
        ms_max, ms, clk = timed(step, args.steps, args.warmup, barrier, dist, uuid)
        algo = 4 * C * n  # every channel's samples once; chunk spectra and sums stay in L2
        gbs = algo / (ms / args.steps / 1e3) / 1e9
        # the library's chunks: at most 48 MiB of half spectra (rows of n/2 + 16 bins)
        chunk = max(2, ((48 << 20) // (C * (fft // 2 + 16) * 8)) & ~1)
        chunks = -(-frames // chunk)
        line.update({"metric": "multi-channel cross-spectral density (Welch): channel samples/s",
                     "value": C * n * world * args.steps / (ms_max / 1e3), "unit": "samples/s",
                     "ms_per_step": ms_max / args.steps,
                     "config": {"workload": "%d channels x %d samples (shared N(0,1) + N(0,1) noise) seeded, "
                                            "fftSize %d, hop %d, Hann, %d frames, %d pairs, per-frame coherence"
                                            % (C, n, fft, hop, frames, pairs),
                                "l2": "input %d MiB; %d chunks of %d frames" % (4 * C * n >> 20, chunks, chunk)},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "algorithmic bytes: the signals once; the per-bin pair products "
                                          "(28 pairs x 3 sums per bin and frame) make it compute-heavy"},
                     "gpu_launches": (2 * chunks + 2) * args.steps, "clocks": clk})
    elif args.workload == "sarfocus":
        prm = M.SARParameters.default(4096, 8192, 1024, 512.0)
        sar = M.SARPipeline(prm)
        raw = sar.simulate(workloads.sar_targets(prm, 64, seed=SEED + rank), 10.0, SEED + rank)
        h, sc = sar.quantize(raw)
        del raw
        phi = torch.zeros(prm.pulses, dtype=torch.float32, device="cuda")
        img, isc = sar.forward(h, sc, phi)
        foc, fsc = sar.focus(img, isc)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731

        def step(i):
            M._check(M.lib.mfft_sar_forward(sar._h, P(h), P(sc), P(phi), P(img), P(isc), st))
            M._check(M.lib.mfft_sar_focus(sar._h, P(img), P(isc), P(foc), P(fsc), 0, st))
        ms_max, ms, clk = timed(step, args.steps, args.warmup, barrier, dist, uuid)
        ns = prm.pulses * prm.range_n
        algo = ns * 32  # four passes, each FP16 in + out
        gbs = algo / (ms / args.steps / 1e3) / 1e9
        line.update({"metric": "FP16 SAR range-Doppler algorithm to a focused image: complex samples/s",
                     "value": ns * world * args.steps / (ms_max / 1e3), "unit": "samples/s",
                     "ms_per_step": ms_max / args.steps, "dtype": "fp16 storage, fp32 compute",
                     "config": {"workload": "4096 pulses x 8192 range, chirp 1024 samples TBP 512, 64 seeded "
                                            "targets, 10 dB SNR; range compression, azimuth FFT, RCMC + azimuth "
                                            "matched filter, inverse azimuth FFT"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "32 B per complex sample: four passes of FP16 in + out"},
                     "gpu_launches": 4 * args.steps, "clocks": clk})
    elif args.workload == "sar":
        prm = M.SARParameters.default(4096, 8192, 1024, 512.0)
        sar = M.SARPipeline(prm)
        raw = sar.simulate(workloads.sar_targets(prm, 64, seed=SEED + rank), 10.0, SEED + rank)
        h, sc = sar.quantize(raw)
        del raw
        phi = torch.from_numpy(workloads.sar_phase(prm.pulses, seed=SEED + rank)).cuda()
        ns = prm.pulses * prm.range_n
        # the FP32 range-compressed intermediate (what the phase adjoint needs to
        # meet FP64 gradients to 1e-5) first, then the default FP16 one (the line)
        sar.set_intermediate(M.RC_FP32)
        out32 = sar.step(h, sc, phi)
        ms32_max, ms32, clk32 = timed(lambda i: sar.step(h, sc, phi, out32), args.steps, args.warmup, barrier, dist,
                                      uuid)
        d32 = out32[2].clone()
        sar.set_intermediate(M.RC_FP16)
        out = sar.step(h, sc, phi)
        ms_max, ms, clk = timed(lambda i: sar.step(h, sc, phi, out), args.steps, args.warmup, barrier, dist, uuid)
        grad_gap = float(torch.linalg.vector_norm(out[2].double() - d32.double()) /
                         torch.linalg.vector_norm(d32.double()))
        modes = {"fp16_intermediate": {"samples_per_s": ns * world * args.steps / (ms_max / 1e3),
                                       "ms_per_step": ms_max / args.steps,
                                       "algorithmic_bytes": ns * 16},
                 "fp32_intermediate": {"samples_per_s": ns * world * args.steps / (ms32_max / 1e3),
                                       "ms_per_step": ms32_max / args.steps,
                                       "algorithmic_bytes": ns * 24, "clocks": clk32},
                 "dphi_rel_l2_fp16_vs_fp32": grad_gap}
        algo = ns * 16  # pass A: FP16 in + out, pass B: FP16 in + out
        gbs = algo / (ms / args.steps / 1e3) / 1e9
        line.update({"metric": "FP16 SAR range-Doppler + phase adjoint: complex samples/s",
                     "value": ns * world * args.steps / (ms_max / 1e3), "unit": "samples/s",
                     "ms_per_step": ms_max / args.steps, "dtype": "fp16 storage, fp32 compute",
                     "loss": float(out[3].item()), "intermediate_modes": modes,
                     "config": {"workload": "4096 pulses x 8192 range, chirp 1024 samples TBP 512, 64 seeded "
                                            "targets, 10 dB SNR, phase N(0,0.3); image + dL/dphi of sum |I|^4",
                                "graph": "one CUDA graph per step (range pass, azimuth+adjoint pass, reduce)"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "16 B per complex sample: two passes of FP16 in + out"},
                     "gpu_launches": 3 * args.steps, "clocks": clk})
    else:
        nx, K, fft = 1 << 24, 4095, 8192
        xh, h, th = workloads.conv_workload(SEED + rank, nx=nx, K=K)
        conv = M.Convolver(h, fft)
        x = torch.from_numpy(xh).cuda()
        t = torch.from_numpy(th).cuda()
        y = torch.empty(nx + K - 1, device="cuda")
        g = torch.empty_like(y)
        dx = torch.empty_like(x)
        dh = torch.empty(K, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731

        def step(i):
            M._check(M.lib.mfft_conv_apply(conv._h, P(x), nx, P(y), M.DEVICE, st))
            torch.sub(y, t, out=g)  # dL/dy for L = 0.5 ||y - t||^2
            M._check(M.lib.mfft_conv_backward(conv._h, P(x), nx, P(g), P(dx), P(dh), M.DEVICE, st))
        ms_max, ms, clk = timed(step, args.steps, args.warmup, barrier, dist, uuid)
        algo = (4 * nx + 4 * (nx + K - 1)) + (4 * nx + 4 * (nx + K - 1) + 4 * nx)  # fwd + bwd bytes
        gbs = algo / (ms / args.steps / 1e3) / 1e9
        line.update({"metric": "fused OLA convolution forward + adjoint: samples/s",
                     "value": nx * world * args.steps / (ms_max / 1e3), "unit": "samples/s",
                     "ms_per_step": ms_max / args.steps,
                     "config": {"workload": "x 2^24 N(0,1), h 4095 taps N(0,1)*exp(-t/800), fftSize 8192, "
                                            "target N(0,1); y, then dx and dh"},
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                  "frac": gbs / peak, "peak_source": peak_src,
                                  "note": "algorithmic bytes: x, y read/written by forward; x, g read and dx "
                                          "written by backward (g = y - t by one torch kernel)"},
                     "gpu_launches": 4 * args.steps, "clocks": clk})
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_other(args.workload)
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import ctypes
    from datetime import timedelta

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    import metalfft_b200 as M
    from metalfft_b200 import dist as D

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    if args.workload != "tc4096":
        run_other(args, M, rank, world, dist, barrier, uuid)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    B = args.batch
    host = make_input(B, rank)
    x = torch.from_numpy(host).cuda()
    y = torch.empty_like(x)
    f = M.MetalFFT(N)
    stream = torch.cuda.current_stream()

    variants = {"fp32": 0, "tc_fp16_split3": M.TC_FP16_SPLIT3, "tc_bf16": M.TC_BF16}

    rows = np.random.default_rng(1).choice(B, 16, replace=False)
    results = {}
    peak, peak_src = peaks()

    for name, tc in list(variants.items()):
        try:
            f.exec(x, y, B, M.FORWARD, tc)
        except M.FFTError as e:
            if name == "fp32":
                raise
            results[name] = {"unavailable": str(e)}
            continue
        torch.cuda.synchronize()
        err = fp64_check(host[rows], y[torch.from_numpy(rows).cuda()].cpu().numpy())
        for _ in range(max(3, args.warmup)):
            f.exec(x, y, B, M.FORWARD, tc)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(uuid) as clk:
            with clk.region():
                e0.record(stream)
                for _ in range(args.steps):
                    f.exec(x, y, B, M.FORWARD, tc)
                e1.record(stream)
                torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        ms_max = D.max_over_ranks(ms, device="cuda")
        per_launch_s = ms / args.steps / 1e3
        gbs = BYTES_PER_TRANSFORM * B / per_launch_s / 1e9
        results[name] = {
            "transforms_per_s": B * world * args.steps / (ms_max / 1e3),
            "gflop_per_s": B * world * args.steps / (ms_max / 1e3) * fft_flops(N) / 1e9,
            "ms_per_step": ms_max / args.steps,
            "rel_rms": err,
            "hbm_gbs": gbs,
            "frac": gbs / peak,
            "clocks": clk.summary(),
        }

    ok = {k: v for k, v in results.items() if "rel_rms" in v and v["rel_rms"] <= ERR_BAR}
    best = max(ok, key=lambda k: ok[k]["transforms_per_s"]) if ok else "fp32"
    r = results[best]

    # e2e through the public C ABI with host buffers (pinned), copies included
    hin = torch.from_numpy(host).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    tc = variants[best]

    def e2e_call():
        if tc:
            st = M.lib.mfft_exec_c2c_tc(f._plan, ctypes.c_void_p(hin.data_ptr()),
                                        ctypes.c_void_p(hout.data_ptr()), B, M.FORWARD, tc,
                                        M.HOST, None)
        else:
            st = M.lib.mfft_exec_c2c(f._plan, ctypes.c_void_p(hin.data_ptr()),
                                     ctypes.c_void_p(hout.data_ptr()), B, M.FORWARD, M.HOST, None)
        M._check(st)

    e2e_call()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_call()
    barrier()
    dt = D.max_over_ranks(time.perf_counter() - t0, device="cuda")
    e2e = {"value": B * world * args.e2e_steps / dt, "unit": "transforms/s",
           "h2d_bytes_per_step": B * N * 8, "d2h_bytes_per_step": B * N * 8,
           "steps": args.e2e_steps, "host_memory": "pinned"}
    e2e.update(link_ceiling(hin, hout, x, y, B * world))
    # the same call on pageable host memory (what a Swift array is)
    hin, hout = None, None
    pin, pout = host, np.empty_like(host)

    def e2e_pageable():
        if tc:
            st = M.lib.mfft_exec_c2c_tc(f._plan, ctypes.c_void_p(pin.ctypes.data), ctypes.c_void_p(pout.ctypes.data),
                                        B, M.FORWARD, tc, M.HOST, None)
        else:
            st = M.lib.mfft_exec_c2c(f._plan, ctypes.c_void_p(pin.ctypes.data), ctypes.c_void_p(pout.ctypes.data),
                                     B, M.FORWARD, M.HOST, None)
        M._check(st)

    e2e_pageable()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_pageable()
    barrier()
    dtp = D.max_over_ranks(time.perf_counter() - t0, device="cuda")
    e2e["pageable"] = {"value": B * world * args.e2e_steps / dtp, "unit": "transforms/s",
                       "steps": args.e2e_steps, "host_memory": "pageable (numpy), same call"}

    kernel_name = "k_fft_batched" if best == "fp32" else "k_fft4096_tcw"
    config = tc4096_config(B)
    line = {
        "metric": METRIC,
        "value": r["transforms_per_s"],
        "unit": "transforms/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32" if best == "fp32" else ("fp16x3->fp32" if best == "tc_fp16_split3" else "bf16->fp32"),
        "data": "synthetic",
        "config": config,
        "variant": best,
        "rel_rms": r["rel_rms"],
        "gflop_per_s": r["gflop_per_s"],
        "gflop_note": "5 N log2 N per transform",
        "variants": results,
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": r["hbm_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": r["hbm_gbs"] / peak, "peak_source": peak_src,
                     "traffic": traffic_per_launch(kernel_name),
                     "algorithmic_bytes_per_launch": BYTES_PER_TRANSFORM * B,
                     "nominal_peak": NOMINAL_HBM_GBS, "frac_nominal": r["hbm_gbs"] / NOMINAL_HBM_GBS},
        "clocks": r["clocks"],
        "e2e": e2e,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(B)
        line["cpu_scipy"] = cpu_scipy(B)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
