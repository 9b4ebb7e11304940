#!/usr/bin/env python
"""Benchmark: AO loop iterations/s at the SAXO-scale 40x40 Shack-Hartmann loop.

One step = one RTC iteration of the ``saxo40`` workload on one GPU: SH image
formation from a resident phase screen (photon + 0.5 e- readout noise),
weighted CoG with threshold fused into the sensor kernel, the 1377 x 2496
command-matrix MVM with the integrator, and the voltage stage (delay ring,
clip).  The L2 cache (126 MB) is flushed before every timed step by writing a
256 MB buffer, so the 13.7 MB float32 command matrix is read from HBM each
iteration.  Each step is bracketed by CUDA events on the launching stream; the
value is steps / (sum of step times).

Other keys of the JSON line:
  e2e       the same step through the C ABI calls a caller makes, with every
            step's phase screen copied in from pinned host memory and its
            voltages written back into pinned host memory by the fused kernel;
            streamed (step k+1's phase crosses the bus while step k computes,
            the pipeline of aob_loop_run), L2 flushed before every step outside
            its span; per_step_sync is the same one step at a time, run_api is
            aob_loop_run itself over all steps in one call;
  roofline  the dominant kernel's algorithmic bytes / measured duration against
            the measured HBM copy bandwidth in MEASURED_PEAKS.json;
  cpu_baseline  the float64 NumPy/SciPy restatement timed on the host cores;
  learned   the same iteration with the learned reconstructor in place of the LS
            matrix (aob_loop_step_mlp, one kernel per step), timed like value;
            its Strehl parity with LS is the c4 workload's;
  closed_loop_extras  the stages around it (screen extrusion, raytrace, DM shape)
            and the whole closed-loop iteration, each in graph replay.

--workload selects what is measured: ``saxo40`` (default, the line above),
or one of the other scope rows, each printing its own JSON line with its own
metric, roofline and CPU baseline: ``mc64`` (64 uneven SH loops advanced by
one persistent launch per step, BF16 MVM), ``pyr50`` (pyramid sensor, 24
modulation points over 512 x 512 FFTs, slopes and a 1600-actuator LS MVM),
``mlp`` (the learned reconstructor: batch-1 inference against the LS MVM and
training throughput on the tensor cores), ``precision`` (the saxo40 closed
loop with its own LS command matrix: command error and residual-wavefront rms
of the F32 / BF16 / FP8 MVM against a float64 reconstruction), ``c4`` (the learned
reconstructor trained at the saxo40 geometry on closed-loop pairs over r0 0.08-0.20 m
and magnitudes 6-10, then its closed-loop long-exposure Strehl against LS).

--impl reference runs the reference's own implementation of the path, its
sutra CUDA code built from its sources into oracle/_ref (oracle/build_ref.py),
on the same GPU through its Python API, as the baseline arm; without that
build or a GPU it falls back to the float64 CPU restatement of its algorithm.  Multi-GPU (torchrun): the path does not shard -- every
rank runs an independent replica; value = total steps / max-over-ranks time.
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
PKG = os.path.join(ROOT, "compass-saxoplus_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "AO loop iters/s at 40x40 SH (learned vs LS recon, same Strehl); % HBM peak"
UNIT = "iters/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic(name):
    """DRAM bytes per launch recorded from an ncu capture (profiles/<name>.txt)."""
    p = os.path.join(ROOT, "profiles", name + ".txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = float(f[2])
                except ValueError:
                    continue
                for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                    "sw_power_cap"), f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # B200 FP32 (non-tensor), nominal


def graph_time(torch, flush, fn, n=20, with_flush=True):
    """Mean device seconds of fn(stream) per launch: n x [flush, fn] minus n x [flush]
    (with_flush=False: n x [fn] alone), each replayed as one CUDA graph (no host
    gaps), best of 5 replays."""
    gs = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(gs):
        for _ in range(2):
            fn(gs.cuda_stream)
    torch.cuda.synchronize()

    def capture(body):
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr, stream=gs):
            for _ in range(n):
                if with_flush:
                    flush.zero_()
                body()
        return gr

    g1 = capture(lambda: fn(gs.cuda_stream))
    # the baseline graph holds the flushes alone; without flushes there is nothing to subtract
    graphs = (g1, capture(lambda: None)) if with_flush else (g1,)
    out = []
    for gr in graphs:
        for _ in range(2):
            gr.replay()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            gr.replay()
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b) / 1000.0)
        out.append(best)
    return (out[0] - (out[1] if with_flush else 0.0)) / n


def max_over_ranks(dist, torch, values, device):
    """Element-wise maximum over the ranks of a list of times (the slowest rank's),
    unchanged without a process group.  Every rank calls it at the same point."""
    if not dist:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_rate(ws, steps, total_ms):
    """Whole-job iterations/s: each of the ws ranks ran ``steps`` iterations and the
    job took the slowest rank's total_ms."""
    return ws * steps / (total_ms / 1000.0)


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(setup, budget_s=12.0, max_iters=400):
    """Time the float64 CPU restatement on a bounded number of iterations."""
    from oracle.loop_cpu import CpuShLoop
    from aob200.workloads import von_karman_screens

    g = setup.geom
    screens = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, 0.14, 25.0, 4, seed=1)
    loop = CpuShLoop(g, setup.cmat, setup.centroider, setup.threshold, setup.weights, setup.noise)
    loop.step(screens[0])
    n = 0
    t0 = time.perf_counter()
    while n < max_iters and (time.perf_counter() - t0) < budget_s:
        loop.step(screens[n % len(screens)])
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": loop.workers, "kind": "port",
            "sample": f"{n} iterations of the saxo40 RTC step (float64 NumPy/SciPy, {loop.workers} threads)"}


def run_reference_gpu(args, setup):
    """The reference's own implementation of the path -- its sutra CUDA code,
    built from its sources into oracle/_ref -- on this GPU, through its Python
    API in the supervisor's order: each step copies the phase from the host,
    forms the SH image with photon and readout noise, computes the wCoG slopes
    with threshold, the LS commands and the voltages, and reads the voltages
    back to the host.  The L2 cache is flushed between steps (outside the
    timed span); the step is timed by the host clock around the calls (they
    end with the voltages on the host)."""
    import torch

    from aob200.workloads import von_karman_screens
    from oracle.ref_sutra import RefShLoop

    g = setup.geom
    loop = RefShLoop(g, setup.cmat, setup.centroider, setup.threshold, setup.weights, noise=setup.noise, seed=1234)
    screens = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, 0.14, 25.0, 8, seed=0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for i in range(args.warmup):
        loop.step(screens[i % 8])
    total = 0.0
    with ClockSampler(0) as clk:
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            loop.step(screens[i % 8])
            total += time.perf_counter() - t0
    v = args.steps / total
    return v, clk.summary()


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from aob200.workloads import sh_loop_setup

    setup = sh_loop_setup("saxo40")
    workload = ("saxo40: 40x40 SH, 1248 valid, 6x6 px, Nfft 32, wCoG+thr, photon+0.5e- noise, "
                "1377x2496 LS MVM")
    from oracle import ref_sutra

    gpu = False
    try:
        import torch

        gpu = torch.cuda.is_available() and ref_sutra.available()
    except Exception:
        gpu = False
    if gpu:
        v, clocks = run_reference_gpu(args, setup)
        g = setup.geom
        sample = (f"{args.steps} RTC iterations of the reference's sutra CUDA build (oracle/_ref) on the GPU, "
                  "driven from one host thread through its Python API")
        line = {
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload, "device": "gpu: the reference's own sutra CUDA code, built from its sources",
                       "l2": "flushed before every timed step (256 MB write)",
                       "timing": "host clock per step: phase from host, comp_image, do_centroids, do_control, "
                                 "comp_voltage, voltages to host"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": g.tel.n * g.tel.n * 4,
                    "d2h_bytes_per_step": setup.nactu * 4},
            "clocks": clocks,
        }
        print(json.dumps(line))
        return 0
    from oracle.loop_cpu import CpuShLoop
    from aob200.workloads import von_karman_screens

    g = setup.geom
    screens = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, 0.14, 25.0, 4, seed=1)
    loop = CpuShLoop(g, setup.cmat, setup.centroider, setup.threshold, setup.weights, setup.noise)
    per_step = 3  # RTC iterations per benchmark step (bounded CPU sample)
    for i in range(args.warmup):
        loop.step(screens[i % 4])
    t0 = time.perf_counter()
    for i in range(args.steps * per_step):
        loop.step(screens[i % 4])
    dt = time.perf_counter() - t0
    v = args.steps * per_step / dt
    res = [{"cores": loop.workers,
            "sample": f"{args.steps * per_step} iterations of the saxo40 RTC step "
                      f"(float64 NumPy/SciPy, {loop.workers} threads)"}]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload, "device": "cpu (the reference's CUDA build is not available here: "
                                                   "its float64 NumPy restatement)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": res[0]["cores"], "kind": "port",
                         "sample": res[0]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# secondary workloads (--workload mc64 | pyr50 | mlp | precision): one JSON line each
def _line(args, workload, metric, value, unit, ms_per_step, dtype, config, **extra):
    d = {"workload": workload, "metric": metric, "value": value, "unit": unit, "n_gpus": 1,
         "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
         "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": config}
    d.update(extra)
    print(json.dumps(d))


def run_mc64(args, torch):
    """64 uneven SH loops (nxsub 24..40, 6x6 / 8x8 px, seeds 0..63, r0 in 0.08..0.20 m,
    photon + readout noise, wCoG, BF16 MVM) advanced by one persistent launch per step."""
    from aob200 import autotune as AT
    from aob200 import workloads as W

    t0 = time.perf_counter()
    insts = W.mc_setup(64)[:args.instances]
    loops, batch = W.build_mc_batch(insts, precision="bf16")
    setup_s = time.perf_counter() - t0
    if args.no_tune:
        batch.set_tuning(16, 256, 96, 16, 2, 0)
        tune = {"tuning": {"subaps": 16, "team": 256, "mvm_kb": 96, "lag": 16, "ctas_per_sm": 2, "order": 0}}
    else:
        tune = AT.tune_batch(batch, noise=True)
    info = batch.info()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    for _ in range(args.warmup):
        batch.step(True, sptr)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for a, b in ev:
            a.record(stream)
            batch.step(True, sptr)
            b.record(stream)
        torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    n = info["instances"]
    peak, peak_kind = _peaks()
    achieved = info["alg_bytes"] / (ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": _profile_traffic("batch_step_mc64"), "kernel": "batch_step_kernel",
                "algorithmic_bytes_per_launch": info["alg_bytes"], "duration_us": ms * 1e3, "peak_source": peak_kind,
                "note": "the sensor stages (54,048 sub-apertures) keep the SMs busy longer than the 240 MB stream"}
    # e2e: all phases in from pinned host memory, all voltages out, every step
    phases = torch.from_numpy(np.concatenate([np.ascontiguousarray(i.phase.ravel(order="F")) for i in insts]))
    h_ph = phases.pin_memory()
    h_v = torch.zeros(info["volt_floats"], dtype=torch.float32).pin_memory()
    for _ in range(3):
        batch.step_host(h_ph.data_ptr(), h_v.data_ptr(), True, sptr)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for a, b in ev2:
        a.record(stream)
        batch.step_host(h_ph.data_ptr(), h_v.data_ptr(), True, sptr)
        b.record(stream)
    torch.cuda.synchronize()
    ms_e2e = sum(a.elapsed_time(b) for a, b in ev2) / args.steps
    e2e = {"value": n / (ms_e2e * 1e-3), "unit": "instance iters/s", "h2d_bytes_per_step": info["phase_floats"] * 4,
           "d2h_bytes_per_step": info["volt_floats"] * 4, "call": "aob_batch_step_host"}
    # the same 64 loops stepped one after another with their own fused kernels
    seq_ms = 0.0
    for (_, _, _, loop) in loops:
        seq_ms += loop.time(noise=True, warmup=2, iters=10)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle.loop_cpu import CpuShLoop

        k, t_cpu = 0, 0.0
        for inst in insts[:4]:
            st = inst.setup
            cl = CpuShLoop(st.geom, st.cmat, st.centroider, st.threshold, st.weights, st.noise)
            cl.step(inst.phase)
            t1 = time.perf_counter()
            for _ in range(5):
                cl.step(inst.phase)
            t_cpu += time.perf_counter() - t1
            k += 5
        cpu = {"value": k / t_cpu, "unit": "instance iters/s", "cores": cl.workers, "kind": "port",
               "sample": f"{k} loop iterations of the first 4 instances (float64 NumPy/SciPy, {cl.workers} threads)"}
    _line(args, "mc64", "Monte Carlo instance iterations/s, %d uneven SH loops, one launch per step" % n, n / (ms * 1e-3),
          "instance iters/s", ms, "f32 sensor, bf16 MVM",
          {"workload": "mc64: %d SH loops, nxsub 24..40, 6x6/8x8 px, Nfft 16/32, photon + 0.5 e- noise, wCoG, " % n +
                       "BF16 LS MVM; %d sub-apertures, %d actuators in total" % (
                           sum(i.setup.geom.nvalid for i in insts), sum(i.setup.nactu for i in insts)),
           "l2": "inputs (%.0f MB) larger than L2" % (info["alg_bytes"] / 1e6), "cuda_graph": True,
           "tuning": tune["tuning"], "setup_s": setup_s},
          roofline=roofline, e2e=e2e, cpu_baseline=cpu, clocks=clk.summary(), gpu_launches=args.steps,
          sequential_loops_ms_per_step=seq_ms, speedup_vs_sequential_loops=seq_ms / ms)


def run_pyr50(args, torch):
    """Pyramid: 50 x 50 pupil samples, 24 modulation points at 3 lambda/D over 512 x 512
    FFTs, photon + 0.3 e- noise, slopes and a 1600-actuator LS MVM."""
    from aob200 import core as C
    from aob200 import geometry as G
    from aob200 import workloads as W

    g = G.pyr_geometry(G.PyrParams(nxsub=50, wavelength_um=1.075, ampl=3.0, npts=24, pup_sep=32, fssize=3.2), 100,
                       diam=8.0, cobs=0.14)
    w = C.PyrWfs.from_geometry(g, noise=0.3, seed=3)
    # the second stage sees the residual of the seeded saxo40 closed loop
    res, pd_in = W.saxo40_residual(niter=200)
    phase = W.resample_pupil(res, pd_in, g.tel.n, g.tel.pupdiam)
    w.set_phase(phase)
    c = C.Centroider(g.nvalid, 0.0, 1.0, "pyr")
    c.load_validpos(g.validsubsx, g.validsubsy)
    c.attach(w)
    ls = C.LsController(2 * g.nvalid, 1600)
    ls.set_cmat((np.random.default_rng(1).standard_normal((1600, 2 * g.nvalid)) * 0.01).astype(np.float32))
    d = ls.buffer("centroids")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step(sp):
        w.comp_image(True, sp)
        c.get_cog(d.ptr, sp)
        ls.comp_com(sp)

    with ClockSampler(0) as clk:
        t_step = graph_time(torch, flush, step, n=max(args.steps, 5))
        t_img = graph_time(torch, flush, lambda sp: w.comp_image(True, sp), n=max(args.steps, 5))
    nfft, npts = g.nfft, g.pyr_cx.size
    flops = (2 * npts + 3) * 5 * nfft * nfft * np.log2(nfft * nfft)  # 2 FFTs per point + the convolution's 2 + 1
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import pyr as opyr

        ncores = len(os.sched_getaffinity(0))
        t1 = time.perf_counter()
        k = 0
        while k < 3:
            opyr.comp_image(phase, g.tel.mpupil, g, g.wavelength_um, g.nphotons, noise=0.3, frame=k, workers=ncores)
            k += 1
        dt = time.perf_counter() - t1
        cpu = {"value": k / dt, "unit": "iters/s", "cores": ncores, "kind": "port",
               "sample": f"{k} pyramid images (float64 scipy.fft, modulation points batched over {ncores} threads)"}
    _line(args, "pyr50", "pyramid loop iters/s (image + slopes + 1600-actuator LS MVM)", 1.0 / t_step, "iters/s",
          t_step * 1e3, "f32",
          {"workload": f"pyr50: {g.nxsub}x{g.nxsub} pupil samples per image, {npts} modulation points at 3 lambda/D, "
                       f"{nfft}x{nfft} FFTs, {g.nvalid} valid, 1600-actuator LS MVM",
           "l2": "flushed before every timed step (256 MB write)",
           "input": "residual phase of the seeded saxo40 closed loop after 200 iterations, resampled to the pupil"},
          # no measured FP32 (non-tensor) peak: nominal 148 SMs x 128 FP32 lanes x 2 FLOP x 1.965 GHz
          roofline={"bound": "fp32 FFT", "achieved": flops / t_img / 1e12, "unit": "TFLOP/s", "peak": FP32_NOMINAL_TFLOPS,
                    "frac": flops / t_img / 1e12 / FP32_NOMINAL_TFLOPS, "peak_source": "nominal (not measured)",
                    "traffic": None, "kernel": "pyramid image kernels",
                    "flops_per_image": flops, "image_us": t_img * 1e6, "step_us": t_step * 1e6},
          cpu_baseline=cpu, clocks=clk.summary(), gpu_launches=None)


def run_mlp(args, torch):
    """Learned reconstructor at the saxo40 geometry: 2496 slopes -> 1024 -> 1024 (GELU)
    -> 1377 commands (+ linear skip), BF16 weights, FP32 accumulation."""
    from aob200 import core as C
    from aob200 import mlp as M
    from aob200.workloads import sh_loop_setup

    setup = sh_loop_setup("saxo40")
    nin, nout = setup.nslope, setup.nactu
    rng = np.random.default_rng(0)
    ls = C.LsController(nin, nout)
    ls.set_cmat(setup.cmat)
    ls.set_gain(0.4)
    ls.set_centroids(rng.standard_normal(nin).astype(np.float32))
    net = M.MlpReconstructor(nin, nout, 1024, 1024, seed=1)
    net.init_from_ls(setup.cmat, 10.0, 1.0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    res = {}
    with ClockSampler(0) as clk:
        res["ls_f32_us"] = graph_time(torch, flush, lambda sp: ls.comp_com(sp)) * 1e6
        ls.set_precision("bf16")
        res["ls_bf16_us"] = graph_time(torch, flush, lambda sp: ls.comp_com(sp)) * 1e6
        ls.set_precision("f32")
        res["mlp_infer_us"] = graph_time(torch, flush, lambda sp: net.comp_com(ls, 3e38, sp)) * 1e6
        params = nin * 1024 + 1024 * 1024 + 1024 * nout + nin * nout
        B = 4096
        X = torch.randn(B, nin, device="cuda")
        T = torch.randn(B, nout, device="cuda")
        t = graph_time(torch, flush, lambda sp: net.train_step(X.data_ptr(), T.data_ptr(), B, 1e-4, None, sp), n=5,
                       with_flush=False)
        res["train_step_B4096_us"] = t * 1e6
        res["train_tflops"] = 6 * params * B / t / 1e12
        # one whole RTC iteration with each reconstructor on the same sensor stages:
        # image with the fused wCoG, slopes to the controller, commands, voltages
        from aob200.workloads import build_sh_loop

        wfs, cen, ls2, loop = build_sh_loop(setup, graph=False)
        cptr = ls2.buffer("centroids").ptr

        def it_learned(sp):
            wfs.comp_image(True, sp)
            cen.get_cog(cptr, sp)
            net.comp_com(ls2, 3e38, sp)
            ls2.comp_voltage(sp)

        def it_ls(sp):
            wfs.comp_image(True, sp)
            cen.get_cog(cptr, sp)
            ls2.comp_com(sp)
            ls2.comp_voltage(sp)

        loop_us = {"learned_fused_kernel": graph_time(torch, flush,
                                                      lambda sp: loop.step_mlp(net, 3e38, None, None, True, sp,
                                                                               wait=False)) * 1e6,
                   "learned": graph_time(torch, flush, it_learned) * 1e6,
                   "ls_same_kernels": graph_time(torch, flush, it_ls) * 1e6,
                   "ls_fused_kernel": graph_time(torch, flush, lambda sp: loop.step(None, None, True, sp)) * 1e6,
                   "what": "one saxo40 RTC iteration (sensor image + wCoG, reconstruction, voltages), graph replay "
                           "with a flushed L2; the learned reconstructor's Strehl parity is the c4 workload's"}
    peak_t = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_t = float(json.load(f)["bf16_tflops"])
    except Exception:
        peak_t = 1590.0
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import mlp as om

        from threadpoolctl import threadpool_info, threadpool_limits

        ncores = len(os.sched_getaffinity(0))
        P = net.get_params()
        x = rng.standard_normal((1, nin)).astype(np.float32)
        with threadpool_limits(limits=ncores, user_api="blas"):
            blas = max([d.get("num_threads", 1) for d in threadpool_info() if d.get("user_api") == "blas"] or [1])
            t1 = time.perf_counter()
            k = 0
            while k < 20:
                om.forward(P, x, net.in_scale)
                k += 1
            dt = time.perf_counter() - t1
        cpu = {"value": k / dt, "unit": "inferences/s", "cores": blas, "kind": "port",
               "sample": f"{k} batch-1 forward passes (NumPy, bfloat16-rounded weights, BLAS on {blas} threads)"}
    _line(args, "mlp", "learned reconstructor batch-1 inferences/s (LS MVM alongside)", 1e6 / res["mlp_infer_us"],
          "inferences/s", res["mlp_infer_us"] / 1e3, "bf16",
          {"workload": f"mlp: {nin} -> 1024 -> 1024 -> {nout} + linear skip, BF16 weights, FP32 accumulation",
           "l2": "flushed before every timed inference (256 MB write)"},
          roofline={"bound": "tensor", "achieved": res["train_tflops"], "peak": peak_t, "unit": "TFLOP/s",
                    "frac": res["train_tflops"] / peak_t, "traffic": None, "kernel": "tc_gemm_kernel (training step)",
                    **res},
          cpu_baseline=cpu, clocks=clk.summary(), gpu_launches=None, loop_us=loop_us)


def run_precision(args, torch):
    """saxo40 with its own LS command matrix (push-pull imat, float64 inverse):
    the command error of one MVM and the closed-loop residual-wavefront rms and
    LE Strehl of each MVM precision against a float64 host reconstruction of
    the same seeded loop (aob200.precision.study)."""
    from aob200 import precision as P

    t0 = time.perf_counter()
    res = P.study(niter=args.loop_iters, nskip=args.loop_iters // 10, sample_every=max(args.loop_iters // 100, 1))
    print(json.dumps({"workload": "precision", "metric": "relative residual-wavefront rms change vs float64 "
                      "reconstruction (noise-free closed loop), LE Strehl (noisy closed loop), and relative "
                      "command error of one MVM",
                      "unit": "relative", "dtype": "f32/bf16/fp8 MVM, f32 sensor", "data": "synthetic",
                      "config": {"workload": "saxo40 closed loop: 3-layer von Karman (r0 0.14 m), noise-free and with "
                                 "photon + 0.5 e- noise at magnitude 8, wCoG + threshold, gain 0.4, LE Strehl at "
                                 "1.65 um",
                                 "iterations": args.loop_iters}, "seconds": round(time.perf_counter() - t0, 1),
                      **res}))
    return 0


def run_c4(args, torch):
    """The learned reconstructor at its configured scale (aob200.learned.c4_experiment):
    the saxo40 geometry, closed-loop training pairs over r0 0.08-0.20 m and magnitudes
    6-10, training on the GPU, the output gain chosen on a validation loop, then the
    long-exposure Strehl of both reconstructors on the held-out loop."""
    from aob200 import learned

    res = learned.c4_experiment(pairs=args.pairs, epochs=args.epochs, loop_iters=args.loop_iters,
                                settle=args.settle)
    print(json.dumps({"workload": "c4", "metric": "long-exposure Strehl at 1.65 um, learned vs LS reconstructor "
                      "(closed loop, same seeded turbulence)", "value": res["mlp"]["strehl_le"], "unit": "Strehl",
                      "ls_value": res["ls"]["strehl_le"], "rel_diff": res["rel_diff"],
                      "dtype": "bf16 weights, f32 accumulation", "data": "synthetic",
                      "config": {"workload": "c4: saxo40 geometry, MLP 2496 -> 1024 -> 1024 (GELU) -> 1352 + linear "
                                 "skip initialised to the LS matrix; pairs from closed LS loops at r0 0.08-0.20 m and "
                                 "magnitudes 6-10; output gain chosen on a validation loop; evaluation at r0 0.14 m, "
                                 "magnitude 8, held-out seeds", "pairs": args.pairs, "epochs": args.epochs,
                                 "loop_iterations": args.loop_iters},
                      **{k: v for k, v in res.items() if k not in ("rel_diff", "net")}}))
    return 0


def run_secondary(args):
    import torch

    torch.cuda.set_device(0)
    fn = {"mc64": run_mc64, "pyr50": run_pyr50, "mlp": run_mlp, "precision": run_precision,
          "c4": run_c4}[args.workload]
    return fn(args, torch) or 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f32", choices=["f32", "bf16", "fp8"])
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="saxo40", choices=["saxo40", "mc64", "pyr50", "mlp", "precision", "c4"])
    ap.add_argument("--loop-iters", type=int, default=5000, help="precision, c4: closed-loop iterations per run")
    ap.add_argument("--pairs", type=int, default=200000, help="c4: training pairs")
    ap.add_argument("--epochs", type=int, default=16, help="c4: training epochs")
    ap.add_argument("--settle", type=int, default=100, help="c4: closed-loop iterations before the long exposure")
    ap.add_argument("--instances", type=int, default=64, help="mc64: number of instances (the first N of the list)")
    ap.add_argument("--no-tune", action="store_true", help="mc64: fixed tile shapes instead of the autotuner")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "saxo40":
        return run_secondary(args)

    ws, rank, local = _dist()
    import torch

    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)

    from aob200 import _lib
    from aob200.workloads import build_sh_loop, sh_loop_setup, von_karman_screens

    setup = sh_loop_setup("saxo40")
    g = setup.geom
    wfs, centro, ls, loop = build_sh_loop(setup, precision=args.precision, device=device,
                                          graph=not args.no_graph, seed=1234 + rank)
    n = g.tel.n
    nscreen = 8
    screens = von_karman_screens(n, 8.0 / g.tel.pupdiam, 0.14, 25.0, nscreen, seed=rank)
    d_screens = torch.from_numpy(np.ascontiguousarray(np.stack([s.ravel(order="F") for s in screens]))).cuda()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    phase_ptr = wfs.d_phase.ptr
    nbytes_phase = n * n * 4

    def load_phase(i):
        _lib.call("aob_memcpy_d2d", phase_ptr, d_screens[i % nscreen].data_ptr(), nbytes_phase, sptr)

    # ---- value: device-resident inputs, L2 flushed before each step --------
    for i in range(args.warmup):
        load_phase(i)
        flush.zero_()
        loop.step(None, None, noise=True, stream=sptr)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(device) as clk:
        for i in range(args.steps):
            load_phase(i)
            flush.zero_()
            starts[i].record(stream)
            loop.step(None, None, noise=True, stream=sptr)
            ends[i].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = max_over_ranks(dist, torch, [sum(s.elapsed_time(e) for s, e in zip(starts, ends))], "cuda")[0]
    clocks = clk.summary()
    ms_per_step = total_ms / args.steps
    value = job_rate(ws, args.steps, total_ms)
    launches = loop.kernels_per_step() * args.steps

    # ---- per-kernel device durations (graph replay, no host gaps) ----------
    loop.use_graph(False)
    t_step = graph_time(torch, flush, lambda sp: loop.step(None, None, True, sp))
    fused = loop.kernels_per_step() == 1
    t_wfs = graph_time(torch, flush, lambda sp: wfs.comp_image(True, sp))
    t_mvm = graph_time(torch, flush, lambda sp: ls.comp_com(sp))
    loop.use_graph(not args.no_graph)
    esize = {"f32": 4, "bf16": 2, "fp8": 1}[args.precision]
    ld = {"f32": 4, "bf16": 8, "fp8": 16}[args.precision]
    ncol_pad = (setup.nslope + ld - 1) // ld * ld
    npix2 = g.npix * g.npix
    # algorithmic bytes: every input read once, every output written once
    mvm_bytes = setup.nactu * ncol_pad * esize + setup.nslope * 4 + setup.nactu * 4 * 5 + \
        (setup.nactu * 4 if args.precision == "fp8" else 0)
    wfs_bytes = 2 * g.nvalid * g.pdiam * g.pdiam * 4 + 2 * g.nvalid * npix2 * 4 + g.nvalid * 4 * 6 + \
        2 * g.nvalid * 4
    peak, peak_kind = _peaks()
    if fused:
        dom, dbytes, dt, prof = "rtc_fused_kernel", mvm_bytes + wfs_bytes, t_step, f"rtc_fused_saxo40_{args.precision}"
    elif t_mvm >= t_wfs:
        dom, dbytes, dt, prof = "ls_mvm_bulk_kernel", mvm_bytes, t_mvm, f"ls_mvm_saxo40_{args.precision}"
    else:
        dom, dbytes, dt, prof = "sh_image_kernel", wfs_bytes, t_wfs, "sh_image_saxo40"
    achieved = dbytes / dt / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": _profile_traffic(prof), "kernel": dom, "algorithmic_bytes_per_launch": dbytes,
                "duration_us": dt * 1e6, "peak_source": peak_kind, "timing": "graph replay, L2 flushed per launch",
                "kernels_us": {"rtc_step": t_step * 1e6, "sh_image": t_wfs * 1e6, "ls_mvm": t_mvm * 1e6}}

    # ---- e2e: host phases in, host voltages out, through the C ABI ----------
    # Streamed, as a real-time controller runs: the phase of step k + 1 crosses
    # the bus (aob_memcpy_h2d on a copy stream, into one of two staging buffers)
    # while step k computes (aob_memcpy_d2d into the sensor's phase, then
    # aob_loop_step_async, whose fused kernel writes the voltages into pinned host
    # memory) -- the pipeline aob_loop_run runs.  L2 is flushed before every step
    # outside its span; span k runs from after the flush until both step k's
    # voltages and step k + 1's phase have landed, so every step's copy is inside
    # a span (step 0's in series with its own compute).
    h_phase = torch.from_numpy(np.ascontiguousarray(np.stack([s.ravel(order="F") for s in screens]))).pin_memory()
    e2e_steps = max(10, args.steps)
    h_volts = torch.zeros((e2e_steps, setup.nactu), dtype=torch.float32).pin_memory()
    h_volt = h_volts[0]  # one step's voltages (pinned)
    cstream = torch.cuda.Stream(device)
    cptr = cstream.cuda_stream
    stage = [torch.empty(n * n, dtype=torch.float32, device="cuda") for _ in range(2)]

    def h2d(k):
        _lib.call("aob_memcpy_h2d_async", stage[k % 2].data_ptr(), h_phase[k % nscreen].data_ptr(), nbytes_phase,
                  cptr)

    for i in range(3):
        loop.step(h_phase[i % nscreen].data_ptr(), h_volt.data_ptr(), noise=True, stream=sptr)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(e2e_steps)]
    copied = [torch.cuda.Event() for _ in range(e2e_steps)]
    for k, (a, b) in enumerate(ev):
        flush.zero_()
        a.record(stream)
        cstream.wait_event(a)  # the copy stream follows the flush (and the last read of its staging buffer)
        if k == 0:
            h2d(0)
            copied[0].record(cstream)
        if k + 1 < e2e_steps:
            h2d(k + 1)
            copied[k + 1].record(cstream)
        stream.wait_event(copied[k])
        _lib.call("aob_memcpy_d2d", phase_ptr, stage[k % 2].data_ptr(), nbytes_phase, sptr)
        loop.step(None, h_volts[k].data_ptr(), noise=True, stream=sptr, wait=False)
        if k + 1 < e2e_steps:
            stream.wait_event(copied[k + 1])
        b.record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in ev)

    # the same steps one at a time: each step's phase copy, kernel and voltages,
    # then the host waits (no overlap), L2 flushed before each
    ev1 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(e2e_steps)]
    wall = 0.0
    for i, (a, b) in enumerate(ev1):
        flush.zero_()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        a.record(stream)
        loop.step(h_phase[i % nscreen].data_ptr(), h_volt.data_ptr(), noise=True, stream=sptr, wait=False)
        b.record(stream)
        b.synchronize()
        wall += time.perf_counter() - w0
    torch.cuda.synchronize()
    sync_ms = sum(a.elapsed_time(b) for a, b in ev1)

    # aob_loop_run itself: e2e_steps streamed steps in one call, no flush between
    # them (the command matrix stays in L2), device span and the call's wall clock
    run_wall = float("nan")
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    torch.cuda.synchronize()
    a.record(stream)
    w0 = time.perf_counter()
    loop.run(h_phase.data_ptr(), e2e_steps, h_volts.data_ptr(), noise=True, stream=sptr, nphases=nscreen)
    run_wall = time.perf_counter() - w0
    b.record(stream)
    torch.cuda.synchronize()
    run_ms = a.elapsed_time(b)
    e2e_ms, sync_ms, run_ms, wall, run_wall = max_over_ranks(dist, torch, [e2e_ms, sync_ms, run_ms, wall, run_wall],
                                                             "cuda")
    e2e = {"value": job_rate(ws, e2e_steps, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": nbytes_phase,
           "d2h_bytes_per_step": setup.nactu * 4, "ms_per_step": e2e_ms / e2e_steps,
           "call": "streamed: aob_memcpy_h2d_async of step k+1's pinned host phase on a copy stream while step k runs "
                   "(aob_memcpy_d2d into the sensor's phase, aob_loop_step_async: the fused kernel writes the voltages "
                   "into pinned host memory); L2 flushed before each step outside its span; span k = until step k's "
                   "voltages and step k+1's phase are both there",
           "per_step_sync": {"value": job_rate(ws, e2e_steps, sync_ms), "wall_clock_value": ws * e2e_steps / wall,
                             "call": "aob_loop_step_async then an event the host waits on, one step at a time "
                                     "(phase copy, kernel, voltages in series), L2 flushed before each"},
           "run_api": {"value": job_rate(ws, e2e_steps, run_ms), "wall_clock_value": ws * e2e_steps / run_wall,
                       "call": f"aob_loop_run: {e2e_steps} streamed steps in one call (pinned phases cycled, pinned "
                               "voltages), no L2 flush between steps"}}

    # ---- the same iteration with the learned reconstructor in place of the LS
    # matrix (2496 -> 1024 -> 1024 -> 1377 + the linear skip; its Strehl parity with
    # LS is the c4 workload's), timed like value: device-resident phase, L2 flushed
    # before every step, one rtc_mlp_kernel launch per step --------------------
    learned, learned_ms, learned_kernels = None, float("nan"), 0
    try:
        from aob200 import mlp as M

        net = M.MlpReconstructor(setup.nslope, setup.nactu, 1024, 1024, device=device, seed=1)
        net.init_from_ls(setup.cmat, 10.0, 1.0)
        wfs_l, _c_l, _ls_l, loop_l = build_sh_loop(setup, precision="f32", device=device, graph=False,
                                                   seed=1234 + rank)
        ph_l = wfs_l.d_phase.ptr
        for i in range(args.warmup):
            _lib.call("aob_memcpy_d2d", ph_l, d_screens[i % nscreen].data_ptr(), nbytes_phase, sptr)
            flush.zero_()
            loop_l.step_mlp(net, 3e38, None, None, True, sptr, wait=False)
        torch.cuda.synchronize()
        st = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        en = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for i in range(args.steps):
            _lib.call("aob_memcpy_d2d", ph_l, d_screens[i % nscreen].data_ptr(), nbytes_phase, sptr)
            flush.zero_()
            st[i].record(stream)
            loop_l.step_mlp(net, 3e38, None, None, True, sptr, wait=False)
            en[i].record(stream)
        torch.cuda.synchronize()
        learned_ms = sum(a.elapsed_time(b) for a, b in zip(st, en))
        learned_kernels = loop_l.kernels_per_step()
        del loop_l, wfs_l, net
    except Exception as e:  # reported, the headline stands
        learned = {"error": str(e)[:300]}
    learned_ms = max_over_ranks(dist, torch, [learned_ms], "cuda")[0]  # every rank, also after an error
    if learned is None and np.isfinite(learned_ms):
        learned = {"value": job_rate(ws, args.steps, learned_ms), "unit": UNIT, "ms_per_step": learned_ms / args.steps,
                   "kernels_per_step": learned_kernels,
                   "call": "aob_loop_step_mlp: one rtc_mlp_kernel per step (sensor stages, the network's control "
                           "step with its LS fallback test, voltages)",
                   "strehl": "long-exposure Strehl within 1 % of LS at this geometry: bench.py --workload c4"}

    # ---- the closed-loop stages around the RTC iteration, each timed alone (graph
    # replay, L2 flushed): the three-layer screen extrusion, the raytrace of the
    # layers and the DM into the sensor's phase, the DM shape from the voltages;
    # then the whole closed-loop iteration (ShAoSystem.next without the PSF) -----
    extras, ex_us, dm_bytes, dm_nact = None, [float("nan")] * 4, 0, 0
    try:
        from aob200 import system as S

        sy = S.ShAoSystem(S.saxo40(), device)
        sy.close(graph=False)
        dm = sy.dm
        dm_bytes, dm_nact = 4 * (dm.influsize * dm.influsize * dm.nact + dm.nact + dm.dim * dm.dim), dm.nact
        ex_us = [graph_time(torch, flush, lambda sp: sy.atmos.move(sp)) * 1e6,
                 graph_time(torch, flush, lambda sp: sy.trace_wfs(sp)) * 1e6,
                 graph_time(torch, flush, lambda sp: dm.comp_shape(None, sp)) * 1e6,
                 graph_time(torch, flush, lambda sp: sy.next(sp, compute_psf=False, noise=True)) * 1e6]
        del sy
    except Exception as e:  # reported, the headline stands
        extras = {"error": str(e)[:300]}
    ex_us = max_over_ranks(dist, torch, ex_us, "cuda")  # every rank, also after an error
    if extras is None and all(np.isfinite(ex_us)):
        extras = {"extrusion_us": ex_us[0], "raytrace_wfs_us": ex_us[1], "dm_shape_us": ex_us[2],
                  "dm_shape_bytes": dm_bytes, "dm_shape_gbs": dm_bytes / ex_us[2] / 1e3, "iteration_us": ex_us[3],
                  "what": f"saxo40 closed loop (3 von Karman layers, {dm_nact}-actuator DM): extrusion of every layer, "
                          "raytrace into the sensor's phase, DM shape, and the whole iteration (extrusion, "
                          "raytrace, fused RTC step, DM shape)"}

    # ---- persistent mode: the fused kernel resident (matrix rows, sensor tables
    # and integrator state in shared memory), one doorbell per step; the L2 flush
    # between steps is written by the resident kernel itself (it holds every
    # SM's registers, no other kernel runs beside it) ------------------------
    persistent, pms, busy_us = None, [float("nan"), float("nan")], float("nan")
    if fused:
        try:
            loop.persist_start(noise=True, host_voltage=h_volt.data_ptr())
            try:
                fptr, fbytes = flush.data_ptr(), flush.numel() * 4
                for i in range(3):
                    loop.persist_step(None, h_volt.data_ptr(), noise=True, stream=sptr, wait=True)

                def timed(host):
                    evs = []
                    for i in range(e2e_steps):
                        loop.persist_flush(fptr, fbytes, stream=sptr)
                        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        a.record(stream)
                        loop.persist_step(h_phase[i % nscreen].data_ptr() if host else None, h_volt.data_ptr(),
                                          noise=True, stream=sptr, wait=False)
                        b.record(stream)
                        evs.append((a, b))
                    # (the stream only: a device-wide synchronise would wait for the resident kernel)
                    stream.synchronize()
                    return sum(a.elapsed_time(b) for a, b in evs)

                n0, t0 = loop.persist_stats()
                pms = [timed(False)]
                n1, t1 = loop.persist_stats()
                pms.append(timed(True))
                busy_us = (t1 - t0) / max(n1 - n0, 1) / 1000.0
            finally:
                loop.persist_stop()
            if ls.status():
                raise RuntimeError(f"controller status {ls.status()} after the persistent steps")
        except Exception as e:  # reported in the line, the launched numbers stand
            persistent = {"error": str(e)[:300]}
            pms = [float("nan"), float("nan")]
    pms = max_over_ranks(dist, torch, pms, "cuda")
    if fused and persistent is None and np.isfinite(pms).all():
        persistent = {
            "value": job_rate(ws, e2e_steps, pms[0]), "unit": UNIT, "ms_per_step": pms[0] / e2e_steps,
            "kernel_busy_us_per_step": busy_us,
            "e2e": {"value": job_rate(ws, e2e_steps, pms[1]), "unit": UNIT, "h2d_bytes_per_step": nbytes_phase,
                    "d2h_bytes_per_step": setup.nactu * 4},
            "call": "aob_loop_persist_step: stream write of the doorbell, stream wait for the kernel's done "
                    "word (e2e: after the phase copy from pinned memory; voltages written into the pinned host "
                    "buffer by the kernel); device-timed per step, the resident kernel's 256 MB L2 flush "
                    "(aob_loop_persist_flush) between steps outside the timed span",
            "resident": "command-matrix rows, sensor tables and integrator state stay in shared memory across "
                        "steps; per step the phase is read from HBM (or copied from the host) and the images, "
                        "slopes, commands and voltages are written"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(setup)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": {"workload": "saxo40: 40x40 SH (1248 valid, 2496 slopes), 6x6 px, Nfft 32, nrebin 3, "
                               "wCoG+threshold, photon + 0.5 e- readout noise, LS 1377x2496 MVM + integrator + "
                               "voltage; one RTC iteration per step",
                   "l2": "flushed before every timed step (256 MB write)",
                   "parallelism": f"replicas x{ws}",
                   "launch": ("one cooperative kernel per step, launched directly" if fused
                              else ("three kernels per step, CUDA graph" if not args.no_graph else "three kernels per step")),
                   "mvm_precision": args.precision},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "gpu_launches": launches,
        "persistent": persistent,
        "learned": learned,
        "closed_loop_extras": extras,
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
