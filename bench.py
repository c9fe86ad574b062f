#!/usr/bin/env python
"""Benchmark of the coupled-standard-map ensemble: orbit-steps/s on one B200.

Workload (the metric's configuration): Froeschle 4D coupled standard maps (nu = kappa = 1.5, coupling mu = 0.05),
65536 orbits with coordinates uniform in [0, 2pi)^4 (seed 1), N = 1e5 steps, tau = 10, two tangent frames carried
along each orbit from W0 = I: QRSpectrum(HouseholderQR) with k = 4, and GALI_4 with SALI read off its first two
columns. A step is one full pass of the hot path over that ensemble (65536 x 1e5 = 6.55e9 orbit-steps).

`value` is the mixed-precision kernel (Float64 orbit and log sums, Float32 frames) with inputs resident in HBM;
the plain Float64 kernel (the reference's arithmetic, bit-identical to the oracle) is timed beside it
(`fp64_kernel`) together with the largest |lambda_1 difference| between the two. `e2e` is the same work through
the C ABI with host buffers (cl_b200_propagate: copies in and out inside the timed region). `cpu_baseline` and
`--impl reference` time the CPU restatement of the reference (the oracle; Julia, the reference's own runtime, is
not installed) on the host cores.

Multi-GPU: orbits are independent, so N ranks run N shards of the same size with no collective in the data path
(weak scaling); the time is the max over ranks.

`--workload` selects one of the other measured configurations (one GPU, one JSON line each, same keys):
  standard  the Chirikov standard map K = 6, 4096 orbits, N = 1e5, k = 2, tau = 1, QRSpectrum(MGS), FP64 kernel
            (bit-identical to the oracle);
  gauss     IntegratorMap(Gauss-3, Henon-Heiles, dt = 0.01), 16384 starts on the E = 1/8 section, N = 1e6,
            k = 2, tau = 10, chain MEGNO + FLI + QRSpectrum(Givens), FP64 kernel: Gauss steps/s;
  lattice   the uneven ensemble: 1,048,576 orbits of standard-map lattices d in {2, 4, 8, 16}, K ~ U[0.5, 3],
            lengths log-uniform in [1e3, 1e6], escape at |p| > 1e3, k = min(d, 8), tau in {5, 10, 20}, mixed
            precision, one CUDA graph of persistent work-queue kernels with autotuned variants: executed
            orbit-steps/s;
  screen    the learned screen on the 2048 x 2048 (x1, p1) grid of Froeschle orbits (x2 = p2 = 0.1), N = 1e5:
            screened orbits/s against the plain full integration of every orbit, with the misclassification
            over the whole grid;
  mlp       the screen's network alone: inference rows/s at a batch of 262144 against the BF16 tensor peak;
  split     IntegratorMap(KahanLi(8), Henon-Heiles, dt = 0.05), 16384 starts on the E = 1/8 section, N = 2e5
            (t = 1e4), k = 2, tau = 10, chain MEGNO + FLI + QRSpectrum(Givens), FP64 kernel: steps/s;
  shadow    the two-trajectory estimator on the coupled-map workload's orbits (65536 x 1e5, tau = 10, d0 = 1e-8);
  record    the study recorder: the wrapped standard map K = 6, 4096 orbits x 1e5 steps, QRSpectrum(MGS), tau = 1,
            100 log-spaced grid rows;
  advance   advance_ensemble(KahanLi(8), Henon-Heiles, tau = 0.05): 1048576 starts on the E = 1/8 section x 1250
            steps, states only;
  indicators the indicator recorder's tangent kind: the chain FLI, MEGNO, SALI with the monitor on the wrapped
            standard map K = 6, 4096 orbits x 1e5 steps, tau = 1, 100 log-spaced grid rows.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ORBITS = 65536
N_STEPS = 100_000
TAU = 10
NU = KAPPA = 1.5
MU = 0.05
SEED = 1
# DRAM bytes per orbit of one launch of the mixed kernel: ncu DRAM read + write of split_frames_kernel on 65536
# orbits x 2000 steps (15.53 MB read, 1.48 MB written: the orbit, both frames and the records once in, once out)
TRAFFIC_PER_ORBIT = 17013504 / 65536
METRIC = "orbit-steps/s (4D coupled standard maps, QRSpectrum(Householder) + GALI_4 + SALI, mixed-precision kernel)"
# the headline kernel: Float64 orbit and GALI / SALI frame, Float32 QRSpectrum frame (the precision every output holds)
HEADLINE = "mixed-ind64"


# ---- algorithmic operation counts ---------------------------------------------------------------------------------
# The counting convention of the hot path's roofline: add, sub, mul = 1, fma = 2, div and sqrt = 1, compares and
# selects 0; the transcendentals (sin, cos, log) are counted apart, by kind and precision. The counts are the
# ALGORITHM's, the same for both kernels (the dense tangent product 2 d^2 k even where a kernel exploits the
# tangent's zeros), split by the precision each kernel computes them in. Per orbit-step of the workload above
# (d = k = 4, tau = 10, two frames: QR and GALI with SALI read off GALI's columns 1-2):
#   map: x' = x + p (2), x1' + x2' (1), _abc (5), forward (8) and the force sums (4): 20 flops + 3 sin + 3 cos
#   tangent products: 2 d^2 k = 128 per frame
#   per handoff: Householder QR 4 d k^2 = 256; window_Gw 2 k^3 / 3 + 2 k^2 = 74; orth_loss (the k (k + 1) / 2
#   distinct dots of Q'Q) 2 d k (k + 1) / 2 = 80; GALI: column norms 2 d k and unit columns d k = 48 (these decide
#   the stop and carry the frame); k + k logs with a Neumaier add (4 flops) each: 32 (Float64 in both kernels)
#   once per run: GALI's values, the twice-orthogonalised Gram-Schmidt 2 sum_j j 4 d = 192, the nested norms 2 d k
#   and scaling d k, the k - 1 products, and SALI 3 d 2 = 24: 267. A handoff's values are overwritten by the next
#   one and read only after the last (gali.jl:156, sali.jl:108), so the algorithm needs them once; the mixed kernel
#   forms them once a launch, the Float64 kernel (the reference's loop, bit for bit) at every handoff
def flops_per_orbit_step(tau: int = TAU, precision: str = "fp64", n_steps: int = N_STEPS) -> dict:
    d, k = 4, 4
    map_flops, trig = 20, 6
    product = 2 * d * d * k
    qr = 4 * d * k * k + (2 * k ** 3 // 3 + 2 * k * k) + d * k * (k + 1)        # Householder, window_Gw, orth_loss
    gali = 2 * d * k + d * k                                                      # norms and unit columns
    values = 2 * sum(j * 4 * d for j in range(k)) + 2 * d * k + d * k + (k - 1) + 6 * d   # GALI's values + SALI
    logsum = k * 4                                                                # per frame: k Neumaier adds
    out = dict(trig_fp64=trig, trig_fp32=0.0, log=2 * k / tau, handoff_flops=qr + gali + 2 * logsum,
               values_flops_per_run=values)
    if precision == "mixed":   # both frames Float32; the orbit, its trigonometry and the log sums Float64
        out.update(fp64=map_flops + 2 * logsum / tau, fp32=2 * product + (qr + gali) / tau + values / n_steps,
                   trig_fp64=trig / 2, trig_fp32=trig / 2)
    elif precision == "mixed-ind64":   # the QR frame Float32; the orbit and the GALI / SALI frame Float64
        out.update(fp64=map_flops + product + (gali + 2 * logsum) / tau + values / n_steps, fp32=product + qr / tau)
    else:
        out.update(fp64=map_flops + 2 * product + (qr + gali + 2 * logsum) / tau + values / n_steps, fp32=0.0)
    return out


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region (200 ms period)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
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
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=mx, reasons=sorted(reasons),
                    samples=len(sm))


def cpu_reference(sample_orbits: int, sample_steps: int, threads: int) -> dict:
    """The oracle (serial C++ restatement of the reference's propagate) on the host cores: orbit-steps/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    from chaos_b200 import FroeschleMap, GALI, HouseholderQR, QRSpectrum, SALI
    from chaos_b200.propagate import FrameSpec
    x0 = np.random.default_rng(SEED).uniform(0, 2 * np.pi, (sample_orbits, 4))
    W0 = np.broadcast_to(np.eye(4), (sample_orbits, 4, 4)).copy()
    frames = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0), FrameSpec(4, (GALI(), SALI()), W0)]
    t = time.perf_counter()
    O.oracle_frames(FroeschleMap(NU, KAPPA, MU), x0, sample_steps, frames, tau=TAU, math="portable", threads=threads,
                    engine="static")
    dt = time.perf_counter() - t
    return dict(value=sample_orbits * sample_steps / dt, seconds=dt, threads=threads)


# The CPU sample of the workload: its first CPU_ORBITS orbits for CPU_STEPS steps (same map, frames, tau and W0), on
# the statically sized oracle (the reference's algorithm specialised on d = k = 4 as StaticArrays specialises it).
CPU_ORBITS, CPU_STEPS = 2048, 20000
CPU_SAMPLE = (f"{CPU_ORBITS} orbits x {CPU_STEPS} steps of the workload (the statically sized oracle, d = k = 4 "
              "compile-time, all host threads; Julia, the reference's runtime, is absent)")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--orbits", type=int, default=None, help="orbits per GPU (default: the workload's own)")
    ap.add_argument("--N", type=int, default=N_STEPS)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--only", choices=["fp64", "mixed", "mixed-ind64"], default=None,
                    help="time one kernel of the default workload and print a short line (a small case for ncu)")
    ap.add_argument("--workload", default="coupled", choices=["coupled", "standard", "gauss", "lattice", "screen", "mlp", "split", "shadow",
                                                             "record", "indicators", "advance", "torus", "record_mixed",
                                                             "coop"])
    args = ap.parse_args()
    if args.workload != "coupled":
        run_workload(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        # a bounded sample of the same workload per step
        so, ss = CPU_ORBITS, CPU_STEPS
        vals = []
        for i in range(args.warmup + args.steps):
            r = cpu_reference(so, ss, threads)
            if i >= args.warmup:
                vals.append(r["value"])
        v = float(np.median(vals))
        line = dict(metric=METRIC, value=v, unit="orbit-steps/s", n_gpus=args.gpus, steps=args.steps,
                    warmup=args.warmup, ms_per_step=so * ss / v * 1e3, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="f64", data="synthetic", impl="reference",
                    config=dict(workload="froeschle-4d-65536x1e5-tau10-qr-householder+gali4+sali", orbits=args.orbits or N_ORBITS,
                                N=args.N, tau=TAU),
                    cpu_baseline=dict(value=v, unit="orbit-steps/s", cores=threads, kind="port", sample=CPU_SAMPLE),
                    e2e=dict(value=v, unit="orbit-steps/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
        print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist

    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        # a short timeout: a rank that waits for a lost peer ends with an error instead of hanging
        dist.init_process_group("nccl", device_id=torch.device("cuda", local), timeout=datetime.timedelta(seconds=180))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    from chaos_b200 import _abi
    from chaos_b200 import FroeschleMap, GALI, HouseholderQR, QRSpectrum, SALI
    from chaos_b200._lib import last_error, lib
    from chaos_b200.propagate import FrameSpec, build_run
    L = lib()

    n, N = args.orbits or N_ORBITS, args.N
    sysm = FroeschleMap(NU, KAPPA, MU)
    # each rank its own shard of the same size (weak scaling): orbit ids rank*n+1 .. (rank+1)*n
    rng = np.random.default_rng(SEED + rank)
    x0_h = rng.uniform(0, 2 * np.pi, (n, 4))
    frames_spec = [FrameSpec(4, (QRSpectrum(HouseholderQR()),)), FrameSpec(4, (GALI(), SALI()))]

    def make_bufs():
        x0 = torch.tensor(x0_h.T.copy(), device=dev)                 # SoA (4, n)
        eye = torch.zeros((16, n), dtype=torch.float64, device=dev)
        eye[[0, 5, 10, 15]] = 1.0
        b = dict(x0=x0, x=torch.empty_like(x0), W0=eye, W=[torch.empty((16, n), dtype=torch.float64, device=dev) for _ in range(2)],
                 st=[], code=[torch.empty(n, dtype=torch.int8, device=dev) for _ in range(2)],
                 hstep=[torch.empty(n, dtype=torch.int64, device=dev) for _ in range(2)])
        return b

    bufs = make_bufs()

    def run_for(precision: str):
        r = build_run(sysm, N, TAU, frames_spec, precision, SEED, orbit_base=rank * n)
        sb = [L.cl_b200_state_bytes(C.byref(r), f) for f in range(2)]
        if not bufs["st"]:
            bufs["st"] = [torch.empty(n * s // 8, dtype=torch.int64, device=dev) for s in sb]
        cb = _abi.cl_buffers()
        cb.x0 = bufs["x0"].data_ptr()
        cb.x = bufs["x"].data_ptr()
        for f in range(2):
            cb.W0[f] = bufs["W0"].data_ptr()
            cb.W[f] = bufs["W"][f].data_ptr()
            cb.states[f] = bufs["st"][f].data_ptr()
            cb.code[f] = bufs["code"][f].data_ptr()
            cb.hstep[f] = bufs["hstep"][f].data_ptr()
        return r, cb

    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # 256 MB > L2

    tuned = {}

    def timed(precision: str, steps: int, warmup: int, sampler=None):
        r, cb = run_for(precision)
        # the autotuner picks the register budget (resident blocks per SM) of this instance on a 2000-step sample
        mb = C.c_int32(0)
        rc = L.cl_b200_tune(C.byref(r), n, C.byref(cb), 1, 2000, C.c_void_p(stream.cuda_stream), C.byref(mb))
        if rc != 0:
            raise RuntimeError(f"cl_b200_tune: {rc} {last_error()}")
        tuned[precision] = int(mb.value)
        for _ in range(warmup):
            rc = L.cl_b200_propagate_device(C.byref(r), n, C.byref(cb), 1, C.c_void_p(stream.cuda_stream))
            if rc != 0:
                raise RuntimeError(f"cl_b200_propagate_device: {rc} {last_error()}")
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        ms = []
        launches0 = L.cl_b200_launch_count()
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            for _ in range(steps):
                flush.fill_(1.0)   # flush L2 between timed iterations (outside the events)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rc = L.cl_b200_propagate_device(C.byref(r), n, C.byref(cb), 1, C.c_void_p(stream.cuda_stream))
                e1.record(stream)
                if rc != 0:
                    raise RuntimeError(f"cl_b200_propagate_device: {rc} {last_error()}")
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize(dev)
        launches = L.cl_b200_launch_count() - launches0
        t = torch.tensor([sum(ms)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.barrier()
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), ms, launches

    from types import SimpleNamespace
    from chaos_b200.reducers import chain_dtype

    def records():
        """Both frames' records on the host (Julia-layout states, status, step) for the error report."""
        out = []
        for f, fs in enumerate(frames_spec):
            dt = chain_dtype(fs.reducers, 4, fs.k)
            st = np.frombuffer(bufs["st"][f].cpu().numpy().tobytes(), dtype=dt).copy()
            out.append(SimpleNamespace(states=st, code=bufs["code"][f].cpu().numpy().copy(),
                                       hstep=bufs["hstep"][f].cpu().numpy().copy(), reducers=fs.reducers))
        return out

    # plain Float64 kernel (the reference's arithmetic), then the mixed kernel
    if args.only:
        tk, msk, launches = timed(args.only, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps(dict(metric=METRIC, kernel=args.only, value=n * N * world * args.steps / (tk / 1e3),
                                  unit="orbit-steps/s", ms_per_step=tk / args.steps, orbits=n, N=N,
                                  tuned_blocks_per_sm=tuned, gpu_launches=int(launches))), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    from chaos_b200.diagnostics import precision_errors
    t64, ms64, _ = timed("fp64", args.steps, args.warmup)
    rec64 = records()
    sampler = ClockSampler(dev.index if world == 1 else local)
    tmx, msmx, launches = timed(HEADLINE, args.steps, args.warmup, sampler)
    recmx = records()
    errs = precision_errors(rec64, recmx, N)
    dl1 = errs[0]["dlambda_max"][0]
    # the all-Float32-frames kernel beside it, with its errors (its GALI / SALI do not hold: see the design notes)
    t32, ms32, _ = timed("mixed", max(1, args.steps // 4), 1)
    errs32 = precision_errors(rec64, records(), N)

    work = n * N * world
    value = work * args.steps / (tmx / 1e3)
    value64 = work * args.steps / (t64 / 1e3)

    # e2e: the C ABI with host buffers (copies in and out inside the timed region)
    from chaos_b200.propagate import propagate_frames
    W0h = np.broadcast_to(np.eye(4), (n, 4, 4)).copy()
    fr_h = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0h), FrameSpec(4, (GALI(), SALI()), W0h)]
    propagate_frames(sysm, x0_h, N, fr_h, tau=TAU, seed=SEED, precision=HEADLINE, finals=True, throw=False)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    # at least five calls; the median call time stands for a call (a host hiccup in one of a few calls -- page
    # faults, another process on the host cores -- moved the mean by up to 20 %), the mean is reported beside it
    te = []
    for _ in range(max(args.steps, 5)):
        t0 = time.perf_counter()
        res = propagate_frames(sysm, x0_h, N, fr_h, tau=TAU, seed=SEED, precision=HEADLINE, finals=True, throw=False)
        te.append(time.perf_counter() - t0)
    tt = torch.tensor([float(np.median(te)), float(np.mean(te))], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    e2e_value = work / float(tt[0].item())
    e2e_mean_value = work / float(tt[1].item())
    h2d = x0_h.nbytes + 2 * W0h.nbytes
    d2h = res[0].x.nbytes + sum(r_.W.nbytes + r_.states.nbytes + r_.code.nbytes + r_.hstep.nbytes for r_ in res)

    fp64_peak = _dgemm_peak(torch, dev)

    fl = flops_per_orbit_step(TAU, HEADLINE, N)
    fl64 = flops_per_orbit_step(TAU, "fp64", N)
    per_launch_ms = float(np.mean(msmx))
    # FP64-pipe equivalent: a Float32 op takes half an FP64 issue slot on B200 (FP32 rate = 2 x FP64 rate)
    achieved = n * N * (fl["fp64"] + fl["fp32"] / 2) / (per_launch_ms / 1e3) / 1e12
    achieved64 = n * N * fl64["fp64"] / (float(np.mean(ms64)) / 1e3) / 1e12

    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cb_ = cpu_reference(CPU_ORBITS, CPU_STEPS, threads)
        cpu = dict(value=cb_["value"], unit="orbit-steps/s", cores=threads, kind="port", sample=CPU_SAMPLE)

    if rank == 0:
        clocks = sampler.summary()
        line = dict(
            metric=METRIC, value=value, unit="orbit-steps/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
            ms_per_step=tmx / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
            dtype="f64 orbit + f64 GALI/SALI frame + f32 QR frame", data="synthetic",
            config=dict(workload="froeschle-4d-65536x1e5-tau10-qr-householder+gali4+sali", orbits_per_gpu=n, N=N,
                        tau=TAU, frames="QRSpectrum(HouseholderQR) k=4 | GALI_4+SALI k=4", W0="I",
                        l2="flushed between timed steps (256 MB write)", parallelism=f"dp{world} (orbit shards)",
                        tuned_blocks_per_sm=tuned),
            fp64_kernel=dict(value=value64, ms_per_step=t64 / args.steps, mixed_over_fp64=value / value64,
                             max_abs_dlambda1=dl1, roofline_tflops=achieved64, frac_of_fp64_peak=achieved64 / fp64_peak),
            mixed_errors=dict(against="the Float64 kernel (bit for bit the oracle) on the same orbits", qr_frame=errs[0],
                              gali_sali_frame=errs[1]),
            fp32_frames_kernel=dict(value=work * max(1, args.steps // 4) / (t32 / 1e3), errors=errs32,
                                    note="both frames Float32: lambda holds, GALI / SALI do not"),
            e2e=dict(value=e2e_value, unit="orbit-steps/s", h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(d2h),
                     calls=len(te), statistic="median call", mean_call_value=e2e_mean_value),
            roofline=dict(bound="fp64", achieved=achieved, peak=fp64_peak, unit="TFLOP/s", frac=achieved / fp64_peak,
                          traffic=TRAFFIC_PER_ORBIT * n,
                          traffic_source="ncu dram__bytes_read + dram__bytes_write of split_frames_kernel on 65536 "
                                         "orbits x 2000 steps (1.701e7 B), scaled by orbits: DRAM bytes grow with the "
                                         "orbits loaded and stored, not with the steps",
                          peak_source="cuBLAS DGEMM 8192^3 measured here (burst)",
                          flops_per_orbit_step=fl,
                          pipes_ncu=dict(fp64=0.448, fma_fp32=0.140, alu=0.234, xu_sfu=0.171, issue_active=0.632,
                                         warps_active=0.171,
                                         source="ncu --set full of split_frames_kernel, 65536 orbits x 2000 steps "
                                                "(profiles/split_frames_kernel_froeschle_65536x2000_ncu.md)")),
            cpu_baseline=cpu, clocks=clocks, gpu_launches=int(launches),
        )
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()

# ---- the other measured configurations (--workload) --------------------------------------------------------------
def _setup():
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    from chaos_b200._lib import lib
    return torch, dev, lib()


def _device_frames(torch, dev, L, sysm, x0_h, N, tau, frames, precision, seed=SEED):
    """SoA device buffers for propagate_device: x0 (s, n), each frame's W0 = I[:, 1:k] as (d k, n), states, codes."""
    from chaos_b200 import _abi
    from chaos_b200.propagate import build_run
    n = len(x0_h)
    r = build_run(sysm, N, tau, frames, precision, seed)
    b = dict(x0=torch.tensor(np.ascontiguousarray(x0_h.T), device=dev))
    b["x"] = torch.empty_like(b["x0"])
    cb = _abi.cl_buffers()
    cb.x0, cb.x = b["x0"].data_ptr(), b["x"].data_ptr()
    d = sysm.d
    for f, fr in enumerate(frames):
        W0 = torch.zeros((d * fr.k, n), dtype=torch.float64, device=dev)
        for j in range(fr.k):
            W0[j * d + j] = 1.0
        sb = L.cl_b200_state_bytes(C.byref(r), f)
        b[f"W0{f}"], b[f"W{f}"] = W0, torch.empty_like(W0)
        b[f"st{f}"] = torch.zeros(max(1, n * sb // 8), dtype=torch.int64, device=dev)
        b[f"code{f}"] = torch.zeros(n, dtype=torch.int8, device=dev)
        b[f"hs{f}"] = torch.zeros(n, dtype=torch.int64, device=dev)
        cb.W0[f], cb.W[f] = W0.data_ptr(), b[f"W{f}"].data_ptr()
        cb.states[f] = b[f"st{f}"].data_ptr() if sb else None
        cb.code[f], cb.hstep[f] = b[f"code{f}"].data_ptr(), b[f"hs{f}"].data_ptr()
    return r, cb, b


def _event_times(torch, dev, stream, fn, steps, warmup, flush, sampler=None):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(dev)
    ms = []
    with (sampler if sampler is not None else _Null()):
        for _ in range(steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    return ms


def _line(metric, value, unit, args, ms, config, **extra):
    out = dict(metric=metric, value=value, unit=unit, n_gpus=1, steps=len(ms), warmup=args.warmup,
               ms_per_step=float(np.mean(ms)) if ms else None, higher_is_better=True, scaling="weak",
               vs_baseline=None, data="synthetic", config=config)
    out.update(extra)
    print(json.dumps(out), flush=True)


def _propagate_workload(args, name, sysm, x0_h, N, tau, frames, unit_name, cpu_fn, config):
    """A plain / mixed pair of propagate_device timings (value = the mixed kernel when compiled, else FP64)."""
    torch, dev, L = _setup()
    from chaos_b200._lib import last_error
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    n = len(x0_h)
    res = {}
    launches = 0
    sampler = ClockSampler(0)
    from chaos_b200.propagate import build_run
    precs = [p for p in ("fp64", "mixed") if L.cl_b200_check(C.byref(build_run(sysm, N, tau, frames, p, SEED))) == 0]
    for prec in precs:
        r, cb, b = _device_frames(torch, dev, L, sysm, x0_h, N, tau, frames, prec)
        mb = C.c_int32(0)
        rc = L.cl_b200_tune(C.byref(r), n, C.byref(cb), 1, min(N, 2000), C.c_void_p(stream.cuda_stream), C.byref(mb))
        if rc != 0:
            raise RuntimeError(f"cl_b200_tune: {rc} {last_error()}")

        def go():
            rc_ = L.cl_b200_propagate_device(C.byref(r), n, C.byref(cb), 1, C.c_void_p(stream.cuda_stream))
            if rc_ != 0:
                raise RuntimeError(f"cl_b200_propagate_device: {rc_} {last_error()}")
        l0 = L.cl_b200_launch_count()
        ms = _event_times(torch, dev, stream, go, args.steps, args.warmup, flush, sampler if prec == precs[-1] else None)
        launches = L.cl_b200_launch_count() - l0 - args.warmup
        st = b["st0"].view(torch.float64).reshape(n, -1).cpu().numpy()
        res[prec] = dict(ms=ms, value=n * N / (np.mean(ms) / 1e3), minb=int(mb.value), st=st,
                         code=b["code0"].cpu().numpy())
    head = res.get("mixed", res["fp64"])
    extra = dict(fp64_kernel=dict(value=res["fp64"]["value"], ms_per_step=float(np.mean(res["fp64"]["ms"]))))
    if "mixed" in res:
        extra["fp64_kernel"]["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    cpu = None if args.no_cpu else cpu_fn()
    config = dict(config, tuned_blocks_per_sm={k: v["minb"] for k, v in res.items()},
                  l2="flushed between timed steps (256 MB write)")
    _line(f"{unit_name}/s ({name})", head["value"], f"{unit_name}/s", args, head["ms"], config,
          dtype="f64 orbit + f32 frames" if "mixed" in res else "f64", cpu_baseline=cpu, clocks=sampler.summary(),
          gpu_launches=int(launches), **extra)
    return res


def _cpu_port(sysm, x0, N, tau, frames, unit, sample):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    O.oracle_frames(sysm, x0, N, frames, tau=tau, math="portable", threads=threads)
    dt = time.perf_counter() - t
    return dict(value=len(x0) * N / dt, unit=unit, cores=threads, kind="port", sample=sample)


def workload_standard(args):
    from chaos_b200 import MGS, QRSpectrum, WrappedStandardMap, torus_state
    from chaos_b200.propagate import FrameSpec
    n, N = 4096, 100_000
    xp = np.random.default_rng(SEED).uniform(0, 2 * np.pi, (n, 2))
    x0 = np.array([torus_state(z) for z in xp])
    sysm = WrappedStandardMap(6.0)
    frames = [FrameSpec(2, (QRSpectrum(MGS()),))]

    def cpu():
        W0 = np.broadcast_to(np.eye(2), (512, 2, 2)).copy()
        return _cpu_port(sysm, x0[:512], 20_000, 1, [FrameSpec(2, (QRSpectrum(MGS()),), W0)], "orbit-steps/s",
                         "512 orbits x 20000 steps of the workload (oracle, all host threads)")
    res = _propagate_workload(args, "Chirikov standard map K=6 mod 2pi, QRSpectrum(MGS) k=2 tau=1", sysm, x0, N, 1,
                              frames, "orbit-steps", cpu,
                              dict(workload="standard-map-k6-4096x1e5-tau1-mgs", orbits=n, N=N, tau=1, W0="I"))
    st = res["fp64"]["st"]
    lam = (st[:, 0:4:2] + st[:, 1:4:2]) / st[:, [4]].view(np.int64)
    print(json.dumps(dict(check="sum of the two exponents", max_abs=float(np.max(np.abs(lam.sum(axis=1)))))),
          file=sys.stderr)


def workload_gauss(args):
    from chaos_b200 import FLI, MEGNO, Gauss, GivensQR, HenonHeilesFlow, IntegratorMap, QRSpectrum, random_energy_starts
    from chaos_b200.propagate import FrameSpec
    n = 16384
    N = args.N if args.N != N_STEPS else 1_000_000
    x0 = random_energy_starts(1 / 8, n, seed=SEED)
    sysm = IntegratorMap(Gauss(3, tol=1e-14), HenonHeilesFlow(), 0.01)
    chain = (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR()))
    frames = [FrameSpec(2, chain)]

    def cpu():
        W0 = np.broadcast_to(np.eye(4)[:, :2], (256, 4, 2)).copy()
        return _cpu_port(sysm, x0[:256], 2000, 10, [FrameSpec(2, chain, W0)], "gauss-steps/s",
                         "256 orbits x 2000 Gauss steps of the workload (oracle, all host threads)")
    _propagate_workload(args, "Henon-Heiles E=1/8, Gauss-3 tol 1e-14 dt 0.01, MEGNO+FLI+QRSpectrum(Givens) k=2 "
                        "tau=10", sysm, x0, N, 10, frames, "gauss-steps", cpu,
                        dict(workload=f"henon-heiles-gauss3-16384x{N:.0e}-tau10", orbits=n, N=N, tau=10, W0="I[:, 1:2]"))


def workload_split(args):
    from chaos_b200 import FLI, MEGNO, GivensQR, HenonHeilesFlow, IntegratorMap, KahanLi, QRSpectrum, random_energy_starts
    from chaos_b200.propagate import FrameSpec
    n = 16384
    N = args.N if args.N != N_STEPS else 200_000
    x0 = random_energy_starts(1 / 8, n, seed=SEED)
    sysm = IntegratorMap(KahanLi(8), HenonHeilesFlow(), 0.05)
    chain = (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR()))

    def cpu():
        W0 = np.broadcast_to(np.eye(4)[:, :2], (256, 4, 2)).copy()
        return _cpu_port(sysm, x0[:256], 4000, 10, [FrameSpec(2, chain, W0)], "steps/s",
                         "256 orbits x 4000 KahanLi-8 steps of the workload (oracle, all host threads)")
    _propagate_workload(args, "Henon-Heiles E=1/8, KahanLi(8) splitting dt 0.05, MEGNO+FLI+QRSpectrum(Givens) k=2 "
                        "tau=10", sysm, x0, N, 10, [FrameSpec(2, chain)], "steps", cpu,
                        dict(workload=f"henon-heiles-kahanli8-16384x{N:.0e}-tau10", orbits=n, N=N, tau=10,
                             W0="I[:, 1:2]", stages=18))


def workload_lattice(args):
    torch, dev, L = _setup()
    from chaos_b200._lib import last_error
    from chaos_b200.ensemble import DeviceClass, device_classes_array, lattice_workload
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    n_total = args.orbits or 1 << 20
    classes = lattice_workload(n_total, seed=SEED, precision="mixed")
    dcs = [DeviceClass(c, torch, dev) for c in classes]
    tuned = []
    for dc in dcs:
        # every queue slot, lengths scaled to 1 % (the longest orbit keeps its share of the class's time)
        rc = L.cl_b200_ensemble_tune(C.byref(dc.cls), 0, max(dc.c.tau, dc.c.N // 100), C.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"cl_b200_ensemble_tune: {rc} {last_error()}")
        tuned.append(dict(d=dc.c.sys.d, blocks_per_sm=int(dc.cls.minb), tau_unroll=int(dc.cls.unroll),
                          lanes_per_orbit=int(dc.cls.lanes)))
    arr = device_classes_array(dcs)
    g = C.c_void_p()
    if L.cl_b200_ensemble_graph_create(arr, len(dcs), C.byref(g)) != 0:
        raise RuntimeError(last_error())
    sampler = ClockSampler(0)
    try:
        def go():
            if L.cl_b200_ensemble_graph_launch(g, C.c_void_p(stream.cuda_stream)) != 0:
                raise RuntimeError(last_error())
        ms = _event_times(torch, dev, stream, go, args.steps, args.warmup, flush, sampler)
    finally:
        L.cl_b200_ensemble_graph_destroy(g)
    executed, escaped, per_d = 0, 0, {}
    for dc in dcs:
        code = dc.t["code"].cpu().numpy()
        hs = dc.t["hs"].cpu().numpy()
        steps = np.where(code != 0, hs, dc.c.lengths)
        executed += int(steps.sum())
        escaped += int((code == 4).sum())
        per_d[str(dc.c.sys.d)] = int(steps.sum())
    value = executed / (np.mean(ms) / 1e3)
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        threads = os.cpu_count() or 1
        m, work, t = 24, 0, 0.0
        for c in classes:
            W0 = c.frame.W0[:m]
            from chaos_b200.propagate import FrameSpec
            t0 = time.perf_counter()
            r = O.oracle_ensemble(c.sys, c.x0[:m], c.N, FrameSpec(c.frame.k, c.frame.reducers, W0), tau=c.tau,
                                  K=c.K[:m], lengths=c.lengths[:m], escape=c.escape, threads=threads)
            t += time.perf_counter() - t0
            work += int(np.where(r["code"] != 0, r["hstep"], c.lengths[:m]).sum())
        cpu = dict(value=work / t, unit="orbit-steps/s", cores=threads, kind="port",
                   sample=f"the first {m} orbits of each d class ({work:.3g} executed orbit-steps; oracle, FP64, all host threads)")
    _line("executed orbit-steps/s (uneven lattice ensemble, one CUDA graph of persistent work-queue kernels)", value,
          "orbit-steps/s", args, ms,
          dict(workload=f"lattice-ensemble-{n_total}-d2/4/8/16-N1e3..1e6-escape1e3", orbits=n_total,
               executed_orbit_steps=executed, escaped=escaped, executed_by_d=per_d, tuned=tuned,
               l2="flushed between timed steps (256 MB write)"),
          dtype="f64 orbit + f32 frames", cpu_baseline=cpu, clocks=sampler.summary(),
          gpu_launches=len(dcs) * len(ms))


def workload_screen(args):
    torch, dev, L = _setup()
    from chaos_b200.screen import FEATURE_STEPS, N_FULL, Screen
    G = int(os.environ.get("SCREEN_GRID", "2048"))
    n_train = int(os.environ.get("SCREEN_TRAIN", "200000"))
    sc = Screen(torch, dev)
    t0 = time.perf_counter()
    X, label, lam = sc.training_set(n_train, N=N_FULL)
    torch.cuda.synchronize(dev)
    t_label = time.perf_counter() - t0
    t0 = time.perf_counter()
    net, info = sc.train(X, label, lam, epochs=12, batch=4096)
    torch.cuda.synchronize(dev)
    t_train = time.perf_counter() - t0
    # warm-up of both paths on a small grid, then one timed run each on the full grid
    sc.screen_grid(net, 128, N=N_FULL)
    sc.full_grid(128, N=N_FULL)
    sampler = ClockSampler(0)
    l0 = L.cl_b200_launch_count()
    with sampler:
        res = sc.screen_grid(net, G, N=N_FULL)
    launches = L.cl_b200_launch_count() - l0
    plain, t_full = sc.full_grid(G, N=N_FULL)
    mis = float((res["labels"] != plain).mean())
    value = res["n"] / res["seconds"]
    base = res["n"] / t_full
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        from chaos_b200.propagate import FrameSpec
        m = 48
        rng = np.random.default_rng(SEED)
        x0 = np.stack([rng.uniform(0, 2 * np.pi, m), np.full(m, 0.1), rng.uniform(0, 2 * np.pi, m),
                       np.full(m, 0.1)], axis=1)
        W0 = np.broadcast_to(np.eye(4)[:, :2], (m, 4, 2)).copy()
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        O.oracle_frames(sc.sys, x0, N_FULL, [FrameSpec(2, sc.frame.reducers, W0)], tau=10, threads=threads)
        cpu = dict(value=m / (time.perf_counter() - t0), unit="orbits/s", cores=threads, kind="port",
                   sample=f"{m} grid orbits classified by full FP64 integration to N = 1e5 (oracle, all host threads)")
    _line("screened orbits/s (learned BF16 MLP screen, 4D coupled-map grid, label final MEGNO > 2.2)", value,
          "orbits/s", args, [res["seconds"] * 1e3],
          dict(workload=f"screen-froeschle-grid{G}x{G}-N1e5", grid=G, N=N_FULL, feature_steps=FEATURE_STEPS,
               training_orbits=n_train, audit=0.05, band=[0.05, 0.95], regular_fraction_in_training_draws=0.1),
          dtype="bf16 mlp (f32 accumulate) + f64/f32 orbits", e2e=dict(value=value, unit="orbits/s",
                                                                       h2d_bytes_per_step=int(res["n"] * 32),
                                                                       d2h_bytes_per_step=int(res["n"] * 64)),
          plain_full_integration=dict(value=base, seconds=t_full), speedup_over_full=value / base,
          misclassification_whole_grid=mis, audit_misclassification=res["audit_misclassification"],
          unsure=res["unsure"], audited=res["audited"], chaotic_fraction=float(plain.mean()),
          orbit_steps_screen=res["orbit_steps"], orbit_steps_full=res["full_orbit_steps"],
          training=dict(label_seconds=t_label, train_seconds=t_train, **{k: v for k, v in info.items() if k != "loss"},
                        final_loss=info["loss"][-1], positives=float(np.mean(label))),
          cpu_baseline=cpu, clocks=sampler.summary(), gpu_launches=int(launches))

def workload_mlp(args):
    """The learned screen's network on the tensor cores at a batch of 262144 rows: inference as one fused persistent
    kernel (the headline), inference layer by layer (4 GEMMs with bias / GELU epilogues), and one training step
    (forward, loss, backward GEMMs, Adam)."""
    torch, dev, L = _setup()
    from chaos_b200.mlp import DIMS, MLP, OUT_PAD
    B = args.orbits or 262144
    net = MLP(torch, dev, seed=0)
    rng = np.random.default_rng(SEED)
    for lay in net.layers:   # nonzero biases, as after training
        lay["b"].copy_(torch.tensor(rng.standard_normal(lay["b"].numel()).astype(np.float32) * 0.1, device=dev))
    X = torch.tensor(rng.standard_normal((B, 64)).astype(np.float32), device=dev).to(torch.bfloat16)
    label = torch.tensor((rng.random(B) < 0.5).astype(np.float32), device=dev)
    target = torch.tensor(rng.standard_normal(B).astype(np.float32), device=dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # algorithmic FLOPs of one forward: 2 B (64*256 + 256*256 + 256*256 + 256*16), the last layer padded to 16
    # outputs as the kernel computes it; a training step adds the weight-gradient GEMM of every layer and the
    # input-gradient GEMM of every layer but the first
    fin = list(DIMS[:-1])
    fout = [DIMS[1], DIMS[2], DIMS[3], OUT_PAD]
    fwd = sum(2 * B * a * b for a, b in zip(fin, fout))
    bwd = sum(2 * B * a * b for a, b in zip(fin, fout)) + sum(2 * B * a * b for a, b in zip(fin[1:], fout[1:]))
    out = torch.empty((B, OUT_PAD), dtype=torch.float32, device=dev)
    net.packed()
    sampler = ClockSampler(0)
    l0 = L.cl_b200_launch_count()
    ms_fused = _event_times(torch, dev, stream, lambda: net.forward_fused(X, out=out), args.steps, args.warmup, flush,
                            sampler)
    n_fwd = (L.cl_b200_launch_count() - l0) // (args.steps + args.warmup) * args.steps   # timed launches only
    ms_layer = _event_times(torch, dev, stream, lambda: net.forward(X), args.steps, args.warmup, flush)
    same = bool(torch.equal(net.forward_fused(X), net.forward(X)))
    ms_train = _event_times(torch, dev, stream, lambda: net.train_step(X, label, target), args.steps, args.warmup,
                            flush)
    # end to end: the rows' features from pinned host memory, the outputs back to it (the public host-data call:
    # chunks of 65536 rows over two streams, copies overlapping the passes)
    Xh = X.cpu().pin_memory()
    oh = torch.empty((B, OUT_PAD), dtype=torch.float32).pin_memory()
    ms_e2e = _event_times(torch, dev, stream, lambda: net.forward_fused_host(Xh, oh), args.steps, args.warmup, flush)
    torch.cuda.synchronize(dev)
    host_same = bool(torch.equal(oh, net.forward_fused(X).cpu()))   # the same weights (after the training step)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("bf16_tflops", 1590.0)
    achieved = fwd / (np.mean(ms_fused) / 1e3) / 1e12
    layered = fwd / (np.mean(ms_layer) / 1e3) / 1e12
    _line("screen-MLP inference rows/s (one fused persistent tcgen05 kernel, BF16 operands, FP32 accumulate)",
          B / (np.mean(ms_fused) / 1e3), "rows/s", args, ms_fused,
          dict(workload=f"mlp-64x256x256x256x2-batch{B}", batch=B, layers=list(DIMS),
               l2="flushed between timed steps (256 MB write)"),
          dtype="bf16 (f32 accumulate)",
          e2e=dict(value=B / (np.mean(ms_e2e) / 1e3), unit="rows/s", h2d_bytes_per_step=int(B * 64 * 2),
                   d2h_bytes_per_step=int(B * OUT_PAD * 4), outputs_equal_device_pass=host_same),
          roofline=dict(bound="tensor", achieved=achieved, peak=peak, unit="TFLOP/s", frac=achieved / peak,
                        traffic=None, peak_source="MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback",
                        flops_per_row=fwd // B),
          layered=dict(ms=float(np.mean(ms_layer)), tflops=layered, frac=layered / peak, bitwise_equal_fused=same),
          training_step=dict(ms=float(np.mean(ms_train)), tflops=(fwd + bwd) / (np.mean(ms_train) / 1e3) / 1e12),
          clocks=sampler.summary(), gpu_launches=int(n_fwd))


def _dgemm_peak(torch, dev) -> float:
    """FP64 peak: cuBLAS DGEMM 8192^3 (the library FP64 rate on this GPU), best of three bursts, TFLOP/s."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.matmul(a, a)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(3):
        e0.record()
        torch.matmul(a, a)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a
    return 2 * 8192 ** 3 / (best / 1e3) / 1e12


def _host_call_workload(args, metric, unit, units_per_call, call, config, cpu, dtype="f64", roofline=None):
    """Steps of the public host entry point: `value` from the device events around its launches (inputs resident),
    `e2e` from the wall clock around the whole call (copies in and out included)."""
    torch, dev, L = _setup()
    sampler = ClockSampler(0)
    for _ in range(args.warmup):
        call()
    gpu, wall = [], []
    with sampler:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ms, h2d, d2h = call()
            wall.append(time.perf_counter() - t0)
            gpu.append(ms)
    l0 = L.cl_b200_launch_count()
    call()
    launches = L.cl_b200_launch_count() - l0
    value = units_per_call / (np.mean(gpu) / 1e3)
    e2e = units_per_call / np.mean(wall)
    extra = {} if roofline is None else dict(roofline=roofline(value, torch, dev))
    _line(metric, value, unit, args, gpu, config, dtype=dtype,
          e2e=dict(value=e2e, unit=unit, h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(d2h)),
          cpu_baseline=None if args.no_cpu else cpu(), clocks=sampler.summary(), gpu_launches=int(launches), **extra)


def workload_shadow(args):
    from chaos_b200 import FroeschleMap
    from chaos_b200.propagate import build_run, FrameSpec
    from chaos_b200.shadow import end_dtype
    import ctypes as C_
    from chaos_b200 import _abi
    torch, dev, L = _setup()
    n, N, tau, d0 = args.orbits or 65536, args.N if args.N != N_STEPS else 100_000, 10, 1e-8
    sysm = FroeschleMap(NU, KAPPA, MU)
    x0 = np.random.default_rng(SEED).uniform(0, 2 * np.pi, (n, 4))
    run = build_run(sysm, N, tau, [FrameSpec(1, ())], "fp64", SEED)

    def call():
        ends = np.zeros(n, dtype=end_dtype(4))
        prov = _abi.cl_prov()
        rc = L.cl_b200_shadow(C_.byref(run), n, x0.ctypes.data_as(C_.POINTER(C_.c_double)), None, ends.ctypes.data,
                              d0, C_.byref(prov))
        if rc != 0:
            raise RuntimeError(rc)
        return prov.gpu_ms, x0.nbytes, ends.nbytes

    def cpu():
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        threads = os.cpu_count() or 1
        t = time.perf_counter()
        O.oracle_shadow(sysm, x0[:1024], 4000, d0=d0, tau=tau, seed=SEED, threads=threads)
        return dict(value=1024 * 4000 / (time.perf_counter() - t), unit="orbit-steps/s", cores=threads, kind="port",
                    sample="1024 orbits x 4000 steps (oracle, all host threads)")
    _host_call_workload(args, "orbit-steps/s (two-trajectory estimator, 4D coupled standard maps, reference and "
                        "shadow orbits)", "orbit-steps/s", n * N, call,
                        dict(workload=f"shadow-froeschle-{n}x{N:.0e}-tau10-d0-1e-8", orbits=n, N=N, tau=tau, d0=d0),
                        cpu)


def workload_record(args, precision="fp64"):
    from chaos_b200 import MGS, QRSpectrum, WrappedStandardMap, torus_state
    from chaos_b200.propagate import build_run, FrameSpec
    import ctypes as C_
    from chaos_b200 import _abi
    torch, dev, L = _setup()
    n, N, tau = args.orbits or 4096, args.N if args.N != N_STEPS else 100_000, 1
    sysm = WrappedStandardMap(6.0)
    xp = np.random.default_rng(SEED).uniform(0, 2 * np.pi, (n, 2))
    x0 = np.array([torus_state(z) for z in xp])
    grid = np.unique(np.round(np.logspace(0, np.log10(N), 100)).astype(np.int64))
    run = build_run(sysm, N, tau, [FrameSpec(2, (QRSpectrum(MGS()),))], precision, SEED)
    ncol = L.cl_b200_record_columns(C_.byref(run))
    sb = L.cl_b200_record_state_bytes(C_.byref(run))

    def call():
        x = x0.copy()
        W = np.broadcast_to(np.eye(2), (n, 2, 2)).copy()
        st = np.zeros((n, sb), np.uint8)
        code = np.zeros(n, np.int8)
        hs = np.zeros(n, np.int64)
        R = np.zeros((n, len(grid), ncol))
        fail = np.zeros(n, np.int64)
        prov = _abi.cl_prov()
        rc = L.cl_b200_record(C_.byref(run), n, x.ctypes.data, W.ctypes.data, st.ctypes.data, code.ctypes.data,
                              hs.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data, fail.ctypes.data,
                              C_.byref(prov))
        if rc != 0:
            raise RuntimeError(rc)
        return prov.gpu_ms, x.nbytes + W.nbytes + grid.nbytes + R.nbytes, R.nbytes + x.nbytes + W.nbytes + st.nbytes

    def cpu():
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        threads = os.cpu_count() or 1
        g = grid[grid <= 20000]
        t = time.perf_counter()
        O.oracle_record(sysm, x0[:512], 20000, tau, QRSpectrum(MGS()), g, threads=threads)
        return dict(value=512 * 20000 / (time.perf_counter() - t), unit="orbit-steps/s", cores=threads, kind="port",
                    sample="512 orbits x 20000 steps with the grid rows up to 20000 (oracle, all host threads)")
    _host_call_workload(args, f"orbit-steps/s (study recorder, wrapped standard map K=6, QRSpectrum(MGS), 100 grid "
                        f"rows, {precision})", "orbit-steps/s", n * N, call,
                        dict(workload=f"record-wrapped-k6-{n}x{N:.0e}-tau1-mgs-{len(grid)}rows", orbits=n, N=N, tau=tau,
                             grid_rows=int(len(grid)), precision=precision), cpu,
                        dtype="f64" if precision == "fp64" else "f64 orbit + f32 frame")


def workload_indicators(args):
    from chaos_b200 import WrappedStandardMap, torus_state
    from chaos_b200.propagate import build_run, FrameSpec
    from chaos_b200.record import indicator_chain
    import ctypes as C_
    from chaos_b200 import _abi
    torch, dev, L = _setup()
    n, N, tau, ns = args.orbits or 4096, args.N if args.N != N_STEPS else 100_000, 1, 2
    members = ["FLI", "MEGNO", "SALI"]
    sysm = WrappedStandardMap(6.0)
    xp = np.random.default_rng(SEED).uniform(0, 2 * np.pi, (n, 2))
    x0 = np.array([torus_state(z) for z in xp])
    grid = np.unique(np.round(np.logspace(0, np.log10(N), 100)).astype(np.int64))
    run = build_run(sysm, N, tau, [FrameSpec(2, indicator_chain(members))], "fp64", SEED)
    ncol = L.cl_b200_indicator_columns(C_.byref(run), ns)
    sb = L.cl_b200_indicator_state_bytes(C_.byref(run))

    def call():
        x = x0.copy()
        W = np.broadcast_to(np.eye(2), (n, 2, 2)).copy()
        st = np.zeros((n, sb), np.uint8)
        code = np.zeros(n, np.int8)
        hs = np.zeros(n, np.int64)
        R = np.zeros((n, len(grid), ncol))
        fail = np.zeros(n, np.int64)
        prov = _abi.cl_prov()
        rc = L.cl_b200_indicator(C_.byref(run), n, ns, x.ctypes.data, W.ctypes.data, st.ctypes.data,
                                 code.ctypes.data, hs.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data,
                                 fail.ctypes.data, C_.byref(prov))
        if rc != 0:
            raise RuntimeError(rc)
        return prov.gpu_ms, x.nbytes + W.nbytes + grid.nbytes + R.nbytes, R.nbytes + x.nbytes + W.nbytes + st.nbytes

    def cpu():
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        threads = os.cpu_count() or 1
        g = grid[grid <= 20000]
        t = time.perf_counter()
        O.oracle_indicators(sysm, x0[:512], 20000, tau, members, g, ns=ns, threads=threads)
        return dict(value=512 * 20000 / (time.perf_counter() - t), unit="orbit-steps/s", cores=threads, kind="port",
                    sample="512 orbits x 20000 steps with the grid rows up to 20000 (oracle, all host threads)")
    _host_call_workload(args, "orbit-steps/s (indicator recorder, tangent kind, chain FLI, MEGNO, SALI + monitor, "
                        "wrapped standard map K=6, 100 grid rows)", "orbit-steps/s", n * N, call,
                        dict(workload=f"indicators-wrapped-k6-{n}x{N:.0e}-tau1-fli-megno-sali-{len(grid)}rows",
                             orbits=n, N=N, tau=tau, grid_rows=int(len(grid))), cpu)


def workload_advance(args):
    from chaos_b200 import HenonHeilesFlow, KahanLi, _abi
    from chaos_b200.systems import IntegratorMap, random_energy_starts
    import ctypes as C_
    torch, dev, L = _setup()
    n = args.orbits or 1_048_576
    N, tau = args.N if args.N != N_STEPS else max(1, 1_310_720_000 // n), 0.05
    m, flow = KahanLi(8), HenonHeilesFlow()
    x0 = np.ascontiguousarray(random_energy_starts(0.125, n, SEED))
    cs = IntegratorMap(m, flow, tau).to_cl()

    def call():
        out = np.empty_like(x0)
        ok = np.zeros(n, np.uint8)
        prov = _abi.cl_prov()
        rc = L.cl_b200_advance_ensemble(C_.byref(cs), n, x0.ctypes.data, out.ctypes.data, ok.ctypes.data, N, 0,
                                        C_.byref(prov))
        if rc != 0:
            raise RuntimeError(rc)
        return prov.gpu_ms, x0.nbytes, out.nbytes + ok.nbytes

    def cpu():
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        threads = os.cpu_count() or 1
        t = time.perf_counter()
        O.oracle_advance(m, flow, x0[:4096], tau, 2000, threads=threads)
        return dict(value=4096 * 2000 / (time.perf_counter() - t), unit="orbit-steps/s", cores=threads, kind="port",
                    sample="4096 orbits x 2000 steps (oracle, all host threads)")
    # FP64 operations per step of advance_n (no contraction: every multiply and add is its own operation): the
    # pending-kick sum per stage, a drift (t = c dt, q += t p: 5), a kick (t = pend dt, the force 7, p -= t F: 12)
    drifts = sum(1 for c in m.c if c != 0.0)
    kicks, pend = 0, 0.0
    for _ in range(2):                        # the second pass counts the steady state (the kick carried over)
        kicks_pass = 0
        for c, d in zip(m.c, m.d):
            if c != 0.0:
                if pend != 0.0:
                    kicks_pass += 1
                    pend = 0.0
            pend += d
        kicks = kicks_pass
    ops = m.stages + 5 * drifts + 12 * kicks

    def roofline(value, torch_, dev_):
        peak = _dgemm_peak(torch_, dev_)
        achieved = value * ops / 1e12
        return dict(bound="fp64", achieved=achieved, peak=peak, unit="TFLOP/s", frac=achieved / peak, traffic=None,
                    peak_source="cuBLAS DGEMM 8192^3 measured here (burst; an FMA counts 2, this kernel has none)",
                    flops_per_orbit_step=ops, drifts=drifts, kicks=kicks)
    _host_call_workload(args, "orbit-steps/s (advance_ensemble, KahanLi(8) on the Henon-Heiles flow, states only)",
                        "orbit-steps/s", n * N, call,
                        dict(workload=f"advance-kahanli8-hh-{n}x{N:.0e}-dt0.05", orbits=n, N=N, tau=tau,
                             stages=m.stages), cpu, roofline=roofline)


def workload_torus(args):
    """The coupled-maps ensemble on the torus: WrappedFroeschleMap(1.5, 1.5, 0.05), coordinates in [0, 2 pi)^4
    with zero winding counts, the same two frames as the default workload (QRSpectrum(Householder) k = 4 and
    GALI_4 + SALI k = 4), 65536 orbits x 1e5 steps, tau = 10."""
    from chaos_b200 import GALI, SALI, HouseholderQR, QRSpectrum, WrappedFroeschleMap, torus_state
    from chaos_b200.propagate import FrameSpec
    n, N = args.orbits or N_ORBITS, args.N
    sysm = WrappedFroeschleMap(NU, KAPPA, MU)
    z = np.random.default_rng(SEED).uniform(0, 2 * np.pi, (n, 4))
    x0 = np.array([torus_state(sysm, v) for v in z])
    frames = [FrameSpec(4, (QRSpectrum(HouseholderQR()),)), FrameSpec(4, (GALI(), SALI()))]

    def cpu():
        W0 = np.broadcast_to(np.eye(4), (512, 4, 4)).copy()
        fr = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0), FrameSpec(4, (GALI(), SALI()), W0)]
        return _cpu_port(sysm, x0[:512], 4000, TAU, fr, "orbit-steps/s",
                         "512 orbits x 4000 steps of the workload (oracle, all host threads)")
    _propagate_workload(args, "WrappedFroeschleMap(1.5, 1.5, 0.05) on the torus, QRSpectrum(Householder) k=4 | "
                        "GALI_4+SALI k=4, tau=10", sysm, x0, N, TAU, frames, "orbit-steps", cpu,
                        dict(workload=f"froeschle-torus-{n}x{N:.0e}-tau10-qr-householder+gali4+sali", orbits=n, N=N,
                             tau=TAU, W0="I"))


def workload_coop(args):
    """`propagate` on a lattice of 8 sites (StandardMapChain, d = 16, k = 8, tau = 10, Float64) through the public
    call: one thread per orbit (variant 1) against one orbit per group of 8 lanes (the cooperative form, variant 8),
    for QRSpectrum(HouseholderQR), QRSpectrum(MGS) and GALI, with the records compared bit for bit. The headline value
    is the cooperative Householder run's orbit-steps/s."""
    torch, dev, L = _setup()
    from chaos_b200 import GALI, MGS, HouseholderQR, QRSpectrum, StandardMapChain
    from chaos_b200.propagate import FrameSpec, build_run, propagate_frames
    n = args.orbits or 2048
    N, tau, d, k = 20000, 10, 16, 8
    sysm = StandardMapChain(8, 1.2, 0.05)
    x0 = np.random.default_rng(SEED).uniform(0, 2 * np.pi, (n, d))
    W0 = np.ascontiguousarray(np.broadcast_to(np.eye(d)[:, :k], (n, d, k)))
    rows, first = {}, None
    for name, chain in (("householder", (QRSpectrum(HouseholderQR()),)), ("mgs", (QRSpectrum(MGS()),)),
                        ("gali", (GALI(),))):
        fr = FrameSpec(k, chain, W0)
        r = build_run(sysm, N, tau, [fr], "fp64", SEED)
        res = {}
        for v in (1, 8):
            L.cl_b200_set_variant(C.byref(r), v)
            out = propagate_frames(sysm, x0, N, [fr], tau=tau, seed=SEED, finals=False, throw=False)[0]
            ms = []
            for _ in range(max(1, args.steps)):
                t0 = time.perf_counter()
                out = propagate_frames(sysm, x0, N, [fr], tau=tau, seed=SEED, finals=False, throw=False)[0]
                ms.append((time.perf_counter() - t0) * 1e3)
            res[v] = (float(np.median(ms)), out, ms)
        L.cl_b200_set_variant(C.byref(r), 0)
        same = bool(np.array_equal(res[1][1].x.view(np.int64), res[8][1].x.view(np.int64)) and
                    np.array_equal(res[1][1].W.view(np.int64), res[8][1].W.view(np.int64)) and
                    res[1][1].states.tobytes() == res[8][1].states.tobytes())
        rows[name] = dict(one_thread=n * N / (res[1][0] / 1e3), cooperative=n * N / (res[8][0] / 1e3),
                          speedup=res[1][0] / res[8][0], bitwise_equal=same)
        if first is None:
            first = res[8][2]
    _line("orbit-steps/s (propagate, StandardMapChain 8 sites d=16 k=8, cooperative lane groups, Float64, host buffers)",
          rows["householder"]["cooperative"], "orbit-steps/s", args, first,
          dict(workload=f"lattice-propagate-d16k8-{n}x{N}-tau{tau}", orbits=n, N=N, tau=tau),
          dtype="f64", per_chain=rows,
          e2e=dict(value=rows["householder"]["cooperative"], unit="orbit-steps/s",
                   h2d_bytes_per_step=int(x0.nbytes + W0.nbytes), d2h_bytes_per_step=int(x0.nbytes + W0.nbytes)),
          gpu_launches=1)


def run_workload(args):
    {"standard": workload_standard, "gauss": workload_gauss, "lattice": workload_lattice,
     "screen": workload_screen, "mlp": workload_mlp, "split": workload_split, "shadow": workload_shadow,
     "record": workload_record, "indicators": workload_indicators, "advance": workload_advance,
     "torus": workload_torus, "record_mixed": lambda a: workload_record(a, "mixed"),
     "coop": workload_coop}[args.workload](args)



class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
