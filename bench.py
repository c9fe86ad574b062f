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
METRIC = "orbit-steps/s (4D coupled standard maps, QRSpectrum(Householder) + GALI_4 + SALI, mixed-precision kernel)"


# ---- algorithmic operation counts ---------------------------------------------------------------------------------
# Counting convention: add, sub, mul = 1, fma = 2, div and sqrt = 1, compare/select = 0. The transcendentals are this
# library's own polynomials, counted by the arithmetic they execute: one FP64 sincos = 3 fma (reduction) + 1 mul
# + 2 x 8 fma + 1 mul/fma (assembly) + 2 mul/sub (quadrant) = 44 flops; one FP64 log = 1 div + 2 add + 9 fma +
# ~10 add/mul = 31 flops. Per orbit-step of the workload above:
def flops_per_orbit_step(tau: int = TAU, mixed: bool = False) -> dict:
    d, k = 4, 4
    log64, sincos64 = 31, 44
    if mixed:
        # the orbit's three values by the split evaluation (reduction 10 + one polynomial 18 = 28 FP64 flops each);
        # the tangent's three complementary values in Float32 (two degree-5 polynomials, 24 flops each)
        map64 = 3 * 28 + 16
        map32 = 3 * 24 + 8
        tangent32 = 2 * k * (2 + 2 * 4)          # per frame: 2 adds + 2 x (2 fma) per column, structured
    else:
        map64 = 3 * sincos64 + 16                # x' (2), x1'+x2' (1), _abc (5), forward (8)
        tangent64 = 2 * d * k * (1 + 2 * (d - 1))  # per frame fused_product: 1 mul + (d-1) fma per entry
    # per handoff: Householder QR d = k = 4 (3 reflectors + Q formation + sign fix), window_Gw, orth_loss
    hh = 3 * (2 * d + 3 + 2 * d + 2 + d + 4 * (2 * d + d)) + 3 * 4 * (2 * d + 2 * d) + 2 * d * k
    gw = 60 + 2 * k * k * 2
    orth = k * k * (2 * d)
    gali = k * (3 * d + 2) + d * k + 2 * sum(j * 4 * d for j in range(k)) + k * (3 * d + 2) + 2 * (3 * d + 2)
    handoff = hh + gw + orth + gali
    nlogs = 2 * k
    if mixed:   # frames, norms, QR and GALI in Float32; logs as hardware log2 times ln 2, sums Float64
        return dict(fp64=map64 + nlogs * (1 + 4) / tau, fp32=map32 + tangent32 + handoff / tau)
    return dict(fp64=map64 + tangent64 + (handoff + nlogs * (log64 + 4)) / tau, fp32=0.0)


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
    O.oracle_frames(FroeschleMap(NU, KAPPA, MU), x0, sample_steps, frames, tau=TAU, math="portable", threads=threads)
    dt = time.perf_counter() - t
    return dict(value=sample_orbits * sample_steps / dt, seconds=dt, threads=threads)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--orbits", type=int, default=N_ORBITS)
    ap.add_argument("--N", type=int, default=N_STEPS)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        # a bounded sample of the same workload per step: 1024 orbits x 4000 steps
        so, ss = 1024, 4000
        vals = []
        for i in range(args.warmup + args.steps):
            r = cpu_reference(so, ss, threads)
            if i >= args.warmup:
                vals.append(r["value"])
        v = float(np.median(vals))
        line = dict(metric=METRIC, value=v, unit="orbit-steps/s", n_gpus=args.gpus, steps=args.steps,
                    warmup=args.warmup, ms_per_step=so * ss / v * 1e3, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="f64", data="synthetic", impl="reference",
                    config=dict(workload="froeschle-4d-65536x1e5-tau10-qr-householder+gali4+sali", orbits=args.orbits,
                                N=args.N, tau=TAU),
                    cpu_baseline=dict(value=v, unit="orbit-steps/s", cores=threads, kind="port",
                                      sample=f"{so} orbits x {ss} steps of the workload per step (oracle, all host threads; Julia absent)"),
                    e2e=dict(value=v, unit="orbit-steps/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
        print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist

    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    from chaos_b200 import _abi
    from chaos_b200 import FroeschleMap, GALI, HouseholderQR, QRSpectrum, SALI
    from chaos_b200._lib import last_error, lib
    from chaos_b200.propagate import FrameSpec, build_run
    L = lib()

    n, N = args.orbits, args.N
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

    def lambdas():
        # QRSpectrum frame states: sums (K=4) then the rest; lambda_1 = (s + c) / n
        st = bufs["st"][0].view(torch.float64).reshape(n, -1)
        s1, c1 = st[:, 0], st[:, 1]
        nn = bufs["st"][0].reshape(n, -1)[:, 8].to(torch.float64)
        return ((s1 + c1) / nn).cpu().numpy(), bufs["code"][0].cpu().numpy().copy()

    # plain Float64 kernel (the reference's arithmetic), then the mixed kernel
    t64, ms64, _ = timed("fp64", args.steps, args.warmup)
    lam64, code64 = lambdas()
    sampler = ClockSampler(dev.index if world == 1 else local)
    tmx, msmx, launches = timed("mixed", args.steps, args.warmup, sampler)
    lammx, codemx = lambdas()
    ok = (code64 == 0) & (codemx == 0)
    dl1 = float(np.max(np.abs(lammx[ok] - lam64[ok]))) if ok.any() else None

    work = n * N * world
    value = work * args.steps / (tmx / 1e3)
    value64 = work * args.steps / (t64 / 1e3)

    # e2e: the C ABI with host buffers (copies in and out inside the timed region)
    from chaos_b200.propagate import propagate_frames
    W0h = np.broadcast_to(np.eye(4), (n, 4, 4)).copy()
    fr_h = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0h), FrameSpec(4, (GALI(), SALI()), W0h)]
    propagate_frames(sysm, x0_h, N, fr_h, tau=TAU, seed=SEED, precision="mixed", finals=False, throw=False)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    te = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = propagate_frames(sysm, x0_h, N, fr_h, tau=TAU, seed=SEED, precision="mixed", finals=False, throw=False)
        te.append(time.perf_counter() - t0)
    tt = torch.tensor([sum(te)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    e2e_value = work * args.steps / float(tt.item())
    h2d = x0_h.nbytes + 2 * W0h.nbytes
    d2h = res[0].x.nbytes + sum(r_.W.nbytes + r_.states.nbytes + r_.code.nbytes + r_.hstep.nbytes for r_ in res)

    # FP64 peak: cuBLAS DGEMM (the library FP64 rate on this GPU), burst
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
    fp64_peak = 2 * 8192 ** 3 / (best / 1e3) / 1e12
    del a

    fl = flops_per_orbit_step(TAU, mixed=True)
    fl64 = flops_per_orbit_step(TAU, mixed=False)
    per_launch_ms = float(np.mean(msmx))
    # FP64-pipe equivalent: a Float32 op takes half an FP64 issue slot on B200 (FP32 rate = 2 x FP64 rate)
    achieved = n * N * (fl["fp64"] + fl["fp32"] / 2) / (per_launch_ms / 1e3) / 1e12
    achieved64 = n * N * fl64["fp64"] / (float(np.mean(ms64)) / 1e3) / 1e12

    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cb_ = cpu_reference(512, 4000, threads)
        cpu = dict(value=cb_["value"], unit="orbit-steps/s", cores=threads, kind="port",
                   sample="512 orbits x 4000 steps of the workload (oracle, all host threads)")

    if rank == 0:
        clocks = sampler.summary()
        line = dict(
            metric=METRIC, value=value, unit="orbit-steps/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
            ms_per_step=tmx / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
            dtype="f64 orbit + f32 frames", data="synthetic",
            config=dict(workload="froeschle-4d-65536x1e5-tau10-qr-householder+gali4+sali", orbits_per_gpu=n, N=N,
                        tau=TAU, frames="QRSpectrum(HouseholderQR) k=4 | GALI_4+SALI k=4", W0="I",
                        l2="flushed between timed steps (256 MB write)", parallelism=f"dp{world} (orbit shards)",
                        tuned_blocks_per_sm=tuned),
            fp64_kernel=dict(value=value64, ms_per_step=t64 / args.steps, mixed_over_fp64=value / value64,
                             max_abs_dlambda1=dl1, roofline_tflops=achieved64, frac_of_fp64_peak=achieved64 / fp64_peak),
            e2e=dict(value=e2e_value, unit="orbit-steps/s", h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(d2h)),
            roofline=dict(bound="fp64", achieved=achieved, peak=fp64_peak, unit="TFLOP/s", frac=achieved / fp64_peak,
                          traffic=None, peak_source="cuBLAS DGEMM 8192^3 measured here (burst)",
                          flops_per_orbit_step=fl),
            cpu_baseline=cpu, clocks=clocks, gpu_launches=int(launches),
        )
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
