#!/usr/bin/env python
"""Throughput benchmark of the B200 minfft engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference] [--workload NAME]

Default workload ("2d2048"): 2-D real DFT + inverse real DFT and 2-D
DCT-2 -> DCT-3 round trips on 2048 x 2048 arrays of i.i.d. standard-normal
data, in double and in single precision.  One step = those 8 transforms
(realdft, invrealdft, dct2, dct3 in f64, then in f32), each through the
engine's C ABI on device-resident data.  Metric: GFLOP/s with the
2.5 * N * log2(N) convention for real-data transforms (N = 2^22 points).

Other workloads (``--workload``): "batch4096" (1024 complex DFTs of length
4096, c128, forward then inverse; 5 N log2 N per transform), "mixed20000"
(20000 1-D transforms of mixed kinds and lengths in one persistent launch),
"3d256" (256^3 c64 DFT, forward then inverse), "long1d" (2^26-point DFTs in
c128 and c64, 2^24-point DCT-4/DST-4 in f64 and f32), "long1d_c64" (the
2^26-point c64 DFT, forward then inverse) and "long1d_t4" (DCT-4 and DST-4
of 2^24 points in f32).  "3d256", "long1d_c64" and "long1d_t4" take
``--precision fp32|tc_f16|tc_bf16`` (CUDA-core or tensor-core split-precision
256-point passes).  The default run also measures every other workload
briefly after the headline and reports them under "configs" (one GPU).

Timing: W untimed warm-up steps, then exactly K steps between CUDA events on
the stream the kernels run on (the legacy default stream), bracketed by a
barrier and a device synchronisation; the maximum over ranks is reported.
Inputs rotate over 4 buffer sets, so each step reads inputs last touched
four steps earlier, with far more than the 126 MB L2 written in between.

Under torchrun every rank runs its own replica of the workload on its own
GPU (the transforms are independent; there is no data-path collective):
value = all ranks' FLOPs / max-over-ranks time, scaling "weak".

``--impl reference`` times the reference's own CPU library (aimukhin/minfft
compiled from its sources into oracle/_ref/, or the oracle restatement if it
was not built) on the host cores: every OpenMP thread runs one independent
instance of the same step with its own plans (a minfft plan is not
re-entrant).  Only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "traffic.json")
FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------------ helpers
def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(dist, x: float, device) -> float:
    """The maximum of x over all ranks (x itself without a process group):
    a multi-rank time is the slowest rank's."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gflops(flops_per_step: float, steps: int, world: int, seconds: float) -> float:
    """Whole-job GFLOP/s: every rank runs `steps` steps of its own replica
    (the same work), all timed by the slowest rank."""
    return flops_per_step * steps * world / seconds / 1e9


_input_cache = {}


def uniform_c64(dims, seed):
    """re/im i.i.d. uniform[-1,1) from numpy PCG64(seed), as complex64
    (kept for the other precisions of the same workload)."""
    key = (tuple(dims), seed)
    if key not in _input_cache:
        rng = np.random.default_rng(seed)
        x = np.empty(dims, dtype=np.complex64)
        x.real = rng.uniform(-1, 1, dims)
        x.imag = rng.uniform(-1, 1, dims)
        _input_cache[key] = x
    return _input_cache[key]


_oracle_cache = {}


def uniform_f32(dims, seed):
    """i.i.d. uniform[-1,1) from numpy PCG64(seed), as float32 (kept for the other precisions)."""
    key = ("f32", tuple(dims), seed)
    if key not in _input_cache:
        _input_cache[key] = np.random.default_rng(seed).uniform(-1, 1, dims).astype(np.float32)
    return _input_cache[key]


def oracle_real(name, seed, op, x, dims):
    """The checker: the FP64 oracle's real transform `op` of x upcast, cached."""
    key = (name, seed, op, tuple(dims))
    if key not in _oracle_cache:
        import oracle

        _oracle_cache[key] = oracle.apply(op, x.astype(np.float64), dims, single=False, kind=oracle.best_kind())
    return _oracle_cache[key]


def oracle_kind_name():
    import oracle

    return {"reference": "reference minfft.c compiled from its sources, double",
            "restatement": "C restatement of minfft.c, double"}[oracle.best_kind()]


def oracle_dft(name, seed, x, dims):
    """The checker (never the measured path): the FP64 oracle's forward DFT
    of x upcast to complex128, cached per workload input."""
    key = (name, seed, tuple(dims))
    if key not in _oracle_cache:
        import oracle

        _oracle_cache[key] = oracle.apply("dft", x.astype(np.complex128), dims, single=False, kind=oracle.best_kind())
    return _oracle_cache[key]


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons while running:
    through NVML every 10 ms (read-only queries), else nvidia-smi every 100 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.samples = []  # (sm_mhz, max_mhz, set of reason names)
        self.source = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def poll():
                while not self.stop.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(sm), float(mx), {n for n, b in bits.items() if rs & b}))
                    except Exception:
                        pass
                    self.stop.wait(0.01)

            self.nvml = pynvml
            self.source = "nvml 10 ms"
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi 100 ms"
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            parts = [p.strip() for p in ln.strip().split(",")]
            if len(parts) < 9:
                continue
            try:
                self.samples.append((float(parts[1]), float(parts[2]),
                                     {nm for nm, v in zip(self.NAMES, parts[5:9]) if v.lower() == "active"}))
            except ValueError:
                continue

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [a for a, _, _ in self.samples]
        mx = self.samples[-1][1] if self.samples else None
        reasons = set()
        for _, _, r in self.samples:
            reasons |= r
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": self.source}


# ---------------------------------------------------------------- workloads
class PerPrecisionStreams:
    """Each precision's plans on its own CUDA stream: a step's f64 and f32
    transforms are independent and run concurrently, while a precision's
    transforms stay in order on its stream.  set_streams(False) puts every
    plan on one stream (used for the per-kernel timing pass)."""

    plan_keys = ()

    def init_streams(self):
        self.streams = [self.torch.cuda.Stream() for _ in self.precs]
        self.set_streams(True)

    def set_streams(self, concurrent: bool):
        self.concurrent = concurrent
        for i, p in enumerate(self.precs):
            st = self.streams[i if concurrent else 0]
            for key in self.plan_keys:
                p[key].set_stream(st.cuda_stream)

    def step_streams(self):
        return self.streams


class Workload2D(PerPrecisionStreams):
    """2048 x 2048 realdft/invrealdft and dct2/dct3 round trips, f64 and f32."""

    name = "2d2048"
    dims = (2048, 2048)
    nsets = 4
    dtype = "f64+f32"
    plan_keys = ("pr", "pt")

    def __init__(self, torch, dev):
        import minfft_b200

        self.torch = torch
        n = int(np.prod(self.dims))
        self.flops_per_transform = 2.5 * n * math.log2(n)
        self.ops_per_step = 8
        rng = np.random.default_rng(2)
        self.precs = []
        for single in (False, True):
            eng = minfft_b200.engine(single)
            rdt = torch.float32 if single else torch.float64
            cdt = torch.complex64 if single else torch.complex128
            spec = (self.dims[0], self.dims[1] // 2 + 1)
            xs = [torch.from_numpy(rng.standard_normal(self.dims)).to(dev, rdt) for _ in range(self.nsets)]
            z = torch.empty(spec, dtype=cdt, device=dev)
            x2 = torch.empty(self.dims, dtype=rdt, device=dev)
            c = torch.empty(self.dims, dtype=rdt, device=dev)
            x3 = torch.empty(self.dims, dtype=rdt, device=dev)
            pr = eng.plan("realdft", self.dims)
            pt = eng.plan("t2t3", self.dims)
            self.precs.append(dict(single=single, eng=eng, pr=pr, pt=pt, xs=xs, z=z, x2=x2, c=c, x3=x3))
        self.init_streams()

    def plans(self):
        for p in self.precs:
            yield p["eng"], p["pr"], ("realdft", "invrealdft")
            yield p["eng"], p["pt"], ("dct2", "dct3")

    def rebuild(self, eng, plan):
        """Replace `plan` by a fresh one (launch lists follow the current tuning table)."""
        for p in self.precs:
            for key in ("pr", "pt"):
                if p[key] is plan:
                    fam = plan.family
                    plan.free()
                    p[key] = eng.plan(fam, self.dims)
        self.set_streams(self.concurrent)

    def step(self, k: int):
        s = k % self.nsets
        for p in self.precs:
            x = p["xs"][s].data_ptr()
            pr, pt = p["pr"], p["pt"]
            pr("realdft", x, p["z"].data_ptr(), check=False)
            pr("invrealdft", p["z"].data_ptr(), p["x2"].data_ptr(), check=False)
            pt("dct2", x, p["c"].data_ptr(), check=False)
            pt("dct3", p["c"].data_ptr(), p["x3"].data_ptr(), check=False)

    def check_errors(self):
        for p in self.precs:
            p["eng"].check()

    def launches_per_step(self):
        tot = 0
        for eng, plan, ops in self.plans():
            tot += sum(eng.launch_count(op, plan.aux) for op in ops)
        return tot

    def e2e_setup(self):
        """Pinned host copies of one input set and two sets of plans and host
        outputs, used on alternate steps.  Every plan has its own stream in
        host-async mode, so within a step the four plans' uploads, transforms
        and downloads overlap, and a step's uploads overlap the previous
        step's downloads; a set waits for its own previous step (two steps
        back) before it is reused."""
        torch = self.torch
        pin = lambda t: torch.empty(t.shape, dtype=t.dtype, pin_memory=True)  # noqa: E731
        self.e2e_sets = []
        for k in range(2):
            plans, host = [], []
            for p in self.precs:
                pr = p["pr"] if k == 0 else p["eng"].plan("realdft", self.dims)
                pt = p["pt"] if k == 0 else p["eng"].plan("t2t3", self.dims)
                streams = []
                for plan in (pr, pt):
                    st = torch.cuda.Stream()
                    plan.set_stream(st.cuda_stream)
                    plan.set_host_async(True)
                    streams.append(st)
                plans.append((pr, pt, streams))
                host.append(dict(z=pin(p["z"]), x2=pin(p["x2"]), c=pin(p["c"]), x3=pin(p["x3"])))
            self.e2e_sets.append((plans, host))
        self.hx = []
        for p in self.precs:
            hx = pin(p["xs"][0])
            hx.copy_(p["xs"][0].cpu())
            self.hx.append(hx)
        self.e2e_k = 0
        h2d = d2h = 0
        for hx, h in zip(self.hx, self.e2e_sets[0][1]):
            # each call stages its input to the device and its output back
            h2d += 2 * hx.numel() * hx.element_size() + h["z"].numel() * h["z"].element_size() + \
                h["c"].numel() * h["c"].element_size()
            d2h += h["z"].numel() * h["z"].element_size() + h["x2"].numel() * h["x2"].element_size() + \
                h["c"].numel() * h["c"].element_size() + h["x3"].numel() * h["x3"].element_size()
        return h2d, d2h

    def e2e_step(self):
        plans, host = self.e2e_sets[self.e2e_k & 1]
        if self.e2e_k >= 2:
            for pr, pt, _ in plans:
                pr.synchronize()
                pt.synchronize()
        self.e2e_k += 1
        for (pr, pt, _), hx, h in zip(plans, self.hx, host):
            pr("realdft", hx.data_ptr(), h["z"].data_ptr(), check=False)
            pr("invrealdft", h["z"].data_ptr(), h["x2"].data_ptr(), check=False)
            pt("dct2", hx.data_ptr(), h["c"].data_ptr(), check=False)
            pt("dct3", h["c"].data_ptr(), h["x3"].data_ptr(), check=False)

    @classmethod
    def config(cls):
        return {"workload": "2-D realdft->invrealdft and dct2->dct3 round trips, 2048x2048, f64 and f32",
                "dims": list(cls.dims), "precisions": ["f64", "f32"], "transforms_per_step": 8,
                "flops": "2.5*N*log2(N) per transform, N=2^22",
                "inputs": "i.i.d. standard normal, numpy PCG64 seed 2",
                "l2": "inputs rotate over 4 buffer sets (192 MiB of inputs; each step writes ~250 MB), "
                      "larger than the 126 MB L2",
                "streams": "one per precision: the f64 and f32 transforms of a step run concurrently, each "
                           "precision's four transforms in order on its stream (per-kernel timings from a "
                           "separate pass with every plan on one stream)"}

    # CPU reference: (family, ops, single) sequences of one step
    cpu_sequences = (("realdft", ("realdft", "invrealdft"), False), ("t2t3", ("dct2", "dct3"), False),
                     ("realdft", ("realdft", "invrealdft"), True), ("t2t3", ("dct2", "dct3"), True))

    @classmethod
    def cpu_measure(cls, kind, threads, warm, reps):
        """Seconds and flops of `reps` steps on the CPU: `threads` independent
        instances of the step, one per OpenMP thread, each with its own plans."""
        t = cpu_run(kind, cls.cpu_sequences, cls.dims, threads, threads, reps, warm)
        n = int(np.prod(cls.dims))
        return t, 2.5 * n * math.log2(n) * 8 * threads * reps


def alternate_plan_sets(torch, plans, like, nout):
    """For each plan: its own CUDA stream, host-async mode and `nout` pinned
    host arrays shaped like `like` (the plan's outputs on the steps it runs)."""
    sets = []
    for plan in plans:
        st = torch.cuda.Stream()
        plan.set_stream(st.cuda_stream)
        plan.set_host_async(True)
        sets.append((plan, st, [torch.empty_like(like, pin_memory=True) for _ in range(nout)]))
    return sets


def next_plan_set(w):
    """The plan and host outputs of the next end-to-end step of workload w
    (alternating between two sets); a set first waits for its previous step."""
    plan, _, outs = w.e2e_sets[w.e2e_k & 1]
    if w.e2e_k >= 2:
        plan.synchronize()
    w.e2e_k += 1
    return plan, outs


class WorkloadBatch4096:
    """1024 independent complex DFTs of length 4096 (c128), forward then inverse."""

    name = "batch4096"
    n, howmany = 4096, 1024
    nsets = 4
    dtype = "f64"

    def __init__(self, torch, dev):
        import minfft_b200

        self.torch = torch
        self.flops_per_transform = 5.0 * self.n * math.log2(self.n) * self.howmany
        self.ops_per_step = 2
        rng = np.random.default_rng(1)
        shape = (self.howmany, self.n)
        self.eng = minfft_b200.engine(False)
        mk = lambda: torch.from_numpy(rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).to(dev)  # noqa
        self.xs = [mk() for _ in range(self.nsets)]
        self.y = torch.empty(shape, dtype=torch.complex128, device=dev)
        self.z = torch.empty(shape, dtype=torch.complex128, device=dev)
        self.plan = self.eng.plan("dft", (self.n,))

    def plans(self):
        yield self.eng, self.plan, ("dft", "invdft")

    def howmany_for(self, op):
        return self.howmany

    def rebuild(self, eng, plan):
        self.plan.free()
        self.plan = eng.plan("dft", (self.n,))

    def step(self, k):
        x = self.xs[k % self.nsets]
        self.plan.batch("dft", x.data_ptr(), self.y.data_ptr(), self.howmany)
        self.plan.batch("invdft", self.y.data_ptr(), self.z.data_ptr(), self.howmany)

    def check_errors(self):
        self.eng.check()

    def launches_per_step(self):
        return 2

    def e2e_setup(self):
        """Two plans on their own streams in host-async mode, used on
        alternate steps (see Workload3D256.e2e_setup)."""
        t = self.torch
        self.hx = t.empty(self.xs[0].shape, dtype=t.complex128, pin_memory=True)
        self.hx.copy_(self.xs[0].cpu())
        self.e2e_sets = alternate_plan_sets(t, [self.plan, self.eng.plan("dft", (self.n,))], self.hx, 2)
        self.e2e_k = 0
        b = self.hx.numel() * 16
        return 2 * b, 2 * b

    def e2e_step(self):
        plan, (hy, hz) = next_plan_set(self)
        plan.batch("dft", self.hx.data_ptr(), hy.data_ptr(), self.howmany)
        plan.batch("invdft", hy.data_ptr(), hz.data_ptr(), self.howmany)

    @classmethod
    def config(cls):
        return {"workload": "1024 x complex DFT N=4096 c128, forward then inverse", "n": cls.n,
                "batch": cls.howmany, "flops": "5*N*log2(N) per transform",
                "inputs": "re/im i.i.d. uniform[-1,1), seed 1",
                "l2": "inputs rotate over 4 sets of 64 MiB (256 MiB), larger than L2"}

    cpu_sequences = (("dft", ("dft", "invdft"), False),)

    @classmethod
    def cpu_sample(cls, P):
        return (f"the whole step: {cls.howmany} transforms forward then inverse, OpenMP over the batch on {P} "
                f"threads, one plan per thread")

    @classmethod
    def cpu_measure(cls, kind, threads, warm, reps):
        """The reference's batched case as its users run it: `omp for` over the
        1024 transforms, one plan per thread (a minfft plan is not re-entrant)."""
        t = cpu_run(kind, cls.cpu_sequences, (cls.n,), cls.howmany, threads, reps, warm)
        return t, 5.0 * cls.n * math.log2(cls.n) * cls.howmany * 2 * reps


class WorkloadMixed:
    """20000 independent 1-D transforms in one persistent graph-launched kernel:
    log2 n uniform in 4..16, kinds uniform over dft, realdft, dct2, dst2,
    dct3, dst3, dct4, dst4, float32, standard-normal inputs."""

    name = "mixed20000"
    count = 20000
    kinds = ("dft", "realdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4")
    dtype = "f32"

    @classmethod
    def job_list(cls):
        rng = np.random.default_rng(4)
        ops = [cls.kinds[k] for k in rng.integers(0, len(cls.kinds), cls.count)]
        ns = [1 << int(v) for v in rng.integers(4, 17, cls.count)]
        return ops, ns

    @classmethod
    def cpu_measure(cls, kind, threads, warm, reps):
        """Seconds and flops of `reps` sweeps of the batch on the CPU: every
        (kind, n) group as one OpenMP batch of the reference library."""
        ops, ns = cls.job_list()
        groups = {}
        for op, n in zip(ops, ns):
            groups[(op, n)] = groups.get((op, n), 0) + 1
        fam = {"dft": "dft", "realdft": "realdft", "dct4": "t4", "dst4": "t4"}
        t = 0.0
        for (op, n), cnt in sorted(groups.items()):
            t += cpu_run(kind, ((fam.get(op, "t2t3"), (op,), True),), (n,), cnt, threads, reps, warm)
        flops = sum((5.0 if op == "dft" else 2.5) * n * math.log2(n) for op, n in zip(ops, ns)) * reps
        return t, flops

    def __init__(self, torch, dev):
        import minfft_b200
        from minfft_b200 import shapes

        self.torch = torch
        self.ops, self.ns = self.job_list()
        self.eng = minfft_b200.engine(True)
        esz = 4
        # all inputs in one region of the pool, all outputs in the next
        # (256-byte aligned slices), so a step's upload and download are one
        # contiguous copy each
        offs_in, offs_out, tot = [], [], 0
        self.in_bytes = self.out_bytes = 0
        sizes = []
        for op, n in zip(self.ops, self.ns):
            ins, inc, outs, outc = shapes(op, (n,))
            sizes.append((int(np.prod(ins)) * esz * (2 if inc else 1), int(np.prod(outs)) * esz * (2 if outc else 1)))
        for bi, _ in sizes:
            offs_in.append((tot, bi))
            tot += (bi + 255) // 256 * 256
            self.in_bytes += bi
        self.in_region = tot
        for _, bo in sizes:
            offs_out.append((tot, bo))
            tot += (bo + 255) // 256 * 256
            self.out_bytes += bo
        self.pool_elems = tot // 4 + 64
        self.pool = torch.empty(self.pool_elems, dtype=torch.float32, device=dev)
        self.pool.normal_(generator=torch.Generator(device=dev).manual_seed(4))
        self.offs_in, self.offs_out = offs_in, offs_out
        self.dev = dev
        self.handle = self.eng.mixed_plan(self._jobs(self.pool))
        self.flops_per_transform = sum((5.0 if op == "dft" else 2.5) * n * math.log2(n)
                                       for op, n in zip(self.ops, self.ns))
        self.ops_per_step = 1

    def _jobs(self, pool):
        base = pool.data_ptr()
        return [(op, n, base + oi, base + oo) for op, n, (oi, _), (oo, _) in zip(self.ops, self.ns, self.offs_in,
                                                                               self.offs_out)]

    def plans(self):
        return iter(())

    @staticmethod
    def cpu_sample(P):
        return f"the whole 20000-transform batch, each (kind, n) group as an OpenMP batch on {P} threads"

    def tune(self):
        self.eng.mixed_autotune(self.handle, 3)
        return self.eng.mixed_items(self.handle)

    def step(self, k):
        self.eng.mixed_execute(self.handle)

    def check_errors(self):
        self.eng.check()

    def launches_per_step(self):
        return 1

    def roofline_stats(self, ms, steps):
        """One graph launch of the persistent kernel per step: its time is the step time."""
        return [("f32 mixed_kernel (graph launch)", steps, ms, float(self.in_bytes + self.out_bytes))]

    def e2e_setup(self):
        """Two device pools with their own plans and streams, used on
        alternate steps: a step uploads its inputs (one copy of the input
        region from pinned host memory), launches the graph and downloads its
        outputs (one copy of the output region), all on its stream, so one
        step's upload overlaps the previous step's download."""
        t = self.torch
        self.pool_b = t.empty(self.pool_elems, dtype=t.float32, device=self.dev)
        self.pool_b.copy_(self.pool)
        self.handle_b = self.eng.mixed_plan(self._jobs(self.pool_b))
        self.eng.mixed_autotune(self.handle_b, 3)
        self.slots = [(self.pool, self.handle, t.cuda.Stream()), (self.pool_b, self.handle_b, t.cuda.Stream())]
        ni = self.in_region // 4
        self.h_in = t.empty(ni, dtype=t.float32, pin_memory=True)
        self.h_in.copy_(self.pool[:ni].cpu())
        self.h_out = [t.empty(self.pool_elems - ni, dtype=t.float32, pin_memory=True) for _ in range(2)]
        self.e2e_k = 0
        return ni * 4, (self.pool_elems - ni) * 4

    def e2e_step(self):
        t = self.torch
        i = self.e2e_k & 1
        self.e2e_k += 1
        pool, handle, st = self.slots[i]
        ni = self.in_region // 4
        with t.cuda.stream(st):
            pool[:ni].copy_(self.h_in, non_blocking=True)
            self.eng.mixed_execute(handle, st.cuda_stream)
            self.h_out[i].copy_(pool[ni:], non_blocking=True)

    @classmethod
    def io_bytes(cls):
        from minfft_b200 import shapes

        tot = 0
        for op, n in zip(*cls.job_list()):
            ins, inc, outs, outc = shapes(op, (n,))
            tot += 4 * (int(np.prod(ins)) * (2 if inc else 1) + int(np.prod(outs)) * (2 if outc else 1))
        return tot

    @classmethod
    def config(cls):
        b = cls.io_bytes()
        return {"workload": "20000 mixed 1-D transforms, one persistent graph-launched kernel",
                "count": cls.count, "log2n": "uniform integer 4..16", "kinds": list(cls.kinds),
                "precision": "f32", "flops": "5*N*log2(N) dft, 2.5*N*log2(N) real-data kinds",
                "inputs": "standard normal (torch generator seed 4)", "bytes_in_out": b,
                "l2": "inputs and outputs total ~%.1f GB, far beyond the 126 MB L2" % (b / 1e9)}

    cpu_sequences = ()


class Workload3D256:
    """256 x 256 x 256 complex DFT, forward then inverse, c64.  The arithmetic
    of its 256-point axis passes follows --precision: "fp32" (CUDA cores) or
    the tensor-core split-precision passes "tc_f16" / "tc_bf16"."""

    name = "3d256"
    dims = (256, 256, 256)
    nsets = 3
    seed = 3
    dtype = "f32"
    precision = "fp32"

    def __init__(self, torch, dev):
        import minfft_b200

        self.torch = torch
        n = int(np.prod(self.dims))
        self.flops_per_transform = 5.0 * n * math.log2(n)
        self.ops_per_step = 2
        self.eng = minfft_b200.engine(True)
        self.xs = [torch.from_numpy(uniform_c64(self.dims, self.seed + i)).to(dev) for i in range(self.nsets)]
        self.y = torch.empty(self.dims, dtype=torch.complex64, device=dev)
        self.z = torch.empty(self.dims, dtype=torch.complex64, device=dev)
        self.plan = self._mkplan()
        self.plan("dft", self.xs[0].data_ptr(), self.y.data_ptr())
        self.plan("invdft", self.y.data_ptr(), self.z.data_ptr())
        torch.cuda.synchronize()
        self.eng.tc_status(self.plan.aux)
        self.accuracy = self._accuracy(self.y.cpu().numpy(), self.z.cpu().numpy())

    def _accuracy(self, y, z):
        """Relative L2 error of the forward result against the FP64 oracle
        (the reference compiled from its sources where available) on the same
        input upcast, and of the round trip against the input."""
        x = self.xs[0].cpu().numpy()
        ref = oracle_dft(self.name, self.seed, x, self.dims)
        err = float(np.linalg.norm((y.astype(np.complex128) - ref).ravel()) / np.linalg.norm(ref.ravel()))
        n = int(np.prod(self.dims))
        rt = float(np.linalg.norm((z.astype(np.complex128) / n - x).ravel()) / np.linalg.norm(x.ravel()))
        return {"rel_l2_vs_fp64_oracle": err, "oracle": oracle_kind_name(), "roundtrip_rel_l2": rt}

    def _mkplan(self):
        plan = self.eng.plan("dft", self.dims)
        self.eng.set_precision(plan.aux, self.precision)
        return plan

    def plans(self):
        yield self.eng, self.plan, ("dft", "invdft")

    def rebuild(self, eng, plan):
        self.plan.free()
        self.plan = self._mkplan()

    def step(self, k):
        x = self.xs[k % self.nsets]
        self.plan("dft", x.data_ptr(), self.y.data_ptr(), check=False)
        self.plan("invdft", self.y.data_ptr(), self.z.data_ptr(), check=False)

    def check_errors(self):
        self.eng.check()
        self.eng.tc_status(self.plan.aux)

    def launches_per_step(self):
        return sum(self.eng.launch_count(op, self.plan.aux) for op in ("dft", "invdft"))

    def e2e_setup(self):
        """Two plans (same precision) on their own streams in host-async mode,
        with their own pinned host outputs, used on alternate steps: a step's
        upload overlaps the previous step's download."""
        t = self.torch
        self.hx = t.empty(self.dims, dtype=t.complex64, pin_memory=True)
        self.hx.copy_(self.xs[0].cpu())
        self.e2e_sets = alternate_plan_sets(t, [self.plan, self._mkplan()], self.hx, 2)
        self.e2e_k = 0
        b = self.hx.numel() * 8
        return 2 * b, 2 * b

    def e2e_step(self):
        plan, (hy, hz) = next_plan_set(self)
        plan("dft", self.hx.data_ptr(), hy.data_ptr(), check=False)
        plan("invdft", hy.data_ptr(), hz.data_ptr(), check=False)

    @classmethod
    def config(cls):
        return {"workload": "3-D complex DFT 256x256x256 c64, forward then inverse", "dims": list(cls.dims),
                "precision": cls.precision, "flops": "5*N*log2(N) per transform, N=2^24",
                "inputs": "re/im i.i.d. uniform[-1,1), numpy PCG64 seeds 3..5",
                "l2": "inputs rotate over 3 sets of 128 MiB, larger than the 126 MB L2"}

    cpu_sequences = (("dft", ("dft", "invdft"), True),)

    @classmethod
    def cpu_measure(cls, kind, threads, warm, reps):
        t = cpu_run(kind, cls.cpu_sequences, cls.dims, threads, threads, reps, warm)
        n = int(np.prod(cls.dims))
        return t, 5.0 * n * math.log2(n) * 2 * threads * reps


class WorkloadLong1D(PerPrecisionStreams):
    """Long 1-D transforms: complex DFT of 2^26 points in c128 and c64, and
    DCT-4 + DST-4 of 2^24 points in f64 and f32."""

    name = "long1d"
    n_dft, n_t4 = 1 << 26, 1 << 24
    nsets = 2
    dtype = "f64+f32"
    plan_keys = ("pd", "p4")

    def __init__(self, torch, dev):
        import minfft_b200

        self.torch = torch
        fd = 5.0 * self.n_dft * math.log2(self.n_dft)
        f4 = 2.5 * self.n_t4 * math.log2(self.n_t4)
        self.flops_per_transform = 2 * fd + 4 * f4  # one step: both DFTs and the four type-4 transforms
        self.ops_per_step = 1
        gen = torch.Generator(device=dev).manual_seed(5)
        self.precs = []
        for single in (False, True):
            eng = minfft_b200.engine(single)
            rdt = torch.float32 if single else torch.float64
            cdt = torch.complex64 if single else torch.complex128
            xs = [torch.randn(self.n_dft, dtype=cdt, device=dev, generator=gen) for _ in range(self.nsets)]
            rs = [torch.randn(self.n_t4, dtype=rdt, device=dev, generator=gen) for _ in range(self.nsets)]
            self.precs.append(dict(eng=eng, single=single, xs=xs, rs=rs,
                                   y=torch.empty(self.n_dft, dtype=cdt, device=dev),
                                   c=torch.empty(self.n_t4, dtype=rdt, device=dev),
                                   s=torch.empty(self.n_t4, dtype=rdt, device=dev),
                                   pd=eng.plan("dft", (self.n_dft,)), p4=eng.plan("t4", (self.n_t4,))))
        self.init_streams()

    def plans(self):
        for p in self.precs:
            yield p["eng"], p["pd"], ("dft",)
            yield p["eng"], p["p4"], ("dct4", "dst4")

    def rebuild(self, eng, plan):
        for p in self.precs:
            for key, fam, n in (("pd", "dft", self.n_dft), ("p4", "t4", self.n_t4)):
                if p[key] is plan:
                    plan.free()
                    p[key] = eng.plan(fam, (n,))
        self.set_streams(self.concurrent)

    def step(self, k):
        s = k % self.nsets
        for p in self.precs:
            p["pd"]("dft", p["xs"][s].data_ptr(), p["y"].data_ptr(), check=False)
            p["p4"]("dct4", p["rs"][s].data_ptr(), p["c"].data_ptr(), check=False)
            p["p4"]("dst4", p["rs"][s].data_ptr(), p["s"].data_ptr(), check=False)

    def check_errors(self):
        for p in self.precs:
            p["eng"].check()

    def launches_per_step(self):
        return sum(eng.launch_count(op, plan.aux) for eng, plan, ops in self.plans() for op in ops)

    def e2e_setup(self):
        """Two sets of plans (each on its own streams, host-async mode) and
        host outputs used on alternate steps, as in the 2-D workload."""
        t = self.torch
        pin = lambda x: t.empty(x.shape, dtype=x.dtype, pin_memory=True)  # noqa: E731
        self.hin = []
        for p in self.precs:
            h = dict(x=pin(p["xs"][0]), r=pin(p["rs"][0]))
            h["x"].copy_(p["xs"][0].cpu())
            h["r"].copy_(p["rs"][0].cpu())
            self.hin.append(h)
        self.e2e_sets = []
        for k in range(2):
            plans, host = [], []
            for p in self.precs:
                pd = p["pd"] if k == 0 else p["eng"].plan("dft", (self.n_dft,))
                p4 = p["p4"] if k == 0 else p["eng"].plan("t4", (self.n_t4,))
                streams = []
                for plan in (pd, p4):
                    st = t.cuda.Stream()
                    plan.set_stream(st.cuda_stream)
                    plan.set_host_async(True)
                    streams.append(st)
                plans.append((pd, p4, streams))
                host.append(dict(y=pin(p["y"]), c=pin(p["c"]), s=pin(p["s"])))
            self.e2e_sets.append((plans, host))
        self.e2e_k = 0
        h2d = d2h = 0
        for hi, h in zip(self.hin, self.e2e_sets[0][1]):
            h2d += hi["x"].numel() * hi["x"].element_size() + 2 * hi["r"].numel() * hi["r"].element_size()
            d2h += h["y"].numel() * h["y"].element_size() + 2 * h["c"].numel() * h["c"].element_size()
        return h2d, d2h

    def e2e_step(self):
        plans, host = self.e2e_sets[self.e2e_k & 1]
        if self.e2e_k >= 2:
            for pd, p4, _ in plans:
                pd.synchronize()
                p4.synchronize()
        self.e2e_k += 1
        for (pd, p4, _), hi, h in zip(plans, self.hin, host):
            pd("dft", hi["x"].data_ptr(), h["y"].data_ptr(), check=False)
            p4("dct4", hi["r"].data_ptr(), h["c"].data_ptr(), check=False)
            p4("dst4", hi["r"].data_ptr(), h["s"].data_ptr(), check=False)

    @classmethod
    def config(cls):
        return {"workload": "1-D dft 2^26 (c128, c64) + dct4/dst4 2^24 (f64, f32)",
                "n_dft": cls.n_dft, "n_t4": cls.n_t4, "transforms_per_step": 6,
                "flops": "5*N*log2(N) dft, 2.5*N*log2(N) dct4/dst4",
                "inputs": "standard normal (torch generator seed 5)",
                "l2": "inputs rotate over 2 sets (1.5 GiB per set), far beyond the 126 MB L2",
                "streams": "one per precision: the f64 and f32 transforms of a step run concurrently (per-kernel "
                           "timings from a separate pass with every plan on one stream)"}

    @classmethod
    def cpu_sample(cls, P):
        return (f"{min(P, 4)} concurrent instances (one per OpenMP thread, own plans) of each transform of one step")

    @classmethod
    def cpu_measure(cls, kind, threads, warm, reps):
        """A bounded sample: min(threads, 4) concurrent instances of each of
        the six transforms (the 2^26 arrays take 1 GiB each)."""
        P = min(threads, 4)
        t = cpu_run(kind, (("dft", ("dft",), False), ("dft", ("dft",), True)), (cls.n_dft,), P, P, reps, warm)
        t += cpu_run(kind, (("t4", ("dct4", "dst4"), False), ("t4", ("dct4", "dst4"), True)), (cls.n_t4,), P, P,
                     reps, warm)
        fd = 5.0 * cls.n_dft * math.log2(cls.n_dft)
        f4 = 2.5 * cls.n_t4 * math.log2(cls.n_t4)
        return t, (2 * fd + 4 * f4) * P * reps


class WorkloadLong1DC64(Workload3D256):
    """Complex DFT of 2^26 points in c64, forward then inverse: a Stockham
    chain of three passes over HBM.  --precision "tc_f16" / "tc_bf16" splits
    the chain into two 256-point tensor-core passes (the second pre-twiddled)
    and one 1024-point CUDA-core pass; "fp32" runs 512-, 512- and 256-point
    CUDA-core passes."""

    name = "long1d_c64"
    dims = (1 << 26,)
    nsets = 3
    seed = 5

    @classmethod
    def config(cls):
        return {"workload": "1-D complex DFT N=2^26 c64, forward then inverse", "dims": list(cls.dims),
                "precision": cls.precision, "flops": "5*N*log2(N) per transform, N=2^26",
                "inputs": "re/im i.i.d. uniform[-1,1), numpy PCG64 seeds 5..7",
                "l2": "inputs rotate over 3 sets of 512 MiB, larger than the 126 MB L2"}

    @classmethod
    def cpu_sample(cls, P):
        return f"{min(P, 4)} concurrent instances (one per OpenMP thread, own plans) of dft + invdft, per timed step"

    @classmethod
    def cpu_measure(cls, kind, threads, warm, reps):
        """A bounded sample: min(threads, 4) concurrent instances (a 2^26
        transform holds 2 GiB of host memory in the single build)."""
        P = min(threads, 4)
        t = cpu_run(kind, cls.cpu_sequences, cls.dims, P, P, reps, warm)
        n = int(np.prod(cls.dims))
        return t, 5.0 * n * math.log2(n) * 2 * P * reps


class WorkloadLong1DT4:
    """DCT-4 and DST-4 of 2^24 points in f32: a pre-rotation, the 2^23-point
    complex chain over HBM and a post-rotation.  --precision "tc_f16" /
    "tc_bf16" runs the chain as two 256-point tensor-core passes and one
    128-point CUDA-core pass; "fp32" as two 2048/4096-point CUDA-core passes."""

    name = "long1d_t4"
    dims = (1 << 24,)
    nsets = 3
    seed = 6
    dtype = "f32"
    precision = "fp32"

    def __init__(self, torch, dev):
        import minfft_b200

        self.torch = torch
        n = self.dims[0]
        self.flops_per_transform = 2.5 * n * math.log2(n)
        self.ops_per_step = 2
        self.eng = minfft_b200.engine(True)
        self.xs = [torch.from_numpy(uniform_f32(self.dims, self.seed + i)).to(dev) for i in range(self.nsets)]
        self.c = torch.empty(self.dims, dtype=torch.float32, device=dev)
        self.s = torch.empty(self.dims, dtype=torch.float32, device=dev)
        self.plan = self._mkplan()
        self.plan("dct4", self.xs[0].data_ptr(), self.c.data_ptr())
        self.plan("dst4", self.xs[0].data_ptr(), self.s.data_ptr())
        torch.cuda.synchronize()
        self.eng.tc_status(self.plan.aux)
        x = self.xs[0].cpu().numpy()
        acc = {}
        for op, y in (("dct4", self.c), ("dst4", self.s)):
            ref = oracle_real(self.name, self.seed, op, x, self.dims)
            acc[f"{op}_rel_l2_vs_fp64_oracle"] = float(np.linalg.norm(y.cpu().numpy().astype(np.float64) - ref) /
                                                       np.linalg.norm(ref))
        acc["oracle"] = oracle_kind_name()
        self.accuracy = acc

    def _mkplan(self):
        plan = self.eng.plan("t4", self.dims)
        self.eng.set_precision(plan.aux, self.precision)
        return plan

    def plans(self):
        yield self.eng, self.plan, ("dct4", "dst4")

    def rebuild(self, eng, plan):
        self.plan.free()
        self.plan = self._mkplan()

    def step(self, k):
        x = self.xs[k % self.nsets]
        self.plan("dct4", x.data_ptr(), self.c.data_ptr(), check=False)
        self.plan("dst4", x.data_ptr(), self.s.data_ptr(), check=False)

    def check_errors(self):
        self.eng.check()
        self.eng.tc_status(self.plan.aux)

    def launches_per_step(self):
        return sum(self.eng.launch_count(op, self.plan.aux) for op in ("dct4", "dst4"))

    def e2e_setup(self):
        t = self.torch
        self.hx = t.empty(self.dims, dtype=t.float32, pin_memory=True)
        self.hx.copy_(self.xs[0].cpu())
        self.e2e_sets = alternate_plan_sets(t, [self.plan, self._mkplan()], self.hx, 2)
        self.e2e_k = 0
        b = self.hx.numel() * 4
        return 2 * b, 2 * b

    def e2e_step(self):
        plan, (hc, hs) = next_plan_set(self)
        plan("dct4", self.hx.data_ptr(), hc.data_ptr(), check=False)
        plan("dst4", self.hx.data_ptr(), hs.data_ptr(), check=False)

    @classmethod
    def config(cls):
        return {"workload": "1-D DCT-4 + DST-4 N=2^24 f32", "dims": list(cls.dims), "precision": cls.precision,
                "flops": "2.5*N*log2(N) per transform, N=2^24",
                "inputs": "i.i.d. uniform[-1,1), numpy PCG64 seeds 6..8",
                "l2": "inputs rotate over 3 sets of 64 MiB; each step writes 128 MiB, beyond the 126 MB L2"}

    cpu_sequences = (("t4", ("dct4", "dst4"), True),)

    @classmethod
    def cpu_sample(cls, P):
        return f"{min(P, 8)} concurrent instances (one per OpenMP thread, own plans) of dct4 + dst4, per timed step"

    @classmethod
    def cpu_measure(cls, kind, threads, warm, reps):
        P = min(threads, 8)
        t = cpu_run(kind, cls.cpu_sequences, cls.dims, P, P, reps, warm)
        n = cls.dims[0]
        return t, 2.5 * n * math.log2(n) * 2 * P * reps


WORKLOADS = {"2d2048": Workload2D, "batch4096": WorkloadBatch4096, "mixed20000": WorkloadMixed,
             "3d256": Workload3D256, "long1d": WorkloadLong1D, "long1d_c64": WorkloadLong1DC64,
             "long1d_t4": WorkloadLong1DT4}


# -------------------------------------------------------------- CPU timing
def cpu_run(kind: str, sequences, dims, batch: int, threads: int, reps: int, warm: int = 1, seed: int = 1):
    """Seconds for `reps` timed sweeps (after `warm` untimed ones) of `batch`
    independent instances of every (family, ops) sequence, on `threads`
    OpenMP threads."""
    import ctypes

    import oracle

    oracle.build()
    cb = ctypes.CDLL(oracle.CPUBENCH_PATH)
    cb.cpubench_run.restype = ctypes.c_double
    cb.cpubench_run.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint]
    fam_code = {"dft": 0, "realdft": 1, "t2t3": 2, "t4": 3}
    op_code = {op: i for i, op in enumerate(("dft", "invdft", "realdft", "invrealdft", "dct2", "dst2", "dct3",
                                             "dst3", "dct4", "dst4"))}
    total = 0.0
    for fam, ops, single in sequences:
        path = oracle._PATHS[(kind, single)]
        arr_ops = (ctypes.c_int * len(ops))(*[op_code[o] for o in ops])
        arr_dims = (ctypes.c_int * len(dims))(*dims)
        t = cb.cpubench_run(path.encode(), int(single), fam_code[fam], len(ops), arr_ops, len(dims), arr_dims,
                            batch, threads, warm, reps, seed)
        if t < 0:
            raise RuntimeError(f"cpubench failed ({t}) for {fam} {ops}")
        total += t
    return total


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_kind():
    import oracle

    return oracle.best_kind()


# ------------------------------------------------------------- reference arm
def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    W = WORKLOADS[args.workload]
    if hasattr(W, "precision"):
        W.precision = args.precision
    if not hasattr(W, "cpu_measure"):
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU reference defined for workload {W.name}"}))
        return 0
    kind = cpu_kind()
    P = cpu_threads()
    t, flops = W.cpu_measure(kind, P, args.warmup, args.steps)
    value = flops / t / 1e9
    line = {"metric": "GFLOP/s (5N log2N complex, 2.5N log2N real-data)", "value": round(value, 3),
            "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1000 * t / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": W.dtype, "data": "synthetic",
            "config": _ref_config(W), "impl": "reference",
            "cpu_baseline": {"value": round(value, 3), "unit": "GFLOP/s", "cores": P, "kind": kind,
                             "sample": W.cpu_sample(P) if hasattr(W, "cpu_sample") else
                             f"{P} concurrent independent instances of the step (one per thread, own plans), "
                             f"per timed step"},
            "e2e": {"value": round(value, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def _ref_config(W):
    """The workload's config, identical to the engine arm's."""
    return W.config()


# ---------------------------------------------------------------- engine arm
def copy_floor_ms(torch, dev, h2d_bytes, d2h_bytes, reps=5):
    """Milliseconds to move one step's input bytes host->device and its
    output bytes device->host at the same time (pinned host memory, one
    stream per direction, no kernels): the transfer floor of an end-to-end
    step."""
    hi = torch.empty(max(int(h2d_bytes), 16), dtype=torch.uint8).pin_memory()
    di = torch.empty(hi.numel(), dtype=torch.uint8, device=dev)
    ho = torch.empty(max(int(d2h_bytes), 16), dtype=torch.uint8).pin_memory()
    do = torch.empty(ho.numel(), dtype=torch.uint8, device=dev)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def once():
        with torch.cuda.stream(s_in):
            di.copy_(hi, non_blocking=True)
        with torch.cuda.stream(s_out):
            ho.copy_(do, non_blocking=True)

    once()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(reps):
        once()
    torch.cuda.synchronize()
    return 1000 * (time.perf_counter() - t) / reps


def measure(torch, dev, dist, W, args, steps, warmup, e2e_seconds=5.0, cpu_seconds=10.0, cpu=True, e2e=True):
    """Tune, time and profile workload W; returns the fields of its JSON line."""
    rank, world, local = rank_info()
    tuned = 0
    tune_path = lambda eng: f"{args.tune_file}.{'f32' if eng.single else 'f64'}"  # noqa: E731
    if args.tune_file and list(W.plans()) and all(os.path.exists(tune_path(e)) for e, _, _ in W.plans()):
        # reuse a saved tuning table (e.g. for deterministic profiling runs)
        for eng, plan, ops in W.plans():
            eng.tune_load(tune_path(eng))
            tuned = max(tuned, eng.tune_size())
        for eng, plan, ops in list(W.plans()):
            W.rebuild(eng, plan)
    elif not args.no_tune:
        # project autotuner: pick kernel form, radix and tile size per launch (setup, untimed)
        for eng, plan, ops in W.plans():
            for op in ops:
                eng.autotune(plan.aux, op, getattr(W, "howmany_for", lambda o: 1)(op), 5)
            tuned = max(tuned, eng.tune_size())
        if hasattr(W, "tune"):
            tuned = W.tune()
        if args.tune_file:
            for eng, plan, ops in W.plans():
                eng.tune_save(tune_path(eng))
    launches_per_step = W.launches_per_step()

    # warm-up
    for k in range(warmup):
        W.step(k)
    torch.cuda.synchronize()
    W.check_errors()

    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    side = W.step_streams() if hasattr(W, "step_streams") else []
    with ClockSampler(local) as clocks:
        start.record()
        for st in side:  # workloads whose plans run on their own streams: fork ...
            st.wait_event(start)
        for k in range(steps):
            W.step(k)
        for st in side:  # ... and join before the end event
            torch.cuda.current_stream().wait_stream(st)
        end.record()
        end.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    W.check_errors()
    ms = max_over_ranks(dist, start.elapsed_time(end), dev)

    # the same steps again with launch-level timing (an event pair around
    # every launch on the plan's stream): per-kernel durations for the
    # roofline.  The events serialise consecutive launches, so these
    # durations are upper bounds and this pass is not the headline number.
    # Plans that run concurrently in the timed loop are put on one stream
    # here, so that each launch's duration is its own.
    prof_steps = min(steps, 500)
    if hasattr(W, "set_streams"):
        W.set_streams(False)
    for eng, plan, ops in W.plans():
        eng.profile(plan.aux, prof_steps * 8 + 64)
    torch.cuda.synchronize()
    for k in range(prof_steps):
        W.step(k)
    torch.cuda.synchronize()
    if hasattr(W, "set_streams"):
        W.set_streams(True)
    flops_step = W.flops_per_transform * W.ops_per_step
    value = job_gflops(flops_step, steps, world, ms / 1e3)

    # per-kernel statistics -> roofline of the dominant kernel
    stats = []
    for eng, plan, ops in W.plans():
        prec = "f32" if eng.single else "f64"
        for lab, cnt, tot, by in eng.profile_stats(plan.aux):
            stats.append((f"{prec} {lab}", cnt, tot, by))
        eng.profile(plan.aux, 0)
    if not stats and hasattr(W, "roofline_stats"):
        stats = W.roofline_stats(ms, steps)  # one launch per step: the timed region itself
    stats.sort(key=lambda r: -r[2])
    hbm, peak_src = peaks()
    roof = None
    if stats:
        lab, cnt, tot, by = stats[0]
        avg_ms = tot / cnt
        achieved = by / (avg_ms / 1e3) / 1e9
        traffic = None
        try:
            with open(TRAFFIC_PATH) as f:
                traffic = json.load(f).get(W.name, {}).get(lab)
        except Exception:
            traffic = None
        roof = {"bound": "hbm", "kernel": lab, "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_source": peak_src,
                "algorithmic_bytes_per_launch": by, "avg_launch_us": round(avg_ms * 1e3, 2),
                "traffic": traffic}
    kernel_table = [{"kernel": lab, "launches": cnt, "total_ms": round(tot, 3),
                     "share": round(tot / sum(s[2] for s in stats), 4),
                     "gbs": round(by / (tot / cnt / 1e3) / 1e9, 1)} for lab, cnt, tot, by in stats]

    # end to end through the C ABI with pinned host buffers
    e2e_rec = None
    if e2e and not args.no_e2e:
        h2d, d2h = W.e2e_setup()
        W.e2e_step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        W.e2e_step()
        torch.cuda.synchronize()
        est = time.perf_counter() - t0
        k_e2e = max(3, min(steps, int(e2e_seconds / max(est, 1e-4))))
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            W.e2e_step()
        torch.cuda.synchronize()
        el = max_over_ranks(dist, time.perf_counter() - t0, dev)
        W.check_errors()
        e2e_rec = {"value": round(job_gflops(flops_step, k_e2e, world, el), 3), "unit": "GFLOP/s",
                   "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": k_e2e,
                   "ms_per_step": round(1000 * el / k_e2e, 3)}
        floor = copy_floor_ms(torch, dev, h2d, d2h)
        e2e_rec["copy_floor_ms_per_step"] = round(floor, 3)
        e2e_rec["frac_of_copy_floor"] = round(floor / (1000 * el / k_e2e), 4)

    # CPU baseline (rank 0, one GPU only): the reference on the host cores
    cpu_rec = None
    if cpu and rank == 0 and world == 1 and not args.no_cpu and hasattr(W, "cpu_measure"):
        cpu_rec = cpu_baseline(W, cpu_seconds)

    rec = {"value": round(value, 3), "ms_per_step": round(ms / steps, 4), "steps": steps, "warmup": warmup,
           "dtype": W.dtype, "config": W.config(), "gpu_launches": int(launches_per_step * steps),
           "clocks": clocks.summary(), "autotuned_launch_configs": tuned, "roofline": roof, "e2e": e2e_rec,
           "cpu_baseline": cpu_rec, "kernels": kernel_table[:8]}
    if getattr(W, "accuracy", None):
        rec["accuracy"] = W.accuracy
    return rec


def cpu_baseline(W, seconds):
    """The reference library on all host cores for workload W: one sample,
    repeated up to about `seconds` of CPU work."""
    P = cpu_threads()
    kind = cpu_kind()
    reps = 1
    t, flops = W.cpu_measure(kind, P, 1, reps)
    if t < seconds / 2:
        reps = min(100, int(math.ceil(seconds / max(t, 1e-3))))
        t, flops = W.cpu_measure(kind, P, 1, reps)
    return {"value": round(flops / t / 1e9, 3), "unit": "GFLOP/s", "cores": P, "kind": kind,
            "sample": (W.cpu_sample(P) if hasattr(W, "cpu_sample") else
                       f"{P} concurrent independent instances of one step (one per OpenMP thread, own plans)")
            + f", {reps} timed repetition(s), {t:.1f} s"}


# Every other workload of the benchmark, measured briefly after the headline
# (one GPU only): (label, workload, precision).
SUB_CONFIGS = (("batch4096", "batch4096", None),
               ("3d256_fp32", "3d256", "fp32"), ("3d256_tc_f16", "3d256", "tc_f16"),
               ("3d256_tc_bf16", "3d256", "tc_bf16"),
               ("mixed20000", "mixed20000", None),
               ("long1d", "long1d", None),
               ("long1d_c64_fp32", "long1d_c64", "fp32"), ("long1d_c64_tc_f16", "long1d_c64", "tc_f16"),
               ("long1d_c64_tc_bf16", "long1d_c64", "tc_bf16"),
               ("long1d_t4_fp32", "long1d_t4", "fp32"), ("long1d_t4_tc_f16", "long1d_t4", "tc_f16"),
               ("long1d_t4_tc_bf16", "long1d_t4", "tc_bf16"))


def single_thread_reference():
    """Seconds per call of the reference on ONE host thread for the
    single-transform workloads (2048^2 real/trig, 256^3 complex, 2^26 complex
    and 2^24 type-4): one untimed and one timed call each."""
    out = {}
    kind = cpu_kind()
    cases = (("2d2048 realdft f64", "realdft", ("realdft",), (2048, 2048), False),
             ("2d2048 invrealdft f64", "realdft", ("invrealdft",), (2048, 2048), False),
             ("2d2048 dct2 f64", "t2t3", ("dct2",), (2048, 2048), False),
             ("2d2048 dct3 f64", "t2t3", ("dct3",), (2048, 2048), False),
             ("2d2048 realdft f32", "realdft", ("realdft",), (2048, 2048), True),
             ("2d2048 dct2 f32", "t2t3", ("dct2",), (2048, 2048), True),
             ("3d256 dft c64", "dft", ("dft",), (256, 256, 256), True),
             ("long1d dft 2^26 c128", "dft", ("dft",), (1 << 26,), False),
             ("long1d dft 2^26 c64", "dft", ("dft",), (1 << 26,), True),
             ("long1d dct4 2^24 f64", "t4", ("dct4",), (1 << 24,), False),
             ("long1d dct4 2^24 f32", "t4", ("dct4",), (1 << 24,), True))
    for label, fam, ops, dims, single in cases:
        t = cpu_run(kind, ((fam, ops, single),), dims, 1, 1, 1, 1)
        n = int(np.prod(dims))
        f = (5.0 if fam == "dft" else 2.5) * n * math.log2(n)
        out[label] = {"ms_per_call": round(1000 * t, 2), "gflops": round(f / t / 1e9, 3)}
    return {"kind": kind, "threads": 1, "calls": out}


def run_engine(args):
    import torch

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    WC = WORKLOADS[args.workload]
    if hasattr(WC, "precision"):
        WC.precision = args.precision
    W = WC(torch, dev)
    rec = measure(torch, dev, dist, W, args, args.steps, args.warmup)
    del W
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    configs = None
    single_ref = None
    if world == 1 and not args.no_configs and args.workload == "2d2048" and args.precision == "fp32":
        configs = {}
        base_vals = {}
        for label, wname, prec in SUB_CONFIGS:
            WS = WORKLOADS[wname]
            if prec is not None:
                WS.precision = prec
            w = WS(torch, dev)
            r = measure(torch, dev, None, w, args, args.sub_steps, 3, e2e_seconds=1.0, cpu_seconds=3.0,
                        cpu=(prec in (None, "fp32")))
            entry = {"value": r["value"], "ms_per_step": r["ms_per_step"], "steps": r["steps"],
                     "config": r["config"], "dtype": r["dtype"], "gpu_launches": r["gpu_launches"],
                     "roofline_frac": r["roofline"]["frac"] if r["roofline"] else None,
                     "top_kernel": r["roofline"]["kernel"] if r["roofline"] else None,
                     "top_kernel_gbs": r["roofline"]["achieved"] if r["roofline"] else None,
                     "e2e": r["e2e"], "reference_cpu": r["cpu_baseline"], "clocks": r["clocks"]}
            if "accuracy" in r:
                entry["accuracy"] = r["accuracy"]
            if prec == "fp32":
                base_vals[wname] = r["value"]
            elif prec is not None and wname in base_vals:
                entry["tc_vs_fp32"] = round(r["value"] / base_vals[wname], 4)
            configs[label] = entry
            del w
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        WC.precision = args.precision
        if not args.no_cpu:
            single_ref = single_thread_reference()

    if rank == 0:
        line = {"metric": "GFLOP/s (5N log2N complex, 2.5N log2N real-data)", "value": rec["value"],
                "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": rec["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": rec["dtype"],
                "data": "synthetic", "config": rec["config"], "parallelism": f"replicas x{world}",
                "gpu_launches": rec["gpu_launches"], "clocks": rec["clocks"],
                "autotuned_launch_configs": rec["autotuned_launch_configs"],
                "roofline": rec["roofline"], "e2e": rec["e2e"], "cpu_baseline": rec["cpu_baseline"],
                "kernels": rec["kernels"]}
        if "accuracy" in rec:
            line["accuracy"] = rec["accuracy"]
        if configs is not None:
            line["configs"] = configs
        if single_ref is not None:
            line["reference_single_thread"] = single_ref
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="2d2048")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (heuristic launch configurations)")
    ap.add_argument("--tune-file", default="", help="tuning table prefix: loaded if present, else saved after tuning")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the short runs of the other workloads after the default headline")
    ap.add_argument("--sub-steps", type=int, default=10, help="timed steps of each other workload")
    ap.add_argument("--precision", choices=["fp32", "tc_f16", "tc_bf16"], default="fp32",
                    help="3d256, long1d_c64, long1d_t4: arithmetic of the 256-point axis passes")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
