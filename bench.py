#!/usr/bin/env python
"""Throughput of the batched scalar spherical harmonic roundtrip on B200.

Workload: 64 scalar fields on a Gauss-Legendre grid, lmax = mmax = 1023,
nlat = 1024, nlon = 2048, orthonormal + Condon-Shortley. One step = one
synthesis of all fields followed by one analysis of the resulting grids
(one "roundtrip" per field). Inputs: synthetic coefficients ~ N(0,1)/(l+1)
(seeded, imag = 0 at m = 0), resident in HBM; every buffer (1 GB of FP64
coefficients, 1 GB of grids) is larger than the 126 MB L2, so no flush is needed.

Paths: "mixed" (tensor-core Legendre GEMMs, FP32 I/O) and "fp64" (plain FP64).
The headline value is the default path; the other path is measured too.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--path mixed|fp64]
  python bench.py --workload uneven     # 256 mixed-size roundtrips as one grouped graph launch

Multi-GPU (torchrun): every rank transforms its own 64 fields (weak scaling, no
collective in the data path); timing is the max over ranks of the device time.
--impl reference times the reference CPU algorithm (the oracle's C port,
all host threads) on a bounded sample of the same workload.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "shtnskit.jl_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "roundtrips/s, lmax=1023×64 fields: mixed vs FP64 GPU @≤1e-6 rel L2; % roofline"
UNIT = "roundtrips/s"
LMAX, NLAT, NLON, NFIELDS = 1023, 1024, 2048, 64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--path", choices=["auto", "mixed", "fp64"], default="auto")
    ap.add_argument("--lmax", type=int, default=LMAX)
    ap.add_argument("--nfields", type=int, default=NFIELDS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-chunks", type=int, default=4, help="field chunks of the pipelined end-to-end step")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", choices=["batched", "uneven"], default="batched",
                    help="batched: the headline 64-field lmax=1023 roundtrip; uneven: 256 roundtrips of "
                         "mixed sizes (lmax uniform in 31..511, seed 7) as one grouped graph launch")
    return ap.parse_args()


def alg_flops_per_field_direction(lmax: int, nlat: int, nlon: int) -> tuple[float, float]:
    """(Legendre, FFT) algorithmic flops of one field in one direction:
    4 * (nlat/2) * nlm for the folded contraction, 2.5 nlat nlon log2 nlon for the real FFT."""
    import math

    nlm = (lmax + 1) * (lmax + 2) // 2
    return 4.0 * (nlat // 2) * nlm, 2.5 * nlat * nlon * math.log2(nlon)


# ---------------------------------------------------------------------------
# clocks sampler
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.gpu_id is not None:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            pass
    return {}


def fp64_peak_tflops(torch, dev) -> float:
    """Measured FP64 peak: cuBLAS DGEMM 4096^3, best of 5 (CUDA events)."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def traffic_table() -> dict:
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            return {}
    return {}


def make_inputs(torch, sht, cfg, nf, dev, seed, complex_dtype):
    """Coefficients ~ N(0,1)/(l+1), imag 0 at m=0, zero for l<m, in column-major layout."""
    g = torch.Generator(device=dev).manual_seed(seed)
    L, M = cfg.lmax, cfg.mmax
    a = sht.julia_empty((L + 1, M + 1, nf), complex_dtype, dev)
    re = torch.randn((nf, M + 1, L + 1), dtype=torch.float64, device=dev, generator=g)
    im = torch.randn((nf, M + 1, L + 1), dtype=torch.float64, device=dev, generator=g)
    l = torch.arange(L + 1, device=dev, dtype=torch.float64)
    mm = torch.arange(M + 1, device=dev).view(-1, 1)
    ll = torch.arange(L + 1, device=dev).view(1, -1)
    mask = (ll >= mm).to(torch.float64)
    re = re / (l + 1.0) * mask
    im = im / (l + 1.0) * mask
    im[:, 0, :] = 0
    a.permute(2, 1, 0).copy_(torch.complex(re, im).to(complex_dtype))
    return a


# ---------------------------------------------------------------------------
# reference arm: the oracle's C port of the reference CPU path
# ---------------------------------------------------------------------------
def cpu_sample(lmax, nlat, nlon, nfields_sample, steps=1, warmup=0):
    import numpy as np

    from oracle import c_oracle as co
    from oracle import sht_oracle as so

    cfg = so.create_gauss_config(lmax, nlat, nlon=nlon)
    rng = np.random.default_rng(0)
    shape = (lmax + 1, lmax + 1, nfields_sample)
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / (np.arange(lmax + 1)[:, None, None] + 1.0)
    a[:, 0, :] = a[:, 0, :].real
    for m in range(lmax + 1):
        a[:m, m, :] = 0
    cores = co.max_threads()
    for _ in range(warmup):
        co.analysis_batch(cfg, co.synthesis_batch(cfg, a))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        f = co.synthesis_batch(cfg, a)
        co.analysis_batch(cfg, f)
        times.append(time.perf_counter() - t0)
    return times, cores


# Fields per CPU roundtrip sample: the reference's batch path computes each P-bar row once per
# (m, latitude) and reuses it for every field of the call (src/batch_transforms.jl:403-425), so
# the sample must hold enough fields for that reuse to be amortised as in the full batch.
CPU_SAMPLE_FIELDS = 16


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    nsample = min(CPU_SAMPLE_FIELDS, args.nfields)
    times, cores = cpu_sample(args.lmax, args.lmax + 1, 2 * (args.lmax + 1), nsample, steps=args.steps,
                              warmup=min(args.warmup, 1))
    t = statistics.median(times)
    value = nsample / t
    sample = (f"{nsample} of {args.nfields} fields per step, one batched roundtrip (P-bar rows shared by "
              f"the {nsample} fields), full lmax={args.lmax} {args.lmax + 1}x{2 * (args.lmax + 1)} grid, "
              f"median of {len(times)} steps after {min(args.warmup, 1)} warm-up")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"batched scalar roundtrip, lmax={args.lmax}, {args.nfields} fields",
                       "engine": "reference CPU algorithm restated in C (oracle/sht_oracle.c), POSIX threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    import shtb200 as sht
    from shtb200 import _lib
    from shtb200 import transforms as T

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from shtb200.distributed import barrier
    from shtb200.distributed import max_over_ranks as _max

    def max_over_ranks(v: float) -> float:
        return _max(v, dev)

    L, nf = args.lmax, args.nfields
    nlat, nlon = L + 1, 2 * (L + 1)
    cfg = sht.create_gauss_config(L, nlat, nlon=nlon)
    plan = cfg.plan(local)
    base_table_bytes = plan.table_bytes()
    paths = ["fp64"]
    mixed_ok = True
    try:
        probe = sht.create_gauss_config(7, 8, nlon=16)
        sht.synthesis(probe, torch.zeros((8, 8), dtype=torch.complex64, device=dev), precision="mixed")
    except sht.BackendUnavailableError:
        mixed_ok = False
    if mixed_ok:
        paths = ["mixed", "fp64"]
    head = args.path if args.path != "auto" else paths[0]
    if head == "mixed" and not mixed_ok:
        raise SystemExit("mixed path not available in this build")

    results = {}
    a64 = make_inputs(torch, sht, cfg, nf, dev, 1234 + rank, torch.complex128)
    lib = _lib.load()

    def run_path(path, timed=True):
        prec = _lib.SHTB_PREC_MIXED if path == "mixed" else _lib.SHTB_PREC_FP64
        rt = torch.float32 if path == "mixed" else torch.float64
        ct = torch.complex64 if path == "mixed" else torch.complex128
        a_in = a64 if path == "fp64" else sht.julia_empty(a64.shape, ct, dev).copy_(a64)
        f = sht.julia_empty((nlat, nlon, nf), rt, dev)
        a_out = sht.julia_empty(a64.shape, ct, dev)
        dcode = _lib.SHTB_F32 if path == "mixed" else _lib.SHTB_F64
        nb = max(plan.workspace_bytes(_lib.SHTB_OP_SYNTHESIS, nf, dcode, prec),
                 plan.workspace_bytes(_lib.SHTB_OP_ANALYSIS, nf, dcode, prec))
        ws = torch.empty(nb, dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream

        def step():
            _lib.check(lib.shtb_synthesis(plan.handle, a_in.data_ptr(), f.data_ptr(), nf, L, dcode, prec,
                                          ws.data_ptr(), nb, stream), "synthesis")
            _lib.check(lib.shtb_analysis(plan.handle, f.data_ptr(), a_out.data_ptr(), nf, L, dcode, prec,
                                         ws.data_ptr(), nb, stream), "analysis")

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        # accuracy of this path's roundtrip against its own input (size-independent check)
        err = float(torch.linalg.vector_norm((a_out.to(torch.complex128) - a64).flatten()) /
                    torch.linalg.vector_norm(a64.flatten()))
        out = {"roundtrip_rel_l2": err, "a_out": a_out, "f": f}
        if not timed:
            return out
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(os.environ.get("SHTB_SMI_INDEX"))
        sampler.start()
        time.sleep(0.3)
        lib.shtb_launch_count(1)
        _lib.profile_enable(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        clocks = sampler.stop()
        launches = int(lib.shtb_launch_count(1))
        prof = _lib.profile_read()
        _lib.profile_enable(False)
        ms = e0.elapsed_time(e1) / args.steps
        out.update(ms=max_over_ranks(ms), clocks=clocks, launches=launches, prof=prof)
        return out

    for p in paths:
        results[p] = run_path(p)
    r = results[head]
    ms = r["ms"]
    value = nf * world * 1000.0 / ms

    # accuracy of the headline path against the FP64 path on the same inputs
    rel_vs_fp64 = None
    if head == "mixed":
        fp = results["fp64"]
        rel_vs_fp64 = {
            "grid": float(torch.linalg.vector_norm((r["f"].to(torch.float64) - fp["f"]).flatten()) /
                          torch.linalg.vector_norm(fp["f"].flatten())),
            "coefficients": float(torch.linalg.vector_norm((r["a_out"].to(torch.complex128) - fp["a_out"]).flatten()) /
                                  torch.linalg.vector_norm(fp["a_out"].flatten())),
        }

    # roofline of the dominant kernel of the headline path
    Fleg, Ffft = alg_flops_per_field_direction(L, nlat, nlon)
    prof = r["prof"]
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_tot, dom_cnt) = dom
    dom_avg_ms = dom_tot / dom_cnt
    peaks = measured_peaks()
    traffic = traffic_table().get(f"{head}:{dom_name}")
    esz = 4 if head == "mixed" else 8
    grid_bytes = nf * nlat * nlon * esz
    coef_bytes = nf * (L + 1) * (L + 1) * 2 * esz
    fourier_bytes = nf * (L + 1) * 2 * (nlat // 2) * 2 * esz
    if "legendre" in dom_name or "gemm" in dom_name:
        flops = Fleg * nf
        if head == "mixed":
            # fp16x3 on kind::f16: three f16 products per logical product, against the
            # dense f16/bf16 tensor peak (the same rate for both types)
            peak = peaks.get("bf16_tflops") or 1590.0
            issued = 3.0 * flops
            roof = {"bound": "tensor", "achieved": issued / (dom_avg_ms * 1e-3) / 1e12, "peak": peak,
                    "unit": "TFLOP/s",
                    "peak_source": "measured (MEASURED_PEAKS.json bf16_tflops, cuBLAS bf16 8192^3 burst)" if peaks
                    else "fallback 1.59 PFLOP/s",
                    "algorithmic_per_launch": f"{issued:.4g} issued f16 flop = 3 x {nf} fields x 4*(nlat/2)*nlm"}
            # the same launch seen from HBM: P table + coefficients + Fourier buffer
            tab = (plan.table_bytes() - base_table_bytes) / 2   # one of the two tile images
            hbm_bytes = coef_bytes + fourier_bytes + tab
            roof["hbm_view"] = {"achieved": hbm_bytes / (dom_avg_ms * 1e-3) / 1e9,
                                "peak": peaks.get("hbm_gbs") or 6650.0, "unit": "GB/s",
                                "bytes_per_launch": hbm_bytes}
            roof["hbm_view"]["frac"] = roof["hbm_view"]["achieved"] / roof["hbm_view"]["peak"]
        else:
            peak = fp64_peak_tflops(torch, dev)
            roof = {"bound": "fp64", "achieved": flops / (dom_avg_ms * 1e-3) / 1e12, "peak": peak,
                    "unit": "TFLOP/s", "peak_source": "measured cuBLAS DGEMM 4096^3 on this GPU",
                    "algorithmic_per_launch": f"{flops:.4g} flop = {nf} fields x 4*(nlat/2)*nlm"}
        roof["frac"] = roof["achieved"] / roof["peak"]
    else:
        byts = grid_bytes + fourier_bytes
        peak = peaks.get("hbm_gbs") or 6650.0
        roof = {"bound": "hbm", "achieved": byts / (dom_avg_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                "peak_source": "measured" if peaks else "fallback"}
        roof["frac"] = roof["achieved"] / roof["peak"]
    roof["kernel"] = dom_name
    roof["avg_launch_ms"] = dom_avg_ms
    roof["traffic"] = traffic
    kernels = {k: {"avg_ms": t / c, "launches": c, "share": t / sum(v[0] for v in prof.values())}
               for k, (t, c) in prof.items()}

    # FP64 path against the FP64 pipe: algorithmic flops of the whole step (Legendre + FFT,
    # both directions) and of each Legendre kernel, over the measured cuBLAS DGEMM rate and
    # over the nominal DFMA rate (148 SMs x 64 FMA/clock x 2 x the max SM clock)
    fp64_roof = None
    if "fp64" in results:
        rf = results["fp64"]
        dgemm = fp64_peak_tflops(torch, dev)
        smx = (r["clocks"] or {}).get("sm_max_mhz") or 1965.0
        nominal = 148 * 64 * 2 * smx * 1e6 / 1e12
        step_flops = nf * 2.0 * (Fleg + Ffft)
        ach = step_flops / (rf["ms"] * 1e-3) / 1e12
        fp64_roof = {"bound": "fp64", "unit": "TFLOP/s", "achieved": ach, "peak": dgemm,
                     "peak_source": "measured cuBLAS DGEMM 4096^3 on this GPU", "frac": ach / dgemm,
                     "nominal_peak": nominal, "frac_of_nominal": ach / nominal,
                     "algorithmic_per_step": f"{step_flops:.4g} flop = {nf} fields x 2 x (4*(nlat/2)*nlm + "
                                             f"2.5*nlat*nlon*log2(nlon))",
                     "kernels": {}}
        for k, (t, c) in rf["prof"].items():
            ent = {"avg_ms": t / c, "launches": c}
            if "legendre" in k:
                a = nf * Fleg / (t / c * 1e-3) / 1e12
                ent.update(achieved_tflops=a, frac=a / dgemm, frac_of_nominal=a / nominal)
            elif "fft" in k:
                gb = (nf * nlat * nlon * 8 + nf * (L + 1) * 2 * (nlat // 2) * 16) / (t / c * 1e-3) / 1e9
                hb = peaks.get("hbm_gbs") or 6650.0
                ent.update(achieved_gbs=gb, frac_hbm=gb / hb)
            fp64_roof["kernels"][k] = ent

    # end to end through the public API with host buffers (pinned), per step:
    # H2D of the coefficients, synthesis_batch + analysis_batch, D2H of the recovered coefficients.
    # The fields go in chunks on three streams (copy in / compute / copy out), so the two
    # PCIe directions and the kernels overlap, within a step and across steps.
    e2e = None
    if not args.no_e2e:
        ct = torch.complex64 if head == "mixed" else torch.complex128
        host_in = torch.empty(a64.permute(2, 1, 0).shape, dtype=ct, pin_memory=True)
        host_in.copy_(a64.permute(2, 1, 0).to(ct).cpu())
        host_out = torch.empty_like(host_in, pin_memory=True)
        a_dev = sht.julia_empty(a64.shape, ct, dev)
        nchunk = max(1, min(args.e2e_chunks, nf))
        bounds = [(c * nf // nchunk, (c + 1) * nf // nchunk) for c in range(nchunk)]
        s_in, s_cmp, s_out = (torch.cuda.Stream(dev) for _ in range(3))
        ev_in = [torch.cuda.Event() for _ in bounds]
        ev_cmp = [torch.cuda.Event() for _ in bounds]

        def e2e_step():
            for c, (c0, c1) in enumerate(bounds):
                with torch.cuda.stream(s_in):
                    s_in.wait_event(ev_cmp[c])   # the previous step's compute has read this chunk
                    a_dev.permute(2, 1, 0)[c0:c1].copy_(host_in[c0:c1], non_blocking=True)
                    ev_in[c].record(s_in)
                with torch.cuda.stream(s_cmp):
                    s_cmp.wait_event(ev_in[c])
                    f = sht.synthesis_batch(cfg, a_dev[:, :, c0:c1], precision=head)
                    b = sht.analysis_batch(cfg, f, precision=head)
                    ev_cmp[c].record(s_cmp)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(ev_cmp[c])
                    host_out[c0:c1].copy_(b.permute(2, 1, 0), non_blocking=True)
                    b.record_stream(s_out)

        main = torch.cuda.current_stream(dev)
        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        k = max(3, min(args.steps, 10))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for st in (s_in, s_cmp, s_out):
            st.wait_stream(main)
        for _ in range(k):
            e2e_step()
        for st in (s_in, s_cmp, s_out):
            main.wait_stream(st)
        e1.record(main)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1) / k)
        err_e2e = float(torch.linalg.vector_norm((host_out.to(torch.complex128) - a64.permute(2, 1, 0).cpu()).flatten()) /
                        torch.linalg.vector_norm(a64.flatten().cpu()))
        nbytes = host_in.numel() * host_in.element_size()
        e2e = {"value": nf * world * 1000.0 / ems, "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "ms_per_step": ems,
               "pipeline": f"{nchunk} field chunks, H2D / synthesis_batch + analysis_batch / D2H on three streams",
               "roundtrip_rel_l2": err_e2e}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ns = min(CPU_SAMPLE_FIELDS, nf)
        times, cores = cpu_sample(L, nlat, nlon, ns, steps=5, warmup=1)
        cpu = {"value": ns / statistics.median(times), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{ns} of {nf} fields per batched roundtrip (P-bar rows shared by the {ns} fields), "
                         f"full lmax={L} {nlat}x{nlon} grid, median of 5 after 1 warm-up "
                         f"(oracle/sht_oracle.c, reference CPU algorithm)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-io/fp16x3-tc" if head == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": f"batched scalar roundtrip (synthesis+analysis), lmax=mmax={L}, nlat={nlat}, "
                                   f"nlon={nlon}, {nf} fields per GPU, Gauss grid, orthonormal+CS",
                       "path": head, "roundtrip": "one field synthesized and analyzed",
                       "l2_flush": "inputs larger than L2 (>1 GB per buffer)", "parallelism": f"fields x{world}"},
            "roofline": roof, "kernels": kernels,
            "cpu_baseline": cpu, "clocks": r["clocks"], "e2e": e2e, "gpu_launches": r["launches"],
            "accuracy": {"roundtrip_rel_l2": r["roundtrip_rel_l2"], "vs_fp64_gpu": rel_vs_fp64},
            "paths": {p: {"value": nf * world * 1000.0 / results[p]["ms"], "ms_per_step": results[p]["ms"],
                          "roundtrip_rel_l2": results[p]["roundtrip_rel_l2"]} for p in results},
        }
        if fp64_roof is not None:
            line["paths"]["fp64"]["roofline"] = fp64_roof
        if "mixed" in results and "fp64" in results:
            line["paths"]["mixed_over_fp64"] = results["fp64"]["ms"] / results["mixed"]["ms"]
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# uneven batches: 256 independent roundtrips of mixed sizes
# ---------------------------------------------------------------------------
UNEVEN_METRIC = ("transforms/s, uneven batch: 256 scalar roundtrips, lmax uniform in 31..511 (seed 7), "
                 "nlat=lmax+1, nlon=smallest 2^a3^b5^c>=2(lmax+1), mixed precision")
UNEVEN_UNIT = "transforms/s"
UNEVEN_N = 256


def uneven_lmaxes(n=UNEVEN_N, seed=7):
    import numpy as np

    return [int(v) for v in np.random.default_rng(seed).integers(31, 512, size=n)]


def pct(v, q):
    import numpy as np

    return float(np.percentile(np.asarray(v, dtype=float), q))


def run_uneven_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from shtb200.group import smooth_nlon

    lm = uneven_lmaxes()[:16]
    cores = 1
    t_all, per = 0.0, []
    for l in lm:
        times, cores = cpu_sample(l, l + 1, smooth_nlon(l), 1, steps=1)
        per.append(times[0] * 1e3)
        t_all += times[0]
    value = len(lm) / t_all
    sample = f"first {len(lm)} of {UNEVEN_N} members (1 field each), one roundtrip each, sequential"
    line = {"impl": "reference", "metric": UNEVEN_METRIC, "value": value, "unit": UNEVEN_UNIT, "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": t_all * 1e3 * UNEVEN_N / len(lm), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "uneven batch (sample)", "engine": "oracle/sht_oracle.c, POSIX threads"},
            "latency_ms": {"p50": pct(per, 50), "p99": pct(per, 99)},
            "cpu_baseline": {"value": value, "unit": UNEVEN_UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNEVEN_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_uneven(args):
    import torch
    import torch.distributed as dist

    import shtb200 as sht
    from shtb200 import _lib
    from shtb200 import transforms as T
    from shtb200.group import UnevenBatch, smooth_nlon

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from shtb200.distributed import max_over_ranks as _max

    def max_over_ranks(v: float) -> float:
        return _max(v, dev)

    lib = _lib.load()
    lmaxes = uneven_lmaxes()
    cfgs = [sht.create_gauss_config(l, l + 1, nlon=smooth_nlon(l)) for l in lmaxes]
    batch = UnevenBatch(cfgs, 1, local)
    for t, (c, a) in enumerate(zip(cfgs, batch.alm_in)):
        a.copy_(make_inputs(torch, sht, c, 1, dev, 7000 + t + 100000 * rank, torch.complex64))
    shape = batch.autotune()
    for _ in range(max(args.warmup, 3)):
        batch.roundtrip()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(os.environ.get("SHTB_SMI_INDEX"))
    sampler.start()
    time.sleep(0.3)
    lib.shtb_launch_count(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        batch.roundtrip()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = int(lib.shtb_launch_count(1))
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    batch.status()
    lat = batch.latencies_ns() / 1e6
    err = max(float(torch.linalg.vector_norm((o - i).flatten()) / torch.linalg.vector_norm(i.flatten()))
              for i, o in zip(batch.alm_in, batch.alm_out))

    # the same 256 roundtrips launched one transform at a time (4 kernels each), back to back
    outs = [(sht.julia_empty((c.nlat, c.nlon, 1), torch.float32, dev),
             sht.julia_empty((c.lmax + 1, c.mmax + 1, 1), torch.complex64, dev)) for c in cfgs]

    def separate(record):
        for t, c in enumerate(cfgs):
            if record:
                ev[t][0].record()
            T.synthesis_device(c, batch.alm_in[t], outs[t][0], c.lmax, _lib.SHTB_PREC_MIXED)
            T.analysis_device(c, outs[t][0], outs[t][1], c.lmax, _lib.SHTB_PREC_MIXED)
            if record:
                ev[t][1].record()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in cfgs]
    separate(False)
    torch.cuda.synchronize()
    separate(True)
    torch.cuda.synchronize()
    sep_lat = [a.elapsed_time(b) for a, b in ev]
    sep_total = ev[0][0].elapsed_time(ev[-1][1])
    same = all(torch.equal(outs[t][1], batch.alm_out[t]) for t in range(len(cfgs)))

    # end to end: pinned host inputs in, recovered coefficients out, every step. Two batches
    # (two sets of device buffers and graphs) alternate, so one batch's copies overlap the
    # other's roundtrip: copy-in, compute and copy-out run on three streams.
    e2e = None
    if not args.no_e2e:
        hin = [torch.empty(a.permute(2, 1, 0).shape, dtype=torch.complex64, pin_memory=True) for a in batch.alm_in]
        hout = [[torch.empty_like(h, pin_memory=True) for h in hin] for _ in range(2)]
        for h, a in zip(hin, batch.alm_in):
            h.copy_(a.permute(2, 1, 0).cpu())
        batch2 = UnevenBatch(cfgs, 1, local)
        batch2.autotune()
        pair = (batch, batch2)
        s_in, s_cmp, s_out = (torch.cuda.Stream(dev) for _ in range(3))
        ev_in = [torch.cuda.Event() for _ in pair]
        ev_cmp = [torch.cuda.Event() for _ in pair]
        ev_out = [torch.cuda.Event() for _ in pair]
        step_no = [0]

        def e2e_step():
            b = step_no[0] & 1
            step_no[0] += 1
            bt = pair[b]
            with torch.cuda.stream(s_in):
                s_in.wait_event(ev_cmp[b])       # this batch's previous roundtrip has read its inputs
                for h, a in zip(hin, bt.alm_in):
                    a.permute(2, 1, 0).copy_(h, non_blocking=True)
                ev_in[b].record(s_in)
            with torch.cuda.stream(s_cmp):
                s_cmp.wait_event(ev_in[b])
                s_cmp.wait_event(ev_out[b])      # its previous results have been copied out
                bt.roundtrip()
                ev_cmp[b].record(s_cmp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_cmp[b])
                for h, a in zip(hout[b], bt.alm_out):
                    h.copy_(a.permute(2, 1, 0), non_blocking=True)
                ev_out[b].record(s_out)

        main_s = torch.cuda.current_stream(dev)
        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        k = max(4, min(args.steps, 10)) // 2 * 2
        e0.record(main_s)
        for st in (s_in, s_cmp, s_out):
            st.wait_stream(main_s)
        for _ in range(k):
            e2e_step()
        for st in (s_in, s_cmp, s_out):
            main_s.wait_stream(st)
        e1.record(main_s)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1) / k)
        e2e_err = max(float(torch.linalg.vector_norm((o.to(torch.complex128) - i.to(torch.complex128)).flatten()) /
                            torch.linalg.vector_norm(i.to(torch.complex128).flatten()))
                      for i, o in zip(hin, hout[(step_no[0] - 1) & 1]))
        nbytes = sum(h.numel() * h.element_size() for h in hin)
        e2e = {"value": UNEVEN_N * world * 1000.0 / ems, "unit": UNEVEN_UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "ms_per_step": ems,
               "pipeline": "two alternating batches; H2D / grouped roundtrip / D2H on three streams",
               "roundtrip_rel_l2_max": e2e_err}
        batch2.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        lm = lmaxes[:8]
        tot, cores = 0.0, 1
        for l in lm:
            times, cores = cpu_sample(l, l + 1, smooth_nlon(l), 1, steps=1)
            tot += times[0]
        cpu = {"value": len(lm) / tot, "unit": UNEVEN_UNIT, "cores": cores, "kind": "port",
               "sample": f"first {len(lm)} of {UNEVEN_N} members, one roundtrip each (oracle/sht_oracle.c)"}

    if rank == 0:
        line = {
            "metric": UNEVEN_METRIC, "value": UNEVEN_N * world * 1000.0 / ms, "unit": UNEVEN_UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-io/fp16x3-tc", "data": "synthetic",
            "config": {"workload": f"{UNEVEN_N} independent scalar roundtrips per GPU, one field each, lmax drawn "
                                   "uniformly from 31..511 (seed 7), Gauss grid nlat=lmax+1, smooth nlon",
                       "launch": "persistent grouped stages in one CUDA graph (shtb_group_roundtrip)",
                       "autotuned_shape": {"fft_pairs_per_cta": shape[0], "fft_ctas": shape[1],
                                           "gemm_ctas": shape[2]},
                       "l2_flush": "none; the batch (~0.3 GB of buffers) is replayed as is",
                       "parallelism": f"batches x{world}"},
            "latency_ms": {"grouped": {"p50": pct(lat, 50), "p99": pct(lat, 99), "max": float(lat.max())},
                           "separate": {"p50": pct(sep_lat, 50), "p99": pct(sep_lat, 99),
                                        "total_ms": sep_total,
                                        "transforms_per_s": UNEVEN_N * 1000.0 / sep_total}},
            "speedup_vs_separate": sep_total / ms, "results_equal_separate": same,
            "accuracy": {"roundtrip_rel_l2_max": err},
            "cpu_baseline": cpu, "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.workload == "uneven":
        if args.impl == "reference":
            run_uneven_reference(args)
        else:
            run_uneven(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
