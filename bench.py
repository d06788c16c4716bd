"""Benchmark of the Cholesky-vector RPA energy path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one RPA correlation energy of one system):
  single_4096: NQ = 4096 Cholesky vectors, NOcc = 64, NVirt = 1024
  (nov = 65536), K = 16 frequencies; synthetic seeded inputs (R = 2.15 GB
  FP64, larger than L2, so no L2 flush is needed between steps).
  Pi(u) in split-BF16 on the tcgen05 tensor cores, FP64 Cholesky log-det,
  double-double quadrature sum.
  N > 1 (torchrun): every rank computes its own independent system (weak
  scaling, no data-path collective); time = max over ranks.

--impl reference times the reference-equivalent CPU restatement (oracle/,
numpy + ILP64 OpenBLAS: 500-column DGEMM blocks per frequency + DGEQRF
log-det, as src/rpa/rpa_THC.f90:313-339 and
src/linear-algebra/real_linalg.f90:793-825 do) on the host cores, on a
bounded sample per step, extrapolated to the full workload.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
METRIC = "RPA E_c/s & Π-build TFLOP/s: split-BF16 vs FP64 on 1 B200 at |ΔE|≤1e-7 Eh"
WORKLOAD = "single_4096"  # default measured workload; --workload selects another (e.g. single_2048 to profile)


def load_package():
    name = "beyond_rpa_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "beyond-rpa_b200"
    spec = importlib.util.spec_from_file_location(name, pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["bf16_tflops"], d["bf16_tflops_sustained"], d["hbm_gbs"], "measured"
    return 1590.0, 1400.0, 6650.0, "fallback"


def profile_traffic(kernel, workload):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / f"{kernel}_{workload}.md"
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        power = [float(r[3]) for r in rows if re.match(r"^[0-9.]+$", r[3])]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(power) if power else None}


# ----------------------------------------------------------------------------- host cores, FP64 peak

def host_cores():
    """(physical cores, logical CPUs) usable by this process: distinct (core, socket) pairs of
    lscpu's table restricted to the CPUs in this process's affinity mask."""
    cpus = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else list(range(os.cpu_count()))
    try:
        out = subprocess.run(["lscpu", "-p=CPU,CORE,SOCKET"], capture_output=True, text=True, timeout=10).stdout
        table = {int(c): (core, sock) for c, core, sock in
                 (line.split(",") for line in out.splitlines() if line and not line.startswith("#"))}
        phys = len({table[c] for c in cpus if c in table}) or len(cpus)
    except (OSError, ValueError, subprocess.SubprocessError):
        phys = len(cpus)
    return phys, len(cpus)


def fp64_peak(stream, seconds=4.0):
    """cuBLAS DGEMM 8192^3 (torch.matmul, float64) on this GPU, the method of the bf16 peaks:
    best of 10 (burst) and back to back for `seconds` (sustained); TFLOP/s, CUDA events."""
    import torch
    n = 8192
    g = torch.Generator(device="cuda").manual_seed(5)
    a = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    c = torch.empty_like(a)
    flop = 2.0 * n ** 3
    for _ in range(2):
        torch.matmul(a, b, out=c)
    best = float("inf")
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        torch.matmul(a, b, out=c)
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    reps = max(1, int(seconds * 1e3 / best))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        torch.matmul(a, b, out=c)
    e1.record(stream)
    e1.synchronize()
    sustained = flop * reps / (e0.elapsed_time(e1) / 1e3) / 1e12
    del a, b, c
    torch.cuda.empty_cache()
    return {"burst_tflops": flop / (best / 1e3) / 1e12, "sustained_tflops": sustained,
            "how": f"torch.matmul float64 {n}^3 (cuBLAS DGEMM, 2 n^3 flop): best of 10 and {reps} back to back, "
                   "CUDA events"}


# ----------------------------------------------------------------------------- CPU restatement timing

def cpu_sample(nq, no, nv, K, budget_s=8.0, seed=0):
    """Time the oracle's FP64 restatement on a bounded sample of the workload
    and extrapolate to one full E_c: Pi blocks of 500 ai columns (DGEMM) for
    one frequency until `budget_s` elapses, plus one DGEQRF log-det."""
    sys.path.insert(0, str(ROOT))
    from oracle import rpa_oracle as O
    rng = np.random.default_rng(seed)
    nov = no * nv
    blk = O.THC_BLOCK_DIM
    nblk_total = math.ceil(nov / blk)
    eo = np.sort(rng.uniform(-1.2, -0.3, no))
    ev = np.sort(np.exp(rng.uniform(math.log(0.02), math.log(5.0), nv)))
    d = O.dai(eo, ev)
    R = rng.standard_normal((nq, blk * 4)) * 0.01
    pi = np.zeros((nq, nq))
    done = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < budget_s and done < nblk_total:
        b = R[:, (done % 4) * blk:(done % 4 + 1) * blk]
        W = b * O.chi_factor(d[:blk], 0.5)[None, :]
        pi += 4.0 * (b @ W.T)
        done += 1
    t_blk = (time.perf_counter() - t0) / done
    A = np.eye(nq) + (R[:, :blk] @ R[:, :blk].T) * 1e-3
    t1 = time.perf_counter()
    O.logdet_qr(A)
    t_qr = time.perf_counter() - t1
    t_full = t_blk * nblk_total * K + t_qr * K
    phys, logical = host_cores()
    sample = (f"{done} DGEMM blocks of 500 ai x NQ={nq} (1 frequency) + 1 DGEQRF log-det of {nq}x{nq}; "
              f"extrapolated to {nblk_total} blocks x {K} frequencies + {K} log-dets")
    return {"value": 1.0 / t_full, "unit": "E_c/s", "cores": phys, "threads": logical, "kind": "port",
            "sample": sample, "seconds_per_Ec": t_full, "t_block_s": t_blk, "t_logdet_s": t_qr}


# ----------------------------------------------------------------------------- inputs

PINNED = ROOT / "tests" / "golden" / "pinned_golden.json"


def pinned_system(pkg, name, rank):
    """Inputs of an oracle-pinned single-system workload (tests/golden/pinned.py, numpy-seeded):
    rank 0 gets the pinned system itself (the fixture's rescale factor and grid, and the oracle's
    E_c to compare with), other ranks another system of the same shape, rescaled here.
    Returns (SyntheticSystem with R on the device, R rows on the host, oracle E_c or None)."""
    import torch
    from beyond_rpa_b200.workloads import SyntheticSystem, lambda_max_pi0
    sys.path.insert(0, str(ROOT))
    from tests.golden import pinned as P
    fix = json.loads(PINNED.read_text()).get(name) if PINNED.exists() else None
    K = P.SINGLE[name][3]
    if rank == 0 and fix is not None:
        Rt, eo, ev = P.single_system(name, fix["factor"])
        x, w, ref = np.array(fix["freqs"]), np.array(fix["weights"]), fix["Ec"]
    else:
        Rt, eo, ev = P.single_system(name, variant=rank)
        Rd = torch.from_numpy(Rt).cuda()
        d = torch.from_numpy((ev[:, None] - eo[None, :]).reshape(-1, order="F")).cuda()
        Rt *= math.sqrt(0.8 / lambda_max_pi0(Rd.T, d))
        del Rd, d
        x, w = pkg.freq_grid(np.concatenate([eo, ev]), len(eo), len(ev), nfixed=K)
        ref = None
    R = torch.from_numpy(Rt).cuda().T  # (NQ, nov) column-major, ld = NQ
    return SyntheticSystem(R=R, eps_o=eo, eps_v=ev, freqs=x, weights=w), Rt, ref


# ----------------------------------------------------------------------------- ours

def run_ours(args):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    pkg = load_package()
    from beyond_rpa_b200.workloads import make_single_system, SINGLE_SYSTEM
    WORKLOAD = args.workload
    nq, no, nv, K, _ = SINGLE_SYSTEM[WORKLOAD]
    nov = no * nv
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()  # the library and the timing events share this stream
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    from tests.golden import pinned as P
    if WORKLOAD in P.SINGLE:
        s, R_host_rows, ec_oracle = pinned_system(pkg, WORKLOAD, rank)
    else:
        s, R_host_rows, ec_oracle = make_single_system(WORKLOAD, seed=1000 + rank), None, None
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        h.ec_rpa(s.R, s.eps_o, s.eps_v, s.freqs, s.weights, prec="split")

    gpu_index = local
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd and all(p.strip().isdigit() for p in cvd.split(",")):
        gpu_index = int(cvd.split(",")[local])
    sampler = ClockSampler(gpu_index)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    contraction, split, logdet, launches, ecs = [], [], [], 0, []
    pi_ms, staging, other = [], [], []
    e0.record(stream)
    for _ in range(args.steps):
        ec, eu = h.ec_rpa(s.R, s.eps_o, s.eps_v, s.freqs, s.weights, prec="split")
        tm = h.timings()
        contraction.append(tm["contraction_ms"])
        split.append(tm["split_ms"])
        logdet.append(tm["logdet_ms"])
        pi_ms.append(tm["pi_ms"])
        staging.append(tm["staging_ms"])
        other.append(tm["other_ms"])
        launches += h.launches()
        ecs.append(ec)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    t_ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * args.steps / (t_ms / 1e3)

    if args.no_extras:
        if rank == 0:
            print(json.dumps({"workload": WORKLOAD, "ms_per_step": t_ms / args.steps, "Ec": ecs[-1],
                              "phase_ms": {"contraction": statistics.mean(contraction),
                                           "scale_split": statistics.mean(split),
                                           "logdet": statistics.mean(logdet)}}), flush=True)
        h.close()
        return
    # end-to-end through the public API with host (pinned) inputs
    Rh_t = torch.empty((nov, nq), dtype=torch.float64, pin_memory=True)
    if R_host_rows is not None:
        Rh_t.copy_(torch.from_numpy(R_host_rows))
        del R_host_rows
    else:
        Rh_t.copy_(s.R.T)
    Rh = Rh_t.T
    h.ec_rpa(Rh, s.eps_o, s.eps_v, s.freqs, s.weights, prec="split")
    e2e_steps = max(1, min(args.steps, 5))
    barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(e2e_steps):
        h.ec_rpa(Rh, s.eps_o, s.eps_v, s.freqs, s.weights, prec="split")
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    t_e2e = max_over_ranks(e2.elapsed_time(e3))
    e2e_value = world * e2e_steps / (t_e2e / 1e3)
    h2d = nq * nov * 8 + (no + nv + 2 * K) * 8
    d2h = 8 * (1 + K)

    # FP64 form of the same path (the split-vs-FP64 comparison), one call
    ec64, _ = h.ec_rpa(s.R, s.eps_o, s.eps_v, s.freqs, s.weights, prec="fp64")
    t64 = h.timings()
    e4 = torch.cuda.Event(enable_timing=True)
    e5 = torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    ec64, _ = h.ec_rpa(s.R, s.eps_o, s.eps_v, s.freqs, s.weights, prec="fp64")
    e5.record(stream)
    torch.cuda.synchronize()
    t64_ms = e4.elapsed_time(e5)
    t64 = h.timings()

    burst, sustained, hbm, src = peaks()
    tc_ms = statistics.mean(contraction)
    flops_tc = 3.0 * nq * nq * nov * K  # three bf16 SYRK products over the lower triangle
    achieved = flops_tc / (tc_ms / 1e3) / 1e12
    pi_flops = float(nq) * nq * nov * K  # FP64-equivalent SYRK flops of the Pi build
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "E_c/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16x3 split (fp32 acc) Pi + f64 log-det",
        "data": "synthetic (seeded; no SCF/Cholesky stack or dataset available)",
        "config": {"workload": f"{WORKLOAD}: NQ={nq} NOcc={no} NVirt={nv} nov={nov} K={K} (one system per rank)",
                   "NQ": nq, "NOcc": no, "NVirt": nv, "K": K,
                   "l2": "inputs larger than L2 (R = %.2f GB FP64), no flush" % (nq * nov * 8 / 1e9),
                   "parallelism": f"dp{world} (independent systems)"},
        "e2e": {"value": e2e_value, "unit": "E_c/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": t_e2e / e2e_steps},
        "gpu_launches": launches,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": sustained, "unit": "TFLOP/s",
                     "frac": achieved / sustained, "frac_of_burst_peak": achieved / burst,
                     "traffic": profile_traffic("syrk_split_bf16", WORKLOAD),
                     "traffic_source": f"profiles/syrk_split_bf16_{WORKLOAD}.md: dram__bytes_read.sum + "
                                       "dram__bytes_write.sum per launch from a committed ncu capture "
                                       "(not measured by this run)",
                     "kernel": "syrk_split_bf16_kernel",
                     "note": f"peak = bf16_tflops_sustained ({src}); achieved = 3 bf16 SYRK products "
                             f"3*NQ^2*nov*K / contraction time"},
        "phase_ms": {"contraction": tc_ms, "scale_split": statistics.mean(split),
                     "logdet": statistics.mean(logdet), "pi_build_total": statistics.mean(pi_ms),
                     "staging": statistics.mean(staging), "result_copies": statistics.mean(other)},
        "pi_build_tflops_fp64_equiv": pi_flops / ((tc_ms + statistics.mean(split)) / 1e3) / 1e12,
        "fp64_form": {"ms_per_step": t64_ms, "contraction_ms": t64["contraction_ms"],
                      "logdet_ms": t64["logdet_ms"], "speedup_split_vs_fp64": t64_ms / (t_ms / args.steps)},
        "energy": {"Ec_split": ecs[-1], "Ec_fp64": ec64, "abs_diff_split_vs_fp64": abs(ecs[-1] - ec64)},
        "clocks": clocks,
    }
    ld_ms = statistics.mean(logdet)
    ld_flops = float(nq) ** 3 / 3.0 * K
    split_bytes = 8.0 * nq * nov + 4.0 * nq * nov * K  # R read once, bf16 hi + lo written per frequency
    out["scale_split_roofline"] = {"bound": "hbm", "achieved": split_bytes / (statistics.mean(split) / 1e3) / 1e9,
                                   "peak": hbm, "unit": "GB/s",
                                   "frac": split_bytes / (statistics.mean(split) / 1e3) / 1e9 / hbm,
                                   "kernel": "scale_split_kernel",
                                   "note": "algorithmic bytes 8 NQ nov + 4 NQ nov K over the pass time"}
    if ec_oracle is not None:
        out["oracle_check"] = {"Ec_oracle": ec_oracle, "abs_err_split": abs(ecs[-1] - ec_oracle),
                               "abs_err_fp64": abs(ec64 - ec_oracle),
                               "source": "tests/golden/pinned_golden.json: the oracle (numpy/LAPACK FP64) on "
                                         "the same seeded inputs"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_sample(nq, no, nv, K)
    if world == 1 and not args.no_mbe:
        # FP64 (DMMA) peak of this GPU, the denominator of the FP64 kernels' fractions
        fp = fp64_peak(stream)
        out["fp64_peak"] = fp
        out["logdet_roofline"] = {"bound": "fp64", "achieved": ld_flops / (ld_ms / 1e3) / 1e12,
                                  "peak": fp["sustained_tflops"], "unit": "TFLOP/s",
                                  "frac": ld_flops / (ld_ms / 1e3) / 1e12 / fp["sustained_tflops"],
                                  "note": "NQ^3/3 K Cholesky flops over the log-det phase; peak = measured "
                                          "sustained cuBLAS DGEMM"}
        out["fp64_form"]["pi_fp64_tflops"] = pi_flops / (t64["contraction_ms"] / 1e3) / 1e12
        # the batched many-body-expansion workload (512 fragments), split-BF16 vs FP64
        del s
        h.close()
        torch.cuda.empty_cache()
        h = pkg.Handle(local)
        h.set_stream(stream.cuda_stream)
        out["mbe_512"] = mbe_measure(pkg, h, stream, 512, steps=2, warmup=1)
        h.close()
        torch.cuda.empty_cache()
        h = pkg.Handle(local)
        # the adjoint and the large single-system shapes of the configuration list, compact legs
        out["adjoint_2560"] = adjoint_leg(pkg, stream)
        out["large_8192"] = single_leg(pkg, stream, "large_8192")
    if rank == 0:
        print(json.dumps(out), flush=True)
    h.close()
    if world > 1:
        dist.destroy_process_group()


def single_leg(pkg, stream, name, steps=2):
    """A compact split-vs-FP64 measurement of one more single-system workload for the default line:
    one warm-up, `steps` timed split-BF16 energies, one timed FP64 energy (R resident)."""
    import torch
    from beyond_rpa_b200.workloads import make_single_system, SINGLE_SYSTEM
    nq, no, nv, K, _ = SINGLE_SYSTEM[name]
    h = pkg.Handle(torch.cuda.current_device())
    h.set_stream(stream.cuda_stream)
    s = make_single_system(name, seed=131)
    torch.cuda.synchronize()
    h.ec_rpa(s.R, s.eps_o, s.eps_v, s.freqs, s.weights, prec="split")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tc = []
    e0.record(stream)
    for _ in range(steps):
        ec, _ = h.ec_rpa(s.R, s.eps_o, s.eps_v, s.freqs, s.weights, prec="split")
        tc.append(h.timings()["contraction_ms"])
    e1.record(stream)
    torch.cuda.synchronize()
    t_split = e0.elapsed_time(e1) / steps
    e0.record(stream)
    ec64, _ = h.ec_rpa(s.R, s.eps_o, s.eps_v, s.freqs, s.weights, prec="fp64")
    e1.record(stream)
    torch.cuda.synchronize()
    t64 = e0.elapsed_time(e1)
    h.close()
    del s
    torch.cuda.empty_cache()
    burst, sustained, hbm, src = peaks()
    tf = 3.0 * nq * nq * no * nv * K / (statistics.mean(tc) * 1e-3) / 1e12
    return {"workload": f"{name}: NQ={nq} NOcc={no} NVirt={nv} K={K}", "ms_split": t_split, "ms_fp64": t64,
            "speedup_split_vs_fp64": t64 / t_split, "Ec_split": ec, "Ec_fp64": ec64,
            "abs_diff_split_vs_fp64": abs(ec - ec64), "contraction_tflops_bf16": tf,
            "contraction_frac_of_sustained": tf / sustained}


def adjoint_leg(pkg, stream, steps=2):
    """The adjoint workload on its oracle-pinned inputs (adjoint_2560): E_c + dE/dR + dE/de per
    step, split-BF16 Pi and FP64 Pi, errors against the oracle fixture."""
    import torch
    sys.path.insert(0, str(ROOT))
    from tests.golden import pinned as P
    fix = json.loads(PINNED.read_text())["adjoint_2560"]
    Rt, eo, ev = P.single_system("adjoint_2560", fix["factor"])
    x, w = np.array(fix["freqs"]), np.array(fix["weights"])
    g = fix["grad"]
    R = torch.from_numpy(Rt).cuda().T
    del Rt
    nq, nov = int(R.shape[0]), int(R.shape[1])
    dR = torch.empty((nov, nq), dtype=torch.float64, device="cuda").T
    dO = torch.empty(len(eo), dtype=torch.float64, device="cuda")
    dV = torch.empty(len(ev), dtype=torch.float64, device="cuda")
    h = pkg.Handle(torch.cuda.current_device())
    h.set_stream(stream.cuda_stream)
    out = {"workload": f"adjoint_2560: NQ={nq} NOcc={len(eo)} NVirt={len(ev)} K={len(x)} (oracle-pinned inputs)"}
    qi = torch.as_tensor(g["q"], device="cuda")
    ai = torch.as_tensor(g["ai"], device="cuda")
    for prec, reps in (("split", steps), ("fp64", 1)):
        h.ec_grad(R, eo, ev, x, w, prec=prec, out=(dR, dO, dV))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            ec, *_ = h.ec_grad(R, eo, ev, x, w, prec=prec, out=(dR, dO, dV))
        e1.record(stream)
        torch.cuda.synchronize()
        samp = dR[qi, ai].cpu().numpy()
        out[prec] = {"ms_per_gradient": e0.elapsed_time(e1) / reps, "Ec": ec,
                     "abs_err_Ec_vs_oracle_qr": abs(ec - fix["Ec"]),
                     "abs_err_Ec_vs_oracle_cholesky": abs(ec - fix["Ec_cholesky"]),
                     "rel_err_dR_vs_oracle": float(np.max(np.abs(samp - np.array(g["dR"]))) / g["dR_max"]),
                     "rel_err_deps_vs_oracle": float(max(
                         np.max(np.abs(dO.cpu().numpy() - np.array(g["deps_o"]))) / np.max(np.abs(g["deps_o"])),
                         np.max(np.abs(dV.cpu().numpy() - np.array(g["deps_v"]))) / np.max(np.abs(g["deps_v"]))))}
    h.close()
    del R, dR
    torch.cuda.empty_cache()
    out["gradients_per_s_split"] = 1e3 / out["split"]["ms_per_gradient"]
    return out


def mbe_measure(pkg, h, stream, n_inst, steps, warmup, rank=0, world=1, fp64_steps=1, gen_cpu=False):
    """Batched many-fragment workload on this rank's share: instances/s of rpa_b200_ec_batched,
    split-BF16 vs FP64 (same batched path), energies gathered over ranks.  gen_cpu: draw the inputs
    on the host and copy them (for profiling runs, whose device launches should be the library's)."""
    import torch
    from beyond_rpa_b200.workloads import make_mbe_batch, mbe_specs
    from beyond_rpa_b200 import distributed as D
    specs = mbe_specs(n_inst, seed=4000)
    mine = D.shard([D.instance_cost(nq, no * nv, K) for no, nv, nq, K in specs], rank, world)
    systems, kinds = make_mbe_batch(n_inst, seed=4000, only=mine, device="cpu" if gen_cpu else "cuda")
    if gen_cpu:
        systems = [(R.T.contiguous().cuda().T, eo, ev, x, w) for R, eo, ev, x, w in systems]
    torch.cuda.synchronize()
    flops = sum(float(R.shape[0]) ** 2 * len(eo) * len(ev) * len(x) for R, eo, ev, x, w in systems)
    ld_flops = sum(float(R.shape[0]) ** 3 / 3 * len(x) for R, eo, ev, x, w in systems)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(warmup):
        h.ec_batched(systems, prec="split")
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ec, _ = h.ec_batched(systems, prec="split")
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    t_ms = D.max_over_ranks(e0.elapsed_time(e1) / steps, device="cuda")
    launches = h.launches()
    h.ec_batched(systems, prec="fp64")
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(fp64_steps):
        ec64, _ = h.ec_batched(systems, prec="fp64")
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    t64 = D.max_over_ranks(e2.elapsed_time(e3) / fp64_steps, device="cuda")
    all_ec = D.gather_energies(mine, ec, n_inst, device="cuda")
    all_ec64 = D.gather_energies(mine, ec64, n_inst, device="cuda")
    del systems
    return {
        "metric": "RPA E_c of a batched many-body-expansion workload",
        "value": n_inst / (t_ms / 1e3), "unit": "instances/s", "ms_per_step": t_ms, "steps": steps,
        "n_gpus": world, "scaling": "strong", "instances": n_inst, "dimers": kinds.count("dimer"),
        "trimers": kinds.count("trimer"),
        "pi_fp64_equiv_tflops_rank0": flops / (t_ms / 1e3) / 1e12, "pi_flops_rank0": flops,
        "logdet_flops_rank0": ld_flops, "gpu_launches_per_step_rank0": launches,
        "fp64_form": {"ms_per_step": t64, "instances_per_s": n_inst / (t64 / 1e3),
                      "speedup_split_vs_fp64": t64 / t_ms},
        "max_abs_dEc_split_vs_fp64": float(np.max(np.abs(all_ec - all_ec64))),
        "dEint_note": "fragments are independent synthetic systems; interaction energies of 16 of them "
                      "are checked against the oracle by tests/test_gpu_pinned.py (<= 1e-7 Eh)",
    }


def run_mbe(args):
    """Batched many-fragment workload: instances/s of rpa_b200_ec_batched, split vs FP64.
    N > 1: fragments dealt out to ranks by cost (strong scaling, no data-path collective)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    pkg = load_package()
    n_inst = int(args.workload.split("_")[1]) if "_" in args.workload else 512
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    res = mbe_measure(pkg, h, stream, n_inst, args.steps, args.warmup, rank, world, gen_cpu=args.gen_cpu)
    if rank == 0:
        print(json.dumps({**res, "workload": args.workload}), flush=True)
    h.close()
    if world > 1:
        dist.destroy_process_group()


def run_adjoint(args):
    """Adjoint workload (adjoint_2560: NQ=2560, NOcc=48, NVirt=640, K=16): time of E_c + dE/dR, dE/de,
    split vs FP64, and a central finite-difference check (step 1e-5, FP64) on 64 random entries of R."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pkg = load_package()
    from beyond_rpa_b200.workloads import make_single_system, SINGLE_SYSTEM
    nq, no, nv, K, _ = SINGLE_SYSTEM[args.workload]
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    s = make_single_system(args.workload, seed=77)
    nov = no * nv
    dR = torch.empty((nov, nq), dtype=torch.float64, device="cuda").T
    dO = torch.empty(no, dtype=torch.float64, device="cuda")
    dV = torch.empty(nv, dtype=torch.float64, device="cuda")
    eo = torch.from_numpy(s.eps_o).cuda()
    ev = torch.from_numpy(s.eps_v).cuda()
    out = {}
    grads = {}
    for prec in ("split", "fp64"):
        for _ in range(args.warmup):
            h.ec_grad(s.R, eo, ev, s.freqs, s.weights, prec=prec, out=(dR, dO, dV))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ec, *_ = h.ec_grad(s.R, eo, ev, s.freqs, s.weights, prec=prec, out=(dR, dO, dV))
        e1.record(stream)
        torch.cuda.synchronize()
        out[prec] = {"ms_per_gradient": e0.elapsed_time(e1) / args.steps, "Ec": ec}
        grads[prec] = (dR.clone(), dO.clone(), dV.clone())
    g64 = grads["fp64"][0]
    out["split_vs_fp64_rel_err_dR"] = float((grads["split"][0] - g64).abs().max() / g64.abs().max())
    out["split_vs_fp64_rel_err_deps"] = float(
        max((grads["split"][1] - grads["fp64"][1]).abs().max() / grads["fp64"][1].abs().max(),
            (grads["split"][2] - grads["fp64"][2]).abs().max() / grads["fp64"][2].abs().max()))
    # central finite differences on 64 random entries (FP64 energies)
    rng = np.random.default_rng(9)
    hstep = 1e-5
    worst = 0.0
    worst_abs = 0.0
    gmax = float(g64.abs().max())
    for _ in range(64):
        q, ai = int(rng.integers(nq)), int(rng.integers(nov))
        old = float(s.R[q, ai])
        s.R[q, ai] = old + hstep
        ep, _ = h.ec_rpa(s.R, eo, ev, s.freqs, s.weights, prec="fp64")
        s.R[q, ai] = old - hstep
        em, _ = h.ec_rpa(s.R, eo, ev, s.freqs, s.weights, prec="fp64")
        s.R[q, ai] = old
        fd = (ep - em) / (2 * hstep)
        worst = max(worst, abs(fd - float(g64[q, ai])) / max(abs(fd), 1e-3 * gmax))
        worst_abs = max(worst_abs, abs(fd - float(g64[q, ai])))
    out["fd_max_rel_err_64_entries"] = worst
    out["fd_max_abs_err_over_max_grad"] = worst_abs / gmax
    print(json.dumps({"metric": "RPA E_c adjoint (dE/dR, dE/de)", "workload": f"{args.workload}: NQ={nq} "
                      f"NOcc={no} NVirt={nv} K={K}", "value": 1e3 / out["split"]["ms_per_gradient"],
                      "unit": "gradients/s", **out}), flush=True)
    h.close()


def run_cc(args):
    """CC-path workload (cc_1024: NQ=1024, NOcc=32, NVirt=256, K=12; cc_2048): one direct-ring T2
    (split Pi, G = 3 NQ guess vectors, cutoff 1e-4) followed by the SOSEX and MBPT3 exchange energies
    from the same amplitudes.  Reports the time of each stage and its FP64 DMMA rate."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pkg = load_package()
    from beyond_rpa_b200.workloads import make_single_system, SINGLE_SYSTEM
    nq, no, nv, K, _ = SINGLE_SYSTEM[args.workload]
    nov = no * nv
    G = min(3 * nq, nov)
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    s = make_single_system(args.workload, seed=91)
    eo = torch.from_numpy(s.eps_o).cuda()
    ev = torch.from_numpy(s.eps_v).cuda()
    u_out = torch.empty((G, nov), dtype=torch.float64, device="cuda").T
    ev_ = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    times = {"t2": [], "sosex": [], "mbpt3": [], "sosex_fp64": [], "mbpt3_fp64": []}
    res = ex_s = ex_m = ex_s64 = ex_m64 = None
    for it in range(args.warmup + args.steps):
        ev_[0].record(stream)
        res = h.dring_t2(s.R, eo, ev, s.freqs, s.weights, prec="split", n_guess=G, seed=5, cutoff_thresh=1e-4,
                         u_out=u_out)
        ev_[1].record(stream)
        ex_s = h.exchange_sosex(s.R, no, nv, res["U"], res["A"], alpha=1.0, prec="split")
        ev_[2].record(stream)
        ex_m = h.exchange_mbpt3(s.R, eo, ev, res["U"], res["A"], prec="split")
        ev_[3].record(stream)
        ex_s64 = h.exchange_sosex(s.R, no, nv, res["U"], res["A"], alpha=1.0, prec="fp64")
        ev_[4].record(stream)
        ex_m64 = h.exchange_mbpt3(s.R, eo, ev, res["U"], res["A"], prec="fp64")
        ev_[5].record(stream)
        torch.cuda.synchronize()
        if it >= args.warmup:
            for k, (a, b) in {"t2": (0, 1), "sosex": (1, 2), "mbpt3": (2, 3), "sosex_fp64": (3, 4),
                              "mbpt3_fp64": (4, 5)}.items():
                times[k].append(ev_[a].elapsed_time(ev_[b]))
    NT = res["NT"]
    ms = {k: statistics.mean(v) for k, v in times.items()}
    pair = 2.0 * no * no * nq * nv * NT
    flops = {"t2": K * (4.0 * nq * nov * G + 2.0 * nq * nq * nov), "sosex": pair, "sosex_fp64": pair,
             "mbpt3": 2.0 * nq * nov * NT + 2.0 * NT * NT * (nq + nov) + 2.0 * nov * NT * NT + pair}
    flops["mbpt3_fp64"] = flops["mbpt3"]
    total = ms["t2"] + ms["sosex"] + ms["mbpt3"]
    print(json.dumps({"metric": "CC-path energies (direct-ring T2 + SOSEX + MBPT3 exchange)",
                      "workload": f"{args.workload}: NQ={nq} NOcc={no} NVirt={nv} nov={nov} K={K} G={G}",
                      "value": 1e3 / total, "unit": "CC-path evaluations/s (split Pi, split exchange contractions)",
                      "steps": args.steps, "warmup": args.warmup, "ms": ms, "NT": NT,
                      "algorithmic_tflops": {k: flops[k] / (ms[k] * 1e-3) / 1e12 for k in ms},
                      "pair_contraction_flops": pair,
                      "Ec_logdet": res["Ec"], "Ec_T2_eig": float(np.sum(res["EigRPA"])),
                      "Ex_sosex": ex_s, "Ex_sosex_fp64": ex_s64, "dEx_sosex": ex_s - ex_s64,
                      "Ex_mbpt3": ex_m, "Ex_mbpt3_fp64": ex_m64, "dEx_mbpt3": ex_m - ex_m64}), flush=True)
    h.close()


def run_exchange_large(args):
    """Beyond-RPA large case, exchange part (exchange_8192: NQ = 8192, NOcc = 128, NVirt = 2048,
    nov = 262144, R = 17.2 GB FP64): the SOSEX exchange contraction -sum (ai|bj) T_aj,bi on ring
    amplitudes of NT = --nt vectors (default 4096), split-BF16 on the tensor cores and FP64 (DMMA)
    on the same amplitudes.  The amplitudes are synthetic (Gaussian vectors, A_mu = -0.1 exp(-mu/400)):
    the direct-ring range finder at this shape (G = 3 NQ = 24576 guess vectors, K = 20) does not fit
    one GPU (its resident split operands alone are 344 GB)."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pkg = load_package()
    from beyond_rpa_b200.workloads import make_single_system, SINGLE_SYSTEM
    nq, no, nv, K, _ = SINGLE_SYSTEM["large_8192"]
    nov = no * nv
    NT = args.nt
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    s = make_single_system("large_8192", seed=131)
    g = torch.Generator(device="cuda").manual_seed(7)
    U = (torch.randn((NT, nov), generator=g, device="cuda", dtype=torch.float64) / math.sqrt(nov)).T
    A = -0.1 * np.exp(-np.arange(NT) / 400.0)
    torch.cuda.synchronize()
    out = {}
    for prec, reps in (("split", max(1, args.steps)), ("fp64", 1)):
        h.exchange_sosex(s.R, no, nv, U, A, prec=prec) if prec == "split" else None  # warm-up (split only)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            ex = h.exchange_sosex(s.R, no, nv, U, A, prec=prec)
        e1.record(stream)
        torch.cuda.synchronize()
        out[prec] = {"ms": e0.elapsed_time(e1) / reps, "Ex": ex}
    pair = 2.0 * no * no * nq * nv * NT  # FP64-equivalent flops of the pair contraction
    burst, sustained, hbm, src = peaks()
    tf_split = pair / (out["split"]["ms"] * 1e-3) / 1e12
    print(json.dumps({
        "metric": "SOSEX exchange contraction at the beyond-RPA large shape",
        "workload": f"exchange_8192: NQ={nq} NOcc={no} NVirt={nv} nov={nov} NT={NT} (synthetic amplitudes)",
        "ms_split": out["split"]["ms"], "ms_fp64": out["fp64"]["ms"],
        "speedup_split_vs_fp64": out["fp64"]["ms"] / out["split"]["ms"],
        "pair_flops_fp64_equiv": pair, "tflops_fp64_equiv_split": tf_split,
        "tensor_pipe_fraction_of_sustained_bf16": 3.0 * tf_split / sustained,
        "tflops_fp64": pair / (out["fp64"]["ms"] * 1e-3) / 1e12,
        "Ex_split": out["split"]["Ex"], "Ex_fp64": out["fp64"]["Ex"],
        "dEx_split_vs_fp64": out["split"]["Ex"] - out["fp64"]["Ex"],
        "note": "tensor-pipe fraction = 3 bf16 products x FP64-equivalent flops / CUDA-event time / "
                f"bf16_tflops_sustained ({src})"}), flush=True)
    h.close()


def run_logdet(args):
    """The FP64 log-det alone (logdet_2048 / logdet_4096: the 16 matrices 1 + Pi(u) of the
    single_2048 / single_4096 workloads, Pi built once in FP64 on the device): time of
    rpa_b200_ec_from_pi's Cholesky phase, its FP64 rate (NQ^3/3 K flops) and the fraction of the
    measured DGEMM peak.  RPA_B200_OZAKI_SLICES=7 or 8 runs the trailing updates on the int8 tensor
    cores instead of DMMA.

    logdet_batch_<n>x<m>: the batched log-det of the many-fragment path (m seeded SPD matrices of
    order n in one variable-size batch, every tile plan timed by rpa_b200_tune_logdet); reports the
    fastest plan's time per step (best of the steps) and its FP64 rate."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pkg = load_package()
    if args.workload.startswith("logdet_batch_"):
        n, m = (int(x) for x in args.workload[len("logdet_batch_"):].split("x"))
        h = pkg.Handle(local)
        best, plans = None, {}
        for it in range(args.warmup + args.steps):
            plan, ms = h.tune_logdet(n, m)
            if it >= args.warmup:
                for k, t in ms.items():
                    plans[str(k)] = min(plans.get(str(k), t), t)
                t = min(ms.values())
                best = t if best is None else min(best, t)
        flops = float(n) ** 3 / 3.0 * m
        print(json.dumps({"metric": "FP64 log-det of a variable-size batch", "workload": f"{m} matrices of order {n}",
                          "logdet_ms": best, "tflops": flops / (best * 1e-3) / 1e12, "plan_ms": plans,
                          "best_plan": list(h.logdet_plan(n))}), flush=True)
        h.close()
        return
    from beyond_rpa_b200.workloads import make_single_system, SINGLE_SYSTEM
    name = "single_" + args.workload.split("_")[1]
    nq, no, nv, K, _ = SINGLE_SYSTEM[name]
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    s = make_single_system(name, seed=17)
    pi = torch.empty((K, nq, nq), dtype=torch.float64, device="cuda")
    h.pi_u(s.R, s.eps_o, s.eps_v, s.freqs, prec="fp64", out=pi)
    del s
    torch.cuda.synchronize()
    ms = []
    for it in range(args.warmup + args.steps):
        ec, _ = h.ec_from_pi(pi, np.ones(K))
        if it >= args.warmup:
            ms.append(h.timings()["logdet_ms"])
    flops = float(nq) ** 3 / 3.0 * K
    fp = fp64_peak(stream, seconds=2.0)
    t = statistics.mean(ms)
    print(json.dumps({"metric": "FP64 log-det of 1 + Pi(u)", "workload": f"{args.workload}: {K} matrices of order {nq}",
                      "logdet_ms": t, "logdet_ms_all": ms, "tflops": flops / (t * 1e-3) / 1e12,
                      "fraction_of_dgemm_sustained": flops / (t * 1e-3) / 1e12 / fp["sustained_tflops"],
                      "fp64_peak": fp, "int8_updates": os.environ.get("RPA_B200_OZAKI_SLICES", "0"),
                      "launches_per_call": h.launches()}), flush=True)
    h.close()


def run_split(args):
    """One system split over the N GPUs (ai columns per rank, reduce-scatter of Pi over the
    frequency index, distributed log-dets): E_c/s of the whole job, strong scaling.
    --workload split_<system> (e.g. split_single_4096)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    group = None
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    pkg = load_package()
    from beyond_rpa_b200.workloads import make_single_system, SINGLE_SYSTEM
    from beyond_rpa_b200 import distributed as D
    system = args.workload[len("split_"):]
    nq, no, nv, K, _ = SINGLE_SYSTEM[system]
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    s = make_single_system(system, seed=1000)  # the same system on every rank
    torch.cuda.synchronize()

    def pi_fn(Rc, eo, ev, fr, out):
        h.pi_u(Rc, eo, ev, fr, prec="split", out=out)

    def ec_fn(pi, wk):
        return h.ec_from_pi(pi, wk)

    def step():
        return D.ec_rpa_ai_split(pi_fn, ec_fn, s.R, s.eps_o, s.eps_v, s.freqs, s.weights, group=group)

    for _ in range(args.warmup):
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ec, eu = step()
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_ms = float(t.item())
    if rank == 0:
        print(json.dumps({"metric": "RPA E_c of one system split over the GPUs (ai columns)", "workload":
                          f"{args.workload}: NQ={nq} NOcc={no} NVirt={nv} K={K}", "value": args.steps / (t_ms / 1e3),
                          "unit": "E_c/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": t_ms / args.steps, "scaling": "strong", "Ec": ec,
                          "collectives": "reduce_scatter (K*NQ^2 FP64) + all_reduce (K+1)"}), flush=True)
    h.close()
    if world > 1:
        dist.destroy_process_group()


def run_thc(args):
    """THC workload (thc_4096: NGrid = 8192, NQ = 4096, NOcc = 64, NVirt = 1024, K = 16): R formed from
    THC factors on the GPU (FP64 tensor-core GEMM) + the split-BF16 energy, per step."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pkg = load_package()
    from beyond_rpa_b200.workloads import SINGLE_SYSTEM, orbital_energies
    from beyond_rpa_b200 import freq_grid
    system = "single_" + args.workload.split("_")[1]
    nq, no, nv, K, kw = SINGLE_SYSTEM[system]
    ng = 2 * nq
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(7)
    Z = torch.randn((nq, ng), generator=g, device="cuda", dtype=torch.float64).T  # column-major NGrid x NQ
    Z *= (0.05 * torch.exp(-torch.arange(nq, device="cuda", dtype=torch.float64) / kw["decay"]))[None, :]
    Xa = torch.randn((nv, ng), generator=g, device="cuda", dtype=torch.float64).T / ng ** 0.5
    Xi = torch.randn((no, ng), generator=g, device="cuda", dtype=torch.float64).T / ng ** 0.5
    eo, ev = orbital_energies(no, nv, 7, kw["occ_range"], kw["virt_range"])
    x, w = freq_grid(np.concatenate([eo, ev]), no, nv)
    x, w = x[:K], w[:K]
    Rbuf = torch.empty((no * nv, nq), dtype=torch.float64, device="cuda").T
    for _ in range(args.warmup):
        h.ec_thc(Z, Xa, Xi, eo, ev, x, w)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record(stream)
    for _ in range(args.steps):
        ec, _ = h.ec_thc(Z, Xa, Xi, eo, ev, x, w)
    e[1].record(stream)
    for _ in range(args.steps):
        h.thc_r(Z, Xa, Xi, out=Rbuf)
    e[2].record(stream)
    torch.cuda.synchronize()
    ms = e[0].elapsed_time(e[1]) / args.steps
    ms_r = e[1].elapsed_time(e[2]) / args.steps
    flops_r = 2.0 * nq * ng * no * nv
    print(json.dumps({"metric": "RPA E_c from THC factors", "workload": f"{args.workload}: NGrid={ng} NQ={nq} "
                      f"NOcc={no} NVirt={nv} K={len(x)}", "value": 1e3 / ms, "unit": "E_c/s", "steps": args.steps,
                      "ms_per_step": ms, "r_formation_ms": ms_r, "r_formation_tflops_fp64": flops_r / ms_r / 1e9,
                      "Ec": ec}), flush=True)
    h.close()


def run_jctc(args):
    """Particle-hole corrections workload (jctc_512: NGrid = 2048, NQ = 512, NOcc = 32, NVirt = 256,
    NVecsT2 = 600, PNO cutoff 1e-5): time of rpa_b200_jctc2024 split into the PNO stage and the
    energy loop (CUDA events inside the library)."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pkg = load_package()
    nq = int(args.workload.split("_")[1])
    ng, no, nv, nt = 4 * nq, 32, 256, 600
    h = pkg.Handle(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h.set_stream(stream.cuda_stream)
    rng = np.random.default_rng(17)
    Z = rng.standard_normal((ng, nq)) * 0.3 * np.exp(-np.arange(nq) / (nq / 3.0))[None, :]
    Xa = rng.standard_normal((ng, nv)) / ng ** 0.5
    Xi = rng.standard_normal((ng, no)) / ng ** 0.5
    U, _ = np.linalg.qr(rng.standard_normal((no * nv, nt)))
    A = -0.05 * rng.uniform(size=nt)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T
    Zd, Xad, Xid, Ud = dev(Z), dev(Xa), dev(Xi), dev(U)
    for _ in range(args.warmup):
        h.jctc2024(Zd, Xid, Xad, Ud, A, cutoff_pno=1e-5)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pno_ms, loop_ms = [], []
    e0.record(stream)
    for _ in range(args.steps):
        en, stats = h.jctc2024(Zd, Xid, Xad, Ud, A, cutoff_pno=1e-5)
        tm = h.timings()
        pno_ms.append(tm["pi_ms"])
        loop_ms.append(tm["logdet_ms"])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"metric": "particle-hole corrections (SOSEX cumulant + PH3) with PNOs", "workload":
                      f"{args.workload}: NGrid={ng} NQ={nq} NOcc={no} NVirt={nv} NVecsT2={nt} cutoff 1e-5",
                      "value": 1e3 / ms, "unit": "evaluations/s", "ms_per_step": ms,
                      "pno_stage_ms": statistics.mean(pno_ms), "energy_loop_ms": statistics.mean(loop_ms),
                      "pno_stats": {"max": stats[0], "avg": stats[1] / (no * (no + 1) // 2), "zero_pairs": stats[2]},
                      "energies": {"EcRPA_PNO": en[0], "Ec1b": en[1], "Ec2bcd": en[2], "Ec2ghij": en[3]}}),
          flush=True)
    h.close()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from importlib import import_module  # noqa: F401
    sys.path.insert(0, str(ROOT / "beyond-rpa_b200"))
    nq, no, nv, K = 4096, 64, 1024, 16
    vals = []
    for _ in range(args.warmup):
        cpu_sample(nq, no, nv, K, budget_s=2.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_sample(nq, no, nv, K, budget_s=6.0)["seconds_per_Ec"])
    wall = time.perf_counter() - t0
    spe = statistics.mean(vals)
    value = 1.0 / spe
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "E_c/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": spe * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{WORKLOAD}: NQ={nq} NOcc={no} NVirt={nv} nov={no * nv} K={K}",
                       "parallelism": "host threads (OpenBLAS)"},
            "cpu_baseline": {"value": value, "unit": "E_c/s", "cores": host_cores()[0],
                             "threads": host_cores()[1], "kind": "port",
                             "sample": "per step: DGEMM blocks of 500 ai for ~6 s (1 frequency) + 1 DGEQRF "
                                       "log-det, extrapolated to the full E_c (reference binary cannot be "
                                       "built: Fortran, no gfortran)"},
            "e2e": {"value": value, "unit": "E_c/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    if args.full_cpu_check:
        # one complete CPU E_c of the same workload (the oracle on the pinned inputs), to validate the
        # per-step extrapolation above
        sys.path.insert(0, str(ROOT))
        from oracle import rpa_oracle as O
        from tests.golden import pinned as P
        fix = json.loads(PINNED.read_text())["single_4096"]
        Rt, eo, ev = P.single_system("single_4096", fix["factor"])
        t0 = time.perf_counter()
        ec, _ = O.ec_rpa(Rt.T, eo, ev, np.array(fix["freqs"]), np.array(fix["weights"]))
        t_full = time.perf_counter() - t0
        line["full_cpu_check"] = {"seconds_per_Ec_measured": t_full, "seconds_per_Ec_extrapolated": spe,
                                  "ratio_measured_over_extrapolated": t_full / spe,
                                  "abs_err_vs_fixture": abs(ec - fix["Ec"])}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default=WORKLOAD, help="single-system workload name (beyond-rpa_b200/workloads.py)")
    ap.add_argument("--full-cpu-check", action="store_true",
                    help="--impl reference: also time one complete CPU E_c to validate the extrapolation")
    ap.add_argument("--nt", type=int, default=4096, help="exchange_8192: ring amplitudes NT")
    ap.add_argument("--gen-cpu", action="store_true", help="mbe workloads: draw the inputs on the host")
    ap.add_argument("--no-mbe", action="store_true",
                    help="skip the extra legs of the default line (FP64 peak, batched fragments, adjoint, "
                         "large system)")
    ap.add_argument("--no-extras", action="store_true",
                    help="profiling runs: print only the timed leg (no e2e, FP64-form or CPU legs)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload.startswith("mbe"):
        run_mbe(args)
    elif args.workload.startswith("adjoint"):
        run_adjoint(args)
    elif args.workload.startswith("cc"):
        run_cc(args)
    elif args.workload == "exchange_8192":
        run_exchange_large(args)
    elif args.workload.startswith("logdet_"):
        run_logdet(args)
    elif args.workload.startswith("split_"):
        run_split(args)
    elif args.workload.startswith("thc_"):
        run_thc(args)
    elif args.workload.startswith("jctc_"):
        run_jctc(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
