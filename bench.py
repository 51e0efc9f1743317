"""Benchmark: Galerkin BEM assembly + solve on B200.

Headline workload (one GPU, the default): the Helmholtz transmission problem
on the unit icosphere of subdivision 5 (20480 panels, 10242 vertices, 30722
unknowns: P1 Dirichlet + P0 Neumann traces), k_out = 5, k_in = 7.5, GaussQR =
5, incident plane wave with a seeded direction.  One step = BEMManager.run
with inputs resident in HBM: the fused Calderon sweep (V, K, K^T, W at both
wavenumbers; separate pairs in FP32, coincident/edge/vertex pairs in FP64)
into A = P-_o + P+_i and P+_i, the identity blocks and right-hand side, and
the reference's least squares on the stacked [A; P+_i]: FP16-split
tensor-core normal matrix (FP64 segment sums), Cholesky with FP64 panels and
tensor-core trailing updates into an FP64 Schur complement, FP64 flexible
GMRES on the normal equations.

  value  = stacked-system entries (2 n^2) / time-to-solution (entries/s),
           device-timed with CUDA events per step, 256 MiB L2 flush between
           steps (the inputs are larger than L2 anyway);
  e2e    = the same metric through the public API (CoreManager with a host
           mesh: mesh upload, set-up, run, solution read back), one full
           lifecycle per step, median of two after one discarded;
  plain_fp64 = the same step on the plain FP64 path (FP64 sweep, FP64
           DMMA normal matrix, Cholesky with DMMA updates, FP64 GMRES), whose
           solution is the FP64 oracle the mixed result's relative error is
           quoted against.

`--workload dirichlet_s4` gives the Helmholtz interior Dirichlet line (5120
panels); the other workloads print their own lines.  `--impl reference`
times the reference's CPU algorithm (the oracle's FP32 restatement of its
loops, all host threads) on a bounded sample of the same workload.
Multi-GPU: one independent replica per rank (the dense solve does not
shard); value = sum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "taichi-bem_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "assembly entries/s + time-to-solution at ≤1e-6 rel err: mixed/batched vs plain GPU"
WORKLOAD = "Helmholtz 3D interior Dirichlet k=3, icosphere s4 (5120 panels), GaussQR=5, plane wave"
# Algorithmic FP32 flops (an FMA counts 2) per kernel evaluation of the fused
# symmetric Helmholtz sweep, counted once from the source of its scalar form
# (far_vkg_sym_kernel<Helmholtz, float>) and kept fixed as the unit of work:
# offsets 3, s = e.(2D+e) 8, r^2 1, r and 1/r with the Newton step 9, d.n_j 6,
# split phase 3, weights 5, k r 1, sine/cosine polynomials 20, (1-ikr) e^{ikr} 4,
# V_ij and (K g)_i accumulation 8, (K g)_j term 10 = 78, plus two MUFU
# operations (reciprocal square root, reciprocal).  One evaluation serves V_ij,
# V_ji, (K g)_i and (K g)_j, so the sweep evaluates each unordered separate
# pair once.  The launched kernel (far_vkg_sym_x2_kernel, packed FP32x2) gets
# the same result with 63 flops per evaluation (s from per-point and
# per-trial-point terms, d.n_j per pair, -d.n_i factored out of the sum over
# test points, shorter polynomials for phases below 0.3); the rate against 78
# is the rate of the unit of work.
FLOPS_PER_EVAL = 78
MUFU_PER_EVAL = 2
# dram__bytes_read.sum + dram__bytes_write.sum of far_vkg_sym_x2_kernel on this
# workload (423.5 MB + 379.3 MB, one ncu capture of --profile-step mixed)
FAR_SWEEP_DRAM_BYTES = 802.8e6

TRANS_WORKLOAD = ("Helmholtz transmission 2x2 block Calderon system, icosphere s5 (20480 panels, 10242 vertices, "
                  "30722 unknowns), k_out=5, k_in=7.5 (n_i=2.25), GaussQR=5, incident plane wave, least squares on "
                  "the stacked [A; P+_i] (61444 x 30722)")
# Algorithmic FP32 work per evaluation of the fused Calderon sweep
# (far_calderon_kernel<float, 2, Helmholtz>), counted once from its scalar
# source and kept fixed: the pair-frame geometry (e, s, r^2, r and 1/r with the
# Newton step, d.n_j, the split phase, w/r, w/r^3, t_j) 24 flops, and per
# wavenumber the phase 1, sine/cosine polynomials 21, k r 1, G 2,
# (1 - ikr) e^{ikr} 4 and the 14 test-point sums 26 = 55; two wavenumbers:
# 134 flops and 3 MUFU operations (reciprocal square root, reciprocal, and
# none per wavenumber).  One evaluation serves V, K, K^T and W of both
# wavenumbers.
CAL_FLOPS_PER_EVAL = 134


def _measured_peaks():
    """The driver-measured peaks of this pool's B200s (MEASURED_PEAKS.json),
    else the fallback figures of the pool's profiling recipe."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


MEASURED = _measured_peaks()


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def replicas_aggregate(ms_local: float, units_per_rank: float, ws: int, device):
    """Whole-job figures of N independent replicas (one per rank): the step
    time is the maximum over ranks and the value is the units of all ranks
    over that time.  Every rank calls this at the same point (one all-reduce
    when ws > 1); `device` is where the reduction runs (the rank's GPU under
    NCCL, the CPU under gloo).  Returns (ms, units per second)."""
    import torch

    ms = float(ms_local)
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, units_per_rank * ws / (ms * 1e-3)


_NVML_CHILD = r"""
import sys, time
try:
    import pynvml
    pynvml.nvmlInit()
    h = pynvml.nvmlDeviceGetHandleByPciBusId(sys.argv[1].encode())
    smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
    # the first query of each counter is the slow one: make it before the timed region
    pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
    pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
except Exception as exc:
    print("fail", exc, flush=True)
    sys.exit(0)
print("ready", smax, flush=True)
sys.stdin.readline()
while True:
    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
    mask = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
    print("S", sm, mask, flush=True)
    time.sleep(0.2)
"""


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of this process's GPU
    during the timed region, polled every 200 ms through NVML by a separate
    Python process (a thread of this process would compete with the
    launching thread for the interpreter lock and delay its launches).  The
    child initialises NVML before the timed region and starts sampling when
    told to; nvidia-smi in loop mode is the fallback when NVML is missing."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.source = None
        self.smax = None

    def start(self):
        import torch
        p = torch.cuda.get_device_properties(self.dev)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", _NVML_CHILD, bus], stdin=subprocess.PIPE,
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            first = self.proc.stdout.readline().split()
            if first and first[0] == "ready":
                self.smax = float(first[1])
                self.source = "nvml"
                self.proc.stdin.write("go\n")
                self.proc.stdin.flush()
                return
            self.proc.wait(timeout=5)
        except (OSError, subprocess.TimeoutExpired, ValueError, IndexError):
            pass
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
            time.sleep(2.0)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, reasons = [], set()
        smax = self.smax
        if self.source == "nvml":
            for line in out.strip().splitlines():
                parts = line.split()
                if len(parts) != 3 or parts[0] != "S":
                    continue
                sm.append(float(parts[1]))
                mask = int(parts[2])
                for name, bit in self.REASONS.items():
                    if mask & bit:
                        reasons.add(name)
        else:
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in out.strip().splitlines():
                parts = [q.strip() for q in line.split(",")]
                if len(parts) < 6:
                    continue
                try:
                    sm.append(float(parts[0]))
                    smax = float(parts[1])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[2:6]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": self.source}


def cpu_reference(steps: int, warmup: int, threads: int | None = None, sample_rows: int | None = None,
                  target_s: float = 10.0):
    """Reference algorithm on the host: the FP32 restatement of the reference's
    loops (one outer iteration per test panel, serial over trial panels x
    GaussQR^4, per-basis recompute) for V and the matrix-free K g of the
    workload, on a sample of test panels; scaled to entries/s."""
    import numpy as np

    from bem_b200 import icosphere
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    O.set_threads(threads)
    v, f = icosphere(4)
    nt, nv = len(f), len(v)
    Q = 5
    k = 3.0
    panels = np.arange(nt, dtype=np.int32)

    def one(rows):
        tp = panels[:rows]
        out = np.zeros((rows, nt), np.complex128)
        t0 = time.perf_counter()
        O.assemble(v, f, O.OP_V, True, k, k * k, Q, True, (tp, 1, tp.copy()), (panels, 1, panels.copy()), out=out,
                   fp32=True)
        g = np.exp(1j * k * (v @ np.array([0.0, 0.0, 1.0])))
        y = np.zeros(rows, np.complex128)
        O.assemble(v, f, O.OP_K, True, k, k * k, Q, True, (tp, 1, tp.copy()),
                   (panels, 3, f.reshape(-1).astype(np.int32)), x=g, y=y, conj_x=True, fp32=True)
        return time.perf_counter() - t0

    # size the sample so that one timed sample is ~`target_s` of CPU work
    t1 = one(threads)
    rows = sample_rows or int(min(nt, threads * max(1, round(target_s / max(t1, 1e-3)))))
    for _ in range(warmup):
        one(max(1, rows // 4))
    times = [one(rows) for _ in range(steps)]
    t = statistics.mean(times)
    # entries/s of V assembled per second of (V + K g) work, as for the GPU step
    value = rows * nt / t
    return {"value": value, "unit": "entries/s", "cores": threads, "kind": "port",
            "sample": f"{rows} of {nt} test panels (rows of V and K g), FP32, {steps} timed samples",
            "seconds_per_sample": t}


def phase_breakdown(b):
    """Device time of each phase of one BEMManager.run step (CUDA events)."""
    import torch
    from bem_b200.utils.types import AssembleType
    out = {}

    def timed(name, fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1)
        return r

    b._mat_A.zero_()
    if b._fusable():
        timed("assemble_V_and_Kg_fused_plus_rhs", b._run_dirichlet_fused)
    else:
        timed("assemble_V", lambda: b.matrix_layer_forward(k=b._k, scope_type=b._scope_type))
        timed("block_add", lambda: b.assemble_matA(assemble_type=int(AssembleType.ADD_M), multiplier=-1.0))
        timed("boundary_data", lambda: b.rhs_constructor.set_boundaries(b._scope_type, b._sqrt_ni, b._sqrt_no))
        timed("rhs_half_M_plus_K_g", lambda: b.rhs_layer_forward(k=b._k, scope_type=b._scope_type))
        timed("rhs_copy", b.assemble_rhs)
    A = b._mat_A
    lo = torch.complex64 if A.is_complex() else torch.float32
    LU = timed("cast_fp32", lambda: A.to(lo))
    piv, dinv, info = timed("lu_factor_fp32_tiled", lambda: b.engine.lu_factor_tiled(LU))
    x = torch.zeros_like(b.rhs)
    # the refinement twice from x = 0, the second one timed (steady state)
    for name in ("refine_fp64_first", "refine_fp64"):
        x.zero_()
        timed(name, lambda: b.engine.refine_solve(A, LU, piv, b.rhs, x, tol=b.refine_tol, maxit=b.refine_maxit,
                                                  dinv=dinv))
    xs = b.rhs.clone()
    timed("lu_solve_fp32_tiled", lambda: b.engine.lu_solve_tiled(LU, piv, dinv, xs))
    LU2 = A.to(lo)
    timed("lu_factor_fp32_partial_pivoting", lambda: b.engine.lu_factor(LU2))
    y = torch.zeros_like(b.rhs)
    timed("gemv_c128", lambda: b.engine.gemv(A, x, y))
    return out


def profile_step(precision: str, workload: str = "dirichlet_s4", subdiv: int = 5, calderon_group: int = 0,
                 gram_form: int = 0):
    """One warm-up and one timed step of the workload, nothing else (the
    command the committed ncu summaries were captured with):
    the Dirichlet problem on 5120 panels, or the transmission least-squares
    problem on the icosphere of subdivision `subdiv` (assembly and solve)."""
    import torch
    from bem_b200.managers import CoreManager
    if workload == "dirichlet_s4":
        from bem_b200.workloads import helmholtz_dirichlet_s4
        params, fD, fN = helmholtz_dirichlet_s4(precision=precision)
    else:
        from bem_b200.workloads import transmission_s5
        params, pw = transmission_s5(precision, subdiv, "lstsq")
        fD, fN = pw.fD, pw.fN
    core = CoreManager(params)
    core.initialization(fD, fN)
    b = core._BEM_manager
    from bem_b200 import _lib as L
    if calderon_group:
        b.engine.set_tuning(L.TUNE_CALDERON_GROUP, calderon_group)
    if gram_form:
        b.engine.set_tuning(L.TUNE_GRAM_PAIR, gram_form)
    b.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.run()
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"profile_step": precision, "ms": e0.elapsed_time(e1), "launches": b.engine.launches}))
    core.kill()


def profile_lu(n: int, lu_update: int = 0):
    """Six tile-pivoted FP32 factorisations of one random complex n x n matrix
    shifted by 40 I (seed 0), each timed with CUDA events (the command the LU
    kernel summaries were captured with)."""
    import torch
    from bem_b200.engine import Engine
    torch.manual_seed(0)
    A = (torch.randn(n, n, dtype=torch.complex64, device="cuda") + 40 * torch.eye(n, device="cuda")).contiguous()
    eng = Engine()
    if lu_update:
        from bem_b200 import _lib as L
        eng.set_tuning(L.TUNE_LU_UPDATE, lu_update)
    ts = []
    for _ in range(6):
        LU = A.clone()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.lu_factor_tiled(LU)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    print(json.dumps({"profile_lu": n, "factor_ms": ts}))
    eng.close()


def shard_wavenumbers(ks, rank: int, ws: int):
    """Rank r's share of a wavenumber sweep: ks[r], ks[r + ws], ... .  Each k
    is an independent unit (its own operators, norm estimate and least
    squares), so the ranks exchange no data while they run."""
    return list(ks[rank::ws])


def sweep_gather(local: dict, ks, rank: int, ws: int) -> dict:
    """Every rank's per-k lists (local[name][i] belongs to
    shard_wavenumbers(ks, rank, ws)[i]) merged in the order of ks, on every
    rank (one all_gather_object when ws > 1; reporting only, after the timed
    region)."""
    parts = [local]
    if ws > 1:
        import torch.distributed as dist
        parts = [None] * ws
        dist.all_gather_object(parts, local)
    out = {}
    for name in local:
        merged = [None] * len(ks)
        for r, part in enumerate(parts):
            for i, v in zip(range(r, len(ks), ws), part[name]):
                merged[i] = v
        out[name] = merged
    return out


def sweep_bench(n_k: int, k_batch: int = 4, ws: int = 1, rank: int = 0, local: int = 0):
    """The wavenumber sweep (managers/sweep.py) of the augmented
    transmission operator over n_k wavenumbers, mixed precision against the
    plain FP64 path, both with the same FP64 block-Krylov norm estimator
    (one fused CGS2 launch per basis column) and the same k-batched assembly
    (k_batch wavenumbers per group); one JSON line with per-k times, phases,
    errors and the norm estimates.  On ws ranks (one GPU each) rank r takes
    the wavenumbers shard_wavenumbers(ks, r, ws) (no data exchange); each arm
    is timed with CUDA events between two barriers and the job time is the
    maximum over ranks.  Each arm first lets the autotuner choose its launch
    shapes (cached per device and problem) and runs one untimed k."""
    import torch
    from bem_b200.managers import CoreManager
    from bem_b200.managers.sweep import wavenumber_sweep
    from bem_b200.tuning import Autotuner
    from bem_b200.workloads import transmission_sweep_s4
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    res, tuned, total_ms = {}, {}, {}
    for prec in ("mixed", "fp64"):
        params, fD, fN, ks = transmission_sweep_s4(prec, n_k)
        mine = shard_wavenumbers(ks, rank, ws)
        params["solver"] = "lstsq"
        core = CoreManager(params)
        core.initialization(fD, fN)
        bm = core._BEM_manager
        bm._k = ks[0]
        tuned[prec] = bm.autotune(Autotuner(bm.engine))
        kw = dict(nrhs=4, seed=0, norm_tol=1e-6, norm_maxit=32, norm_method="iterative", k_batch=k_batch)
        wavenumber_sweep(bm, mine[:1] or ks[:1], **kw)  # warm-up
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res[prec] = wavenumber_sweep(bm, mine, **kw) if mine else {
            "k": [], "inv_norm": [], "cond": [], "solutions": [], "ms": [], "phase_ms": [], "iterations": []}
        e1.record()
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        total_ms[prec], _ = replicas_aggregate(e0.elapsed_time(e1), 1.0, ws, dev)
        res[prec]["launches"] = bm.engine.launches
        core.kill()
    local_lists = {
        "sol_err": [float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
                    for a, b in zip(res["mixed"]["solutions"], res["fp64"]["solutions"])],
        "norm_diff": [abs(a - b) / b for a, b in zip(res["mixed"]["inv_norm"], res["fp64"]["inv_norm"])],
        "inv_norm": res["mixed"]["inv_norm"], "cond": res["mixed"]["cond"],
        "blocks": res["mixed"]["iterations"],
        "ms_mixed": res["mixed"]["ms"], "ms_fp64": res["fp64"]["ms"],
        "phase_mixed": res["mixed"]["phase_ms"], "phase_fp64": res["fp64"]["phase_ms"],
    }
    g = sweep_gather(local_lists, ks, rank, ws)
    launches = sweep_gather({"l": [[res["mixed"]["launches"], res["fp64"]["launches"]]]}, list(range(ws)), rank, ws)
    if ws > 1:
        dist.destroy_process_group()
    if rank != 0:
        return

    def phases(lst):
        return {ph: statistics.mean(x[ph] for x in lst) for ph in ("assemble", "norm", "lstsq")}

    mixed_s, fp64_s = total_ms["mixed"] * 1e-3, total_ms["fp64"] * 1e-3
    print(json.dumps({
        "workload": "augmented transmission sweep A_I, icosphere s4, P1/P1 (5124 unknowns, stacked 10248 x 5124), "
                    "GaussQR=3, n_i=3, n_o=1, k = 16 + i/30, 4 complex Gaussian RHS per k",
        "n_k": len(ks), "k_range": [ks[0], ks[-1]], "n_gpus": ws,
        "scaling": "strong" if ws > 1 else None,
        "sharding": "rank r takes k_r, k_(r+N), ... (independent units, no data-path collective); job time = max over "
                    "ranks of the CUDA-event time between two barriers",
        "mixed_s": mixed_s, "plain_fp64_s": fp64_s, "speedup": fp64_s / mixed_s,
        "ms_per_k_mixed": mixed_s * 1e3 / len(ks), "ms_per_k_fp64": fp64_s * 1e3 / len(ks),
        "phase_ms_per_k": {"mixed": phases(g["phase_mixed"]), "fp64": phases(g["phase_fp64"])},
        "solution_rel_err_max": max(g["sol_err"]), "inv_norm_rel_diff_max": max(g["norm_diff"]),
        "inv_norm": g["inv_norm"], "cond": g["cond"],
        "norm_method": "both arms: energy-scaled operator by FP64 DMMA products, block Krylov of (S^H S)^{-1} "
                       "(8-vector blocks, the FP64 Cholesky inverse of the scaled S^H S) and of S^H S, CGS2 bases "
                       "(one cooperative launch per column), Ritz values from the CGS2 R of S Q, stop at 1e-6 "
                       "relative change or 32 blocks",
        "lstsq": {"mixed": "FP32 far-field assembly, FP16-split tcgen05 normal matrix, Cholesky with tcgen05 updates, "
                           "FP64 flexible GMRES per RHS",
                  "fp64": "FP64 assembly, DMMA normal matrix, Cholesky with DMMA updates, FP64 flexible GMRES "
                          "per RHS"},
        "autotuned": tuned,
        "norm_krylov_blocks": g["blocks"],
        "k_batch": k_batch,
        "assembly": "per group of k_batch wavenumbers k: V, K (with -K^T) and W each by one bem_assemble_batch call "
                    "over the 2 k_batch media wavenumbers (one far launch per pair of wavenumbers, geometry shared)",
        "gpu_launches": {"mixed": sum(x[0] for x in launches["l"]), "fp64": sum(x[1] for x in launches["l"])},
    }))


def shape_bench(subdiv: int, n_check: int):
    """The shape gradient of the Laplace Dirichlet problem on a radially
    perturbed icosphere (real spherical harmonics of degree <= 6, max |dr| =
    0.05), J = ||t - t_target||^2 with t_target from the unperturbed sphere,
    GaussQR = 5.  Times the mixed forward solve and the adjoint pass, and
    checks the adjoint gradient against central differences (h = 1e-6) of the
    FP64-assembled problem along seeded random directions at n_check vertices."""
    import numpy as np
    import torch
    from bem_b200 import icosphere
    from bem_b200.meshes import perturbed_sphere
    from bem_b200.shape import DirichletShape, DirichletShapeSolve, point_source
    v0, f = icosphere(subdiv)
    v, _ = perturbed_sphere(subdiv, lmax=6, amplitude=0.05, seed=0)
    u, gu = point_source()
    dev = torch.device("cuda")
    X0, X = torch.as_tensor(v0, device=dev), torch.as_tensor(v, device=dev)

    def grad_of(prob, t_target):
        Xg = X.clone().requires_grad_(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t = DirichletShapeSolve.apply(Xg, prob)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ((t - t_target) ** 2).sum().backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        return Xg.grad, (t1 - t0) * 1e3, (t2 - t1) * 1e3

    pm = DirichletShape(f, u, gu, gauss_qr=5, precision="mixed")
    tm = pm.forward(X0).clone()
    grad_of(pm, tm)  # warm-up
    Gm, fwd_ms, bwd_ms = grad_of(pm, tm)
    p64 = DirichletShape(f, u, gu, gauss_qr=5, precision="fp64", solver="mixed")
    t64 = p64.forward(X0).clone()
    G64, fwd64_ms, _ = grad_of(p64, t64)
    rng = np.random.default_rng(0)
    h = 1e-6
    errs = []
    for vi in rng.choice(len(v), size=n_check, replace=False):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        dt = torch.as_tensor(d, device=dev)
        Js = []
        for sgn in (1.0, -1.0):
            Xs = X.clone()
            Xs[int(vi)] += sgn * h * dt
            Js.append(float(((p64.forward(Xs) - t64) ** 2).sum()))
        fd = (Js[0] - Js[1]) / (2 * h)
        ad = float(G64[int(vi)] @ dt)
        errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
    gmax = float(G64.abs().max())
    print(json.dumps({
        "workload": f"shape gradient, Laplace Dirichlet, perturbed icosphere s{subdiv} ({len(f)} panels), "
                    "GaussQR=5, J = ||t - t_target||^2",
        "forward_ms_mixed": fwd_ms, "adjoint_ms": bwd_ms, "forward_ms_fp64_assembly": fwd64_ms,
        "fd_check": {"vertices": n_check, "h": h, "max_rel_err": max(errs), "median_rel_err": float(np.median(errs))},
        "mixed_vs_fp64_gradient_rel": float((Gm - G64).norm() / G64.norm()), "grad_max": gmax,
    }))


def transmission_bench(subdiv: int, plain: bool, solver: str = "lstsq"):
    """The Helmholtz transmission system (k_out = 5, k_in = 7.5) on
    icosphere s<subdiv> in mixed precision (solver "lstsq": the reference's
    least squares, tensor-core normal matrix and Cholesky, FP64 GMRES;
    "square": TF32 tile LU + FP64 refinement of the square system), its error
    against the FP64 path, and dJ/dk of J = ||x||^2 by the adjoint with the
    analytic operator derivative (managers/kderiv.py), in mixed precision and
    in FP64, against the fourth-order central difference of the FP64 J
    (delta = 1e-3)."""
    import torch
    from bem_b200.managers import CoreManager
    from bem_b200.managers.kderiv import solution_norm_k_gradient
    from bem_b200.workloads import transmission_s5
    res = {}
    params, pw = transmission_s5("mixed", subdiv, solver)
    core = CoreManager(params)
    core.initialization(pw.fD, pw.fN)
    b = core._BEM_manager
    b.run()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run()
    torch.cuda.synchronize()
    res["mixed_ms"] = (time.perf_counter() - t0) * 1e3
    res["refinement"] = {k: (v if not hasattr(v, "item") else v.item()) for k, v in b.solve_info.items()}
    x_mixed = b.raw_solved.clone()
    n = b.N_Neumann + b.M_Dirichlet
    gm = solution_norm_k_gradient(b, pw, check=False)
    core.kill()
    params, pw = transmission_s5("fp64", subdiv, solver)
    if solver == "square":
        params.update(solve_precision="mixed", refine_tol=1e-13)
    core = CoreManager(params)
    core.initialization(pw.fD, pw.fN)
    core._BEM_manager.run()
    x64 = core._BEM_manager.raw_solved.clone()
    g64 = solution_norm_k_gradient(core._BEM_manager, pw, check=True, delta=1e-3)
    core.kill()
    cd = g64["dJdk_central_difference"]
    res["dJdk"] = {"J": g64["J"], "central_difference_fp64": cd, "central_difference": g64["central_difference"],
                   "adjoint_mixed": gm["dJdk"], "rel_diff_mixed": abs(gm["dJdk"] - cd) / abs(cd),
                   "adjoint_fp64": g64["dJdk"], "rel_diff_fp64": abs(g64["dJdk"] - cd) / abs(cd),
                   "mixed_ms": {k: gm[k] for k in ("solve_ms", "adjoint_solve_ms", "derivative_assembly_ms",
                                                    "contraction_ms")},
                   "fp64_ms": {k: g64[k] for k in ("solve_ms", "adjoint_solve_ms", "derivative_assembly_ms",
                                                    "contraction_ms")}}
    res["rel_err_vs_fp64"] = {"l2": float(torch.linalg.norm(x_mixed - x64) / torch.linalg.norm(x64)),
                              "max": float((x_mixed - x64).abs().max() / x64.abs().max())}
    if plain:
        params, pw = transmission_s5("fp64", subdiv, solver)
        core = CoreManager(params)
        core.initialization(pw.fD, pw.fN)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        core._BEM_manager.run()
        torch.cuda.synchronize()
        res["plain_fp64_ms"] = (time.perf_counter() - t0) * 1e3
        res["speedup"] = res["plain_fp64_ms"] / res["mixed_ms"]
        core.kill()
    print(json.dumps(dict(workload=f"Helmholtz transmission, icosphere s{subdiv}, {n} unknowns, k_out=5, "
                                   f"k_in=7.5, GaussQR=5, solver {solver}", **res)))


def disk2d_bench(n_seg: int, gauss_qr: int, k: float, reps: int = 5):
    """The 2D path: Helmholtz interior Dirichlet on the reference's analytical
    disk (radius 1) with n_seg segments, P0 Neumann unknowns, P1 Dirichlet
    data of a plane wave.  Times the V block alone (CUDA events, mean of
    `reps` launches; entries/s = n_seg^2 / time), the whole assembly of the
    system (V + (1/2 M + K) g), the FP64 LU solve and the mixed solve, and
    times the oracle's numpy restatement of the same V rows on a 16-row
    sample on one host core."""
    import numpy as np
    import torch
    from bem_b200 import _lib as L
    from bem_b200.managers import CoreManager
    from bem_b200.meshes import analytical_disk
    from bem_b200.workloads import PlaneWave
    rng = np.random.default_rng(0)
    d = rng.standard_normal(2)
    d /= np.linalg.norm(d)
    pw = PlaneWave(k, d)
    v, f = analytical_disk(1.0, n_seg)
    # quirk=False: the right-hand side takes g, not conj(g), so that the
    # solution can be compared with the exact Neumann trace of the plane wave
    params = dict(dim=2, vertices=v, panels=f, kernel="Helmholtz", boundary="Dirichlet", scope="Interior",
                  GaussQR=gauss_qr, k=k, Q_Neumann=0, Q_Dirichlet=1, precision="fp64", solve_precision="fp64",
                  fuse=True, quirk=False)
    res = {}
    for solve in ("fp64", "mixed"):
        core = CoreManager(dict(params, solve_precision=solve))
        core.initialization(pw.fD, pw.fN)
        b = core._BEM_manager
        b.run()  # warm-up
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record()
        b.assemble_system()
        ev[1].record()
        b.solve()
        ev[2].record()
        torch.cuda.synchronize()
        res[solve] = {"assemble_ms": ev[0].elapsed_time(ev[1]), "solve_ms": ev[1].elapsed_time(ev[2]),
                      "x": b.raw_solved.clone(), "exact": b.raw_analytical_solved.clone(),
                      "info": {kk: (vv.item() if hasattr(vv, "item") else vv) for kk, vv in b.solve_info.items()}}
        if solve == "fp64":
            sp = b.space("charge", 0, "N", 0)
            V = torch.zeros(n_seg, n_seg, dtype=torch.complex128, device="cuda")
            desc = b.op_desc(L.OP_V, k, 1.0)
            b.engine.assemble(desc, sp, sp, V)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                b.engine.assemble(desc, sp, sp, V)
            e1.record()
            torch.cuda.synchronize()
            res["v_block_ms"] = e0.elapsed_time(e1) / reps
            del V
        core.kill()
    x64, xmx, ex = res["fp64"]["x"], res["mixed"]["x"], res["fp64"]["exact"]
    # CPU: the oracle's V rows for a sample of test segments
    from oracle import oracle2d as O2
    rows = 16
    p = np.arange(n_seg, dtype=np.int32)
    out = np.zeros((n_seg, n_seg), np.complex128)
    t0 = time.perf_counter()
    O2.assemble(v, f, 0, True, k, k * k, gauss_qr, (p[:rows], 1, p[:rows].copy()), (p, 1, p.copy()), out=out)
    cpu_s = time.perf_counter() - t0
    cpu_rate = rows * n_seg / cpu_s
    gpu_rate = n_seg * n_seg / (res["v_block_ms"] * 1e-3)
    print(json.dumps({
        "workload": f"2D Helmholtz interior Dirichlet, analytical disk r=1, {n_seg} segments, k={k}, "
                    f"GaussQR={gauss_qr}, P0 Neumann unknowns, plane-wave data, quirk=False",
        "v_block_ms": res["v_block_ms"], "v_entries_per_s": gpu_rate,
        "v_pair_points_per_s": gpu_rate * gauss_qr ** 2,
        "assemble_system_ms": res["fp64"]["assemble_ms"],
        "solve_fp64_lu_ms": res["fp64"]["solve_ms"], "solve_mixed_ms": res["mixed"]["solve_ms"],
        "mixed_refinement": res["mixed"]["info"],
        "mixed_vs_fp64_rel_err": float(torch.linalg.norm(xmx - x64) / torch.linalg.norm(x64)),
        "fp64_vs_exact_trace_rel_err": float(torch.linalg.norm(x64 - ex) / torch.linalg.norm(ex)),
        "cpu_baseline": {"value": cpu_rate, "unit": "entries/s", "cores": 1, "kind": "port",
                         "sample": f"oracle/oracle2d.py (numpy, scipy Hankel) V rows 0..{rows - 1} x {n_seg}"},
        "gpu_vs_cpu_entries": gpu_rate / cpu_rate,
    }))


def reference_line(args, workload, fn):
    """The reference arm: the reference's algorithm on the host cores (the
    oracle's FP32 restatement of its loops), one JSON line."""
    base = {"metric": METRIC, "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": {"workload": workload, "host": "cpu"}}
    cb = fn(args.steps, max(1, min(args.warmup, 1)))
    base.update(value=cb["value"], unit="entries/s", ms_per_step=cb["seconds_per_sample"] * 1e3,
                cpu_baseline=cb, e2e={"value": cb["value"], "unit": "entries/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0})
    print(json.dumps(base))


def cpu_reference_transmission(steps: int, warmup: int, threads: int | None = None, target_s: float = 10.0):
    """The reference's transmission assembly on the host: the oracle's FP32
    restatement of its loops (one outer iteration per test panel, serial
    over trial panels x GaussQR^4, per-basis recompute) for V, K and W at both
    wavenumbers, on a sample of test panels; its time is scaled by the
    sampled fraction of the test panels to the whole assembly, and the rate
    is the stacked system's 2 n^2 entries over that time (the assembly alone,
    without the reference's least-squares solve: a bound in the CPU's
    favour)."""
    import numpy as np

    from bem_b200 import icosphere
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    O.set_threads(threads)
    v, f = icosphere(5)
    nt, nv = len(f), len(v)
    n = nt + nv
    Q = 5
    panels = np.arange(nt, dtype=np.int32)
    p1dof = f.reshape(-1).astype(np.int32)

    def one(rows):
        tp = panels[:rows]
        t0 = time.perf_counter()
        for sqrt_n in (1.0, 1.5):
            k = 5.0 * sqrt_n
            V = np.zeros((rows, nt), np.complex128)
            O.assemble(v, f, O.OP_V, True, k, k * k, Q, True, (tp, 1, tp.copy()), (panels, 1, panels.copy()), out=V,
                       fp32=True)
            K = np.zeros((rows, nv), np.complex128)
            O.assemble(v, f, O.OP_K, True, k, k * k, Q, True, (tp, 1, tp.copy()), (panels, 3, p1dof), out=K,
                       fp32=True)
            # W rows per (test panel, vertex) slot: the same work as the vertex rows, in a compact output
            W = np.zeros((3 * rows, nv), np.complex128)
            O.assemble(v, f, O.OP_W, True, k, k * k, Q, True, (tp, 3, np.arange(3 * rows, dtype=np.int32)),
                       (panels, 3, p1dof), out=W, fp32=True)
        return time.perf_counter() - t0

    t1 = one(threads)
    rows = int(min(nt, threads * max(1, round(target_s / max(t1, 1e-3)))))
    for _ in range(warmup):
        one(max(1, rows // 4))
    times = [one(rows) for _ in range(steps)]
    t = statistics.mean(times)
    full_s = t * nt / rows
    value = 2.0 * n * n / full_s
    return {"value": value, "unit": "entries/s", "cores": threads, "kind": "port",
            "sample": f"V, K and W rows of {rows} of {nt} test panels at both wavenumbers, FP32, {steps} timed "
                      f"samples; whole assembly extrapolated to {full_s:.1f} s",
            "seconds_per_sample": t}


def transmission_headline(args, ws, rank, local):
    """The north-star line: the Helmholtz transmission problem on icosphere s5
    (TRANS_WORKLOAD), mixed precision (FP32 far field in the fused Calderon
    sweep, FP64 near field, FP16-split tensor-core normal matrix, Cholesky
    with tensor-core updates into an FP64 Schur complement, FP64 flexible
    GMRES on the normal equations) against the plain FP64 path (FP64 sweep,
    DMMA normal matrix, Cholesky with DMMA updates, the same FP64
    iteration), whose solution is the FP64 oracle of the error."""
    import torch
    import torch.distributed as dist

    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from bem_b200.engine import measure_peaks
    from bem_b200.managers import CoreManager
    from bem_b200.workloads import transmission_s5
    subdiv = args.trans_subdiv

    def make(precision, vertices=None, panels=None):
        params, pw = transmission_s5(precision, subdiv, "lstsq")
        params["device"] = f"cuda:{local}"
        if vertices is not None:
            params.update(vertices=vertices, panels=panels)
        core = CoreManager(params)
        core.initialization(pw.fD, pw.fN)
        return core

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    # ---- mixed path: device-timed steps ----
    core = make("mixed")
    b = core._BEM_manager
    eng = b.engine
    n = b.N_Neumann + b.M_Dirichlet
    nt = b.num_of_panels
    entries = 2 * n * n  # the stacked system [A; P+_i]
    peaks = measure_peaks(eng)
    # launch shapes chosen by the autotuner (timed here, in the warm-up, unless cached)
    tuned = {"mixed": b.autotune()}
    for _ in range(args.warmup):
        b.run()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = eng.launches
    evs = [(ev(), ev()) for _ in range(args.steps)]
    for s_ in range(args.steps):
        flush.fill_(1.0)
        evs[s_][0].record()
        b.run()
        evs[s_][1].record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = eng.launches - launches0
    step_ms = [a.elapsed_time(z) for a, z in evs]
    info = {k: (v.item() if hasattr(v, "item") else v) for k, v in b.solve_info.items()}
    sol_mixed = b.raw_solved.clone()
    ms, value = replicas_aggregate(statistics.mean(step_ms), entries, ws, dev)

    # ---- phases of one step, each kernel phase timed on its own ----
    phases = {}

    def timed(name, fn):
        e0, e1 = ev(), ev()
        torch.cuda.synchronize()
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        phases[name] = e0.elapsed_time(e1)
        return r

    timed("assemble_calderon_mass_rhs", b.assemble_system)
    A, P = b._mat_A, b._mat_P
    d = torch.empty(n, dtype=torch.float64, device=dev)
    Nm = torch.empty(n, n, dtype=torch.complex128, device=dev)
    timed("normal_matrix_tensor_cores", lambda: eng.gram(A, P, Nm, d, tensor_cores=True))
    piv, dinv, _ = timed("cholesky_tensor_cores", lambda: eng.chol_factor(Nm, tensor_cores=True))
    x = torch.zeros(n, dtype=A.dtype, device=dev)
    timed("fgmres_fp64", lambda: eng.lstsq_refine(A, P, d, Nm, piv, dinv, b.rhs, x, tol=b.lstsq_tol,
                                                  maxit=b.lstsq_maxit, accept=b.lstsq_accept))
    del Nm, piv, dinv
    # the far-field sweep alone (both wavenumbers in one launch), for its roofline
    neu = b.space("charge", 0, "N", 0, offset=b._Neumann_offset_i)
    dir_ = b.space("charge", 1, "D", 1, offset=b._Dirichlet_offset_i)
    from bem_b200 import _lib as L
    desc = b.op_desc(L.OP_V, b._k, 1.0)
    ks, k2s = [], []
    for sqrt_n in (b._sqrt_no, b._sqrt_ni):
        dd = b.op_desc(L.OP_V, b._k, sqrt_n)
        ks.append(dd.k)
        k2s.append(dd.k2)
    A.zero_()
    P.zero_()
    timed("calderon_sweep_with_near", lambda: eng.assemble_calderon(desc, ks, k2s, neu, dir_, [A, P], [-1.0, 1.0]))
    near = eng.near_pairs
    core.kill()
    del core, b, A, P
    torch.cuda.empty_cache()

    # ---- e2e through the public API: host mesh in, solution out, one lifecycle per step ----
    from bem_b200 import icosphere
    vh, fh = icosphere(subdiv)
    vpin = torch.as_tensor(vh).pin_memory()
    fpin = torch.as_tensor(fh).pin_memory()
    e2e_ms, d2h = [], 0
    h2d = vh.nbytes + fh.nbytes
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c2 = make("mixed", vpin.numpy(), fpin.numpy())
        c2._BEM_manager.autotune()  # the cached choices
        c2._BEM_manager.run()
        host = c2._BEM_manager.raw_solved.to("cpu")
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        d2h = host.numel() * host.element_size()
        c2.kill()
        del c2
        torch.cuda.empty_cache()
    e2e, e2e_value = replicas_aggregate(statistics.median(e2e_ms[1:]), entries, ws, dev)

    # ---- plain FP64 path (its solution is the FP64 oracle of the error) ----
    core64 = make("fp64")
    b64 = core64._BEM_manager
    tuned["fp64"] = b64.autotune()
    b64.run()
    torch.cuda.synchronize()
    ms64 = []
    for _ in range(args.plain_steps):
        flush.fill_(1.0)
        e0, e1 = ev(), ev()
        e0.record()
        b64.run()
        e1.record()
        torch.cuda.synchronize()
        ms64.append(e0.elapsed_time(e1))
    sol64 = b64.raw_solved.clone()
    info64 = {k: (v.item() if hasattr(v, "item") else v) for k, v in b64.solve_info.items()}
    p64 = {}
    e0, e1 = ev(), ev()
    e0.record()
    b64.assemble_system()
    e1.record()
    torch.cuda.synchronize()
    p64["assemble_calderon_mass_rhs"] = e0.elapsed_time(e1)
    A64, P64 = b64._mat_A, b64._mat_P
    N64 = torch.empty(n, n, dtype=torch.complex128, device=dev)
    d64 = torch.empty(n, dtype=torch.float64, device=dev)
    e0, e1 = ev(), ev()
    e0.record()
    b64.engine.gram(A64, P64, N64, d64, tensor_cores=False)
    e1.record()
    torch.cuda.synchronize()
    p64["normal_matrix_fp64_dmma"] = e0.elapsed_time(e1)
    e0, e1 = ev(), ev()
    e0.record()
    b64.engine.chol_factor(N64, tensor_cores=False)
    e1.record()
    torch.cuda.synchronize()
    p64["cholesky_fp64_dmma"] = e0.elapsed_time(e1)
    del N64
    qr = None
    if args.qr_check:
        # numpy-free FP64 QR least squares of the same stacked system (cuSOLVER
        # via torch, used here only as the checker of the normal-equation solution)
        G = torch.cat([A64, P64], 0)
        xq = torch.linalg.lstsq(G, b64.rhs.unsqueeze(1)).solution.squeeze(1)
        qr = {"fp64_normal_eq_vs_qr_l2": float(torch.linalg.norm(sol64 - xq) / torch.linalg.norm(xq)),
              "mixed_vs_qr_l2": float(torch.linalg.norm(sol_mixed - xq) / torch.linalg.norm(xq)),
              "mixed_vs_qr_max": float((sol_mixed - xq).abs().max() / xq.abs().max())}
        del G, xq
    core64.kill()
    del core64, b64, A64, P64
    torch.cuda.empty_cache()
    rel2 = float(torch.linalg.norm(sol_mixed - sol64) / torch.linalg.norm(sol64))
    relm = float((sol_mixed - sol64).abs().max() / sol64.abs().max())

    # ---- rooflines of the kernels of the step ----
    tr = (2 * n + 127) // 128
    gram_flops = 8.0 * n ** 3  # the Hermitian product (A^H A + P^H P): 2n x n complex
    q4 = 625
    evals = (nt * nt - near) // 2 * q4
    kern = {
        "gram_tc_kernel": {"bound": "tensor", "ms": phases["normal_matrix_tensor_cores"],
                           "achieved": gram_flops / (phases["normal_matrix_tensor_cores"] * 1e-3) / 1e12,
                           "peak": MEASURED["bf16_tflops"], "unit": "TFLOP/s",
                           "note": "algorithmic 8 n^3 flops of the Hermitian product; the tensor pipe executes "
                                   "three FP16 products per product (hi hi, hi lo, lo hi) on "
                                   f"{tr * (tr + 1) // 2} lower 128 x 128 real tiles"},
        "cholesky": {"bound": "tensor", "ms": phases["cholesky_tensor_cores"],
                     "achieved": 4.0 / 3.0 * n ** 3 / (phases["cholesky_tensor_cores"] * 1e-3) / 1e12,
                     "peak": MEASURED["bf16_tflops"], "unit": "TFLOP/s",
                     "note": "4/3 n^3 flops of the complex Cholesky; panels in FP64 on DMMA, trailing rank-1024 "
                             "updates on tcgen05 (three FP16 products per product) into the FP64 Schur complement"},
        "far_calderon_kernel": {"bound": "fp32", "ms": phases["calderon_sweep_with_near"],
                                "achieved": evals * CAL_FLOPS_PER_EVAL / (phases["calderon_sweep_with_near"] * 1e-3)
                                / 1e12, "peak": peaks[0], "unit": "TFLOP/s",
                                "note": f"{CAL_FLOPS_PER_EVAL} flops per evaluation, {evals} evaluations; timed "
                                        "with its FP64 near-pair kernels in one call"},
    }
    for kv in kern.values():
        kv["frac"] = kv["achieved"] / kv["peak"]
    top = max(kern, key=lambda k_: kern[k_]["ms"])
    roof = dict(kern[top])
    roof["kernel"] = top
    roof["traffic"] = None
    roof["peak_source"] = {"tensor": "MEASURED_PEAKS.json bf16_tflops (burst)",
                           "fp32": "bem_measure_peaks FP32 FMA probe on this GPU",
                           "fp64": "bem_measure_peaks FP64 FMA probe on this GPU"}[roof["bound"]]

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            cpu = cpu_reference_transmission(1, 0)
        except Exception as exc:  # the baseline never blocks the GPU line
            cpu = {"value": None, "error": repr(exc)}
    if ws > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "entries/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "c64 far field / c128 near field, FP16-split tensor-core normal matrix and Cholesky updates "
                     "(FP64 sums), FP64 refinement",
            "data": "synthetic (generated icosphere, analytic plane wave)",
            "config": {"workload": TRANS_WORKLOAD, "unknowns": n, "stacked_entries": entries, "precision": "mixed",
                       "quirk": "reference quadrature", "l2": "inputs larger than L2; 256 MiB flush between steps",
                       "parallelism": f"replicas x{ws}"},
            "time_to_solution_ms": ms, "step_ms": step_ms, "ms_per_step_median": statistics.median(step_ms),
            "breakdown_ms": phases,
            "plain_fp64": {"time_to_solution_ms": statistics.mean(ms64), "step_ms": ms64, "breakdown_ms": p64,
                           "solve": info64},
            "speedup_vs_plain_fp64": statistics.mean(ms64) / ms,
            "autotuned": tuned,
            "rel_err_vs_fp64": {"l2_rel": rel2, "max_abs_rel": relm},
            "qr_check": qr,
            "solve": info,
            "e2e": {"value": e2e_value, "unit": "entries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e},
            "roofline": roof, "kernels": kern,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--profile-step", default=None, choices=["mixed", "fp64"],
                    help="run one warm-up and one step of the workload and exit (for ncu captures)")
    ap.add_argument("--calderon-group", type=int, default=0,
                    help="form of the fused Calderon sweep in --profile-step (the BEM_TUNE_CALDERON_GROUP value)")
    ap.add_argument("--gram-form", type=int, default=0,
                    help="form of the tensor-core normal matrix in --profile-step (BEM_TUNE_GRAM_PAIR value)")
    ap.add_argument("--lu-update", type=int, default=0,
                    help="form of the tile LU's large trailing updates in --profile-lu (BEM_TUNE_LU_UPDATE value)")
    ap.add_argument("--profile-lu", type=int, default=0,
                    help="time six tiled FP32 factorisations of a random complex matrix of this size and exit")
    ap.add_argument("--workload", default="transmission_s5",
                    choices=["transmission_s5", "dirichlet_s4", "sweep", "shape", "transmission_dk", "disk2d"],
                    help="transmission_s5: the headline line (the 20480-panel transmission problem); dirichlet_s4: "
                         "Helmholtz interior Dirichlet on 5120 panels; sweep: the wavenumber sweep of the "
                         "augmented transmission operator; shape: the shape gradient on a perturbed sphere; "
                         "transmission_dk: the transmission solve with dJ/dk through the adjoint; disk2d: the 2D operators "
                         "(each its own JSON line)")
    ap.add_argument("--plain-steps", type=int, default=1, help="timed steps of the plain FP64 comparator")
    ap.add_argument("--qr-check", action="store_true",
                    help="also solve the FP64 stacked system by QR (torch.linalg.lstsq) as a checker")
    ap.add_argument("--no-cpu", action="store_true", help="skip the timed CPU baseline")
    ap.add_argument("--disk-n", type=int, default=8192, help="segments of the disk2d workload")
    ap.add_argument("--shape-subdiv", type=int, default=5, help="icosphere subdivision of the shape workload")
    ap.add_argument("--shape-check", type=int, default=32, help="vertices of the finite-difference check")
    ap.add_argument("--trans-subdiv", type=int, default=5, help="icosphere subdivision of the transmission workload")
    ap.add_argument("--trans-plain", action="store_true", help="also time the plain FP64 path (FP64 LU)")
    ap.add_argument("--trans-solver", default="lstsq", choices=["square", "lstsq"],
                    help="solver of the transmission_dk workload")
    ap.add_argument("--sweep-k", type=int, default=60, help="number of wavenumbers of the sweep workload")
    ap.add_argument("--k-batch", type=int, default=4,
                    help="wavenumbers assembled together by the sweep workload (1: one k at a time)")
    args = ap.parse_args()
    ws, rank, local = _dist()
    if args.workload == "sweep":
        sweep_bench(args.sweep_k, args.k_batch, ws, rank, local)
        return
    if args.workload == "shape":
        if rank == 0:
            shape_bench(args.shape_subdiv, args.shape_check)
        return
    if args.workload == "transmission_dk":
        if rank == 0:
            transmission_bench(args.trans_subdiv, args.trans_plain, args.trans_solver)
        return
    if args.workload == "disk2d":
        if rank == 0:
            disk2d_bench(args.disk_n, 5, 3.0)
        return
    if args.profile_step:
        profile_step(args.profile_step, args.workload, args.trans_subdiv, args.calderon_group, args.gram_form)
        return
    if args.profile_lu:
        profile_lu(args.profile_lu, args.lu_update)
        return

    if args.workload == "dirichlet_s4":
        if args.impl == "reference":
            if rank == 0:
                reference_line(args, WORKLOAD, cpu_reference)
            return
        dirichlet_headline(args, ws, rank, local)
        return
    if args.impl == "reference":
        if rank == 0:
            reference_line(args, TRANS_WORKLOAD, cpu_reference_transmission)
        return
    transmission_headline(args, ws, rank, local)


def dirichlet_headline(args, ws, rank, local):
    """The config-2 line (Helmholtz interior Dirichlet, icosphere s4): see
    WORKLOAD."""
    import torch
    import torch.distributed as dist

    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    from bem_b200.engine import measure_peaks
    from bem_b200.managers import CoreManager
    from bem_b200.workloads import helmholtz_dirichlet_s4

    def make(precision, extra=None):
        params, fD, fN = helmholtz_dirichlet_s4(precision=precision)
        params["device"] = f"cuda:{local}"
        if extra:
            params.update(extra)
        core = CoreManager(params)
        core.initialization(fD, fN)
        return core

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush_l2():
        flush.fill_(1.0)

    # ---- mixed path: device-timed steps ----
    core = make("mixed")
    b = core._BEM_manager
    nt = b.num_of_panels
    entries = nt * nt
    eng = b.engine
    peaks = measure_peaks(eng)
    for _ in range(args.warmup):
        b.run()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = eng.launches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    factors = []
    for s in range(args.steps):
        flush_l2()
        ev[s][0].record()
        b.run()
        ev[s][1].record()
        factors.append(b.solve_info.get("factor"))
    torch.cuda.synchronize()
    launches = eng.launches - launches0
    step_ms = [a.elapsed_time(z) for a, z in ev]
    # the dominant kernel of the step, the fused far-field sweep, through its
    # C-ABI call (bem_assemble_dirichlet, which also launches the FP64
    # near-pair kernels on the same stream), for the roofline
    va = []
    for s in range(args.steps):
        flush_l2()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.fused_assembly_call()
        e1.record()
        torch.cuda.synchronize()
        va.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    breakdown = phase_breakdown(b)
    info = dict(b.solve_info)
    sol_mixed = b.raw_solved.clone()
    ms, value = replicas_aggregate(statistics.mean(step_ms), entries, ws, dev)

    # ---- e2e through the public API, host inputs, solution read back ----
    from bem_b200 import icosphere
    vh, fh = icosphere(4)
    vpin = torch.as_tensor(vh).pin_memory()
    fpin = torch.as_tensor(fh).pin_memory()
    e2e_ms = []
    h2d = vh.nbytes + fh.nbytes
    d2h = 0
    for s in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        params, fD, fN = helmholtz_dirichlet_s4(precision="mixed")
        params.update(device=f"cuda:{local}", vertices=vpin.numpy(), panels=fpin.numpy())
        c2 = CoreManager(params)
        c2.initialization(fD, fN)
        c2._BEM_manager.run()
        host = c2._BEM_manager.raw_solved.to("cpu")
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        d2h = host.numel() * host.element_size()
        c2.kill()
    # the first lifecycle of the loop is discarded; whole job: max over ranks
    e2e, e2e_value = replicas_aggregate(statistics.median(e2e_ms[1:]), entries, ws, dev)

    # ---- plain FP64 path (the FP64 oracle of the mixed result) ----
    core64 = make("fp64")
    b64 = core64._BEM_manager
    b64.run()
    torch.cuda.synchronize()
    ms64 = []
    for _ in range(2):
        flush_l2()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b64.run()
        e1.record()
        torch.cuda.synchronize()
        ms64.append(e0.elapsed_time(e1))
    # the same assembly work on the plain path: V (one kernel per operator)
    # and the right-hand side 1/2 M g + K g (matrix-free)
    va64 = []
    for _ in range(2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b64.single_layer.forward(b64._scope_type, b64._k, 1.0)
        b64.rhs_layer_forward(k=b64._k, scope_type=b64._scope_type)
        e1.record()
        torch.cuda.synchronize()
        va64.append(e0.elapsed_time(e1))
    sol64 = b64.raw_solved
    rel = float((sol_mixed - sol64).abs().max() / sol64.abs().max())
    rel2 = float(torch.linalg.norm(sol_mixed - sol64) / torch.linalg.norm(sol64))
    core64.kill()
    del core64, b64
    torch.cuda.empty_cache()

    # roofline of the dominant kernel: the fused symmetric far-field sweep
    q4 = 625
    near = eng.near_pairs
    evals = (nt * nt - near) // 2 * q4  # unordered separate pairs x GaussQR^4
    va_ms = statistics.mean(va)
    achieved = evals * FLOPS_PER_EVAL / (va_ms * 1e-3) / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peaks[0], "unit": "TFLOP/s",
            "frac": achieved / peaks[0],
            # DRAM read + write of one far_vkg_sym_x2_kernel launch of this workload, one ncu capture
            "traffic": FAR_SWEEP_DRAM_BYTES,
            "kernel": "far_vkg_sym_x2_kernel<Helmholtz> (packed FP32x2; timed with its FP64 near-pair kernels "
                      "in one call)",
            "peak_source": "bem_measure_peaks FP32 FMA probe on this GPU (MEASURED_PEAKS.json has HBM and bf16 only)",
            "flops_per_eval": FLOPS_PER_EVAL, "flops_per_eval_executed": 63, "evals_per_launch": evals,
            "call_ms": va_ms,
            "mufu": {"achieved_gops": evals * MUFU_PER_EVAL / (va_ms * 1e-3) / 1e9, "peak_gops": peaks[2]},
            "fp64_peak_tflops": peaks[1]}

    cpu = None
    if rank == 0 and ws == 1:
        try:
            cpu = cpu_reference(1, 0)
        except Exception as exc:  # the baseline never blocks the GPU line
            cpu = {"value": None, "error": repr(exc)}

    if ws > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "entries/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 far field / c128 near field + FP32 LU + FP64 refinement",
            "data": "synthetic (generated icosphere, analytic plane wave)",
            "config": {"workload": WORKLOAD, "panels": nt, "entries": entries, "precision": "mixed",
                       "quirk": "reference quadrature", "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas x{ws}"},
            "time_to_solution_ms": ms,
            "step_ms": step_ms,
            "ms_per_step_median": statistics.median(step_ms),
            "step_factor": factors,
            "assembly_entries_per_s": entries / (va_ms * 1e-3),
            "assembly_ms": va_ms,
            "assembly": "V and K g in one symmetric FP32 far sweep + FP64 near pairs",
            "plain_fp64": {"time_to_solution_ms": statistics.mean(ms64),
                           "assembly_entries_per_s": entries / (statistics.mean(va64) * 1e-3),
                           "assembly_ms": statistics.mean(va64),
                           "assembly": "V (FP64, all ordered pairs) + matrix-free 1/2 M g + K g"},
            "speedup_vs_plain_fp64": statistics.mean(ms64) / ms,
            "rel_err_vs_fp64": {"max_abs_rel": rel, "l2_rel": rel2},
            "refinement": {k: (v if not hasattr(v, "item") else v.item()) for k, v in info.items()},
            "e2e": {"value": e2e_value, "unit": "entries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e},
            "roofline": roof,
            "cpu_baseline": cpu,
            "breakdown_ms": breakdown,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line))
    core.kill()
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
