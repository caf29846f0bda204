"""Benchmark of the determinant-space Hamiltonian hot path on B200.

Workload (one GPU, N=1): a synthetic 30-orbital, 24-electron (12 alpha /
12 beta) system with Cholesky-form integrals (K = 60), 1,000,000 unique
determinants from seeded iterated heat-bath sampling (excitation level <= 4
from HF), static heat-bath screening eps1 = 1e-6.

One step = the hot path of one outer iteration on that space:
  1. screened build of H_VV (singles + heat-bath doubles, Slater-Condon
     elements, V lookup, CSR assembly) on the device;
  2. H.psi with FP64 values -> local energies E_loc,i = (H psi)_i / psi_i
     and the Rayleigh quotient;
  3. the same with FP32 values and compensated FP32 accumulation
     (|dE| against step 2 reported).

`value` = screened H elements (nnz of H_VV) per second over the whole step,
inputs resident in HBM; `e2e` = the same through the C ABI with host
buffers (pinned host -> device copy of the determinants and psi, local
energies copied back).  Under torchrun each rank builds its own system of
the same size (seed + rank): weak scaling, no collective on the data path.

`--workload batched`: 64 systems of uneven size (n_orb 10..40, 1e3..2e5
determinants each, eps1 = 1e-7) rebuilt and contracted together in one
graph-replayed step with FP32-compensated H.psi and autotuned tunables,
beside the plain FP64 path that builds and contracts one system at a time.

`--workload serving`: a Poisson stream (200 req/s) of screened-H builds and
local-energy requests over 54 systems (the batched size distribution plus
bond-scan families) served by the device-resident loop with continuous
batching, beside the same stream served one request at a time in FP64;
p50/p99 latency.

`--workload downfold`: 100 orbitals (two-word determinants), S = 1e5,
dynamic amplitude screening at eps1 = 1e-5 into C ~ 1e7 external
determinants, and the downfolded H_eff in FP64 and FP32 values; |dE| of the
lowest eigenvalue (device Lanczos) between the two.

`--workload det_batch`: the neural models' determinant batch features
(prepare_det_batch) for the single workload's 1e6 determinants, every
field, relative to HF.

`--workload slogdet`: sign, log|det| and its gradient for 32768 10x10 FP64
matrices (the batched log-det of the neural models).

`--impl reference` times the reference DetNQS C++ core (compiled from its
sources into oracle/_ref) on a bounded sample of rows of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ORB, N_ALPHA, N_BETA, N_CHOL = 30, 12, 12, 60
N_DETS = 1_000_000
EPS1 = 1e-6
SMS = 148          # B200 streaming multiprocessors
INT_SEED, DET_SEED, PSI_SEED = 1001, 2002, 3003
CACHE = os.path.join(tempfile.gettempdir(), "detnqs_b200_bench")
_T0 = time.perf_counter()


def _log(msg: str) -> None:
    """Progress on stderr (the JSON line is the only stdout output)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def workload(rank: int, n_dets: int):
    from detnqs_b200 import synthetic as S
    si, sd, sp = rank_seeds(rank)
    sysm = S.make_system(N_ORB, N_ALPHA, N_BETA, N_CHOL, si)
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"dets_{N_ORB}_{n_dets}_{sd}_{si}.npy")
    if os.path.exists(path):
        V = np.load(path)
    else:
        V = S.heat_bath_sample(sysm, n_dets, sd)
        np.save(path, V)
    psi = S.normalized_psi(n_dets, sp)
    return sysm, V, psi


class ClockSampler:
    """nvidia-smi sampling during the timed region.

    nvidia-smi's start-up (driver queries) stalls CUDA calls of the same
    process for up to a few hundred milliseconds, so start() returns only
    after the first sample has arrived: callers start it before their
    warm-up steps and bracket the timed steps with begin() / end(); the
    statistics use the samples taken between the two (all samples when the
    timed region was shorter than one sampling interval)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[tuple[float, str]] = []
        self.t_begin = None
        self.t_end = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None

    def begin(self):
        self.t_begin = time.perf_counter()

    def end(self):
        self.t_end = time.perf_counter()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        lines = [ln for t, ln in self.lines
                 if (self.t_begin is None or t >= self.t_begin)
                 and (self.t_end is None or t <= self.t_end + 0.25)]
        if not lines:
            lines = [ln for _, ln in self.lines]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Max of a per-rank timing over all ranks (all_reduce MAX); identity
    when running alone.  `device` is the tensor device of the process
    group's backend (cuda for NCCL, cpu for gloo)."""
    if world <= 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def rank_seeds(rank: int):
    """(integral, determinant, psi) seeds of a rank: every rank gets its own
    system of the same size (weak scaling)."""
    return INT_SEED + rank, DET_SEED + rank, PSI_SEED + rank


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(kernel)


# ---------------------------------------------------------------------------
# reference CPU path
# ---------------------------------------------------------------------------

def cpu_reference_sample(sysm, V, target_s: float = 15.0, min_rows: int = 64,
                         probe_rows: int = 1024):
    """Time the reference core's static heat-bath H_VV rows on a bounded
    sample of rows of the same workload.  Returns (elements/s, rows, nnz,
    seconds, threads, kind)."""
    import oracle
    if not os.path.exists(oracle.PORT_LIB):
        oracle.build(None)
    kind = "reference" if oracle.Checker.reference_available() else "port"
    chk = oracle.Checker.reference() if kind == "reference" else oracle.Checker.port()
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    with tempfile.TemporaryDirectory() as d:
        from detnqs_b200 import synthetic as S
        if kind == "reference":
            fd = os.path.join(d, "sys.fcidump")
            S.write_fcidump(fd, sysm)
            ctx = chk.ctx_from_fcidump(fd, N_ORB)
        else:
            ctx = chk.ctx_from_arrays(N_ORB, sysm.h1e, sysm.eri, sysm.e_core)
        ctx.hb_prepare(1e-15)
        rng = np.random.default_rng(77)
        rows = np.sort(rng.choice(len(V), min(probe_rows, len(V)), replace=False))
        t0 = time.perf_counter()
        r = ctx.vv_hb_rows(V, rows, EPS1)
        t_probe = time.perf_counter() - t0
        # the map of V is built inside each call; time it separately (the
        # faster of two calls: host noise only adds time)
        t_map = t_probe
        for _ in range(2):
            t0 = time.perf_counter()
            ctx.vv_hb_rows(V, rows[:1], EPS1)
            t_map = min(t_map, time.perf_counter() - t0)
        # a noisy probe must not size the sample past its bound: a row costs
        # at least a quarter of the probe's time per row
        per_row = max(t_probe - t_map, 0.25 * t_probe) / len(rows)
        n_rows = int(min(len(V), max(min_rows, (target_s - t_map) / per_row)))
        rows = np.sort(rng.choice(len(V), n_rows, replace=False))
        t0 = time.perf_counter()
        r = ctx.vv_hb_rows(V, rows, EPS1)
        t = time.perf_counter() - t0
        nnz = len(r["val"])
    return nnz / t, n_rows, nnz, t, threads, kind


def cpu_reference_rows(systems, target_s: float = 15.0, probe_rows: int = 1024, seed: int = 77):
    """Reference core's static heat-bath H_VV rows on a sample of rows drawn
    uniformly from the concatenated rows of many systems (sysm, V, eps1).
    Context creation and the per-call map of V stay outside the timing.
    Returns (elements/s, rows, elements, seconds, threads, kind)."""
    import oracle
    from detnqs_b200 import synthetic as S
    if not os.path.exists(oracle.PORT_LIB):
        oracle.build(None)
    kind = "reference" if oracle.Checker.reference_available() else "port"
    chk = oracle.Checker.reference() if kind == "reference" else oracle.Checker.port()
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    sizes = np.array([len(V) for _, V, _ in systems], np.int64)
    off = np.concatenate([[0], np.cumsum(sizes)])
    rng = np.random.default_rng(seed)
    with tempfile.TemporaryDirectory() as d:
        ctxs = {}

        def ctx_of(k):
            if k not in ctxs:
                sysm = systems[k][0]
                if kind == "reference":
                    fd = os.path.join(d, f"sys{k}.fcidump")
                    S.write_fcidump(fd, sysm)
                    c = chk.ctx_from_fcidump(fd, sysm.n_orb)
                else:
                    c = chk.ctx_from_arrays(sysm.n_orb, sysm.h1e, sysm.eri, sysm.e_core)
                c.hb_prepare(1e-15)
                ctxs[k] = c
            return ctxs[k]

        def run(n_rows):
            g = np.sort(rng.choice(off[-1], min(n_rows, off[-1]), replace=False))
            which = np.searchsorted(off, g, side="right") - 1
            t_all = 0.0
            t_calls = 0.0
            nnz = 0
            for k in np.unique(which):
                _, V, eps = systems[k]
                rows = g[which == k] - off[k]
                c = ctx_of(k)
                # the map of V is built inside each call: the faster of two
                # one-row calls (host noise only adds time)
                t_map = float("inf")
                for _ in range(2):
                    t0 = time.perf_counter()
                    c.vv_hb_rows(V, rows[:1], eps)
                    t_map = min(t_map, time.perf_counter() - t0)
                t0 = time.perf_counter()
                r = c.vv_hb_rows(V, rows, eps)
                t_call = time.perf_counter() - t0
                t_calls += t_call
                t_all += max(t_call - t_map, 0.0)
                nnz += len(r["val"])
            return len(g), nnz, t_all, t_calls

        rows, nnz, t, t_calls = run(probe_rows)
        # a noisy probe must not size the sample past its bound: a row costs
        # at least a quarter of the probe's whole call time per row
        per_row = max(t, 0.25 * t_calls) / max(rows, 1)
        rows, nnz, t, _ = run(int(max(probe_rows, target_s / per_row)))
    return nnz / max(t, 1e-9), rows, nnz, t, threads, kind


def scipy_eloc_rate(H, psi, reps: int = 3):
    """SciPy CSR matvec, exactly detnqs/operator/kernel.py:75-78 (one core)."""
    A = H.to_scipy(0)
    A.dot(psi)
    t0 = time.perf_counter()
    for _ in range(reps):
        A.dot(psi)
    t = (time.perf_counter() - t0) / reps
    return len(psi) / t, t


# ---------------------------------------------------------------------------
# GPU step
# ---------------------------------------------------------------------------

def run_ours(args, rank: int, world: int):
    import torch
    from detnqs_b200 import core, device, native

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_dets = args.n_dets
    _log("sampling the determinant space")
    sysm, V, psi = workload(rank, n_dets)
    _log("context")
    ctx = core.IntCtx.from_arrays(N_ORB, sysm.h1e, sysm.eri, sysm.e_core, device=local)
    ctx.hb_prepare(1e-15)
    # the step runs FP32 H.psi on every build: its FP32 copy is written by the build
    native.check(native.lib.dnq_set_option(native.OPT_BUILD_F32, 1))
    V_dev = torch.from_numpy(V.view(np.int64)).to(dev)
    psi_dev = torch.from_numpy(psi).to(dev)
    eloc = torch.empty(n_dets, dtype=torch.float64, device=dev)
    eloc32 = torch.empty(n_dets, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        H = device.build(ctx, V_dev, n_orb=N_ORB, policy=native.POLICY_STATIC,
                         use_heatbath=True, eps1=EPS1, want_vp=False)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        e64 = H.local_energy(psi_dev, eloc=eloc, precision=native.F64)
        ev[1].record()
        e32 = H.local_energy(psi_dev, eloc=eloc32, precision=native.F32)
        ev[2].record()
        return H, e64, e32, ev

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    clk = ClockSampler(local)   # before the warm-up: see ClockSampler
    clk.start()
    _log("warm-up steps")
    for _ in range(args.warmup):
        H, *_ = step()
        H.close()
    barrier()
    _log("timed steps")

    launches0 = native.lib.dnq_launch_count()
    clk.begin()
    t_steps, t_build, t_fill, t_count, t_e64, t_e32 = [], [], [], [], [], []
    nnz = cand = 0
    dE = 0.0
    for _ in range(args.steps):
        flush.zero_()                         # L2 flush between timed steps
        barrier()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record()
        H, e64, e32, ev = step()
        s1.record()
        torch.cuda.synchronize()
        t_steps.append(s0.elapsed_time(s1))
        tm = H.timings()
        t_build.append(tm["total"])
        t_fill.append(tm["fill"])
        t_count.append(tm["count"])
        t_e64.append(ev[0].elapsed_time(ev[1]))
        t_e32.append(ev[1].elapsed_time(ev[2]))
        nnz, cand = H.nnz_vv, H.candidates
        dE = abs(e32[0] / e32[1] - e64[0] / e64[1])
        if _ == args.steps - 1:
            last = H
        else:
            H.close()
    clk.end()
    clocks = clk.stop()
    launches = (native.lib.dnq_launch_count() - launches0) // args.steps
    ms_step = max_over_ranks(float(np.mean(t_steps)), world, dev)

    # ---- steady state of the inner loop: repeated H.psi on the resident H
    _log("steady-state H.psi")
    ss = {}
    for prec, key in ((native.F64, "f64"), (native.F32, "f32")):
        for _ in range(2):   # FP32 values prepared outside timing
            last.local_energy(psi_dev, eloc=eloc, precision=prec)
        reps = 20
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            last.spmv(psi_dev, out=eloc32, precision=prec)
        b.record()
        torch.cuda.synchronize()
        ss[key] = a.elapsed_time(b) / reps

    # ---- several amplitude sets per pass: k vectors gathered interleaved
    # (8 FP32 or 4 FP64 per 32-byte sector), each column equal to the
    # single-vector result bit for bit
    from detnqs_b200 import synthetic as S
    multi = {}
    for prec, key, kv in ((native.F32, "f32_k8", 8), (native.F64, "f64_k4", 4)):
        Xk = torch.from_numpy(np.stack([S.normalized_psi(n_dets, PSI_SEED + 100 + j)
                                        for j in range(kv)], 1)).to(dev)
        Yk = torch.empty_like(Xk)
        for _ in range(2):
            last.spmv_multi(Xk, out=Yk, precision=prec)
        reps = 20
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            last.spmv_multi(Xk, out=Yk, precision=prec)
        b.record()
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / reps
        multi[key] = {"vectors": kv, "ms_per_pass": t,
                      "e_loc_per_s": kv * n_dets / (t * 1e-3),
                      "speedup_vs_fp64_single_vector": kv * ss["f64"] / t}
        del Xk, Yk

    # ---- end to end through the C ABI with host buffers
    _log("end-to-end steps")
    pin_V = torch.from_numpy(V.view(np.int64)).pin_memory()
    pin_psi = torch.from_numpy(psi).pin_memory()
    pin_eloc = torch.empty(n_dets, dtype=torch.float64).pin_memory()
    Vh = pin_V.numpy().view(np.uint64)
    ph = pin_psi.numpy()
    eh = pin_eloc.numpy()
    e2e = []
    # the host-buffer path needs a little more device memory than the
    # resident one: untimed warm-up steps let the pool reach its size first
    for k in range(args.warmup + max(1, args.steps)):
        flush.zero_()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        H = device.build(ctx, Vh, n_orb=N_ORB, policy=native.POLICY_STATIC,
                         use_heatbath=True, eps1=EPS1, want_vp=False)
        H.local_energy(ph, eloc=eh, precision=native.F64)
        H.local_energy(ph, eloc=eh, precision=native.F32)
        b.record()
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e.append(a.elapsed_time(b))
        H.close()
    e2e_ms = max_over_ranks(float(np.mean(e2e)), world, dev)

    peak, peak_kind = measured_peaks()
    fill_ms = float(np.mean(t_fill))
    # dets in; column, FP64 and FP32 value of every entry and each row's
    # arena position and length out
    alg_fill = n_dets * 16 + nnz * (4 + 8 + 4) + n_dets * 12
    spmv_ms = float(np.mean(t_e64))
    alg_spmv = nnz * (4 + 8) + n_dets * (8 + 8 + 8)                 # CSR, rowptr, x, y
    result = {
        "metric": "screened H elements/s (H_VV nnz per second of build + FP64 and FP32 "
                  "local-energy passes)",
        "value": world * nnz / (ms_step * 1e-3),
        "unit": "elements/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 build; f64 and f32-compensated H.psi",
        "data": "synthetic (seeded integrals, heat-bath sampled determinants)",
        "config": {"workload": "30 orbitals, 12a/12b, K=60, 1e6 heat-bath-sampled dets, "
                               "eps1=1e-6 static heat-bath, H_VV build + E_loc",
                   "n_orb": N_ORB, "n_dets": n_dets, "eps1": EPS1, "nnz_H_VV": nnz,
                   "candidates_per_step": cand, "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed steps"},
        "e_loc_per_s": n_dets / (spmv_ms * 1e-3),
        "e_loc_per_s_fp32": n_dets / (float(np.mean(t_e32)) * 1e-3),
        "hpsi_steady_ms": ss,
        "e_loc_per_s_steady": {k: n_dets / (v * 1e-3) for k, v in ss.items()},
        "hpsi_multi_vector": multi,
        "build_elements_per_s": nnz / (float(np.mean(t_build)) * 1e-3),
        "candidates_per_s": cand / (float(np.mean(t_build)) * 1e-3),
        "dE_fp32_vs_fp64_Ha": dE,
        "build_phase_ms": {k: float(v) for k, v in last.timings().items()},
        "ms_steps": [round(x, 3) for x in t_steps],
        "roofline": {"bound": "hbm",
                     "kernel": "V->V fill: k_vv_arena (members) + k_vv_singles + k_vv_eval "
                               "(entries) + long rows",
                     "achieved": alg_fill / (fill_ms * 1e-3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg_fill / (fill_ms * 1e-3) / 1e9 / peak,
                     "traffic": ncu_traffic("vv_fill"),
                     "peak_kind": peak_kind,
                     "note": "the walk is integer-issue bound and the evaluation L2-latency "
                             "bound; bytes are the determinants read and the block written "
                             "(column, FP64 and FP32 value per entry, arena position and "
                             "length per row); traffic (walk + evaluation) adds the 8-byte "
                             "member records written and read back"},
        "roofline_spmv": {"bound": "hbm", "kernel": "k_spmv_f64 (steady state)", "achieved":
                          alg_spmv / (ss["f64"] * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": alg_spmv / (ss["f64"] * 1e-3) / 1e9 / peak,
                          "traffic": ncu_traffic("k_spmv_f64"), "peak_kind": peak_kind},
        "roofline_spmv_f32": {"bound": "hbm", "kernel": "k_spmv_f32c (steady state)",
                              "achieved": (nnz * 8 + n_dets * 36) / (ss["f32"] * 1e-3) / 1e9,
                              "peak": peak, "unit": "GB/s",
                              "frac": (nnz * 8 + n_dets * 36) / (ss["f32"] * 1e-3) / 1e9 / peak,
                              "traffic": ncu_traffic("k_spmv_f32c"), "peak_kind": peak_kind},
        # every x gather of H.psi is its own 32-byte L1 sector; an SM's L1
        # returns about one sector per clock, which bounds both precisions
        "gather_bound_spmv": {
            "unit": "sectors/s",
            "sectors_per_launch": {"f64": nnz + (nnz * 12 + n_dets * 24) / 32,
                                   "f32": nnz + (nnz * 8 + n_dets * 36) / 32},
            "peak": SMS * (clocks.get("sm_mhz") or 1965.0) * 1e6,
            "achieved": {k: sec / (ss[k] * 1e-3) for k, sec in
                         (("f64", nnz + (nnz * 12 + n_dets * 24) / 32),
                          ("f32", nnz + (nnz * 8 + n_dets * 36) / 32))},
            "frac": {k: sec / (ss[k] * 1e-3) / (SMS * (clocks.get("sm_mhz") or 1965.0) * 1e6)
                     for k, sec in (("f64", nnz + (nnz * 12 + n_dets * 24) / 32),
                                    ("f32", nnz + (nnz * 8 + n_dets * 36) / 32))},
            "note": "one L1 sector per gathered x value plus the streamed CSR sectors; peak = 1 "
                    "sector per SM clock, the rate ncu measured for the FP32 kernel on the 200k "
                    "case"},
        "e2e": {"value": world * nnz / (e2e_ms * 1e-3), "unit": "elements/s",
                "ms_per_step": e2e_ms, "ms_steps": [round(x, 3) for x in e2e],
                "h2d_bytes_per_step": n_dets * 16 + 2 * n_dets * 8,
                "d2h_bytes_per_step": 2 * n_dets * 8 + 32},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        _log("CPU baseline: reference rows")
        rate, rows, cnnz, t, threads, kind = cpu_reference_sample(sysm, V, args.cpu_seconds)
        _log("CPU baseline: SciPy H.psi")
        er, et = scipy_eloc_rate(last, psi)
        _log("CPU baseline done")
        result["cpu_baseline"] = {
            "value": rate, "unit": "elements/s", "cores": threads, "kind": kind,
            "sample": f"{rows} random rows of the same 1e6-det space, static heat-bath "
                      f"eps1=1e-6, H_VV rows ({cnnz} elements) in {t:.1f} s",
            "e_loc_per_s_scipy_1core": er}
    last.close()
    return result


# ---------------------------------------------------------------------------
# Batched workload: 64 systems of uneven size in one graph-replayed step
# ---------------------------------------------------------------------------

BATCH_N_SYS, BATCH_SEED, BATCH_EPS = 64, 77, 1e-7
BATCH_WORKLOAD = ("64 synthetic systems, n_orb uniform 10..40, n_elec 40-60% of 2 n_orb "
                  "(alpha = beta), K = 2 n_orb, dets log-uniform 1e3..2e5 (HF + heat-bath "
                  "sampled up to triples), eps1 = 1e-7 static heat-bath, FP32-compensated "
                  "H.psi, autotuned, whole step as one CUDA graph")


def batch_workload(rank: int):
    """Systems of one rank (seed + rank) and their normalised amplitudes,
    concatenated in system order."""
    from detnqs_b200 import batch as B
    from detnqs_b200 import synthetic as S
    W = B.make_batch_workload(BATCH_N_SYS, seed=BATCH_SEED + rank,
                              cache_dir=os.path.join(CACHE, "batch"))
    psi = np.concatenate([S.normalized_psi(len(w.dets), PSI_SEED + 1000 * rank + k)
                          for k, w in enumerate(W)])
    return W, psi


def run_batched(args, rank: int, world: int):
    W, psi = batch_workload(rank)        # sampled in spawned processes, before CUDA
    import torch
    from detnqs_b200 import batch as B
    from detnqs_b200 import core, device, native

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_orbs = [w.sysm.n_orb for w in W]
    ctxs = []
    for w in W:
        c = core.IntCtx.from_arrays(w.sysm.n_orb, w.sysm.h1e, w.sysm.eri, w.sysm.e_core,
                                    device=local)
        c.hb_prepare(1e-15)
        ctxs.append(c)
    t0 = time.perf_counter()
    bt = B.Batch(ctxs, [w.dets for w in W], n_orbs, eps1=BATCH_EPS, device=local)
    create_s = time.perf_counter() - t0
    total, nnz, off = bt.total, bt.nnz, bt.offsets
    stream = torch.cuda.Stream(dev)
    sp = stream.cuda_stream
    psi_dev = torch.from_numpy(psi).to(dev)
    eloc_dev = torch.empty(total, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    tune = B.autotune(bt, psi_dev, precision=native.F32,
                      cache=os.path.join(CACHE, f"autotune_dev{local}.json"))

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # phase split from eager steps (same kernels as the graph)
    phases = []
    l0 = native.lib.dnq_launch_count()
    for _ in range(3):
        flush.zero_()
        barrier()
        bt.step(psi_dev, precision=native.F32, stream=sp, eloc=eloc_dev)
        phases.append(bt.timings())
    launches_per_step = (native.lib.dnq_launch_count() - l0) // 3
    phase = {k: float(np.mean([p[k] for p in phases])) for k in phases[0]}

    clk = ClockSampler(local)   # before the warm-up: see ClockSampler
    clk.start()
    for _ in range(args.warmup):
        bt.step(psi_dev, precision=native.F32, graph=True, stream=sp, eloc=eloc_dev)
    barrier()
    clk.begin()
    t_step = []
    for _ in range(args.steps):
        flush.zero_()
        barrier()
        e32, ms = bt.step(psi_dev, precision=native.F32, graph=True, stream=sp, eloc=eloc_dev)
        t_step.append(ms)
    t_apply = {}
    for prec, key in ((native.F32, "f32"), (native.F64, "f64")):
        bt.apply(psi_dev, precision=prec, graph=True, stream=sp, eloc=eloc_dev)
        ts = []
        for _ in range(max(args.steps, 5)):
            flush.zero_()
            barrier()
            _, ms = bt.apply(psi_dev, precision=prec, graph=True, stream=sp, eloc=eloc_dev)
            ts.append(ms)
        t_apply[key] = float(np.mean(ts))
    # several amplitude sets per system in one pass (8 FP32 sets per sector)
    Xk = torch.stack([psi_dev] + [torch.roll(psi_dev, 17 * j) for j in range(1, 8)], 1)
    bt.apply_multi(Xk, precision=native.F32)
    ts = []
    for _ in range(max(args.steps, 5)):
        flush.zero_()
        barrier()
        _, ms = bt.apply_multi(Xk, precision=native.F32)
        ts.append(ms)
    t_multi = float(np.mean(ts))
    del Xk
    clk.end()
    clocks = clk.stop()
    ms_step = max_over_ranks(float(np.mean(t_step)), world, dev)
    e64b, _ = bt.step(psi_dev, precision=native.F64, stream=sp)

    # ---- plain FP64 path: one system at a time, build + E_loc
    V_dev = [torch.from_numpy(w.dets.view(np.int64)).to(dev) for w in W]
    parts = [psi_dev[off[k]:off[k + 1]] for k in range(len(W))]
    outs = [torch.empty_like(p) for p in parts]

    def plain_step():
        Hs, es = [], []
        for k in range(len(W)):
            H = device.build(ctxs[k], V_dev[k], n_orb=n_orbs[k], policy=native.POLICY_STATIC,
                             use_heatbath=True, eps1=BATCH_EPS, want_vp=False)
            es.append(H.local_energy(parts[k], precision=native.F64))
            Hs.append(H)
        return Hs, es

    Hs, _ = plain_step()
    for H in Hs:
        H.close()
    t_plain = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.zero_()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        Hs, e_plain = plain_step()
        b.record()
        torch.cuda.synchronize()
        t_plain.append(a.elapsed_time(b))
        if _ < max(1, min(args.steps, 3)) - 1:
            for H in Hs:
                H.close()
    for k, H in enumerate(Hs):            # conversion outside the timing
        H.spmv(parts[k], out=outs[k], precision=native.F64)
    barrier()
    ts = []
    for _ in range(5):
        flush.zero_()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for k, H in enumerate(Hs):
            H.spmv(parts[k], out=outs[k], precision=native.F64)
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    t_plain_hpsi = float(np.mean(ts))
    for H in Hs:
        H.close()
    ms_plain = float(np.mean(t_plain))
    E_plain = np.array([n / d for n, d in e_plain])
    dE32 = float(np.max(np.abs(e32[:, 0] / e32[:, 1] - E_plain)))
    dE64 = float(np.max(np.abs(e64b[:, 0] / e64b[:, 1] - E_plain)))

    # ---- end to end through the public API: psi from pinned host memory,
    # local energies and per-system energies back to the host
    pin_psi = torch.from_numpy(psi).pin_memory()
    pin_eloc = torch.empty(total, dtype=torch.float64).pin_memory()
    ph, eh = pin_psi.numpy(), pin_eloc.numpy()
    e2e = []
    for k in range(args.warmup + max(1, args.steps)):
        flush.zero_()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        bt.step(ph, precision=native.F32, graph=True, stream=sp, eloc=eh)
        b.record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e.append(a.elapsed_time(b))
    e2e_ms = max_over_ranks(float(np.mean(e2e)), world, dev)

    peak, peak_kind = measured_peaks()
    alg_build = total * 16 + (total + 1) * 8 + nnz * 12
    alg_hpsi = nnz * 8 + total * 36
    build_ms = phase["build"]
    roof_build = {"bound": "hbm", "kernel": "k_vv_arena + k_vv_big (batched build)",
                  "achieved": alg_build / (build_ms * 1e-3) / 1e9, "peak": peak,
                  "unit": "GB/s", "frac": alg_build / (build_ms * 1e-3) / 1e9 / peak,
                  "traffic": ncu_traffic("k_vv_arena_batch"), "peak_kind": peak_kind,
                  "note": "generation is integer/L2-latency bound; bytes are the CSR "
                          "written and determinants read"}
    roof_hpsi = {"bound": "hbm", "kernel": "k_spmv_f32c (batched, graph replay)",
                 "achieved": alg_hpsi / (t_apply["f32"] * 1e-3) / 1e9, "peak": peak,
                 "unit": "GB/s", "frac": alg_hpsi / (t_apply["f32"] * 1e-3) / 1e9 / peak,
                 "traffic": ncu_traffic("k_spmv_f32c_batch"), "peak_kind": peak_kind}
    result = {
        "metric": "screened H elements/s (H_VV nnz per second of the batched step: build of "
                  "every system + FP32-compensated local energies)",
        "value": world * nnz / (ms_step * 1e-3),
        "unit": "elements/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 build; f32-compensated H.psi (f64 diagonal and energies)",
        "data": "synthetic (seeded integrals, heat-bath sampled determinants)",
        "config": {"workload": BATCH_WORKLOAD, "n_sys": len(W), "rows": total,
                   "nnz_H_VV": nnz, "n_orb_range": [min(n_orbs), max(n_orbs)],
                   "eps1": BATCH_EPS, "autotuned_config": list(bt.config),
                   "autotune": {"tune_seconds": tune.get("tune_seconds"),
                                "tried": len(tune.get("tried", []))},
                   "batch_create_s": create_s, "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed steps"},
        "e_loc_per_s": world * total / (ms_step * 1e-3),
        "hpsi_ms": t_apply,
        "e_loc_per_s_hpsi": {k: total / (v * 1e-3) for k, v in t_apply.items()},
        "phase_ms_eager": phase,
        "plain_fp64": {"step_ms": ms_plain, "hpsi_ms": t_plain_hpsi,
                       "what": "one system at a time: dnq_build + FP64 local energy; H.psi "
                               "alone on the resident blocks"},
        "hpsi_multi_8sets_ms": t_multi,
        "speedup_vs_plain_fp64": {"step": ms_plain / ms_step,
                                  "hpsi": t_plain_hpsi / t_apply["f32"],
                                  "hpsi_per_set_8sets": 8 * t_plain_hpsi / t_multi},
        "dE_fp32_vs_fp64_Ha": dE32,
        "dE_batched_fp64_vs_plain_Ha": dE64,
        "roofline": roof_build if build_ms >= phase["hpsi"] else roof_hpsi,
        "roofline_hpsi": roof_hpsi,
        "e2e": {"value": world * nnz / (e2e_ms * 1e-3), "unit": "elements/s",
                "ms_per_step": e2e_ms, "h2d_bytes_per_step": total * 8,
                "d2h_bytes_per_step": total * 8 + 16 * len(W)},
        "gpu_launches": int(launches_per_step) * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, rows, cnnz, t, threads, kind = cpu_reference_rows(
            [(w.sysm, w.dets, BATCH_EPS) for w in W], args.cpu_seconds)
        result["cpu_baseline"] = {
            "value": rate, "unit": "elements/s", "cores": threads, "kind": kind,
            "sample": f"{rows} rows drawn uniformly over the 64 systems' rows, static "
                      f"heat-bath eps1=1e-7 H_VV rows ({cnnz} elements) in {t:.1f} s"}
        result["build_speedup_vs_cpu"] = (nnz / (phase["build"] + phase["compact"]) * 1e3) / rate
    bt.close()
    return result


# ---------------------------------------------------------------------------
# Serving workload: Poisson stream of build / local-energy requests
# ---------------------------------------------------------------------------

SERVE_RATE, SERVE_REQUESTS, SERVE_SEED = 200.0, 1200, 505
SERVE_BUDGET = 150e9
SERVE_WORKLOAD = ("Poisson request stream, 200 req/s, 1200 requests: 25% screened-H builds, "
                  "75% local-energy requests, over 24 systems of the batched size distribution "
                  "plus 3 bond-scan families x 10 points (integrals scaled element-wise up to "
                  "+-2%); eps1 = 1e-7; 150 GB admission budget; served FP32-compensated with "
                  "continuous batching vs one request at a time in FP64")


def serving_workload(rank: int):
    """Systems (sysm, dets), the request list (arrival s, kind, system, psi
    pool index) and a pool of 3 normalised psi per system."""
    from detnqs_b200 import batch as B
    from detnqs_b200 import synthetic as S
    seed = SERVE_SEED + rank
    W = B.make_batch_workload(24, seed=seed, cache_dir=os.path.join(CACHE, "serve"))
    systems = [(w.sysm, w.dets) for w in W]
    rng = np.random.default_rng(seed)
    for f in range(3):
        n = int(rng.integers(10, 41))
        na = int(rng.integers(int(np.ceil(0.4 * n)), int(np.floor(0.6 * n)) + 1))
        nd = int(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
        fam = S.scan_family(n, na, na, 2 * n, seed * 10 + f, points=10)
        path = os.path.join(CACHE, "serve", f"scan_{seed}_{f}_{n}_{na}_{nd}.npy")
        if os.path.exists(path):
            V = np.load(path)
        else:
            V = S.heat_bath_sample(fam[0], nd, seed * 31 + f, max_level=3)
            np.save(path, V)
        systems += [(sysm, V) for sysm in fam]
    arrivals = np.cumsum(rng.exponential(1.0 / SERVE_RATE, size=SERVE_REQUESTS))
    kinds = (rng.random(SERVE_REQUESTS) >= 0.25).astype(int)     # 1 = ELOC, 0 = BUILD
    targets = rng.integers(0, len(systems), size=SERVE_REQUESTS)
    which = rng.integers(0, 3, size=SERVE_REQUESTS)
    pool = [[S.normalized_psi(len(d), seed * 1000 + 3 * k + j) for j in range(3)]
            for k, (_, d) in enumerate(systems)]
    reqs = list(zip(arrivals.tolist(), kinds.tolist(), targets.tolist(), which.tolist()))
    return systems, reqs, pool


def _pct(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def run_serving(args, rank: int, world: int):
    systems, reqs, pool = serving_workload(rank)
    import torch
    from detnqs_b200 import core, device, native
    from detnqs_b200 import serve as V

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctxs = []
    for sysm, _ in systems:
        c = core.IntCtx.from_arrays(sysm.n_orb, sysm.h1e, sysm.eri, sysm.e_core, device=local)
        c.hb_prepare(1e-15)
        ctxs.append(c)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # warm-up: every system built once (its context then sizes later builds
    # as the plain path's will be), and one small system through both paths
    for k, (sysm, d) in enumerate(systems):
        H = device.build(ctxs[k], d, n_orb=sysm.n_orb, policy=native.POLICY_STATIC,
                         use_heatbath=True, eps1=1e-7, want_vp=False)
        H.close()
    clk = ClockSampler(local)   # before the warm-up: see ClockSampler
    clk.start()
    small = int(np.argmin([len(d) for _, d in systems]))
    for _ in range(max(1, args.warmup)):
        with V.Server(device=local, budget_bytes=SERVE_BUDGET, build_slots=4) as srv:
            k = srv.add_system(ctxs[small], systems[small][1], systems[small][0].n_orb, eps1=1e-7)
            srv.wait(srv.submit(V.ELOC, k, pool[small][0], precision=native.F32))
        H = device.build(ctxs[small], systems[small][1], n_orb=systems[small][0].n_orb,
                         policy=native.POLICY_STATIC, use_heatbath=True, eps1=1e-7,
                         want_vp=False)
        H.local_energy(pool[small][0], precision=native.F64)
        H.close()
    barrier()

    # ---- served: continuous batching, FP32-compensated, HBM admission
    import threading
    clk.begin()
    l0 = native.lib.dnq_launch_count()
    srv = V.Server(device=local, budget_bytes=SERVE_BUDGET, build_slots=args.serve_slots,
                   max_group=64)
    ids = [srv.add_system(c, d, s.n_orb, eps1=1e-7) for (s, d), c in zip(systems, ctxs)]
    tickets = [None] * len(reqs)
    t0 = time.perf_counter() + 0.05

    def submitter():
        for i, (ta, kind, k, j) in enumerate(reqs):
            dt = t0 + ta - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            tickets[i] = srv.submit(kind, ids[k], pool[k][j], precision=native.F32)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    served = [srv.wait(t) for t in tickets]
    t_end = time.perf_counter()
    st = srv.stats()
    srv.close()
    launches = native.lib.dnq_launch_count() - l0
    barrier()
    clk.end()
    clocks = clk.stop()
    span_served = t_end - t0

    # ---- plain: one request at a time, FP64, blocks kept resident
    resident = {}
    plain_lat, plain_e = [], []
    plain_build_s = 0.0
    t0p = time.perf_counter() + 0.05
    for ta, kind, k, j in reqs:
        dt = t0p + ta - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        sysm, dets = systems[k]
        if kind == V.BUILD or k not in resident:
            if k in resident:
                resident[k].close()
            tb = time.perf_counter()
            resident[k] = device.build(ctxs[k], dets, n_orb=sysm.n_orb,
                                       policy=native.POLICY_STATIC, use_heatbath=True,
                                       eps1=1e-7, want_vp=False)
            plain_build_s += time.perf_counter() - tb
        num = den = None
        if kind == V.ELOC:
            el = np.empty(len(dets))
            num, den = resident[k].local_energy(pool[k][j], eloc=el, precision=native.F64)
        plain_lat.append(time.perf_counter() - (t0p + ta))
        plain_e.append(None if num is None else num / den)
    span_plain = time.perf_counter() - t0p
    for H in resident.values():
        H.close()

    lat = [r["latency_s"] for r in served]
    lat_e = [r["latency_s"] for r, q in zip(served, reqs) if q[1] == V.ELOC]
    lat_b = [r["latency_s"] for r, q in zip(served, reqs) if q[1] == V.BUILD]
    dE = max(abs(r["energy"] - e) for r, e, q in zip(served, plain_e, reqs)
             if q[1] == V.ELOC)
    rows = sum(len(systems[q[2]][1]) for q in reqs if q[1] == V.ELOC)
    built = sum(r["nnz"] for r in served)
    n = len(reqs)
    p50, p99 = _pct(lat, 50) * 1e3, _pct(lat, 99) * 1e3
    result = {
        "metric": "p99 latency of the served request stream (build + local-energy requests)",
        "value": p99,
        "unit": "ms",
        "n_gpus": world,
        "steps": n,
        "warmup": args.warmup,
        "ms_per_step": span_served / n * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 build; f32-compensated H.psi (f64 diagonal and energies)",
        "data": "synthetic (seeded integrals, heat-bath sampled determinants, Poisson arrivals)",
        "config": {"workload": SERVE_WORKLOAD, "systems": len(systems), "requests": n,
                   "rate_per_s": SERVE_RATE, "budget_bytes": SERVE_BUDGET,
                   "build_slots": args.serve_slots,
                   "max_group": 64, "parallelism": f"replicas x{world}",
                   "l2": "requests arrive in real time; inputs (1e3..2e5-row blocks) larger "
                         "than L2 in aggregate"},
        "latency_ms": {"p50": p50, "p99": p99, "eloc_p50": _pct(lat_e, 50) * 1e3,
                       "eloc_p99": _pct(lat_e, 99) * 1e3, "build_p50": _pct(lat_b, 50) * 1e3,
                       "build_p99": _pct(lat_b, 99) * 1e3},
        "throughput": {"requests_per_s": n / span_served, "e_loc_per_s": rows / span_served,
                       "built_elements_per_s": built / span_served},
        "plain_fp64": {"latency_ms": {"p50": _pct(plain_lat, 50) * 1e3,
                                      "p99": _pct(plain_lat, 99) * 1e3},
                       "requests_per_s": n / span_plain, "build_seconds": plain_build_s,
                       "what": "same stream, one request at a time: dnq_build + FP64 local "
                               "energy, blocks kept resident, no overlap or grouping"},
        "speedup_vs_plain_fp64": {"p50": _pct(plain_lat, 50) * 1e3 / p50,
                                  "p99": _pct(plain_lat, 99) * 1e3 / p99,
                                  "throughput": span_plain / span_served},
        "server": st,
        "dE_fp32_vs_fp64_Ha": dE,
        "roofline": None,
        "e2e": {"value": p99, "unit": "ms",
                "h2d_bytes_per_step": int(8 * rows / n),
                "d2h_bytes_per_step": int(8 * rows / n + 16),
                "note": "latencies are host-to-host: psi from host memory, energies back"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    return result


# ---------------------------------------------------------------------------
# Downfolding workload: 100 orbitals, two-word determinants
# ---------------------------------------------------------------------------

DF_N, DF_NE, DF_K, DF_S = 100, 20, 200, 100_000
DF_EPS, DF_TAIL, DF_SIGMA = 1e-5, 2e-6, 0.1
DF_WORKLOAD = ("100 orbitals, 20a/20b, K=200, two-word determinants; S = 1e5 heat-bath-sampled "
               "dets (<= 4 excitations); psi_S: HF amplitude 1 and a N(0,1) tail of scale 2e-6 "
               "(normalised); C = screened singles/doubles of S with dynamic amplitude "
               "screening eps1 = 1e-5; H_eff = H_SS + H_SC (e_ref - D_CC)^-1 H_CS with "
               "e_ref = <psi|H_SS|psi>, sigma regularisation 0.1 Ha, FP64 and FP32 values")


def downfold_workload(rank: int, n_s: int = DF_S):
    from detnqs_b200 import synthetic as S
    seed = 4004 + 10 * rank
    sysm = S.make_system(DF_N, DF_NE, DF_NE, DF_K, seed)
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"df_{DF_N}_{n_s}_{seed}.npy")
    if os.path.exists(path):
        V = np.load(path)
    else:
        V = S.heat_bath_sample_wide(sysm, n_s, seed + 1, max_level=4)
        np.save(path, V)
    rng = np.random.default_rng(seed + 2)
    psi = DF_TAIL * rng.normal(size=len(V))
    psi[0] = 1.0
    psi /= np.linalg.norm(psi)
    return sysm, V, psi


def cpu_wide_rows(sysm, V, psi, target_s: float = 15.0, seed: int = 5):
    """Two-word restatement (oracle/wide.cpp, the only CPU form: the
    reference stops at 64 orbitals) on a sample of rows.  Returns
    (elements/s, rows, elements, seconds, threads)."""
    from oracle import WideChecker
    chk = WideChecker(DF_N, sysm.h1e, sysm.eri, sysm.e_core)
    chk.hb_prepare(1e-15)
    rng = np.random.default_rng(seed)
    order = rng.permutation(np.arange(1, len(V)))
    nnz = 0
    t_all = 0.0
    rows = 0
    for r in order:
        t0 = time.perf_counter()
        o = chk.build(V, psi, eps1=DF_EPS, rows=(int(r), int(r) + 1))
        t_all += time.perf_counter() - t0
        nnz += len(o["H_VV"]["val"]) + len(o["H_VP"]["val"])
        rows += 1
        if t_all >= target_s:
            break
    return nnz / t_all, rows, nnz, t_all, os.cpu_count() or 1


def run_downfold(args, rank: int, world: int):
    sysm, V, psi = downfold_workload(rank, args.df_dets)
    import torch
    from detnqs_b200 import eigen as E
    from detnqs_b200 import native
    from detnqs_b200 import wide as Wd

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    t0 = time.perf_counter()
    ctx = Wd.IntCtxWide.from_arrays(DF_N, sysm.h1e, sysm.eri, sysm.e_core, device=local)
    ctx.hb_prepare(1e-15)
    ctx_s = time.perf_counter() - t0
    Vd = torch.from_numpy(V.view(np.int64)).to(dev)
    pd = torch.from_numpy(psi).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def step():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        ev[0].record()
        H = Wd.build_wide(ctx, Vd, pd, n_orb=DF_N, eps1=DF_EPS)
        ev[1].record()
        hpp = torch.empty(H.n_p, dtype=torch.float64, device=dev)
        Wd.p_diag(H, ctx, hpp)
        num, den = H.local_energy(pd)
        e_ref = num / den
        ev[2].record()
        E64 = Wd.ham_eff_wide(H, hpp, e_ref, epsilon=DF_SIGMA, precision=native.F64)
        ev[3].record()
        E32 = Wd.ham_eff_wide(H, hpp, e_ref, epsilon=DF_SIGMA, precision=native.F32)
        ev[4].record()
        ev[5].record()
        return H, hpp, e_ref, E64, E32, ev

    clk = ClockSampler(local)   # before the warm-up: see ClockSampler
    clk.start()
    for _ in range(args.warmup):
        H, hpp, e_ref, E64, E32, _ = step()
        for h in (H, E64, E32):
            h.close()
    barrier()
    clk.begin()
    l0 = native.lib.dnq_launch_count()
    t_step, t_build, t_diag, t_h64, t_h32 = [], [], [], [], []
    for k in range(args.steps):
        flush.zero_()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        H, hpp, e_ref, E64, E32, ev = step()
        b.record()
        torch.cuda.synchronize()
        t_step.append(a.elapsed_time(b))
        t_build.append(ev[0].elapsed_time(ev[1]))
        t_diag.append(ev[1].elapsed_time(ev[2]))
        t_h64.append(ev[2].elapsed_time(ev[3]))
        t_h32.append(ev[3].elapsed_time(ev[4]))
        if k < args.steps - 1:
            for h in (H, E64, E32):
                h.close()
    clk.end()
    clocks = clk.stop()
    launches = (native.lib.dnq_launch_count() - l0) // max(1, args.steps)
    ms_step = max_over_ranks(float(np.mean(t_step)), world, dev)
    n_s, nnz_ss, n_c, nnz_sc = H.n_v, H.nnz_vv, H.n_p, H.nnz_vp
    # SpGEMM work: sum over C columns of (entries in the column)^2
    _, ccols, _ = H.to_csr_arrays(1)
    m_k = np.bincount(ccols.astype(np.int64), minlength=n_c)
    work = int((m_k.astype(np.int64) ** 2).sum())
    nnz_eff = E32.nnz_vv

    # lowest eigenvalue of the symmetric part of each H_eff (device Lanczos)
    te = time.perf_counter()
    S64, S32 = E.symmetric_part(E64), E.symmetric_part(E32)
    lam64, it64 = E.lowest_eigenvalue(S64, device=local)
    lam32, it32 = E.lowest_eigenvalue(S32, device=local)
    eig_s = time.perf_counter() - te
    for h in (S64, S32):
        h.close()

    # end to end through the public API: host determinants and psi in,
    # host diag(H_CC) and the FP32 H_eff (CSR) out
    pin_V = torch.from_numpy(V.view(np.int64)).pin_memory().numpy().view(np.uint64)
    pin_p = torch.from_numpy(psi).pin_memory().numpy()
    e2e = []
    d2h = 0
    for k in range(min(args.warmup, 1) + max(1, args.steps)):
        flush.zero_()
        barrier()
        a = time.perf_counter()
        He = Wd.build_wide(ctx, pin_V, pin_p, n_orb=DF_N, eps1=DF_EPS)
        hp = Wd.p_diag(He, ctx)
        nu, de = He.local_energy(pin_p)
        Ee = Wd.ham_eff_wide(He, hp, nu / de, epsilon=DF_SIGMA, precision=native.F32)
        rp, cc, vv = Ee.to_csr_arrays(0)
        if k >= min(args.warmup, 1):
            e2e.append((time.perf_counter() - a) * 1e3)
        d2h = hp.nbytes + rp.nbytes + cc.nbytes + vv.nbytes + 16
        for h in (He, Ee):
            h.close()
    e2e_ms = max_over_ranks(float(np.mean(e2e)), world, dev)

    peak, peak_kind = measured_peaks()
    build_ms, h32_ms = float(np.mean(t_build)), float(np.mean(t_h32))
    alg_build = n_s * 32 + (n_s + 1) * 16 + (nnz_ss + nnz_sc) * 12 + nnz_sc * 32
    alg_spgemm = nnz_sc * (4 + 4) * 2 + n_c * 8 + nnz_eff * (4 + 8) + n_s * 8
    result = {
        "metric": "screened H elements/s (H_SS + H_SC nnz per second of the downfolding step: "
                  "build, diag(H_CC), FP64 and FP32 H_eff)",
        "value": world * (nnz_ss + nnz_sc) / (ms_step * 1e-3),
        "unit": "elements/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 build; H_eff in f64 and in f32 values with float-float accumulation",
        "data": "synthetic (seeded integrals, heat-bath sampled two-word determinants)",
        "config": {"workload": DF_WORKLOAD, "n_orb": DF_N, "S": n_s, "C": n_c,
                   "nnz_H_SS": nnz_ss, "nnz_H_SC": nnz_sc, "nnz_H_eff": nnz_eff,
                   "spgemm_multiply_adds": work, "e_ref": e_ref, "context_s": ctx_s,
                   "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed steps"},
        "phase_ms": {"build": build_ms, "diag_cc_and_e_ref": float(np.mean(t_diag)),
                     "h_eff_f64": float(np.mean(t_h64)), "h_eff_f32": h32_ms},
        "lowest_eigenvalue": {"f64": lam64, "f32": lam32, "lanczos_steps": [it64, it32],
                              "seconds": eig_s,
                              "of": "0.5 (H_eff + H_eff^T), device Lanczos in FP64"},
        "dE_fp32_vs_fp64_Ha": abs(lam32 - lam64),
        "spgemm_multiply_adds_per_s": work / (h32_ms * 1e-3),
        "roofline": {"bound": "hbm", "kernel": "k_wide_build (count + fill)",
                     "achieved": alg_build / (build_ms * 1e-3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg_build / (build_ms * 1e-3) / 1e9 / peak,
                     "traffic": ncu_traffic("k_wide_build"), "peak_kind": peak_kind,
                     "note": "generation is integer/L2-latency bound; bytes are dets read, "
                             "CSR and C keys written"},
        "roofline_spgemm": {"bound": "hbm", "kernel": "k_heff<F32> (FP32 H_eff)",
                            "achieved": alg_spgemm / (h32_ms * 1e-3) / 1e9, "peak": peak,
                            "unit": "GB/s",
                            "frac": alg_spgemm / (h32_ms * 1e-3) / 1e9 / peak,
                            "traffic": ncu_traffic("k_heff_f32"), "peak_kind": peak_kind},
        "e2e": {"value": world * (nnz_ss + nnz_sc) / (e2e_ms * 1e-3), "unit": "elements/s",
                "ms_per_step": e2e_ms, "h2d_bytes_per_step": n_s * 40 + n_c * 8,
                "d2h_bytes_per_step": int(d2h),
                "note": "FP32 H_eff only; host dets/psi in, diag(H_CC) and H_eff CSR out"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, rows, cnnz, t, threads = cpu_wide_rows(sysm, V, psi, args.cpu_seconds)
        result["cpu_baseline"] = {
            "value": rate, "unit": "elements/s", "cores": threads, "kind": "port",
            "sample": f"{rows} random non-HF rows of S (two-word restatement; the reference "
                      f"cannot represent 100 orbitals), {cnnz} elements in {t:.1f} s"}
    for h in (H, E64, E32):
        h.close()
    return result


# ---------------------------------------------------------------------------
# Determinant batch features: the single workload's 1e6 determinants
# ---------------------------------------------------------------------------

DB_KMAX = 8          # holes/particles kept: twice the deepest excitation of the space
DB_WORKLOAD = ("30 orbitals, 12a/12b, the 1e6 heat-bath-sampled dets of the single "
               "workload; every feature (occ, k, phase, holes/parts kmax=8, hp_mask, "
               "positions) relative to HF")


def det_batch_inputs(rank: int, n_dets: int):
    _, V, _ = workload(rank, n_dets)
    hf = np.array([(1 << N_ALPHA) - 1, (1 << N_BETA) - 1], np.uint64)
    return V, hf


def det_batch_bytes(n: int) -> int:
    """Algorithmic bytes: dets read; occ, k, phase, holes, parts, positions
    and mask written."""
    return n * (16 + 4 * (N_ALPHA + N_BETA) + 2 + DB_KMAX * (4 * 4 + 1))


def run_det_batch(args, rank: int, world: int):
    import torch
    from detnqs_b200 import core, native

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V, hf = det_batch_inputs(rank, args.n_dets)
    n = len(V)
    Vd = torch.from_numpy(V.view(np.int64)).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    kw = dict(kmax=DB_KMAX, need_k=True, need_phase=True, need_hp=True, need_hp_pos=True,
              device=local)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    clk = ClockSampler(local)   # before the warm-up: see ClockSampler
    clk.start()
    for _ in range(args.warmup):
        core.prepare_det_batch(Vd, hf, N_ORB, N_ALPHA, N_BETA, **kw)
    barrier()
    clk.begin()
    l0 = native.lib.dnq_launch_count()
    ts = []
    for _ in range(args.steps):
        flush.zero_()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        out = core.prepare_det_batch(Vd, hf, N_ORB, N_ALPHA, N_BETA, **kw)
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    clk.end()
    clocks = clk.stop()
    launches = (native.lib.dnq_launch_count() - l0) // max(1, args.steps)
    ms = max_over_ranks(float(np.mean(ts)), world, dev)
    # end to end: host determinants in, host features out
    pin_V = torch.from_numpy(V.view(np.int64)).pin_memory().numpy().view(np.uint64)
    e2e = []
    for k in range(1 + max(1, args.steps)):
        flush.zero_()
        barrier()
        t0 = time.perf_counter()
        host = core.prepare_det_batch(pin_V, hf, N_ORB, N_ALPHA, N_BETA, **kw)
        if k:
            e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(float(np.mean(e2e)), world, dev)
    d2h = sum(v.nbytes for v in host.values())
    peak, peak_kind = measured_peaks()
    alg = det_batch_bytes(n)
    result = {
        "metric": "determinant batch features per second (occ, k, phase, holes/parts, "
                  "positions, mask)",
        "value": world * n / (ms * 1e-3), "unit": "dets/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (heat-bath sampled determinants)",
        "config": {"workload": DB_WORKLOAD, "n_dets": n, "kmax": DB_KMAX,
                   "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed steps"},
        "roofline": {"bound": "hbm", "kernel": "k_det_batch", "achieved": alg / (ms * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": alg / (ms * 1e-3) / 1e9 / peak,
                     "traffic": ncu_traffic("k_det_batch"), "peak_kind": peak_kind,
                     "note": "timed over the whole call (staging, kernel, error read-back)"},
        "e2e": {"value": world * n / (e2e_ms * 1e-3), "unit": "dets/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": n * 16, "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    for k, v in out.items():   # the last timed batch equals the host one
        assert np.array_equal(v.cpu().numpy(), host[k]), k
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, m, t, kind = cpu_det_batch(V, hf)
        result["cpu_baseline"] = {"value": rate, "unit": "dets/s", "cores": 1, "kind": kind,
                                  "sample": f"{m} dets of the batch in {t:.2f} s "
                                            "(prepare_det_batch is a serial loop)"}
    return result


def cpu_det_batch(V, hf, seconds: float = 10.0):
    """The reference's prepare_det_batch (oracle/_ref) on the host, every
    feature, over repeated passes of the batch for about `seconds`."""
    from oracle import Checker
    kind = "reference" if Checker.reference_available() else "port"
    chk = Checker.reference() if kind == "reference" else Checker.port()
    m, t0 = 0, time.perf_counter()
    while True:
        chk.prepare_det_batch(V, hf, N_ORB, N_ALPHA, N_BETA, DB_KMAX, True, True, True, True)
        m += len(V)
        t = time.perf_counter() - t0
        if t >= seconds:
            return m / t, m, t, kind


# ---------------------------------------------------------------------------
# Batched log-determinant: sign, log|det| and its gradient
# ---------------------------------------------------------------------------

SL_B, SL_N = 32768, 10     # the reference's largest "typical SPO" case (test_logdet.py:195-200)
SL_WORKLOAD = ("32768 FP64 10x10 matrices N(0,1) + 10 I (the reference's largest typical-SPO "
               "benchmark case); sign, log|det| and the gradient of log|det|")


def slogdet_inputs(rank: int):
    rng = np.random.default_rng(4242 + rank)
    a = rng.normal(size=(SL_B, SL_N, SL_N)) + np.eye(SL_N) * SL_N
    return a, rng.normal(size=SL_B)


def run_slogdet(args, rank: int, world: int):
    import torch
    from detnqs_b200 import native
    from detnqs_b200 import slogdet as L

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    a, cot = slogdet_inputs(rank)
    ad = torch.from_numpy(a).to(dev)
    cd = torch.from_numpy(cot).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def step(x, c):
        sign, logabs = L.slogdet(x, device=local)
        return sign, logabs, L.slogdet_grad(x, c, device=local)

    clk = ClockSampler(local)   # before the warm-up: see ClockSampler
    clk.start()
    for _ in range(args.warmup):
        step(ad, cd)
    barrier()
    clk.begin()
    l0 = native.lib.dnq_launch_count()
    ts = []
    for _ in range(args.steps):
        flush.zero_()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        out = step(ad, cd)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    clk.end()
    clocks = clk.stop()
    launches = (native.lib.dnq_launch_count() - l0) // max(1, args.steps)
    ms = max_over_ranks(float(np.mean(ts)), world, dev)
    pin_a = torch.from_numpy(a).pin_memory().numpy()
    pin_c = torch.from_numpy(cot).pin_memory().numpy()
    e2e = []
    for k in range(1 + max(1, args.steps)):
        barrier()
        t0 = time.perf_counter()
        host = step(pin_a, pin_c)
        if k:
            e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(float(np.mean(e2e)), world, dev)
    for got, want in zip(out, host):
        assert np.array_equal(got.cpu().numpy(), want)
    peak, peak_kind = measured_peaks()
    alg = SL_B * (8 * SL_N * SL_N * 2 + 8 * 3 + 8 * SL_N * SL_N)   # a read twice, cot, sign, log, grad
    result = {
        "metric": "matrices per second (sign, log|det| and the gradient of log|det|)",
        "value": world * SL_B / (ms * 1e-3), "unit": "matrices/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded N(0,1) + n I matrices)",
        "config": {"workload": SL_WORKLOAD, "batch": SL_B, "n": SL_N,
                   "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed steps"},
        "roofline": {"bound": "hbm", "kernel": "k_slogdet + k_slogdet_grad",
                     "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (ms * 1e-3) / 1e9 / peak, "traffic": None,
                     "peak_kind": peak_kind,
                     "note": "timed over both calls; the LU is shared-memory FMA work"},
        "e2e": {"value": world * SL_B / (e2e_ms * 1e-3), "unit": "matrices/s",
                "ms_per_step": e2e_ms, "h2d_bytes_per_step": 2 * a.nbytes + cot.nbytes,
                "d2h_bytes_per_step": 2 * 8 * SL_B + a.nbytes},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, m, t = cpu_slogdet(a, cot)
        result["cpu_baseline"] = {
            "value": rate, "unit": "matrices/s", "cores": 1, "kind": "port",
            "sample": f"{m} matrices in {t:.2f} s: numpy (LAPACK) slogdet and inverse, the "
                      "CPU path of the reference's slogdet (use_fast_kernel=False under XLA)"}
    return result


def cpu_slogdet(a, cot, seconds: float = 10.0):
    """LAPACK slogdet + inverse on one host thread over repeated passes."""
    try:
        from threadpoolctl import threadpool_limits
        lim = threadpool_limits(1)
    except ImportError:
        lim = None
    m, t0 = 0, time.perf_counter()
    while True:
        np.linalg.slogdet(a)
        cot[:, None, None] * np.swapaxes(np.linalg.inv(a), -1, -2)
        m += len(a)
        t = time.perf_counter() - t0
        if t >= seconds:
            break
    if lim is not None:
        lim.unregister()
    return m / t, m, t


def run_reference(args, rank: int, world: int):
    """Reference CPU implementation on the same workload (rank 0 only)."""
    if rank != 0:
        return None
    if args.workload == "slogdet":
        a, cot = slogdet_inputs(0)
        vals, info = [], None
        for _ in range(max(1, args.steps)):
            rate, m, t = cpu_slogdet(a, cot, max(1.0, args.cpu_seconds / max(1, args.steps)))
            vals.append(rate)
            info = (m, t)
        m, t = info
        v = float(np.mean(vals))
        return {
            "impl": "reference",
            "metric": "matrices per second (sign, log|det| and the gradient of log|det|)",
            "value": v, "unit": "matrices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": SL_WORKLOAD, "batch": SL_B, "n": SL_N},
            "cpu_baseline": {"value": v, "unit": "matrices/s", "cores": 1, "kind": "port",
                             "sample": f"{m} matrices per step in {t:.2f} s: LAPACK slogdet and "
                                       "inverse (the reference's fused kernel needs cuSolverDx, "
                                       "absent here; its XLA fallback is LAPACK on the host)"},
            "e2e": {"value": v, "unit": "matrices/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
    if args.workload == "det_batch":
        V, hf = det_batch_inputs(0, args.n_dets)
        vals, info = [], None
        for _ in range(max(1, args.steps)):
            rate, m, t, kind = cpu_det_batch(V, hf, max(1.0, args.cpu_seconds / max(1, args.steps)))
            vals.append(rate)
            info = (m, t, kind)
        m, t, kind = info
        v = float(np.mean(vals))
        return {
            "impl": "reference",
            "metric": "determinant batch features per second (occ, k, phase, holes/parts, "
                      "positions, mask)",
            "value": v, "unit": "dets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": DB_WORKLOAD, "n_dets": len(V), "kmax": DB_KMAX},
            "cpu_baseline": {"value": v, "unit": "dets/s", "cores": 1, "kind": kind,
                             "sample": f"{m} dets per step in {t:.2f} s (serial loop)"},
            "e2e": {"value": v, "unit": "dets/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
    if args.workload in ("batched", "serving"):
        if args.workload == "batched":
            W, _ = batch_workload(0)
            sys_list = [(w.sysm, w.dets, BATCH_EPS) for w in W]
            desc = BATCH_WORKLOAD
        else:
            systems, _, _ = serving_workload(0)
            sys_list = [(sy, d, 1e-7) for sy, d in systems]
            desc = SERVE_WORKLOAD + " (reference: CPU build rate over the served systems)"
        vals, info = [], None
        for _ in range(max(1, args.steps)):
            rate, rows, nnz, t, threads, kind = cpu_reference_rows(
                sys_list, max(2.0, args.cpu_seconds / max(1, args.steps)), seed=77 + _)
            vals.append(rate)
            info = (rows, nnz, t, threads, kind)
        rows, nnz, t, threads, kind = info
        v = float(np.mean(vals))
        return {
            "impl": "reference",
            "metric": "screened H elements/s (H_VV nnz per second of the batched step: build "
                      "of every system + FP32-compensated local energies)",
            "value": v, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "n_sys": len(sys_list), "eps1": sys_list[0][2]},
            "cpu_baseline": {"value": v, "unit": "elements/s", "cores": threads, "kind": kind,
                             "sample": f"{rows} rows per step drawn over all systems, H_VV "
                                       "rows of the static heat-bath policy (reference C++ "
                                       "core, OpenMP)"},
            "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
    sysm, V, psi = workload(0, args.n_dets)
    vals = []
    info = None
    for _ in range(args.warmup if args.warmup < 2 else 1):
        pass
    for _ in range(max(1, args.steps)):
        rate, rows, nnz, t, threads, kind = cpu_reference_sample(
            sysm, V, max(2.0, args.cpu_seconds / max(1, args.steps)))
        vals.append(rate)
        info = (rows, nnz, t, threads, kind)
    rows, nnz, t, threads, kind = info
    v = float(np.mean(vals))
    return {
        "impl": "reference",
        "metric": "screened H elements/s (H_VV nnz per second of build + FP64 and FP32 "
                  "local-energy passes)",
        "value": v, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "30 orbitals, 12a/12b, K=60, 1e6 heat-bath-sampled dets, "
                               "eps1=1e-6 static heat-bath, H_VV build + E_loc",
                   "n_orb": N_ORB, "n_dets": args.n_dets, "eps1": EPS1},
        "cpu_baseline": {"value": v, "unit": "elements/s", "cores": threads, "kind": kind,
                         "sample": f"{rows} random rows per step, H_VV rows of the "
                                   "static heat-bath policy (reference C++ core, OpenMP)"},
        "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# The default single-GPU run also measures the other workloads briefly, each
# in its own process (3 timed steps after 2 warm-up steps, 3 s of CPU
# baseline; the serving stream three times for its tail), and reports them
# under "extras" beside the headline numbers.
EXTRAS = (("batched", 1), ("serving", 3), ("downfold", 1), ("slogdet", 1), ("det_batch", 1))


def _extra_summary(w: str, runs: list) -> dict:
    def pick(d, *keys):
        return {k: d.get(k) for k in keys if k in d}
    ok = [d for d in runs if "error" not in d]
    out = {"wall_s": [round(d.get("_wall_s", 0.0), 1) for d in runs]}
    if not ok:
        out["error"] = runs[-1].get("error") if runs else "not run"
        return out
    d = ok[-1]
    out.update(pick(d, "metric", "value", "unit", "ms_per_step", "ms_steps", "dtype",
                    "dE_fp32_vs_fp64_Ha", "gpu_launches", "clocks"))
    out["config"] = {"workload": d.get("config", {}).get("workload")}
    if "cpu_baseline" in d:
        out["cpu_baseline"] = d["cpu_baseline"]
    if "e2e" in d:
        out["e2e"] = d["e2e"]
    if w == "batched":
        out.update(pick(d, "plain_fp64", "speedup_vs_plain_fp64", "hpsi_ms",
                        "hpsi_multi_8sets_ms", "phase_ms_eager", "build_speedup_vs_cpu"))
    elif w == "serving":
        out["repeats"] = [{"p50_ms": r["latency_ms"]["p50"], "p99_ms": r["latency_ms"]["p99"],
                           "plain_p50_ms": r["plain_fp64"]["latency_ms"]["p50"],
                           "plain_p99_ms": r["plain_fp64"]["latency_ms"]["p99"],
                           "requests_per_s": r["throughput"]["requests_per_s"]} for r in ok]
        out["p99_ms_median"] = float(np.median([r["latency_ms"]["p99"] for r in ok]))
        out["plain_p99_ms_median"] = float(np.median(
            [r["plain_fp64"]["latency_ms"]["p99"] for r in ok]))
    elif w == "downfold":
        out.update(pick(d, "heff_ms", "build_ms", "phase_ms"))
    return out


def run_extras(args) -> dict:
    import subprocess
    out = {}
    for w, reps in EXTRAS:
        runs = []
        for _ in range(reps):
            _log(f"extra: {w}")
            t0 = time.perf_counter()
            try:
                p = subprocess.run([sys.executable, os.path.abspath(__file__), "--workload", w,
                                    "--steps", "3", "--warmup", "2", "--cpu-seconds", "3"],
                                   capture_output=True, text=True, timeout=args.extras_timeout)
                lines = [x for x in p.stdout.strip().splitlines() if x.startswith("{")]
                d = json.loads(lines[-1]) if lines else {
                    "error": f"rc={p.returncode}: {p.stderr.strip()[-300:]}"}
            except Exception as e:   # an extra never takes the headline line down
                d = {"error": f"{type(e).__name__}: {e}"[:300]}
            d["_wall_s"] = time.perf_counter() - t0
            runs.append(d)
        out[w] = _extra_summary(w, runs)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-dets", type=int, default=N_DETS)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--df-dets", type=int, default=DF_S,
                    help="size of S for --workload downfold (a smaller S for profiling)")
    ap.add_argument("--serve-slots", type=int, default=2,
                    help="build worker streams of the served path")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the short runs of the other workloads (default single-GPU "
                         "run only)")
    ap.add_argument("--extras-timeout", type=float, default=600.0)
    ap.add_argument("--workload", choices=["single", "batched", "serving", "downfold",
                                           "det_batch", "slogdet"],
                    default="single",
                    help="single: one 30-orbital system, 1e6 dets (default); batched: 64 "
                         "systems of uneven size per step; serving: Poisson request stream")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    run = {"single": run_ours, "batched": run_batched, "serving": run_serving,
           "downfold": run_downfold, "det_batch": run_det_batch,
           "slogdet": run_slogdet}[args.workload]
    res = run(args, rank, world)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        if args.workload == "single" and world == 1 and not args.no_extras:
            res["extras"] = run_extras(args)
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
