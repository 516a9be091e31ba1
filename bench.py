#!/usr/bin/env python
"""Benchmark of the pseudo-spectral SAV vesicle time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (N=1): 2D, 1024^2 grid, 8 vesicles (seeded non-overlapping ellipses,
radii U[0.4,0.7]), dt = 1e-5 (the largest probed step at which the reference
scheme stays stable), one time step = Steps 1-7 of the reference
(src/Solvers.jl) + state update + the per-step monitoring of
src/simulation.jl:146-148 (modified energy, area ratio).

The headline value is the arm named by --arm (default "mixed_krylov_diag":
FP64 fields, FFTs and SAV scalars; the psi solve -- the dominant cost -- as
the reference's left-preconditioned diagonal BiCGSTAB in FP32 inside FP64
iterative refinement).  Every comparison arm solves psi to the same TRUE
relative residual ||b - A x|| / ||b|| <= 1e-8 (the Krylov-form arms with the
true-residual stop, the flexible arms by construction) and is timed over the
same --steps; each arm reports the residual it actually reached (measured in
FP64 on a separate short run) and its per-field error against the FP64
reference-form solver after the same number of steps:
  mixed_krylov_diag   mixed precision, diagonal, Krylov.jl-form BiCGSTAB
  learned             mixed precision, flexible BiCGSTAB, diagonal + learned correction
  flex_diag           mixed precision, flexible BiCGSTAB, diagonal alone
  fp64_diag_rtol1e-8  the plain FP64 diagonal BiCGSTAB GPU solver at the same residual
  fp64_diag           the FP64 reference-form solve at the reference's settings
                      (conf.tol = 1e-12, Krylov.jl's preconditioned stop)
  fp32_bulk_learned   FP32 fields and FFTs, learned flexible BiCGSTAB (FP32 reaches 1e-6)

N>1 (torchrun): replicas only -- each rank advances its own seeded run, no
data-path collective; value = all ranks' steps / max-over-ranks device time.

--impl reference: the CPU restatement of the reference (the oracle, NumPy
FP64 on multi-threaded pocketfft) on the host cores, rank 0 only, on the
same configuration: every step is the whole coupled 8-vesicle step.
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
PKG = os.path.join(ROOT, "julia-vesicles-growth-and-shrinkage_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "steps/s at 1024²×8 vesicles, learned vs diagonal precond, same GPU, ≤1e-5 err"
WORKLOAD = "multi2d_1024x8"
DT = 1e-5


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Cfg:
    def __init__(self, **kw):
        self.__dict__.update(kw)
        self.Nz = kw.get("Nz", 0)
        self.Lz = kw.get("Lz", 0.0)


def workload(seed, n_vesicles=None):
    from vsav import ics
    kw, phi, psi, _ = ics.workload(WORKLOAD, seed=seed, N_override=n_vesicles)
    kw["dt"] = DT
    return kw, phi, psi


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        # the raw samples (set VSAV_CLOCKS_DIR to keep them); the JSON line carries the summary
        self.path = os.path.join(os.environ.get("VSAV_CLOCKS_DIR", tempfile.gettempdir()), f"vsav_clocks_rank{gpu_index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------- dist
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(x, ws, device="cuda"):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(steps, ms, ws, device="cuda"):
    """Whole-job rate of ws replicas that each timed `steps` steps in `ms` ms of
    device time: all replicas' steps over the slowest replica's time."""
    ms_max = max_over_ranks(ms, ws, device)
    return ws * steps / (ms_max / 1000.0), ms_max


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------- CPU
def class_roofline(prof, nsteps, hbm, peak_kind, traffic_file=False):
    """HBM roofline of the kernel class with the most device time in a profile
    (CUDA events around every launch, algorithmic bytes per launch)."""
    byte_classes = {k: v for k, v in prof.items() if k != "psi_net"}
    dom = max(byte_classes, key=lambda k: byte_classes[k]["ms"])
    d = prof[dom]
    per_launch_bytes = d["bytes"] / max(d["launches"], 1)
    per_launch_ms = d["ms"] / max(d["launches"], 1)
    achieved = per_launch_bytes / (per_launch_ms / 1000.0) / 1e9 if per_launch_ms > 0 else 0.0
    # DRAM bytes of one ncu-captured launch of the class (profiles/traffic.json, headline
    # workload only), scaled by algorithmic bytes to this class's average launch
    traffic, traffic_note = None, None
    tr_path = os.path.join(ROOT, "profiles", "traffic.json")
    if traffic_file and os.path.exists(tr_path):
        try:
            tr = json.load(open(tr_path)).get(dom)
            if tr:
                traffic = tr["dram_bytes"] / tr["algorithmic_bytes"] * per_launch_bytes
                traffic_note = (f"ncu dram__bytes_read+write of one {tr['kernel']} launch ({tr['dram_bytes']:.4g} B for "
                                f"{tr['algorithmic_bytes']:.4g} algorithmic B), scaled to the class's mean launch")
        except Exception:
            traffic = None
    tot_ms = max(sum(p["ms"] for p in prof.values()), 1e-9)
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": traffic, "traffic_note": traffic_note,
            "algorithmic_bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms,
            "launches_per_step": d["launches"] / nsteps, "share_of_profiled_time": d["ms"] / tot_ms,
            "classes": prof}


def headline_config(V, ws, arm):
    """The `config` object of the headline line (shared with the reference arm,
    which runs the same workload)."""
    return {"workload": WORKLOAD, "grid": [1024, 1024], "vesicles": V, "runs_per_gpu": 1, "dt": DT,
            "step": "Steps 1-7 + update + modified energy + area ratio",
            "psi_tolerance": "true relative residual 1e-8 (comparison arms)",
            "arm": arm, "parallelism": f"replicas x{ws}",
            "l2": "inputs larger than L2 (device state ~3 GB per run)"}


def step_roofline(prof, nsteps, ms_per_step, hbm, psi_iters=None, psi_fp32=False):
    """Whole-step HBM figures.  implementation: the algorithmic bytes of every
    launch of the step (the per-launch accounting of class_roofline, summed) over
    the step time.  reference_logical: the reference's own transforms and Krylov
    vector passes per step (profiles/algorithmic_bytes.json, counted by the
    oracle; pointwise work excluded, a lower bound) with the psi iteration counts
    `psi_iters` (iterations per system of one step), in the full-complex form the
    reference solves in and in the half-spectrum real-equivalent form."""
    impl = sum(p["bytes"] for k, p in prof.items() if k != "psi_net") / nsteps
    sec = ms_per_step / 1000.0
    out = {"unit": "GB/s", "peak": hbm, "ms_per_step": ms_per_step,
           "implementation_bytes_per_step": impl, "implementation_achieved": impl / sec / 1e9,
           "implementation_frac": impl / sec / 1e9 / hbm}
    try:
        ab = json.load(open(os.path.join(ROOT, "profiles", "algorithmic_bytes.json")))[WORKLOAD]
    except Exception:
        return out
    if psi_iters is not None:
        base = ab["fp64"]
        ps = ab["fp32" if psi_fp32 else "fp64"]
        it = float(sum(psi_iters))
        for conv in ("full", "half"):
            b = base["nonpsi_transform_bytes"] + ps["psi_fixed_bytes_" + conv] + it * ps["psi_bytes_per_iteration_" + conv]
            out["reference_logical_bytes_per_step_" + conv] = b
            out["reference_logical_achieved_" + conv] = b / sec / 1e9
            out["reference_logical_frac_" + conv] = b / sec / 1e9 / hbm
        out["psi_iters_per_system"] = list(psi_iters)
        out["psi_bytes_precision"] = "fp32" if psi_fp32 else "fp64"
    return out


def cpu_reference(steps, warmup, rank_seed=0):
    """The oracle (NumPy FP64, scipy pocketfft with all host threads) on the
    whole workload: every step advances all 8 coupled vesicle fields of the
    1024^2 run (Steps 1-7, update, monitor), as the reference's loop does."""
    from oracle import vsav_oracle as O
    kw, phi, psi = workload(rank_seed)
    cfg = O.Config(**kw)
    cores = os.cpu_count() or 1
    orc = O.Oracle(cfg, workers=cores)
    pres = O.make_state(cfg, phi, psi, orc.ops)
    O.init_state(cfg, pres, orc.ops)
    old = pres.copy()
    n = 1
    for _ in range(warmup):
        orc.step(pres, old, n, DT)
        orc.monitor(pres, old)
        n += 1
    t0 = time.perf_counter()
    for _ in range(steps):
        orc.step(pres, old, n, DT)
        orc.monitor(pres, old)
        n += 1
    dt = time.perf_counter() - t0
    iters = orc.counter.psi_iters
    return dict(value=steps / dt, unit="steps/s", cores=cores, kind="port",
                sample=f"the whole 1024^2 x 8 workload: {steps} coupled steps after {warmup} warm-up steps; "
                       f"FP64 NumPy/pocketfft (scipy.fft) with {cores} threads",
                sec_per_step=dt / steps, mean_psi_iters=float(np.mean(iters)) if iters else None)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_reference(args.steps, args.warmup)
    from vsav import ics
    kw, _, _, _ = ics.workload(WORKLOAD, seed=0)
    out = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "steps/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / cb["value"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": headline_config(kw["N"], args.gpus, args.arm),
           "reference_impl": "CPU restatement of the reference (oracle/vsav_oracle.py; Julia is absent)",
           "cpu_baseline": cb,
           "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------- ours
NET_FLOP_PER_PIXEL = 2 * (2 * 16 * 9 + 3 * 16 * 16 * 9 + 16 * 9)     # 14688: five 3x3 conv layers
WEIGHTS = os.path.join(PKG, "vsav", "precond_weights.npz")
TUNE_FILE = os.path.join(PKG, "vsav", "tuning_b200.json")
# the configurations timed on the same workload (the headline is --arm); the comparison
# arms solve psi to the same true relative residual 1e-8
ARMS = {
    "mixed_krylov_diag": dict(precision="mixed", psi_precond="diag", psi_rtol=1e-8, psi_stop="true"),
    "learned": dict(precision="mixed", psi_precond="learned", psi_net=WEIGHTS, psi_rtol=1e-8),
    "flex_diag": dict(precision="mixed", psi_precond="flex_diag", psi_rtol=1e-8),
    "fp64_diag_rtol1e-8": dict(precision="fp64", psi_precond="diag", psi_rtol=1e-8, psi_stop="true"),
    "fp64_diag": dict(precision="fp64", psi_precond="diag"),
    "fp32_bulk_learned": dict(precision="fp32", psi_precond="learned", psi_net=WEIGHTS, psi_rtol=1e-6, psi_itmax=60),
}
ARM_TEXT = {
    "mixed_krylov_diag": ("f64+f32", "FP64 fields, FFTs and SAV scalars; psi BiCGSTAB in FP32 inside FP64 iterative "
                          "refinement; Krylov.jl-form left-preconditioned diagonal BiCGSTAB, stopped on the true "
                          "residual 1e-8"),
    "learned": ("f64+f32+bf16", "FP64 fields, FFTs and SAV scalars; flexible BiCGSTAB in FP32 inside FP64 "
                "refinement, diagonal + learned correction (BF16 tensor-core network), true residual 1e-8"),
    "flex_diag": ("f64+f32", "FP64 fields, FFTs and SAV scalars; flexible BiCGSTAB in FP32 inside FP64 "
                  "refinement, diagonal, true residual 1e-8"),
    "fp64_diag_rtol1e-8": ("f64", "FP64 throughout; Krylov.jl-form diagonal BiCGSTAB, true residual 1e-8"),
    "fp64_diag": ("f64", "FP64 throughout; the reference's solve (Krylov.jl form, conf.tol 1e-12)"),
    "fp32_bulk_learned": ("f32+bf16", "FP32 fields and FFTs, FP64 SAV scalars; learned flexible BiCGSTAB, 1e-6"),
}


def field_errors(hh, Ea, ref, sb, Eb):
    """Relative L2 error of every field, the SAV scalars and the energy history
    of a handle against the FP64 reference-form state after the same steps."""
    acc = {}
    for k in ref:
        acc[k] = float(np.linalg.norm(hh.get_field(k) - ref[k]) / max(np.linalg.norm(ref[k]), 1e-300))
    sa = hh.get_scalars()[0]
    for i, k in enumerate(("Q", "R1", "R2", "R3")):
        acc[k] = float(abs(sa[i] - sb[i]) / max(abs(sb[i]), 1e-300))
    acc["energy"] = float(np.max(np.abs(Ea - Eb) / np.abs(Eb)))
    acc["energy_non_increasing"] = bool(np.all(np.diff(Ea) <= 0))
    acc["max_field_err"] = max(acc[k] for k in ("phi", "psi", "mu", "nu", "u", "p"))
    return acc


def run_ours(args):
    ws, rank, local = dist_init()
    os.environ.setdefault("VSAV_TUNE_FILE", TUNE_FILE)
    from vsav import Handle, _lib
    hbm, peak_kind = peaks()
    try:
        tflops_peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
    except Exception:
        tflops_peak = 1590.0
    kw, phi, psi = workload(rank, args.vesicles)
    V = kw["N"]
    head = args.arm
    K, W = args.steps, args.warmup
    h = Handle(Cfg(**kw), device=local, **ARMS[head])
    h.init_state(phi, psi)
    n = 1
    E_head = list(h.run(n, W, monitor=True)[0][:, 0])
    n += W
    clk = ClockSampler(local)
    barrier(ws)
    clk.start()
    l0 = _lib.load().vsav_launch_count()
    ms = h.time_run(n, K, monitor=True)
    launches = _lib.load().vsav_launch_count() - l0
    n += K
    clocks = clk.stop()
    barrier(ws)
    value, ms_max = aggregate(K, ms, ws)
    iters = h.psi_stats()[:, 0].tolist()
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": K,
                              "warmup": W, "ms_per_step": ms_max / K, "quick": True, "arm": head, "vesicles": V,
                              "gpu_launches": int(launches), "clocks": clocks, "psi_iters_last_step": iters,
                              "tuning": h.tuning()}), flush=True)
        h.close()
        return

    # end to end through the public API, host buffers: per step dt in (pinned
    # host memory), energy + area ratio out, as run_simulation's loop does
    import ctypes as ct
    try:
        import torch
        dt_host = torch.full((h.R,), DT, dtype=torch.float64).pin_memory()
        dt_ptr = ct.cast(dt_host.data_ptr(), ct.POINTER(ct.c_double))
        out_host = torch.zeros(2 * h.R, dtype=torch.float64).pin_memory()
        e_ptr = ct.cast(out_host.data_ptr(), ct.POINTER(ct.c_double))
        a_ptr = ct.cast(out_host.data_ptr() + 8 * h.R, ct.POINTER(ct.c_double))
        pinned = True
    except Exception:
        dt_np = np.full(h.R, DT)
        out_np = np.zeros(2 * h.R)
        dt_ptr = dt_np.ctypes.data_as(ct.POINTER(ct.c_double))
        e_ptr = out_np.ctypes.data_as(ct.POINTER(ct.c_double))
        a_ptr = ct.cast(out_np.ctypes.data + 8 * h.R, ct.POINTER(ct.c_double))
        pinned = False
    lib = _lib.load()
    st = _lib.VsavStatus()
    barrier(ws)
    t0 = time.perf_counter()
    for k in range(K):
        rc = lib.vsav_run(h.h, n, 1, dt_ptr, e_ptr, a_ptr, ct.byref(st))
        if rc < 0:
            raise RuntimeError(lib.vsav_last_error(h.h).decode())
        n += 1
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, ws)
    e2e = {"value": ws * K / e2e_s, "unit": "steps/s", "h2d_bytes_per_step": 8 * h.R,
           "d2h_bytes_per_step": 16 * h.R,
           "api": "vsav_run(h, n, 1, dt, energy, area_ratio) per step (the run_simulation loop body), "
                  + ("pinned" if pinned else "pageable") + " host buffers"}

    # per-kernel-class device time over K more steps (CUDA events per launch)
    h.profile("reset")
    h.profile(True)
    E_prof, _ = h.run(n, K, monitor=True)
    n += K
    h.profile(False)
    prof = h.profile_read()
    h.profile("reset")
    tuning = h.tuning()
    head_state = {k: h.get_field(k) for k in ("phi", "psi", "mu", "nu", "u", "p")}
    head_scalars = h.get_scalars()[0]
    h.close()
    head_steps = n - 1                                   # W + 3K steps from step 1
    roofline = class_roofline(prof, K, hbm, peak_kind, traffic_file=True)
    step_bytes = step_roofline(prof, K, ms_max / K, hbm, psi_iters=iters,
                               psi_fp32=ARMS[head]["precision"] != "fp64")

    def net_roofline(prof, nsteps, arm):
        pn = prof.get("psi_net", {})
        if not pn.get("launches"):
            return None
        px = 3 * V * kw["Nx"] * kw["Ny"]
        tf = pn["launches"] * px * NET_FLOP_PER_PIXEL / (pn["ms"] / 1000.0) / 1e12
        tot = max(sum(p["ms"] for p in prof.values()), 1e-9)
        kern = "k_net_apply_tc (tcgen05 bf16)" if os.environ.get("VSAV_NET_TC", "0") != "0" else "k_net_apply (mma.sync bf16)"
        return {"bound": "tensor", "kernel": kern, "arm": arm, "achieved": tf,
                "peak": tflops_peak, "unit": "TFLOP/s", "frac": tf / tflops_peak, "peak_kind": "measured bf16 burst",
                "ms_per_launch": pn["ms"] / pn["launches"], "launches_per_step": pn["launches"] / nsteps,
                "share_of_profiled_time": pn["ms"] / tot, "flop_per_pixel": NET_FLOP_PER_PIXEL}

    net_roof = net_roofline(prof, K, head)

    # the FP64 reference-form solve over the same steps: its state after W + K steps
    # (every arm's end point) and after W + 3K steps (the headline handle's end point)
    hb = Handle(Cfg(**kw), precision="fp64", psi_form="full", device=local)
    hb.init_state(phi, psi)
    Eb1, _ = hb.run(1, W + K, monitor=True)
    ref1 = {k: hb.get_field(k) for k in head_state}
    sb1 = hb.get_scalars()[0]
    Eb2, _ = hb.run(W + K + 1, 2 * K, monitor=True)
    ref2 = {k: hb.get_field(k) for k in head_state}
    sb2 = hb.get_scalars()[0]
    hb.close()

    class _State:                                        # the headline's end state, as a handle-like view
        def get_field(self, k):
            return head_state[k]

        def get_scalars(self):
            return [head_scalars]
    # fields and scalars after the headline's W + 3K steps; energies of its last K (profiled) steps
    head_acc = field_errors(_State(), E_prof[:, 0], ref2, sb2, Eb2[-K:, 0])
    head_acc["steps"] = head_steps

    # every arm: W warm-up + K timed steps, accuracy after those W + K steps, and the
    # true residual its psi solves reach (a separate 2-step run with the FP64 check)
    arms = {}
    for name, opts in ARMS.items():
        if args.arms and name not in args.arms.split(","):
            continue
        ha = Handle(Cfg(**kw), device=local, **opts)
        ha.init_state(phi, psi)
        Ew, _ = ha.run(1, W, monitor=True)
        msa = ha.time_run(1 + W, K, monitor=True)
        msa = max_over_ranks(msa, ws)
        it_last = ha.psi_stats()[:, 0].tolist()
        # the timed steps ran without monitor output to the host; the energy history of
        # the arm's W + K steps is compared at the warm-up steps and the end state
        acc = field_errors(ha, Ew[:, 0], ref1, sb1, Eb1[:W, 0])
        if net_roof is None and opts.get("psi_precond") == "learned":
            ha.profile("reset")
            ha.profile(True)
            ha.run(1 + W + K, 1, monitor=True)
            ha.profile(False)
            net_roof = net_roofline(ha.profile_read(), 1, name)
            ha.profile("reset")
        ha.close()
        hc = Handle(Cfg(**kw), device=local, psi_check=True, **opts)
        hc.init_state(phi, psi)
        hc.run(1, 2, monitor=False)
        true_res = hc.true_residuals().tolist()
        hc.close()
        arms[name] = {"value": ws * K / (msa / 1000.0), "unit": "steps/s", "steps": K, "warmup": W,
                      "psi_iters_last_step": it_last, "psi_true_residual_step2": true_res,
                      "rel_err_vs_fp64_after_steps": W + K, "rel_err_vs_fp64": acc,
                      "options": {k: v for k, v in opts.items() if k != "psi_net"}}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_reference(steps=1, warmup=1)
        cpu["sample"] = "the whole 1024^2 x 8 workload: 1 coupled step after 1 warm-up step; " +                         cpu["sample"].split("; ", 1)[1]

    if rank == 0:
        dtype, text = ARM_TEXT[head]
        cfg_out = headline_config(V, ws, head)
        cfg_out["precision"] = text
        out = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": K,
               "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
               "config": cfg_out, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
               "roofline": roofline, "roofline_step": step_bytes, "roofline_net": net_roof, "cpu_baseline": cpu,
               "psi_iters_last_step": iters, "accuracy_vs_fp64": head_acc, "tuning": tuning, "arms": arms}
        if "fp64_diag_rtol1e-8" in arms:
            out["speedup_vs_fp64_diag_same_residual"] = value / arms["fp64_diag_rtol1e-8"]["value"]
        if "fp64_diag" in arms:
            out["speedup_vs_fp64_reference_settings"] = value / arms["fp64_diag"]["value"]
        if "learned" in arms and "flex_diag" in arms:
            out["learned_vs_same_solver_diag"] = arms["learned"]["value"] / arms["flex_diag"]["value"]
            # why the learned arm wins or loses: iterations it saves against what its
            # network costs (two applications per flexible BiCGSTAB iteration)
            la, fa = arms["learned"], arms["flex_diag"]
            it_l, it_d = sum(la["psi_iters_last_step"]), sum(fa["psi_iters_last_step"])
            ms_l, ms_d = 1000.0 / la["value"], 1000.0 / fa["value"]
            budget = {"iterations_last_sweep_learned": la["psi_iters_last_step"],
                      "iterations_last_sweep_diag": fa["psi_iters_last_step"],
                      "iterations_saved_per_sweep": it_d - it_l,
                      "ms_per_step_learned": ms_l, "ms_per_step_diag": ms_d}
            if net_roof:
                budget["network_ms_per_application"] = net_roof["ms_per_launch"]
                budget["diag_ms_per_iteration_estimate"] = ms_d / max(1, 2 * it_d)
                budget["verdict"] = ("the network pays for itself only if it saves more iterations than its two "
                                     "applications per iteration cost: here it saves %d per sweep and adds %.2f ms "
                                     "per iteration" % (it_d - it_l, 2 * net_roof["ms_per_launch"]))
            out["learned_budget"] = budget
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def run_ensemble(args):
    """Batched ensemble (64 independent runs at 256^2, N ~ U{1..4}, FP32 bulk):
    one handle advancing all runs with one launch per sub-step, against the
    same 64 runs solved one after another, each in its own handle."""
    from vsav import Handle, ics
    kw, sizes, phi, psi = ics.ensemble(64)
    opts = dict(precision="fp32", psi_rtol=1e-6, psi_itmax=60)
    h = Handle(Cfg(**kw), run_sizes=sizes, **opts)
    h.init_state(phi, psi)
    h.run(1, args.warmup, monitor=True)
    ms = h.time_run(1 + args.warmup, args.steps, monitor=True)
    h.close()
    R = len(sizes)
    batched = R * args.steps / (ms / 1000.0)
    seq_ms = 0.0
    v0 = 0
    for r, N in enumerate(sizes):
        kr = dict(kw, N=N, psi_in_v=kw["psi_in_v"][v0:v0 + N], psi_out_v=kw["psi_out_v"][v0:v0 + N])
        hr = Handle(Cfg(**kr), **opts)
        hr.init_state(phi[v0:v0 + N], psi[v0:v0 + N])
        hr.run(1, args.warmup, monitor=True)
        seq_ms += hr.time_run(1 + args.warmup, args.steps, monitor=True)
        hr.close()
        v0 += N
    seq = R * args.steps / (seq_ms / 1000.0)
    print(json.dumps({"workload": "ensemble_256x64", "metric": "aggregate run-steps/s", "unit": "run-steps/s",
                      "runs": R, "vesicles": int(sum(sizes)), "grid": [256, 256], "precision": "fp32",
                      "steps": args.steps, "warmup": args.warmup,
                      "batched": {"value": batched, "ms_per_step": ms / args.steps},
                      "sequential": {"value": seq, "ms_per_run_step": seq_ms / (R * args.steps)},
                      "speedup": batched / seq}), flush=True)


def run_config(args):
    """Other configurations of the path, each its own JSON line (not the headline):
    multi2d_512x4 (2D 512^2, 4 vesicles), single3d_128 (3D 128^3, spectral-direct
    psi) and single3d_128_psivar (the same with the variable psi mobility and its
    BiCGSTAB, an extension): FP64 GPU, the faster GPU precision with its per-field
    error against the FP64 GPU path, and the CPU restatement (oracle) on a
    bounded sample."""
    from vsav import Handle, ics
    from oracle import vsav_oracle as O
    variable = args.workload.endswith("_psivar")
    hbm, peak_kind = peaks()
    kw, phi, psi, _ = ics.workload(args.workload.replace("_psivar", ""), seed=0)
    # the workloads' dt (vsav/ics.py: the largest probed step that stays stable)
    kw["dt"] = ics.DT_2D if kw.get("Nz", 0) == 0 else ics.DT_3D
    fast = "mixed" if args.workload == "multi2d_512x4" else "fp32"
    out = {"workload": args.workload, "metric": "steps/s", "unit": "steps/s", "steps": args.steps,
           "warmup": args.warmup, "dt": kw["dt"], "grid": [kw["Nx"], kw["Ny"]] + ([kw["Nz"]] if kw.get("Nz") else []),
           "vesicles": kw["N"], "psi3d_variable": variable}
    ref = None
    for prec in ("fp64", fast) + (("mixed",) if variable else ()):
        xo = dict(psi3d_variable=True) if variable else {}
        if variable and prec == "fp32":
            # the tightest tolerance one FP32 solve reaches reliably (the mixed 2D mode's sweep floor)
            xo.update(psi_rtol=1e-6, psi_itmax=60)
        h = Handle(Cfg(**kw), precision=prec, **xo)
        h.init_state(phi, psi)
        E, _ = h.run(1, args.warmup, monitor=True)
        fields = {k: h.get_field(k) for k in ("phi", "psi", "mu", "nu", "u", "p")}
        ms = h.time_run(1 + args.warmup, args.steps, monitor=True)
        res = {"value": args.steps / (ms / 1000.0), "ms_per_step": ms / args.steps,
               "energy_non_increasing": bool(np.all(np.diff(E[:, 0]) <= 0))}
        if variable:
            res["psi_iters_last_step"] = [int(x) for x in h.psi_stats()[:, 0]]
        # dominant kernel class over 2 more steps (CUDA events around every launch)
        h.profile("reset")
        h.profile(True)
        h.run(1 + args.warmup + args.steps, 2, monitor=True)
        h.profile(False)
        rf = class_roofline(h.profile_read(), 2, hbm, peak_kind)
        rf.pop("classes")
        res["roofline"] = rf
        h.close()
        if ref is None:
            ref = fields
        else:
            res["rel_err_vs_fp64_after_warmup_steps"] = {
                k: float(np.linalg.norm(fields[k] - ref[k]) / max(np.linalg.norm(ref[k]), 1e-300)) for k in ref}
        out[prec] = res
    if not args.no_cpu:
        cfg = O.Config(**kw)
        cores = os.cpu_count() or 1
        orc = O.Oracle(cfg, workers=cores, psi3d_variable=variable)
        pres = O.make_state(cfg, phi, psi, orc.ops)
        O.init_state(cfg, pres, orc.ops)
        old = pres.copy()
        orc.step(pres, old, 1, kw["dt"])
        t0 = time.perf_counter()
        orc.step(pres, old, 2, kw["dt"])
        orc.monitor(pres, old)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "steps/s", "cores": cores, "kind": "port",
                               "sample": "1 step after 1 warm-up step, FP64 NumPy/pocketfft"}
        out["speedup_fp64_gpu_vs_cpu"] = out["fp64"]["value"] / out["cpu_baseline"]["value"]
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--quick", action="store_true", help="main timed region only (for profiler runs)")
    ap.add_argument("--arm", default="mixed_krylov_diag", choices=list(ARMS),
                    help="the configuration of the headline value")
    ap.add_argument("--arms", default="", help="comma-separated subset of the compared configurations")
    ap.add_argument("--vesicles", type=int, default=None,
                    help="with --quick: fewer vesicles on the 1024^2 grid (smaller profiler captures)")
    ap.add_argument("--workload", default="multi2d_1024x8",
                    choices=["multi2d_1024x8", "ensemble_256x64", "multi2d_512x4", "single3d_128",
                             "single3d_128_psivar"],
                    help="anything but multi2d_1024x8 prints its own comparison line, not the headline")
    args = ap.parse_args()
    if args.vesicles is not None and not args.quick:
        ap.error("--vesicles changes the workload: --quick runs only")
    if args.workload == "ensemble_256x64":
        run_ensemble(args)
        return
    if args.workload in ("multi2d_512x4", "single3d_128", "single3d_128_psivar"):
        run_config(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
