"""Benchmark: turbulent-channel RK3/CN steps per second at 128 x 129 x 128 modes.

Workload (one step = one RK3/Crank-Nicolson step of the full velocity-vorticity
Navier-Stokes equations): box 4 pi x 2 x 4 pi/3, 129 x 129 x 129 Fourier /
Chebyshev modes (the reference's 128 x 129 x 128 configuration; its dealiased
physical grid is 194 x 129 x 194), Re_tau = 180, dt = 0.002, constant mass
flux, initial field = Reichardt mean profile + seeded solenoidal perturbation
(|kx|, |kz| <= 16, 10% of the centreline velocity).

Two forms are timed: plain FP64, and mixed precision (FP32 transforms and
products, split-TF32 y-derivatives on the tensor cores, FP64-accurate solves).
The headline is the mixed form when its energy after a fixed 1000-step run
agrees with the FP64 form's to 1e-6, else the FP64 form. Side legs (adjoint
gradients/s, the 48x65x48 perturbation case, gain ascent, the 256-run ensemble
on mixed boxes at a tenth of its horizons) print their own JSON lines first;
the headline line comes last and repeats the ensemble leg's rates.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun) runs independent replicas, one per GPU (the step does not
shard: no data-path collective); value = total steps of all ranks / max rank
time. `--impl reference` times the CPU restatement of the reference algorithm
(oracle/) on the host cores on a bounded sample of the same workload.
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

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "jax-spectral-dns_b200"))

SHAPE = (128, 129, 128)
LX, LZ = 4 * 3.141592653589793, 4 * 3.141592653589793 / 3
RE_TAU, DT = 180.0, 0.002
KMAX = (16, 16)
METRIC = "steps/s at 128x129x128 (turbulent channel RK3/CN step)"
WORKLOAD = "turbulent channel Re_tau=180, 129x129x129 modes, constant mass flux, dt=0.002"


def _dist():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def aggregate_over_ranks(local_ms: float, local_steps: int, device=None):
    """(max of the ranks' times, sum of the ranks' steps): the timing is the
    slowest replica's and the work is all replicas'. One MAX and one SUM
    all-reduce when a process group of more than one rank is up; the local
    values otherwise."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1):
        return float(local_ms), int(local_steps)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    n = torch.tensor([float(local_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), int(round(n.item()))


def split_runs(specs, rank: int, world: int):
    """This rank's share of an ensemble's independent runs (round robin): the
    replicas need no collective to step them."""
    return list(specs)[rank::world]


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# kernel class -> summary file stem under profiles/ (<stem>_channel_128x129x128.md)
KERNEL_NAMES = {"gemm": "k_dgemm", "sgemm": "k_tc05_split", "zinv": "k_zinv_sq", "xmid": "k_xmid", "zfwd": "k_zfwd_sq",
                "eigen": "k_eigen_update"}


def _ncu_traffic(kernel: str, form: str):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary of the benchmark workload, or None when there is none."""
    import re
    path = os.path.join(REPO, "profiles", f"{kernel}_channel_128x129x128.md")
    try:
        text = open(path).read()
    except OSError:
        return None
    m = re.search(r"DRAM traffic per launch \(read \+ write, MB\):(.*)", text)
    if not m:
        return None
    vals = dict(kv.split("=") for kv in m.group(1).split())
    if form in vals:
        return float(vals[form]) * 1e6
    launches = [float(v) for k, v in vals.items() if k.startswith("launch")]
    return sum(launches) / len(launches) * 1e6 if launches else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _seed_state():
    from jax_spectral_dns.seeds import turbulent_channel_hat

    return turbulent_channel_hat(SHAPE, (LX, LZ), RE_TAU, KMAX, seed=0)


def cpu_reference_leg(n_samples: int, warmup: int):
    """The oracle (CPU restatement of the reference step) on host cores.
    Returns (steps/s, seconds per step, sample description, threads)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np
    import jsd_oracle as O

    u0 = _seed_state()
    g = O.Grid(SHAPE, LX, LZ)
    st = O.Stepper(g, RE_TAU, DT, kind="ns", constant_mass_flux=True, flow_rate_target=g.flow_rate(u0[0]))
    dp = -g.flow_rate(u0[0]) * 3 / 2 / RE_TAU
    u = u0
    for t in range(warmup):
        u, dp = st.rk_step(u, dp, t)
    t0 = time.perf_counter()
    for t in range(n_samples):
        u, dp = st.rk_step(u, dp, warmup + t)
    dt = (time.perf_counter() - t0) / n_samples
    threads = os.cpu_count() or 1
    sample = (f"{n_samples} full RK3 step(s) of the 128x129x128 channel on the NumPy FP64 oracle "
              f"(OpenBLAS threads for the per-wavenumber matmuls, pocketfft single-threaded)")
    return 1.0 / dt, dt, sample, threads


def run_reference(args):
    rank, world, _ = _dist()
    if rank != 0:
        return
    # bounded sample: whole run within a few minutes (one oracle step is ~1 minute on 8 cores)
    n = max(1, min(args.steps, 2))
    rate, sec, sample, threads = cpu_reference_leg(n, 0)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": n, "warmup": 0, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Reichardt + solenoidal perturbation)",
        "config": {"workload": WORKLOAD, "modes": [129, 129, 129], "parallelism": "host cores"},
        "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


ACC_STEPS, ACC_EVERY = 1000, 50


def accuracy_leg(plans, u0_dev, dpdx0, n_steps=ACC_STEPS, every=ACC_EVERY):
    """Every form stepped n_steps (1000) from the same seeded field, whatever
    --steps is, with the energy recorded every `every` steps: the mixed form's
    relative energy error against the FP64 form (which the tests pin to the
    reference) after n_steps and over the history, and the relative error of
    the mean profile u_00(y)."""
    import torch
    from jax_spectral_dns._plan import GraphedSteps, to_reference_layout

    out, hist, final = {"steps": n_steps}, {}, {}
    dev = u0_dev.device
    for pr, plan in plans.items():
        st = u0_dev.clone()
        dp = torch.tensor([dpdx0], dtype=torch.float64, device=dev)
        g = GraphedSteps(plan, st, dp, 0, every)
        energies = [plan.energy(st)]
        for _ in range(n_steps // every):
            g.replay()
            energies.append(plan.energy(st))
        plan.check_device_errors()
        hist[pr] = torch.cat(energies).cpu()
        final[pr] = to_reference_layout(st)[0, 0, :, 0].real.clone()
        del g
    if "fp64" in hist and "mixed" in hist:
        rel = (hist["mixed"] / hist["fp64"] - 1).abs()
        out["mixed_energy_rel_err_vs_fp64"] = float(rel[-1])
        out["mixed_energy_history_max_rel_err"] = float(rel.max())
        out["mixed_mean_profile_rel_err_vs_fp64"] = float(
            torch.linalg.norm(final["mixed"] - final["fp64"]) / torch.linalg.norm(final["fp64"]))
    out["energy_final"] = {pr: float(h[-1]) for pr, h in hist.items()}
    out["energy_growth"] = {pr: float(h[-1] / h[0]) for pr, h in hist.items()}
    return out


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    from jax_spectral_dns._plan import GraphedSteps, StepPlan, to_device_layout, to_reference_layout
    from jax_spectral_dns.seeds import mode_counts

    modes, phys = mode_counts(SHAPE)
    u0 = _seed_state()
    u0_dev = to_device_layout(u0, device=dev)
    probe = StepPlan(modes, phys, LX, LZ, 0, RE_TAU, DT, device=dev)
    q0 = probe.flow_rate(u0_dev[0]).item()
    del probe
    dpdx0 = -q0 * 3 / 2 / RE_TAU
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return aggregate_over_ranks(x, 0, device=dev)[0]

    def timed(plan):
        """W warm-up steps, then K steps timed with CUDA events on the
        launching stream, barrier + synchronize on both sides. The K steps
        are one CUDA-graph replay (captured before the timed region)."""
        state = u0_dev.clone()
        dpdx = torch.tensor([dpdx0], dtype=torch.float64, device=dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        plan.step(state, dpdx, 0, args.warmup)
        graph = GraphedSteps(plan, state, dpdx, args.warmup, args.steps) if args.graph else None
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        if graph is not None:
            graph.replay()
        else:
            plan.step(state, dpdx, args.warmup, args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        # a kernel that gave up a bounded wait or a non-finite state voids the leg
        plan.check_device_errors()
        return max_over_ranks(ev0.elapsed_time(ev1)), state, dpdx

    forms = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    plans, results = {}, {}
    with ClockSampler(local) as clocks:
        time.sleep(0.3)  # let the sampler start before the GPU is loaded
        for pr in forms:
            plans[pr] = StepPlan(modes, phys, LX, LZ, 0, RE_TAU, DT, constant_mass_flux=True, flow_rate_target=q0,
                                 device=dev, precision=pr, autotune=args.autotune)
            ms, state, dpdx = timed(plans[pr])
            results[pr] = {"ms": ms, "state": state, "dpdx": dpdx, "energy": plans[pr].energy(state).item()}
    clock_summary = clocks.summary()
    finite = all(bool(torch.isfinite(torch.view_as_real(r["state"])).all()) for r in results.values())
    acc = accuracy_leg(plans, u0_dev, dpdx0, n_steps=args.accuracy_steps) if args.accuracy_steps > 0 else None
    mixed_err = acc.get("mixed_energy_rel_err_vs_fp64") if acc else None
    # headline form: mixed when its 1000-step energy error against FP64 meets the 1e-6 bar
    if args.precision == "both":
        head = "mixed" if (mixed_err is not None and mixed_err <= 1e-6) else "fp64"
    else:
        head = forms[0]
    plan = plans[head]
    ms_max = results[head]["ms"]
    value = world * args.steps / (ms_max / 1e3)
    state, dpdx = results[head]["state"], results[head]["dpdx"]

    # per-kernel-class timing with CUDA events on the launching stream (same workload)
    plan.profile(True)
    plan.step(state, dpdx, args.warmup + args.steps, args.steps)
    torch.cuda.synchronize()
    kernels = {}
    for name in ("gemm", "sgemm", "zinv", "xmid", "zfwd", "eigen"):
        tms, n, work = plan.profile_read(name)
        if n:
            kernels[name] = {"ms": tms, "launches": n, "work": work}
    plan.profile(False)
    plan.check_device_errors()

    # end to end through the public host-state call: every step copies a
    # state host->device from pinned memory, steps it and copies the result
    # back (StepPlan.step_host_stream overlaps the copies of the neighbouring
    # states with each step)
    host_in = to_reference_layout(state).cpu().pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    n_e2e = max(1, min(args.steps, 20))
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    plan.step_host_stream([host_in] * n_e2e, [host_out] * n_e2e, dpdx, 0, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    plan.check_device_errors()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / n_e2e)
    e2e_value = world / (e2e_ms / 1e3)
    state_bytes = host_in.numel() * host_in.element_size()

    if rank == 0:
        peaks, peak_src = _peaks()
        dom = max(kernels, key=lambda k: kernels[k]["ms"]) if kernels else None
        total_k = sum(v["ms"] for v in kernels.values())
        roofline = None
        if dom is not None:
            k = kernels[dom]
            ozaki = head == "mixed" and all(plans[head].eig_kernel(i)[0] == 1 for i in (1, 2))
            if dom == "gemm" and ozaki:
                # the mixed form's only GEMM-class launches are the eigenbasis
                # products, here on the int8 tensor cores: FP64-equivalent
                # throughput against the FP64 GEMM peak they replace, and the
                # int8 pipe's own use (36 slice products of 128 x 128 tensor
                # tiles per FP64-equivalent (Ny-2) x Ny product)
                fp64_peak = measure_fp64_peak(dev)
                achieved = k["work"] / (k["ms"] / 1e3) / 1e12
                ny = modes[1]
                int8_tops = achieved * 36 * 128 * 128 / ((ny - 2) * ny)
                int8_peak = 2 * peaks["bf16_tflops"]
                roofline = {"kernel": "k_oz8_gemm (FP64-accurate eigenbasis products, Ozaki int8 on tcgen05)",
                            "bound": "tensor", "achieved": achieved, "peak": fp64_peak,
                            "unit": "TFLOP/s (FP64-equivalent)", "frac": achieved / fp64_peak,
                            "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run (FP64 has no "
                                           "entry in MEASURED_PEAKS.json)",
                            "int8_pipe": {"achieved_tops": int8_tops, "peak_tops": int8_peak,
                                          "frac": int8_tops / int8_peak,
                                          "peak_source": "2 x bf16_tflops of MEASURED_PEAKS.json (dense int8 "
                                                         "issues at twice the bf16 rate)"},
                            "traffic": _ncu_traffic("k_oz8_gemm", head), "share_of_kernel_time": k["ms"] / total_k}
            elif dom == "gemm":
                fp64_peak = measure_fp64_peak(dev)
                ny = modes[1]
                same_shape = measure_fp64_same_shape(dev, ny - 2, ny, 3 * 2 * modes[0] * modes[2])
                achieved = k["work"] / (k["ms"] / 1e3) / 1e12
                mixed_sites = head == "mixed" and any(plans[head].eig_kernel(i)[0] == 1 for i in (1, 2))
                label = ("k_dgemm + k_oz8_gemm (eigenbasis products: FP64 DMMA at one site, FP64-accurate "
                         "int8 Ozaki at the other)" if mixed_sites else "k_dgemm (FP64 DMMA y-contractions)")
                roofline = {"kernel": label, "bound": "tensor",
                            "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                            "frac": achieved / fp64_peak,
                            "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run (FP64 has no "
                                           "entry in MEASURED_PEAKS.json)",
                            "cublas_same_shape_tflops": same_shape,
                            "traffic": _ncu_traffic("k_dgemm", head), "share_of_kernel_time": k["ms"] / total_k}
            elif dom == "sgemm":
                # split-TF32 products (y-derivatives, eigenbasis-in of the
                # nonlinear terms): three TF32 tensor products per FP32-level
                # product, against the dense TF32 rate (half the bf16 rate)
                achieved = 3 * k["work"] / (k["ms"] / 1e3) / 1e12
                tf32_peak = peaks["bf16_tflops"] / 2
                roofline = {"kernel": "k_tc05_split (split-TF32 products on tcgen05)", "bound": "tensor",
                            "achieved": achieved, "peak": tf32_peak, "unit": "TFLOP/s (TF32)",
                            "frac": achieved / tf32_peak,
                            "peak_source": peak_src + " (MEASURED_PEAKS.json bf16_tflops / 2)",
                            "traffic": _ncu_traffic("k_tc05_split", head),
                            "share_of_kernel_time": k["ms"] / total_k}
            else:
                achieved = k["work"] / (k["ms"] / 1e3) / 1e9
                roofline = {"kernel": KERNEL_NAMES[dom], "bound": "hbm", "achieved": achieved,
                            "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                            "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)",
                            "traffic": _ncu_traffic(KERNEL_NAMES[dom], head),
                            "algorithmic_bytes_per_launch": k["work"] / k["launches"],
                            "share_of_kernel_time": k["ms"] / total_k}
                if dom == "xmid":
                    # its bytes are small next to its FFT arithmetic: the HBM
                    # fraction is low because instruction issue limits it
                    roofline["limiter"] = ("instruction issue (ncu: 62% issue active, 12 warps per SM, 92 M warp "
                                           "instructions per launch; profiles/k_xmid_channel_128x129x128.md)")
            if roofline["traffic"] is not None:
                roofline["traffic_source"] = ("dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                                              f"profiles/{roofline['kernel'].split()[0]}_channel_128x129x128.md")
        per_kernel = {k: {"avg_us": round(1e3 * v["ms"] / v["launches"], 2), "launches": v["launches"],
                          "share": round(v["ms"] / total_k, 4)} for k, v in kernels.items()}
        for k, v in kernels.items():
            if k in ("gemm", "sgemm"):
                per_kernel[k]["tflops"] = round(v["work"] / (v["ms"] / 1e3) / 1e12, 2)
            else:
                per_kernel[k]["gbs"] = round(v["work"] / (v["ms"] / 1e3) / 1e9, 1)
        # side legs and kernel choices on their own lines, before the headline
        details = {pr: {"gemm_configs": {site: cfg for site, (cfg, _) in plans[pr].gemm_configs().items()},
                        "split_kernel": plans[pr].split_kernel(), "split_eig_in": plans[pr].split_eig_in(),
                        "xmid_variant": plans[pr].xmid_variant(),
                        "eig_kernels": {site: plans[pr].eig_kernel(i) for i, site in ((1, "eig_in"), (2, "eig_out"))}}
                   for pr in plans}
        print(json.dumps({"leg": "kernel_choices", "forms": details, "kernels": per_kernel}), flush=True)
        if not args.no_adjoint:
            print(json.dumps({"leg": "adjoint", **adjoint_leg(dev)}), flush=True)
        if not args.no_mixed_check:
            print(json.dumps({"leg": "perturbation_48x65x48", **mixed_check_leg(dev, args.autotune)}), flush=True)
        if not args.no_ascent:
            print(json.dumps({"leg": "gain_ascent", **ascent_leg(dev)}), flush=True)
        ens = None
        if world == 1 and args.ensemble_leg_runs > 0:
            ens = ensemble_leg(args.ensemble_leg_runs, args.ensemble_leg_scale)
            print(json.dumps({"leg": "ensemble", **ens}), flush=True)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            rate, sec, sample, threads = cpu_reference_leg(1, 0)
            cpu = {"value": rate, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample}
        forms_out = {pr: {"steps_per_s": round(world * args.steps / (r["ms"] / 1e3), 2),
                          "ms_per_step": round(r["ms"] / args.steps, 4)} for pr, r in results.items()}
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head == "fp64" else "mixed: f32 transforms/products, 3xtf32 y-derivatives, f64 solves",
            "data": "synthetic (seeded Reichardt mean + solenoidal perturbation)",
            "config": {"workload": WORKLOAD, "modes": list(modes), "fft_sizes": list(plan.fft_sizes),
                       "parallelism": f"replicas x{world}",
                       "l2": "working set per step ~1 GB > 126 MB L2 (no flush needed)",
                       "cuda_graph": bool(args.graph), "precision": head},
            "forms": forms_out,
            "mixed_over_fp64": (forms_out["mixed"]["steps_per_s"] / forms_out["fp64"]["steps_per_s"]
                                if len(forms_out) == 2 else None),
            "accuracy": acc,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "api": "StepPlan.step_host_stream on pinned host states (copies overlapped with the steps)"},
            "gpu_launches": plan.launches(args.steps),
            "ensemble": ({k: ens[k] for k in ("runs", "horizon_scale", "total_steps", "steps_per_s",
                                              "sequential_steps_per_s", "speedup_over_sequential")}
                         if ens else None),
            "roofline": roofline, "clocks": clock_summary, "cpu_baseline": cpu, "finite": finite,
            "device_errors": "none (jsd_device_error read after every timed region)",
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def adjoint_leg(dev, checkpoints=(10, 50, 150, 1500)):
    """Gain gradients per second on the 32x65x32 adjoint configuration
    (Re = 3000, Lx = 2 pi, Lz = pi, T = 15, dt = 0.01: 1500 steps), timed with
    CUDA events against a forward-only pass of the same horizon. Linear: the
    exact gradient by the discrete adjoint (no checkpoints needed: the
    linearised step is a fixed linear map). Nonlinear (E0 = 1e-4): the
    reference's continuous dual with checkpoints every K steps and recompute
    (K = 1500: one segment, the trajectory recorded in the forward pass)."""
    import torch
    from jax_spectral_dns.adjoint import GainProblem
    from jax_spectral_dns._plan import to_device_layout
    from jax_spectral_dns.seeds import mode_counts, seeded_velocity_hat

    shape, lx, lz, re, dt, T = (32, 65, 32), 2 * 3.141592653589793, 3.141592653589793, 3000.0, 0.01, 15.0
    modes, phys = mode_counts(shape)
    out = {"config": "32x65x32 (33x65x33 modes), Re=3000, T=15, dt=0.01 (1500 steps), seeded |k|<=8",
           "unit": "gradients/s"}

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, r

    u0 = to_device_layout(seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-6, seed=0), device=dev)
    p = GainProblem(modes, phys, lx, lz, re, dt, T, True, checkpoint_every=150, device=dev)
    p.discrete_gradient(u0)  # warm-up (captures the graphs)
    fwd_s, _ = timed(lambda: p.forward_only(u0))
    grad_s, (g, _) = timed(lambda: p.discrete_gradient(u0))
    out["linear_discrete"] = {"grads_per_s": 1.0 / grad_s, "grad_s": grad_s, "forward_s": fwd_s,
                              "cost_over_forward": grad_s / fwd_s, "gain": float(g.item()),
                              "note": "exact derivative of the discrete gain (jsd_step_adjoint)"}
    del p
    torch.cuda.empty_cache()
    u0 = to_device_layout(seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-4, seed=0), device=dev)
    per_k = {}
    for K in checkpoints:
        p = GainProblem(modes, phys, lx, lz, re, dt, T, False, checkpoint_every=K, device=dev)
        p.gain_and_dual(u0)  # warm-up (captures the segment graphs)
        fwd_s, _ = timed(lambda: p.forward_checkpoints(u0))
        grad_s, (g, _, _) = timed(lambda: p.gain_and_dual(u0))
        per_k[str(K)] = {"grads_per_s": 1.0 / grad_s, "grad_s": grad_s, "forward_s": fwd_s,
                         "cost_over_forward": grad_s / fwd_s, "gain": float(g.item())}
        del p
        torch.cuda.empty_cache()
    out["nonlinear_dual"] = per_k
    return out


def mixed_check_leg(dev, autotune=True, n_steps=2000, every=20):
    """Nonlinear perturbation about the laminar base U = 1 - y^2: Re = 5000,
    48x65x48 grid (49x65x49 modes), Lx = 2 pi, Lz = pi, dt = 0.005, 2000 steps,
    seeded solenoidal field over |kx|, |kz| <= 8 with E0 = 1e-3; run in the FP64
    and the mixed form, energy recorded every `every` steps. Reports steps/s of
    both forms and the largest relative energy difference of the mixed history
    from the FP64 one (the FP64 form is pinned to the oracle by the tests)."""
    import torch
    from jax_spectral_dns import _native
    from jax_spectral_dns._plan import GraphedSteps, StepPlan, to_device_layout
    from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

    shape, lx, lz, re, dt = (48, 65, 48), 2 * 3.141592653589793, 3.141592653589793, 5000.0, 0.005
    modes, phys = mode_counts(shape)
    u0 = to_device_layout(seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-3, seed=0), device=dev)
    base = 1 - cheb_points(modes[1]) ** 2
    out = {"config": "48x65x48 (49x65x49 modes), Re=5000, Lx=2pi, Lz=pi, dt=0.005, 2000 steps, E0=1e-3, "
                     "laminar base", "steps": n_steps}
    hist = {}
    for pr in ("fp64", "mixed"):
        plan = StepPlan(modes, phys, lx, lz, _native.JSD_KIND_PERTURBATION, re, dt, linearise=False,
                        base_u=base, precision=pr, device=dev, autotune=autotune)
        st, dp = u0.clone(), torch.zeros(1, dtype=torch.float64, device=dev)
        g = GraphedSteps(plan, st, dp, 0, every)
        energies = [plan.energy(st)]
        for _ in range(n_steps // every):
            g.replay()
            energies.append(plan.energy(st))
        hist[pr] = torch.cat(energies).cpu().numpy()
        # timing on a fresh copy: one graph of all steps, no energy evaluations inside
        st.copy_(u0)
        dp.zero_()
        gt = GraphedSteps(plan, st, dp, 0, n_steps)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        gt.replay()
        e1.record()
        torch.cuda.synchronize()
        out[pr] = {"steps_per_s": n_steps / (e0.elapsed_time(e1) / 1e3), "fft_sizes": list(plan.fft_sizes),
                   "energy_final": float(hist[pr][-1])}
        del gt, g, plan
    rel = abs(hist["mixed"] / hist["fp64"] - 1)
    out["mixed_over_fp64"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    out["energy_history_max_rel_err"] = float(rel.max())
    out["energy_growth"] = float(hist["fp64"][-1] / hist["fp64"][0])
    return out


def ascent_leg(dev, iterations=20):
    """Gain ascent on the 32x65x32 linear adjoint configuration (Re = 3000,
    T = 15, dt = 0.01, E0 = 1e-6) through the drop-in classes: dual problem from
    the forward perturbation equation and the conjugate-gradient solver, 20
    iterations. Reports the gain history and seconds per iteration."""
    import torch
    from jax_spectral_dns.domain import PhysicalDomain
    from jax_spectral_dns.field import FourierField, VectorField
    from jax_spectral_dns.gradient_descent_solver import ConjugateGradientDescentSolver
    from jax_spectral_dns.navier_stokes_perturbation import NavierStokesVelVortPerturbation
    from jax_spectral_dns.navier_stokes_perturbation_dual import NavierStokesVelVortPerturbationDual
    from jax_spectral_dns.seeds import seeded_velocity_hat

    shape, lx, lz, re, dt, T = (32, 65, 32), 2 * 3.141592653589793, 3.141592653589793, 3000.0, 0.01, 15.0
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(lx, 1.0, lz), aliasing=3 / 2)
    u0 = torch.as_tensor(seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-6, seed=0), device=dev)
    vel = VectorField.FromData(FourierField, dom, u0, name="velocity_hat")
    nse = NavierStokesVelVortPerturbation(vel, Re=re, dt=dt, end_time=T, linearise=True)
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse)
    solver = ConjugateGradientDescentSolver(dual, max_iterations=iterations, step_size=1e-2)
    solver.initialise()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while not solver.is_done(solver.i):
        solver.update()
        solver.i += 1
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    return {"config": "32x65x32, Re=3000, T=15, dt=0.01, linear, E0=1e-6, ConjugateGradientDescentSolver",
            "iterations": solver.i, "seconds_per_iteration": sec / max(1, solver.i),
            "gains": [float(g) for g in solver.history],
            "note": "host wall clock around whole iterations (forward run, dual run, projection, renormalisation)"}


def ensemble_leg(n_runs: int, horizon_scale: float):
    """The ensemble workload on one GPU: n_runs independent perturbation runs
    on mixed boxes (draw_ensemble), stepped as one batch plan per box (the
    product: one launch set per RK stage for all runs of a box) against the
    same runs one plan each, one after another on one stream. Device time
    (CUDA events) of one full pass each, after a warm-up pass of the batched
    form; the per-run plans' graphs are captured and warmed when they are
    built. Horizons are scaled by horizon_scale to bound the leg's time."""
    import numpy as np
    import torch

    from jax_spectral_dns.ensemble import BatchedEnsemble, Ensemble, draw_ensemble

    specs = draw_ensemble(n_runs, seed=0, horizon_scale=horizon_scale)
    steps = sum(s.steps for s in specs)
    bat = BatchedEnsemble(specs, streams=4, chunk=100)
    bat.run()
    bat.reset()
    ms = bat.run()
    e_bat = bat.energies()
    groups = len(bat.groups)
    del bat
    torch.cuda.empty_cache()
    seq = Ensemble(specs, streams=1, chunk=50)
    seq.reset()
    ms_seq = seq.run_sequential()
    e_seq = seq.energies()
    del seq
    torch.cuda.empty_cache()
    return {"runs": n_runs, "horizon_scale": horizon_scale, "total_steps": steps, "groups": groups,
            "steps_per_s": steps / (ms / 1e3), "sequential_steps_per_s": steps / (ms_seq / 1e3),
            "speedup_over_sequential": ms_seq / ms,
            "energy_max_rel_diff_vs_one_plan_per_run": float(np.abs(e_bat / e_seq - 1).max()),
            "dtype": "f64",
            "config": "Nx=Nz in {16,32,48,64} x Ny in {49,65,97}, Re U[2000,6000], E0 logU[1e-6,1e-2], "
                      "T in {5,10,15,20} x horizon_scale, dt=0.01, nonlinear perturbation runs"}


def run_ensemble(args):
    """Aggregate steps/s of an ensemble of independent perturbation runs:
    runs sharing a box stepped as one batch plan per group (the product), the
    same runs one plan each on a stream pool, and one after another."""
    import numpy as np
    import torch

    from jax_spectral_dns.ensemble import BatchedEnsemble, Ensemble, draw_ensemble

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    specs = draw_ensemble(args.ensemble, seed=0, horizon_scale=args.ensemble_horizon_scale)
    mine = split_runs(specs, rank, world)  # replicas: runs split across GPUs, no collective while stepping
    bat = BatchedEnsemble(mine, streams=4, chunk=100)
    bat.run()  # warm-up
    bat.reset()
    ms = bat.run()
    e_bat = bat.energies()
    del bat
    torch.cuda.empty_cache()
    ens = Ensemble(mine, streams=args.ensemble_streams, chunk=50)
    ens.run()  # warm-up
    ens.reset()
    ms_pool = ens.run()
    e_pool = ens.energies()
    ens.reset()
    ms_seq = ens.run_sequential()
    local_steps = sum(s.steps for s in mine)
    ms, steps = aggregate_over_ranks(ms, local_steps, device=torch.device("cuda", local))
    ms_pool, _ = aggregate_over_ranks(ms_pool, 0, device=torch.device("cuda", local))
    ms_seq, _ = aggregate_over_ranks(ms_seq, 0, device=torch.device("cuda", local))
    if rank == 0:
        print(json.dumps({
            "metric": "ensemble steps/s (independent perturbation runs, mixed grids)",
            "value": steps / (ms / 1e3), "unit": "steps/s", "n_gpus": world, "runs": len(specs),
            "total_steps": steps, "ms": ms, "groups_rank0": len({(s.n, s.ny) for s in mine}),
            "stream_pool_steps_per_s": steps / (ms_pool / 1e3), "sequential_steps_per_s": steps / (ms_seq / 1e3),
            "speedup_over_stream_pool": ms_pool / ms, "speedup_over_sequential": ms_seq / ms,
            "energy_max_rel_diff_vs_one_plan_per_run": float(np.abs(e_bat / e_pool - 1).max()),
            "horizon_scale": args.ensemble_horizon_scale, "dtype": "f64",
            "config": {"workload": "Nx=Nz in {16,32,48,64} x Ny in {49,65,97}, Re U[2000,6000], "
                                   "E0 logU[1e-6,1e-2], T in {5,10,15,20} x horizon_scale, dt=0.01",
                       "product": "one batch plan per box, one launch set per RK stage for all its runs"},
        }), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()

def measure_fp64_peak(dev) -> float:
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return 2 * n ** 3 / (best / 1e3) / 1e12


def measure_fp64_same_shape(dev, m: int, k: int, n: int) -> float:
    """cuBLAS FP64 (torch.matmul) TFLOP/s on the eigenbasis products' own
    shape: an m x k operator times k x n fields (n = 3 fields' columns)."""
    import torch

    a = torch.randn(m, k, dtype=torch.float64, device=dev)
    b = torch.randn(k, n, dtype=torch.float64, device=dev)
    for _ in range(3):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return 2.0 * m * k * n / (best / 1e3) / 1e12


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=ACC_STEPS,
                    help="steps of the mixed-vs-FP64 accuracy run (0 skips it; the headline is then FP64)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint gradients/s leg")
    ap.add_argument("--no-mixed-check", action="store_true",
                    help="skip the 48x65x48 perturbation leg (FP64 vs mixed energy history)")
    ap.add_argument("--no-ascent", action="store_true", help="skip the 20-iteration gain-ascent leg")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default GEMM tile configurations instead of autotuning them at plan creation")
    ap.add_argument("--ensemble", type=int, default=0, help="run the ensemble benchmark with this many runs")
    ap.add_argument("--ensemble-horizon-scale", type=float, default=0.25)
    ap.add_argument("--ensemble-streams", type=int, default=16)
    ap.add_argument("--ensemble-leg-runs", type=int, default=256,
                    help="runs of the ensemble leg of the default run (0 skips it)")
    ap.add_argument("--ensemble-leg-scale", type=float, default=0.1,
                    help="horizon scale of the ensemble leg of the default run")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="launch the timed steps directly instead of replaying a captured CUDA graph")
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"],
                    help="headline form; 'both' times FP64 and mixed and reports mixed beside FP64")
    args = ap.parse_args()
    world = _dist()[1]
    if 0 < args.ensemble < world:
        # every rank must own at least one run: an empty rank would skip the
        # stepping but its peers would still wait for it in the aggregation
        ap.error(f"--ensemble {args.ensemble} is smaller than the number of ranks ({world})")
    if args.impl == "reference":
        run_reference(args)
    elif args.ensemble > 0:
        run_ensemble(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
