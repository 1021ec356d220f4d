"""Benchmark: THC-GW iteration time (and RPA E_c time) on one B200, mixed vs FP64.

One step = one THC-GW iteration of the RPA + GW workload ``rpa_gw_k6_nb96_np1024``
(6x6x6 k-grid = 216 k, 96 orbitals / 48 occupied, N_mu = 1024, beta = 1000, IR
Lambda = 1e5 "low" -> 61 tau points, 6,696 (q, iW) Dyson problems): Pi(tau) -> Pi(iW) ->
Dyson W(iW) -> W(tau) -> Sigma(tau), i.e. scr_coulomb_t::update_w + gw_t::evaluate.  It is
the largest of the reference-shaped configurations and fits one B200 (Pi/W as complex64,
56 GB).  ``--workload`` selects another (``g0w0_k4_nb64_np512``, ``batch32_gamma``,
``scgw_k3_nb48_np384``).

* ``value``: device time per iteration with G resident in HBM (CUDA events on the
  library's stream), mixed precision; ``e2e``: the same through the public C ABI with the
  host G copied in and Sigma copied out every step (pinned host buffers).
* ``rpa_energy_ms``: the RPA E_c time (Pi -> Pi(iW) -> FP64 log-det), resident G.
* ``fp64_form``: the same path in FP64, its times, and the mixed path's errors against it.
* ``--impl reference``: the FP64 oracle (numpy/OpenBLAS restatement of the reference
  algorithm) on the host cores, per-unit samples extrapolated to one iteration.
* Multi-GPU (torchrun): the path does not shard; ranks run independent replicas.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "rpa_gw_k6_nb96_np1024"
METRIC = "THC-GW iteration time (mixed precision, 1 B200)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default=WORKLOAD)
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64-form comparison")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--only-iteration", action="store_true",
                   help="the timed GW iterations alone (no side legs), e.g. under a profiler")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(vals, world, device="cuda"):
    """Element-wise maximum of per-rank timings over the process group (identity for one rank):
    the replicas' step time is that of the slowest rank."""
    if world <= 1:
        return [float(v) for v in vals]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


class Clocks:
    """Samples the SM clock and the throttle reasons during the timed region (NVML in-process
    every 10 ms, one sample as the region starts and one as it ends; nvidia-smi when NVML is
    unavailable)."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.rows, self.stop = device, [], threading.Event()
        self.nvml = None
        try:  # in-process NVML reads: one sample costs microseconds, not a process start
            import pynvml
            import torch
            pynvml.nvmlInit()
            p = torch.cuda.get_device_properties(device)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            self.nvml = (pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus))
        except Exception:
            self.nvml = None

    def _nvml_row(self):
        nv, h = self.nvml

        def q(f, *a):
            try:
                return f(h, *a)
            except Exception:
                return None
        bits = q(nv.nvmlDeviceGetCurrentClocksEventReasons)
        sm = q(nv.nvmlDeviceGetClockInfo, nv.NVML_CLOCK_SM)
        if bits is None or sm is None:
            raise RuntimeError("NVML clock query failed")
        mx = q(nv.nvmlDeviceGetMaxClockInfo, nv.NVML_CLOCK_SM)
        pw = q(nv.nvmlDeviceGetPowerUsage)
        flags = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                 nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        return ([str(sm), str(mx) if mx is not None else "", str(pw / 1000.0) if pw else ""]
                + ["Active" if bits & f else "Not Active" for f in flags])

    def _sample_nvml(self):
        try:
            self.rows.append(self._nvml_row())
            self.src.add("nvml")
            return True
        except Exception:
            self.fails += 1
            return False

    def _run(self):
        bad = 0
        while self.nvml is not None and not self.stop.is_set():
            bad = 0 if self._sample_nvml() else bad + 1
            if bad >= 5:  # NVML keeps failing: fall back to nvidia-smi
                self.nvml = None
                break
            self.stop.wait(0.01)
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([v.strip() for v in out.split(",")])
                    self.src.add("nvidia-smi")
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.src, self.fails = set(), 0
        if self.nvml is not None:
            self._sample_nvml()  # the state as the timed region starts
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)
        if self.nvml is not None:
            self._sample_nvml()  # and as it ends

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows),
                "source": sorted(self.src), "failed_queries": self.fails}


def make_case(name):
    from coqui_b200.iaft import IAFT
    from coqui_b200.synthetic import WORKLOADS, make_system
    w = WORKLOADS[name]
    s = make_system(w["n"], w["nb"], w["nocc"], w["Np"], beta=w["beta"], seed=2024)
    ft = IAFT(w["beta"], w["lam"] / w["beta"], w["prec"])
    return w, s, ft


def make_ctx(s, ft, mode):
    from coqui_b200 import capi
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=mode)
    c.set_ir(ft)
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    return c


def total_ms(ctx):
    return sum(ms for _, ms in ctx.timings())


def gemm_flops_c(M, N, K):
    return 8.0 * M * N * K  # complex MAC = 8 real flops (FP64-equivalent count)


def algorithmic_work(w, s, ft):
    """Algorithmic work of each kernel group: (kind, amount per launch group or None,
    amount per iteration or None, amount per work unit or None).  Flops count a complex
    multiply-add as 8 (FP64-equivalent count of the product actually formed, triangular
    structure included); bytes are the compulsory complex64 reads + writes.  The projections
    count per (tau, k) problem, times the problems the library reports (a G(tau) whose
    projection does not fit the cache is projected again for the self-energy)."""
    nk, nb, Np, nth, nwh, nt = s.nk, s.nb, s.Np, ft.nt_half, ft.nw_half, ft.nt_f
    ncol, P = Np * Np, nk * nwh  # Dyson problems per iteration
    n3 = float(Np) ** 3
    return {
        # per (tau, k) problem: T = X G (Np x nb, K = nb), T X^H (Np x Np, K = nb); and
        # U = S X (Np x nb, K = Np), X^H U (nb x nb, K = Np)
        "proj_p2a": ("tensor", None, None, gemm_flops_c(Np, nb, nb) + gemm_flops_c(Np, Np, nb)),
        "proj_a2p": ("tensor", None, None, gemm_flops_c(Np, nb, Np) + gemm_flops_c(nb, nb, Np)),
        "pi_fused": ("hbm", 3 * nk * ncol * 8, None),
        "sigma_fused": ("hbm", 5 * nk * ncol * 8, None),
        "dft_w": ("hbm", 2 * nth * nk * ncol * 8, None),
        "ir_transform": ("hbm", (nth + nwh) * nk * ncol * 8, None),
        # M = L^H Pi L: the part of P1 = L^H Pi on and above the diagonal (Np^3 / 3; the
        # lower triangle of M reads no other) and the lower triangle of L^H P1^H (Np^3 / 6)
        # complex multiply-adds
        "dyson_M_gemm": ("tensor", None, (1 / 3 + 1 / 6) * 8 * n3 * P),
        # lower triangles of F = D^H D (1/6), T = L E (1/3) and W = T L^H (1/6)
        "dyson_W_gemm": ("tensor", None, (1 / 6 + 1 / 3 + 1 / 6) * 8 * n3 * P),
        # FP64 Cholesky (Np^3 / 6 complex multiply-adds) + inverse of the 128 x 128 diagonal
        # groups (Np 128^2 / 6); the whole inverse (Np^3 / 6) when Np <= 128
        "dyson_chol_inv": ("fp64", None, 8 * (n3 / 6 + (Np * min(Np, 128) ** 2) / 6) * P),
        # the rest of the triangular inverse on the tensor cores
        "dyson_tc_inverse": ("tensor", None, 8 * max(0.0, n3 - Np * min(Np, 128) ** 2) / 6 * P),
    }


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count()


def _best(fn, reps=2):
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best


def reference_unit_counts(s, ft):
    """How often the reference algorithm performs each unit in one GW iteration without
    symmetry (nq = nk): the polarizability (rpa_pi.icc:102-176), the IR transforms
    (IAFT.icc:49-128), the LU Dyson solve (scr_coulomb_t.cpp:171-199) and the R-space
    self-energy with its aux -> primary step (thc_gw.icc:70-213, 37-65)."""
    nk, nth, nwh = s.nk, ft.nt_half, ft.nw_half
    return {
        # G(tau) and G(beta - tau) for every tau < beta/2, once for Pi and again for Sigma
        "proj_p2a": 4 * nth * nk,
        "proj_a2p": 2 * nth * nk,
        # (nk x nk) x (nk x Np^2) DFT GEMMs: Pi 3 per tau; Sigma: W q->R and back (nth
        # each) plus 2 per tau and half
        "dft": 3 * nth + 6 * nth,
        "hadamard": nth + 2 * nth,
        "ir_columns": 2,  # tau -> iW and iW -> tau over all nq Np^2 columns
        "dyson": nk * nwh,
    }


def cpu_sample(s, ft, reps=2):
    """One GW iteration of the FP64 oracle (numpy complex128 on OpenBLAS, every host core),
    extrapolated from timed samples of its units: each unit is timed on a bounded sample
    (best of `reps`) and scaled by the number of times the reference algorithm performs it
    (`reference_unit_counts`).  Returns (total ms, {unit: ms per iteration})."""
    from oracle import thc_oracle as O
    nk, Np, nt, nth, nwh = s.nk, s.Np, ft.nt_f, ft.nt_half, ft.nw_half
    ncol = Np * Np
    G = s.G0(ft)
    f_Rk = O.k_to_R_coefficients(s.kpts, s.lattv, s.kp_grid)
    kk = min(nk, 4)
    cols = min(ncol, 1 << 15)
    rng = np.random.default_rng(1)
    slab = (rng.standard_normal((nk, cols)) + 1j * rng.standard_normal((nk, cols)))
    S_k = (rng.standard_normal((1, kk, Np, Np)) + 1j * rng.standard_normal((1, kk, Np, Np)))
    tslab = np.resize(slab, (nth, cols))
    per = {
        "proj_p2a": _best(lambda: O.primary_to_aux(G[0][:, :kk], s.X[:, :kk]), reps) / kk,
        "proj_a2p": _best(lambda: O.aux_to_primary(S_k, s.X[:, :kk]), reps) / kk,
        "dft": _best(lambda: f_Rk @ slab, reps) * ncol / cols,
        "hadamard": _best(lambda: -2.0 * slab * np.conj(slab), reps) * ncol / cols,
        "ir_columns": _best(lambda: ft.Twt_pos() @ tslab, reps)
        * nk * ncol / cols,
        "dyson": _best(lambda: O.dyson_W_in_place(S_k[:, :1] * 1e-3, s.V[:1]), reps),
    }
    counts = reference_unit_counts(s, ft)
    parts = {k: per[k] * counts[k] * 1e3 for k in per}
    return float(sum(parts.values())), parts


CPU_SAMPLE_NOTE = ("FP64 numpy/OpenBLAS oracle, extrapolated: per-unit times (projections of 4 "
                   "k-points, one DFT and one Hadamard product over 32768 columns, one IR "
                   "transform over the same columns, one (q, iW) LU Dyson solve) scaled by the "
                   "reference algorithm's unit counts for one GW iteration")


def run_reference(args, rank):
    if rank != 0:
        return
    w, s, ft = make_case(args.workload)
    cores = host_cores()
    vals = []
    for i in range(args.warmup + args.steps):
        t, parts = cpu_sample(s, ft, reps=1)
        if i >= args.warmup:
            vals.append(t)
    v = float(np.median(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": v,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic", "config": config_of(args.workload, w, s, ft),
        "cpu_baseline": {"value": v, "unit": "ms", "cores": cores, "kind": "port",
                         "extrapolated": True, "sample": CPU_SAMPLE_NOTE,
                         "parts_ms": {k: round(x, 1) for k, x in parts.items()}},
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_of(name, w, s, ft):
    return {"workload": name, "nk": s.nk, "nb": s.nb, "Np": s.Np, "nt": ft.nt_f,
            "nw_b": ft.nw_b, "prec": w["prec"], "beta": w["beta"], "lambda": w["lam"],
            "parallelism": "replicas",
            "l2": "working set (Pi/W %.1f GB) far above L2 (126 MB); no flush" % (
                max(ft.nt_half, ft.nw_half) * s.nk * s.Np ** 2 * 8 / 1e9)}


def measure_fp64_peak(device):
    """Dense FP64 rate of cuBLAS on this GPU (TFLOP/s): DGEMM 8192^3 (2 N^3 flop) and ZGEMM
    4096^3 (8 N^3 flop), best of 8 each, CUDA events; the larger of the two."""
    import torch
    out = {}
    for name, n, dt, fl in (("dgemm", 8192, torch.float64, 2.0), ("zgemm", 4096, torch.complex128,
                                                                    8.0)):
        a = torch.randn(n, n, dtype=dt, device=device)
        b = torch.randn(n, n, dtype=dt, device=device)
        c = a @ b
        best = float("inf")
        for _ in range(8):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b, out=c)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        out[name + "_tflops"] = fl * n ** 3 / (best * 1e-3) / 1e12
        if name == "zgemm":
            # sustained: back to back for ~2.5 s, so that the clocks settle under the power
            # cap as they do inside a GW iteration (the denominator for kernels timed there)
            reps = max(8, int(2.5e3 / best))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with Clocks(device) as clk:
                e0.record()
                for _ in range(reps):
                    torch.matmul(a, b, out=c)
                e1.record()
                e1.synchronize()
            out["zgemm_sustained_tflops"] = fl * n ** 3 * reps / (e0.elapsed_time(e1) * 1e-3) / 1e12
            out["sustained_sm_mhz"] = clk.summary().get("sm_mhz")
        del a, b, c
    torch.cuda.empty_cache()
    out["tflops"] = max(out["dgemm_tflops"], out["zgemm_tflops"])
    out["sustained_tflops"] = out["zgemm_sustained_tflops"]
    out["how"] = ("cuBLAS through torch.matmul: DGEMM 8192^3 and ZGEMM 4096^3, best of 8 (burst); "
                  "ZGEMM 4096^3 back to back for ~2.5 s (sustained)")
    return out


def group_rates(stats, steps, work, hbm, bf16, fp64, fp64_sustained=None, units=None):
    """Per-kernel-group time and achieved rate against its own roof (HBM copy, bf16 tensor,
    or the measured FP64 rate, burst and sustained)."""
    groups = {}
    units = units or {}
    for name, (ms_tot, n) in stats.items():
        ms_it = ms_tot / steps
        kind, per_launch, per_iter, per_unit = (tuple(work.get(name, ())) + (None,) * 4)[:4]
        u = units.get(name, 0)
        if per_iter is not None:
            amount = per_iter
        elif per_launch is not None:
            amount = per_launch * n / steps
        elif per_unit is not None and u > 0:
            amount = per_unit * u / steps
        else:
            amount = None
        g = {"ms_per_step": ms_it, "launch_groups_per_step": n / steps, "bound": kind}
        if per_unit is not None and u > 0:
            g["units_per_step"] = u / steps
        if amount and ms_it > 0:
            if kind == "hbm":
                g["achieved_GBps"] = amount / (ms_it * 1e-3) / 1e9
                g["frac_of_hbm"] = g["achieved_GBps"] / hbm
            else:
                g["achieved_TFLOPs"] = amount / (ms_it * 1e-3) / 1e12
                if kind == "tensor":
                    g["frac_of_bf16"] = g["achieved_TFLOPs"] / bf16
                    g["frac_of_split_tf32_ceiling"] = g["achieved_TFLOPs"] / (bf16 / 6.0)
                elif kind == "fp64":
                    g["frac_of_fp64_measured"] = g["achieved_TFLOPs"] / fp64
                    if fp64_sustained:
                        g["frac_of_fp64_sustained"] = g["achieved_TFLOPs"] / fp64_sustained
        groups[name] = g
    return groups


def profile_traffic(kernel, Np):
    """DRAM bytes per (q, iW) problem of a kernel group from a committed ncu summary
    (`profiles/dram_traffic_<group>_np<Np>.md`, line `bytes_per_problem: B`), or None."""
    path = os.path.join(ROOT, "profiles", f"dram_traffic_{kernel}_np{Np}.md")
    try:
        for ln in open(path):
            if ln.startswith("bytes_per_problem:"):
                return float(ln.split(":")[1]), os.path.relpath(path, ROOT)
    except OSError:
        pass
    return None, None


def run_ours(args, rank, world, local):
    import torch
    from coqui_b200 import capi

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    w, s, ft = make_case(args.workload)
    G = s.G0(ft)
    side = max(1, min(args.steps, 3))  # repetitions of the legs beside the headline

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    fp64_peak = measure_fp64_peak(local)
    ctx = make_ctx(s, ft, capi.MIXED)

    # warm-up (resident G)
    ctx.gw_iteration(G, want_sigma=False)
    for _ in range(max(args.warmup - 1, 0)):
        ctx.gw_iteration(None, want_sigma=False)
    barrier()
    launches0 = ctx.kernel_launches()
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            ctx.gw_iteration(None, want_sigma=False)
            times.append(total_ms(ctx))
    barrier()
    launches = (ctx.kernel_launches() - launches0) // max(args.steps, 1)
    t_step = float(np.sum(times)) / args.steps
    phases = dict(ctx.timings())
    if args.only_iteration:
        ctx.close()
        t_step = max_over_ranks([t_step], world)[0]
        if rank == 0:
            print(json.dumps({
                "metric": METRIC, "value": t_step / world, "unit": "ms", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "c64/f64", "data": "synthetic", "legs": "iteration only",
                "config": config_of(args.workload, w, s, ft), "gpu_launches": int(launches),
                "steps_ms": [round(t, 3) for t in times], "clocks": clk.summary()}), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    # per-kernel-group CUDA-event timing in separate steps (the events add host work between
    # launches, so they stay out of the timed steps above)
    ctx.set_profiling(True)
    for _ in range(side):
        ctx.gw_iteration(None, want_sigma=False)
    barrier()
    stats = ctx.kernel_stats()
    stat_units = ctx.kernel_units()
    ctx.set_profiling(False)

    # e2e through the public API with pinned host buffers
    Gh = torch.empty(G.shape, dtype=torch.complex128, pin_memory=True).numpy()
    Gh[...] = G
    Sh = torch.empty(G.shape, dtype=torch.complex128, pin_memory=True).numpy()
    ctx.gw_iteration(Gh, sigma_out=Sh)
    e2e, e2e_wall = [], []
    with Clocks(local) as clk_e2e:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ctx.gw_iteration(Gh, sigma_out=Sh)  # returns with Sigma in Sh
            e2e_wall.append((time.perf_counter() - t0) * 1e3)
            e2e.append(total_ms(ctx))
    t_e2e = float(np.mean(e2e))
    e2e_phases = dict(ctx.timings())

    # RPA energy time (resident G) and E_c
    ctx.rpa_energy(Gh)
    rpa = []
    with Clocks(local) as clk_rpa:
        for _ in range(max(1, args.steps)):
            e_c = ctx.rpa_energy(None)
            rpa.append(total_ms(ctx))
    t_rpa = float(np.mean(rpa))
    rpa_phases = dict(ctx.timings())

    # THC Hartree-Fock F = J + K (gygi) of the density matrix of G, FP64 in both precision
    # modes: the device phase and the public call with the host Dm in and F out
    Dm = -np.tensordot(ft.T_beta_t_ff, G, axes=(0, 0))
    Dm = np.ascontiguousarray(0.5 * (Dm + np.conj(np.swapaxes(Dm, -1, -2))))
    S_ov = np.ascontiguousarray(np.broadcast_to(np.eye(s.nb, dtype=np.complex128), Dm.shape))
    hf_dev, hf_e2e, hf_wall = [], [], []
    l0 = ctx.kernel_launches()
    for i in range(1 + side):
        t0 = time.perf_counter()
        F_hf = ctx.hf_evaluate(Dm, S_ov, True, True, "gygi", 0.5)
        wall = (time.perf_counter() - t0) * 1e3
        if i >= 1:
            hf_dev.append(dict(ctx.timings())["HF"])
            hf_e2e.append(total_ms(ctx))
            hf_wall.append(wall)
    hf = {"what": "THC Hartree-Fock J + K with the gygi term (hf_t::evaluate), FP64",
          "ms": float(np.mean(hf_dev)), "e2e_ms": float(np.mean(hf_e2e)),
          "e2e_wall_ms": float(np.mean(hf_wall)),
          "gpu_launches": int((ctx.kernel_launches() - l0) // (1 + side)),
          "h2d_bytes": int(Dm.nbytes + S_ov.nbytes),
          "d2h_bytes": int(F_hf.nbytes)}

    # the gygi treatment (head at the smallest nonzero |q| and Sigma_div_correction): the
    # iteration with the correction (it takes the plain path: the head goes through the host)
    # and the correction's own device time
    ctx.set_div_treatment("gygi", 0.5, s.chi_bar[0])
    gy = []
    for i in range(1 + side):
        ctx.gw_iteration(None, want_sigma=False)
        if i >= 1:
            gy.append(total_ms(ctx))
    ctx.set_profiling(True)
    ctx.gw_iteration(None, want_sigma=False)
    gst = ctx.kernel_stats()
    ctx.set_profiling(False)
    ctx.set_div_treatment("ignore_g0")
    gygi = {"what": "GW iteration with div_treatment gygi (Sigma_div_correction, FP64)",
            "gw_iteration_ms": float(np.mean(gy)),
            "correction_ms": float(gst.get("sigma_div", (0.0, 0))[0]),
            "eps_head_ms": float(gst.get("eps_head", (0.0, 0))[0])}

    # the dielectric head of the mixed iteration (it reads all of W) for the accuracy figures
    _, head_mixed = ctx.gw_iteration(None, want_sigma=False, want_head=True)

    # the oracle on a bounded sample at this size: the projection of G(tau = 0) for every k
    oracle_sample = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import thc_oracle as O
        got = ctx.primary_to_aux(G[:1])
        ref = O.primary_to_aux(G[:1], s.X[None])
        oracle_sample = {"what": "primary -> aux projection X G(tau_0) X^H, all k, mixed path "
                                 "against the FP64 oracle", "max_abs_diff":
                         float(np.abs(got - ref).max()), "max_abs": float(np.abs(ref).max())}
        del got, ref
    ctx.close()  # the FP64 form needs the memory

    fp64 = None
    fp64_stats = {}
    if not args.no_fp64:
        c64 = make_ctx(s, ft, capi.FP64)
        S64, head64 = c64.gw_iteration(Gh, want_head=True)
        c64.set_profiling(True)
        c64.gw_iteration(None, want_sigma=False)
        fp64_stats = c64.kernel_stats()
        c64.set_profiling(False)
        c64.gw_iteration(None, want_sigma=False)
        t64 = total_ms(c64)
        e64 = c64.rpa_energy(None)
        r64 = total_ms(c64)
        fp64 = {"what": "the same algorithm in FP64 on the library's own kernels: complex128 "
                        "storage, FP64 tensor-core (DMMA) products with the same triangular "
                        "structure, the same batched FP64 factorisation (whole inverse in FP64) "
                        "and W = L E L^H, chunks of all (q, iW) problems",
                "gw_iteration_ms": t64, "rpa_energy_ms": r64, "E_c": e64,
                "max_abs_dSigma_mixed_vs_fp64": float(np.abs(Sh - S64).max()),
                "max_abs_Sigma": float(np.abs(S64).max()),
                "max_abs_d_eps_inv_head_mixed_vs_fp64": float(np.abs(head_mixed - head64).max()),
                "abs_dE_c_mixed_vs_fp64": abs(e_c - e64),
                "speedup_gw_iteration": t64 / t_step, "speedup_rpa": r64 / t_rpa,
                "note": "the FP64 form is checked against the FP64 oracle at the 2x2x2 / 128 and "
                        "4x4x4 / 512 configurations by tests/test_gpu_configs.py"}
        c64.close()
        del S64

    # max over ranks
    t_step, t_e2e = max_over_ranks([t_step, t_e2e], world)

    # per-group achieved rates and the roofline of the dominant group
    work = algorithmic_work(w, s, ft)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    bf16 = peaks.get("bf16_tflops", 1590.0)
    fp64_tf = fp64_peak["tflops"]
    peak_src = "measured" if peaks else "fallback"
    fp64_sus = fp64_peak.get("sustained_tflops")
    groups = group_rates(stats, side, work, hbm, bf16, fp64_tf, fp64_sus, stat_units)
    if fp64_stats:
        fp64["kernel_groups_ms"] = {k: v[0] for k, v in fp64_stats.items()}
    roof = None
    cand = [(g["ms_per_step"], k) for k, g in groups.items()
            if "achieved_GBps" in g or "achieved_TFLOPs" in g]
    if cand:
        _, name = max(cand)
        g = groups[name]
        n_l = max(g["launch_groups_per_step"], 1e-9)
        per_ms = g["ms_per_step"] / n_l
        nprob = s.nk * ft.nw_half
        traffic, tsrc = profile_traffic(name, s.Np)
        if g["bound"] == "hbm":
            roof = {"kernel": name, "bound": "hbm", "achieved": g["achieved_GBps"], "peak": hbm,
                    "unit": "GB/s", "frac": g["achieved_GBps"] / hbm, "traffic": None,
                    "avg_launch_ms": per_ms, "peak_source": peak_src + " HBM copy"}
        elif g["bound"] == "fp64":
            # timed inside a long step: the sustained FP64 rate is the denominator (the
            # burst fraction is kept beside it)
            pk = fp64_sus or fp64_tf
            roof = {"kernel": name, "bound": "tensor", "pipe": "FP64 tensor cores (DMMA)",
                    "achieved": g["achieved_TFLOPs"], "peak": pk, "unit": "TFLOP/s",
                    "frac": g["achieved_TFLOPs"] / pk,
                    "frac_of_burst": g["achieved_TFLOPs"] / fp64_tf,
                    "traffic": traffic * nprob / n_l if traffic else None,
                    "traffic_source": tsrc, "avg_launch_ms": per_ms,
                    "peak_source": "measured in this run (" + ("sustained" if fp64_sus else
                                   "burst") + "): " + fp64_peak["how"]}
            # the FP64 pipe's rate scales with the SM clock: the same peak at the clock the
            # timed iterations ran at (power-capped by their tensor-core phases), as context
            it_mhz, pk_mhz = clk.summary().get("sm_mhz"), fp64_peak.get("sustained_sm_mhz")
            if it_mhz and pk_mhz:
                roof["peak_at_iteration_clock"] = pk * it_mhz / pk_mhz
                roof["frac_at_iteration_clock"] = g["achieved_TFLOPs"] / roof["peak_at_iteration_clock"]
                roof["clocks_mhz"] = {"iteration": it_mhz, "peak_measurement": pk_mhz}
        else:
            roof = {"kernel": name, "bound": "tensor", "achieved": g["achieved_TFLOPs"],
                    "peak": bf16, "unit": "TFLOP/s", "frac": g["achieved_TFLOPs"] / bf16,
                    "traffic": traffic * nprob / n_l if traffic else None,
                    "traffic_source": tsrc, "avg_launch_ms": per_ms,
                    "peak_source": peak_src + " dense bf16 cuBLAS; split-TF32 complex products "
                                   "issue 3 TF32 MMAs at half the bf16 rate per counted flop",
                    "split_tf32_ceiling": bf16 / 6.0,
                    "frac_of_split_tf32_ceiling": g["achieved_TFLOPs"] / (bf16 / 6.0)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, parts = cpu_sample(s, ft, reps=2)
        cpu = {"value": v, "unit": "ms", "cores": host_cores(), "kind": "port",
               "extrapolated": True, "sample": CPU_SAMPLE_NOTE,
               "parts_ms": {k: round(x, 1) for k, x in parts.items()}}
        # the oracle's Hartree-Fock on the same density matrix: time and full-size parity
        from oracle import thc_oracle as O
        t0 = time.perf_counter()
        F_ref = O.thc_hf(Dm, s.X, s.V, s.kpts, s.lattv, s.kp_grid, S_ov, True, True, "gygi", 0.5)
        hf["cpu_oracle_ms"] = (time.perf_counter() - t0) * 1e3
        hf["max_abs_dF_vs_oracle"] = float(np.abs(F_hf - F_ref).max())
        hf["max_abs_F"] = float(np.abs(F_ref).max())

    gbytes = G.nbytes
    line = {
        "metric": METRIC, "value": t_step / world, "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c64/f64",
        "data": "synthetic", "config": config_of(args.workload, w, s, ft),
        "e2e": {"value": t_e2e / world, "unit": "ms", "h2d_bytes_per_step": gbytes,
                "d2h_bytes_per_step": gbytes},
        "gpu_launches": int(launches),
        "rpa_energy_ms": t_rpa, "E_c": e_c, "rpa_clocks": clk_rpa.summary(),
        "fp64_form": fp64,
        "oracle_sample": oracle_sample,
        "fp64_peak_measured": fp64_peak,
        "hartree_fock": hf,
        "div_gygi": gygi,
        "phases_ms": phases,
        "steps_ms": [round(t, 3) for t in times],
        "e2e_steps_ms": [round(t, 3) for t in e2e],
        # wall clock of each public-API call (host G in, Sigma out, returns after the copy)
        "e2e_wall_steps_ms": [round(t, 3) for t in e2e_wall],
        "e2e_clocks": clk_e2e.summary(),
        "e2e_phases_ms": e2e_phases,
        "rpa_phases_ms": rpa_phases,
        "kernel_groups": groups,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def batch_molecules(n=32, seed=4040):
    """Uneven batch of Gamma-only molecules: orbitals uniform in 30..300, N_mu = 6 x orbitals,
    beta = 500, Lambda = 1e4 ("low")."""
    from coqui_b200.iaft import IAFT
    from coqui_b200.synthetic import make_system
    rng = np.random.default_rng(seed)
    nbs = rng.integers(30, 301, n)
    ft = IAFT(500.0, 20.0, "low")
    mols = [make_system(1, int(nb), int(nb) // 2, 6 * int(nb), beta=500.0, seed=seed + i,
                        gamma_only=True) for i, nb in enumerate(nbs)]
    return ft, mols


def run_batch(args, rank):
    """Fused batch of Gamma-only molecules against one single-system context per molecule."""
    from coqui_b200 import capi
    if rank != 0:
        return
    import torch
    ft, mols = batch_molecules()

    def pinned_like(a):  # page-locked host buffers, as in the single-system e2e
        h = torch.empty(a.shape, dtype=torch.complex128, pin_memory=True).numpy()
        h[...] = a
        return h
    Gs = [pinned_like(m.G0(ft)[:, 0, 0]) for m in mols]
    b = capi.Batch([m.nb for m in mols], [m.Np for m in mols], ft.nt_f, ft.nw_b)
    b.set_ir(ft)
    for i, m in enumerate(mols):
        b.set_thc(i, m.X[0, 0], m.V[0])
    out = [pinned_like(np.zeros_like(G)) for G in Gs]
    for _ in range(args.warmup):
        b.gw_iteration(Gs, out)
    dev, wall = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        b.gw_iteration(Gs, out)
        wall.append((time.perf_counter() - t0) * 1e3)
        dev.append(b.last_ms())
    b.close()
    # per molecule: the single-system context (nk = 1), one call each (skipped with
    # --only-iteration, e.g. for a launch list of the fused iteration alone)
    per, diff = 0.0, 0.0
    for m, S in zip(mols, [] if args.only_iteration else out):
        c = make_ctx(m, ft, capi.MIXED)
        G = m.G0(ft)
        for _ in range(2):
            S1, _ = c.gw_iteration(G)
        per += total_ms(c)
        diff = max(diff, float(np.abs(S1[:, 0, 0] - S).max()))
        c.close()
    line = {
        "metric": "fused GW iteration time, 32 Gamma-only molecules (mixed precision, 1 B200)",
        "value": float(np.mean(dev)), "unit": "ms", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(dev)), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64/f64", "data": "synthetic",
        "config": {"workload": "batch32_gamma", "orbitals": [m.nb for m in mols],
                   "Np": [m.Np for m in mols], "nt": ft.nt_f, "nw_b": ft.nw_b, "beta": 500.0},
        "e2e": {"value": float(np.mean(wall)), "unit": "ms",
                "h2d_bytes_per_step": int(sum(G.nbytes for G in Gs)),
                "d2h_bytes_per_step": int(sum(G.nbytes for G in Gs))},
    }
    if not args.only_iteration:
        line.update({"per_molecule_contexts_ms": per, "fused_speedup": per / float(np.mean(dev)),
                     "max_abs_diff_fused_vs_per_molecule": diff})
    print(json.dumps(line), flush=True)


def run_scgw(args, rank):
    """Self-consistent GW with the learned update (3x3x3 k, 48 orbitals, N_mu 384): the network
    is trained on the plain damped loop's trajectories of seeded training systems, then a
    held-out system is iterated in mixed precision to a 1e-6 residual (and |dE| < 1e-6 Ha) with
    plain damping, damping + network and commutator DIIS."""
    from coqui_b200 import learned
    from coqui_b200.iaft import IAFT
    from coqui_b200.synthetic import WORKLOADS, make_system
    from coqui_b200 import capi
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    ft = IAFT(w["beta"], w["lam"] / w["beta"], w["prec"])
    n_train = 16
    t0 = time.perf_counter()
    trajs = [learned.trajectory(make_system(w["n"], w["nb"], w["nocc"], w["Np"], seed=1000 + i), ft)
             for i in range(n_train)]
    t_traj = time.perf_counter() - t0
    X, T = learned.dataset(trajs)
    t0 = time.perf_counter()
    net, loss = learned.train(X, T, epochs=20)
    t_train = time.perf_counter() - t0
    s = make_system(w["n"], w["nb"], w["nocc"], w["Np"], seed=5000)
    G0 = s.G0(ft)
    c = learned.make_context(s, ft, capi.MIXED)
    runs = {}
    for name, kw in (("damping", dict()), ("damping+mlp", dict(mlp=net)),
                     ("diis", dict(alg="diis", mixing=0.2))):
        for _ in range(max(args.warmup, 0) if name == "damping" else 0):
            learned.run_loop(c, G0, max_iter=2)  # warm-up: tiles tuned, buffers allocated
        best = None
        for _ in range(max(args.steps, 1)):
            r = learned.run_loop(c, G0, tol_e=1e-6, tol_r=1e-6, **kw)
            if best is None or r["wall_s"] < best["wall_s"]:
                best = r
        runs[name] = {"iterations": best["iterations"], "gw_evaluations": best["evaluations"],
                      "wall_s": best["wall_s"], "e_tot": best["e_tot"],
                      "learned_steps": best["learned_steps"], "withdrawn": best["withdrawn"],
                      "final_residual": best["history"][-1]["residual"]}
    c.close()
    net.close()
    print(json.dumps({
        "metric": "scGW wall time to a 1e-6 residual, damping + learned update (mixed precision, "
                  "1 B200)",
        "value": runs["damping+mlp"]["wall_s"] * 1e3, "unit": "ms", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
        "dtype": "c64/f64", "data": "synthetic",
        "config": {"workload": args.workload, "nk": s.nk, "nb": s.nb, "Np": s.Np,
                   "train_systems": n_train, "train_samples": int(X.shape[0])},
        "runs": runs, "trajectories_s": t_traj, "train_s": t_train,
        "loss_first": float(loss[0]), "loss_last": float(loss[-1]),
        "max_abs_dE_between_runs": max(abs(runs[a]["e_tot"] - runs[b]["e_tot"])
                                       for a in runs for b in runs)}), flush=True)


def run_factor(args, rank):
    """The batched FP64 factorisation of the Dyson step alone (coqui_b200_factor_dielectric) on
    random Hermitian M with I - M positive definite: workload factor_np<Np>_x<problems>."""
    import torch
    from coqui_b200 import capi
    if rank != 0:
        return
    parts = args.workload.split("_")
    n, nprob = int(parts[1][2:]), int(parts[2][1:])
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(5)
    H = torch.randn((nprob, n, n), dtype=torch.complex64, device=dev, generator=g)
    M = (H + H.conj().transpose(1, 2)) * (0.15 / np.sqrt(n))
    del H
    A = torch.empty((nprob, n, n), dtype=torch.complex128, device=dev)
    ld = torch.empty(nprob, dtype=torch.float64, device=dev)
    tr = torch.empty(nprob, dtype=torch.complex128, device=dev)
    info = torch.empty(nprob, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        capi.factor_dielectric(M.data_ptr(), A.data_ptr(), ld.data_ptr(), tr.data_ptr(),
                               info.data_ptr(), n, nprob, ctypes_stream)
    import ctypes
    ctypes_stream = ctypes.c_void_p(stream.cuda_stream)
    for _ in range(args.warmup):
        step()
    times = []
    with Clocks(0) as clk:
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    assert int(info.abs().sum()) == 0
    ms = float(np.mean(times))
    g128 = min(n, 128)
    flop = 8.0 * (n ** 3 / 6 + n * g128 ** 2 / 6) * nprob
    peak = measure_fp64_peak(0)
    print(json.dumps({
        "metric": "batched FP64 factorisation of I - M (Cholesky, log det, group inverse)",
        "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "Np": n, "problems": nprob},
        "achieved_TFLOPs": flop / (ms * 1e-3) / 1e12,
        "frac_of_fp64_measured": flop / (ms * 1e-3) / 1e12 / peak["tflops"],
        "fp64_peak_measured": peak, "steps_ms": [round(t, 3) for t in times],
        "clocks": clk.summary()}), flush=True)


def run_ibz(args, rank):
    """The symmetry-reduced k-space path (coqui_b200_set_symmetry) against the full-BZ path of
    the same system: workload ibz_<trev|swap>_k<n0><n1><n2>_nb<nb>_np<Np> on seeded symmetric
    inputs (coqui_b200.symmetry.symmetric_system), beta = 1000, Lambda = 1e4 "low", mixed
    precision.  One step = one GW iteration (update_w + evaluate) through the C ABI, host G in
    and Sigma out; device time = the sum of the call's CUDA-event phases, e2e = wall clock."""
    from coqui_b200 import capi
    from coqui_b200.iaft import IAFT
    from coqui_b200.symmetry import symmetric_system
    if rank != 0:
        return
    parts = args.workload.split("_")
    kind, grid = parts[1], tuple(int(ch) for ch in parts[2][1:])
    nb, Np = int(parts[3][2:]), int(parts[4][2:])
    ft = IAFT(1000.0, 10.0, "low")
    d = symmetric_system(kind, grid, nb, Np, ft, seed=11)
    sym = d["sym"]
    c = capi.Context(sym["nk"], nb, Np, ft.nt_f, ft.nw_b, grid, mode=capi.MIXED)
    c.set_ir(ft)
    c.set_kmesh(d["kpts_lex"], d["lattv"])
    c.set_thc(d["X_lex"], d["V_lex"])

    def timed(G):
        for _ in range(max(args.warmup, 1)):
            c.gw_iteration(G)
        dev, wall, l0 = [], [], c.kernel_launches()
        for _ in range(max(args.steps, 1)):
            t0 = time.perf_counter()
            S, _ = c.gw_iteration(G)
            wall.append((time.perf_counter() - t0) * 1e3)
            dev.append(sum(ms for _, ms in c.timings()))
        return S, float(np.median(dev)), float(np.median(wall)), \
            (c.kernel_launches() - l0) // max(args.steps, 1)

    with Clocks(0) as clk:
        S_full, dev_full, wall_full, n_full = timed(d["G_lex"])
        e_full = c.rpa_energy(d["G_lex"])
        c.set_symmetry(sym, d["D"])
        S_ibz, dev_ibz, wall_ibz, n_ibz = timed(d["G_ibz"])
        e_ibz = c.rpa_energy(d["G_ibz"])
    kl = d["lex"][:sym["nk_ibz"]]
    out = {
        "metric": "GW iteration time on the IBZ k-space path (mixed precision, 1 B200)",
        "value": dev_ibz, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ibz, "higher_is_better": False, "dtype": "c64/f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "symmetry": kind, "kp_grid": list(grid),
                   "nk": sym["nk"], "nk_ibz": sym["nk_ibz"], "nq_ibz": sym["nq_ibz"],
                   "nsym": int(len(sym["qsymms"])), "nb": nb, "Np": Np, "nt": ft.nt_f,
                   "nw_b": ft.nw_b},
        "e2e": {"value": wall_ibz, "unit": "ms"},
        "full_bz": {"device_ms": dev_full, "e2e_ms": wall_full, "gpu_launches": n_full},
        "gpu_launches": n_ibz, "speedup_vs_full_bz": dev_full / dev_ibz,
        "e_rpa_ibz": e_ibz, "e_rpa_full": e_full, "abs_dE_rpa": abs(e_ibz - e_full),
        "clocks": clk.summary()}
    if kind == "trev":  # with time reversal both routes give the same self-energy
        out["max_abs_dSigma_vs_full_bz"] = float(np.abs(S_ibz - S_full[:, :, kl]).max())
    c.close()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload.startswith("ibz_"):
        run_ibz(args, rank)
        return
    if args.workload.startswith("batch"):
        run_batch(args, rank)
        return
    if args.workload.startswith("factor_"):
        run_factor(args, rank)
        return
    if args.workload.startswith("scgw"):
        run_scgw(args, rank)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
