#!/usr/bin/env python
"""VMC-iteration benchmark on B200: MinSR iteration over persistent walkers (configuration 2:
N=16 electrons, 4096 walkers, width 64, 4 blocks, K=4 determinants, RBF Jastrow, Ewald Coulomb).

One step = 10 Metropolis sweeps (1 joint move + 2 spin flips per sweep) + forward-Laplacian local
energies with the Ewald term + the per-sample Jacobian + the median-MAD clip + the MinSR update.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config 1|2]

Rank 0 prints ONE JSON line. The headline `value` is VMC iterations/s of the mixed-precision
path (float32 network, float32 O, BF16 tcgen05 Gram, float64 determinants / Cholesky / energies);
the plain float64 GPU path is timed in the same run for the mixed-vs-fp64 comparison. With N>1
every rank runs an independent replica (the path's only cross-walker coupling, the MinSR Gram,
is solved per GPU), so value = N x per-replica iterations / max-over-ranks time ("weak").
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "continuum-nqs_b200"))

import torch  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--walkers", type=int, default=None)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU sample work")
    ap.add_argument("--bf16-steps", type=int, default=2)
    ap.add_argument("--no-bf16", action="store_true",
                    help="skip the BF16-operand network variant")
    ap.add_argument("--trajectory", type=int, default=5,
                    help="iterations of the mixed-vs-float64 trajectory comparison (0: skip)")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.index), "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][2]), "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows), "reasons": reasons}


# ---------------------------------------------------------------------------------------------
# algorithmic work (flops) of one iteration, for the roofline
# ---------------------------------------------------------------------------------------------
def gram_flops(W, P):
    """Lower-triangular SYRK of the 2W x P Jacobian: (2W)(2W+1) P flops (never the mirror)."""
    n = 2 * W
    return n * (n + 1) * P


def forward_flops(model):
    N, d, H, K, F = model.n_elec, model.embed_dim, model.n_heads, model.n_dets, 4 * model.n_freq + 2
    D = model.ff_mult * d
    g = 2 * N * F * d + model.depth * (2 * N * d * 3 * d + 2 * N * d * d + 2 * N * d * D + 2 * N * D * d
                                       + 4 * N * N * d)
    g += 4 * N * d * K * N + 8 * N ** 3 + K * (8 * N ** 3) // 3
    return g


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------
def max_over_ranks(value, device=None):
    """The largest `value` over the ranks of the default process group (the value itself without
    one): every rank reports the slowest rank's step time."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist = torch.distributed
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(ms_max, world):
    """Whole-job VMC iterations per second: each of the `world` ranks runs one replica, and the
    job's step takes the slowest rank's time."""
    return world * 1000.0 / ms_max


def run_ours(a, rank, world):
    from nqs import _lib
    from nqs.configs import config
    from nqs.ewald import make_ewald
    from nqs.minsr import VMCIteration
    from nqs.sampler import init_walkers_uniform

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    model, params, su = config(a.config, a.walkers)
    theta = model.theta(params)
    R0, S0 = init_walkers_uniform(1234 + rank, su.n_walkers, su.N, su.L)
    _, _, coul = make_ewald(su.L, alpha=1.0, ewald_alpha=su.ewald_eta, n_real=su.n_real,
                            n_recip=su.n_recip)
    common = dict(m_star=1.0, lambda_r=su.lambda_r, h_z=su.h_z, coulomb=coul, lr=su.lr,
                  lam=su.lam, n_sweeps=su.n_sweeps, step_size=su.step, clip_k=5.0, seed=7 + rank,
                  checkpoint_blocks=su.checkpoint_blocks)
    it = VMCIteration(model, theta, R0, S0, precision="mixed", gram="bf16", **common)
    it.sample(40)  # thermalise once before timing
    torch.cuda.synchronize()
    L = _lib.lib()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # the clock sampler starts before the warm-up steps, so that its start-up (a process launch
    # competing for the host) does not fall into the timed steps; it samples through them
    clocks = Clocks(dev.index)
    clocks.start()
    for _ in range(a.warmup):
        it.step()
    torch.cuda.synchronize()
    # ------------------------------------------------ timed region (device time, events)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(a.steps)]
    for e0_, e1_ in gev:  # create the CUDA events now; the library re-records them
        e0_.record()
        e1_.record()
    launches0 = L.nqs_kernel_launches()
    L.nqs_profile_gemm_read(None, None, None)  # clear
    L.nqs_profile_block_read(None, None, None, None)
    barrier()
    torch.cuda.synchronize()
    L.nqs_profile_gemm(1)  # event pair around every tensor-core row GEMM launch of the timed steps
    torch.cuda.nvtx.range_push("timed")  # lets ncu --nvtx-include "timed/" select these launches
    ev[0].record()
    for k in range(a.steps):
        # events recorded on the stream right before / after the Gram kernel of this step
        L.nqs_profile_events(gev[k][0].cuda_event, gev[k][1].cuda_event)
        it.step()
    ev[1].record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    L.nqs_profile_gemm(0)
    L.nqs_profile_events(None, None)
    g_ms_c, g_bytes_c, g_n_c = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
    _lib.check(L.nqs_profile_gemm_read(ctypes.byref(g_ms_c), ctypes.byref(g_bytes_c),
                                       ctypes.byref(g_n_c)), "nqs_profile_gemm_read")
    gemm_prof = (g_ms_c.value, g_bytes_c.value, g_n_c.value)
    b_ms_c, b_bytes_c, b_flops_c, b_n_c = (ctypes.c_double(), ctypes.c_double(), ctypes.c_double(),
                                           ctypes.c_longlong())
    _lib.check(L.nqs_profile_block_read(ctypes.byref(b_ms_c), ctypes.byref(b_bytes_c),
                                        ctypes.byref(b_flops_c), ctypes.byref(b_n_c)),
               "nqs_profile_block_read")
    block_prof = (b_ms_c.value, b_bytes_c.value, b_flops_c.value, b_n_c.value)
    gram_ms = [g0.elapsed_time(g1) for g0, g1 in gev]
    barrier()
    clk = clocks.stop()
    launches = (L.nqs_kernel_launches() - launches0) // a.steps
    ms = max_over_ranks(ev[0].elapsed_time(ev[1]) / a.steps, dev)
    # ------------------------------------------------ phase breakdown (one extra step)
    pe = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    pe[0].record()
    it.sample()
    pe[1].record()
    it.energies()
    pe[2].record()
    it.jacobian()
    pe[3].record()
    it.update()
    pe[4].record()
    torch.cuda.synchronize()
    phases = {k: pe[i].elapsed_time(pe[i + 1]) for i, k in
              enumerate(["sample_ms", "local_energy_ms", "jacobian_ms", "minsr_ms"])}
    stats = it.stats.cpu().tolist()
    # ------------------------------------------------ end to end through host buffers
    e2e = None
    if a.steps > 0:
        Rh = it.R.cpu().pin_memory()
        Sh = it.S.cpu().pin_memory()
        Th = it.theta.cpu().pin_memory()
        st_h = torch.empty(5, dtype=torch.float64).pin_memory()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            it.R.copy_(Rh, non_blocking=True)
            it.S.copy_(Sh, non_blocking=True)
            it.theta.copy_(Th, non_blocking=True)
            it.step()
            Th.copy_(it.theta, non_blocking=True)
            Rh.copy_(it.R, non_blocking=True)
            Sh.copy_(it.S, non_blocking=True)
            st_h.copy_(it.stats, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / a.steps, dev)
        h2d = Rh.numel() * 8 + Sh.numel() * 4 + Th.numel() * 8
        d2h = h2d + 5 * 8
        e2e = {"value": job_throughput(e2e_ms, world), "unit": "VMC iter/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms}
    # ------------------------------------------------ plain float64 GPU path + accuracy gates
    fp64 = None
    acc = None
    bf16net = None
    if not a.no_fp64 and a.fp64_steps > 0:
        from nqs.minsr import minsr_step
        # accuracy of the mixed paths against float64 on identical walkers and parameters, all
        # solved at the configured damping lam; one Jacobian resident at a time (configuration
        # 5's float64 Jacobian alone is 118 GB)
        def mixed_direction(r):
            r.energies()
            e_r = r.e.clone()
            r.jacobian()
            dl = torch.zeros(1, dtype=torch.float64, device=dev)
            inf_ = torch.zeros(5, dtype=torch.int32, device=dev)
            d_r = minsr_step(r.O, e_r, su.lam, "bf16", n_refine=r.n_refine, damping_out=dl,
                             info=inf_)
            r.release_jacobian()
            torch.cuda.empty_cache()
            return e_r.real.double(), d_r, float(dl.item()), inf_.tolist()

        em, d_mixed, dshift, inf = mixed_direction(it)
        itb = None
        if not a.no_bf16:
            itb = VMCIteration(model, it.theta, it.R, it.S, precision="mixed_bf16", **common)
            eb, d_bf, _, infb = mixed_direction(itb)
        it64 = VMCIteration(model, it.theta, it.R, it.S, precision="fp64", **common)
        it64.energies()
        e64 = it64.e.real.double()
        it64.jacobian()
        d_64 = minsr_step(it64.O, it64.e, su.lam, "fp64")
        n64 = float(d_64.norm())

        def gates(e_r, d_r, inf_):
            return {"dE_per_electron": float((e_r.mean() - e64.mean()).abs()) / su.N,
                    "dE_target": 1e-4,
                    "dvar_rel": float((e_r.var() - e64.var()).abs() / e64.var()),
                    "dvar_target": 0.05,
                    "lam": su.lam,
                    "dtheta_rel_vs_fp64_lam": float((d_r - d_64).norm()) / n64,
                    "dtheta_cos_vs_fp64_lam": float((d_r * d_64).sum()) / (float(d_r.norm()) * n64),
                    "dtheta_target": 1e-2,
                    "pcg_iterations": inf_[3],
                    "pcg_stop": ["limit", "converged", "breakdown"][inf_[4]]}

        acc = gates(em, d_mixed, inf)
        acc.update(bf16_preconditioner_shift=dshift, E_fp64=float(e64.mean()),
                   E_mixed=float(em.mean()))
        if itb is not None:
            acc_bf = gates(eb, d_bf, infb)
            acc_bf["E_mixed_bf16"] = float(eb.mean())
        it64.step()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(a.fp64_steps):
            it64.step()
        f1.record()
        torch.cuda.synchronize()
        ms64 = f0.elapsed_time(f1) / a.fp64_steps
        fp64 = {"ms_per_step": ms64, "VMC_iter_per_s": 1000.0 / ms64,
                "mixed_speedup": ms64 / ms, "E": float(it64.stats[0])}
        del it64
        torch.cuda.empty_cache()
        if itb is not None:
            # the same iteration with BF16 operands in the network's Dense layers (TF32 is the
            # headline's comparison precision)
            itb.step()
            torch.cuda.synchronize()
            b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b0.record()
            for _ in range(a.bf16_steps):
                itb.step()
            b1.record()
            torch.cuda.synchronize()
            msb = b0.elapsed_time(b1) / a.bf16_steps
            bf16net = {"ms_per_step": msb, "VMC_iter_per_s": 1000.0 / msb,
                       "speedup_vs_fp64": ms64 / msb, "accuracy_vs_fp64": acc_bf,
                       "network": "Dense layers with BF16 operands on tcgen05 kind::f16 "
                                  "(float32 accumulation); the rest as the mixed path"}
            del itb
            torch.cuda.empty_cache()

    traj = None
    if not a.no_fp64 and a.trajectory > 0:
        if 2 * su.n_walkers * it.P * 12 < 100e9:  # both runs' Jacobians resident at once
            traj = trajectories(model, it, common, a.trajectory, su)
        else:
            traj = {"skipped": "the two runs' Jacobians (float32 + float64) do not fit together"}
    # ------------------------------------------------ roofline of the dominant kernel: the
    # tensor-core row GEMMs of the network (HBM-bound), timed per launch over the timed steps
    peaks, src = load_peaks()
    t_ms, t_bytes, t_n = gemm_prof
    per_launch_bytes = t_bytes / max(t_n, 1)
    per_launch_ms = t_ms / max(t_n, 1)
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9 if t_n else float("nan")
    hbm = peaks.get("hbm_gbs", 6650.0)
    ratio = traffic_ratio()
    roof = {"kernel": "k_rowgemm_tc (persistent tcgen05 TF32 row GEMMs of the network)",
            "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_source": f"{src} (HBM copy)",
            "traffic": per_launch_bytes * ratio if ratio else None,
            "algorithmic_bytes_per_launch": per_launch_bytes, "avg_launch_ms": per_launch_ms,
            "launches_per_step": t_n / a.steps, "share_of_step": t_ms / a.steps / ms,
            "traffic_source": "ncu DRAM bytes / algorithmic bytes of all row-GEMM launches of one "
                              "timed step at W = 1024 (profiles/rowgemm_traffic.json), times "
                              "this run's algorithmic bytes per launch" if ratio else None}
    # the fused value-pass transformer blocks: bytes in/out + weights against HBM, with their
    # tensor-core + attention flops alongside
    b_ms, b_bytes, b_flops, b_n = block_prof
    roof_blk = None
    if b_n:
        bl_ms, bl_bytes = b_ms / b_n, b_bytes / b_n
        b_ach = bl_bytes / (bl_ms * 1e-3) / 1e9
        roof_blk = {"kernel": "k_block_value_tc (one transformer block of the value passes per "
                              "launch: LN, QKV, attention, projection, MLP; tcgen05 TF32)",
                    "bound": "hbm", "achieved": b_ach, "peak": hbm, "unit": "GB/s",
                    "frac": b_ach / hbm, "peak_source": f"{src} (HBM copy)", "traffic": None,
                    "algorithmic_bytes_per_launch": bl_bytes, "avg_launch_ms": bl_ms,
                    "flops_per_launch": b_flops / b_n,
                    "achieved_tflops": b_flops / b_n / (bl_ms * 1e-3) / 1e12,
                    "launches_per_step": b_n / a.steps, "share_of_step": b_ms / a.steps / ms,
                    "note": "latency-bound: per-row CUDA-core work (attention, LayerNorm, GELU) "
                            "between MMA round trips, 8 warps per SM"}
    # the dominant kernel of the step (larger share of the timed region) is the headline roofline
    roof_other = None
    if roof_blk and roof_blk["share_of_step"] > roof["share_of_step"]:
        roof, roof_other = roof_blk, roof
    else:
        roof_other = roof_blk
    # the MinSR Gram on the tensor cores, for reference
    gflop = gram_flops(su.n_walkers, it.P)
    g_ms = sorted(gram_ms)[len(gram_ms) // 2] if gram_ms else float("nan")
    g_ach = gflop / (g_ms * 1e-3) / 1e12
    # timed inside a long step: against the sustained (power-capped) BF16 figure, burst beside it
    g_peak = peaks.get("bf16_tflops_sustained", 1400.0)
    g_burst = peaks.get("bf16_tflops", 1590.0)
    roof_gram = {"kernel": "k_gram_tc_wide<bf16> (tcgen05 SYRK of the 2W x P Jacobian, 256 x 256 "
                           "tiles, two TMEM accumulators per CTA)",
                 "bound": "tensor", "achieved": g_ach, "peak": g_peak, "unit": "TFLOP/s",
                 "frac": g_ach / g_peak, "peak_source": f"{src} (sustained bf16)",
                 "frac_of_burst": g_ach / g_burst, "gram_ms": g_ms, "algorithmic_flops": gflop}
    return dict(ms=ms, phases=phases, stats=stats, e2e=e2e, fp64=fp64, roofline=roof,
                roofline_second=roof_other, roofline_gram=roof_gram, clocks=clk,
                launches=launches, su=su, model=model, P=it.P, acc=acc, traj=traj,
                bf16net=bf16net)


def trajectories(model, it, common, n_iter, su):
    """n_iter VMC iterations of the mixed path and of the all-float64 path, interleaved, from the
    same theta, walkers and random stream (seed, counter). Per iteration: |dE|/N and its
    statistical error sqrt(err_mixed^2 + err_fp64^2)/N, the relative difference of var(E_loc),
    the relative difference of theta, and how many walkers' configurations differ between the
    two runs (an accept decision that flips with the precision moves that walker onto its own
    chain; beyond that point the two energies are no longer paired samples)."""
    from nqs.minsr import VMCIteration
    st = it.state_dict()
    runs = {}
    for prec in ("mixed", "fp64"):
        r = VMCIteration(model, st["theta"], st["R"], st["S"], precision=prec, **common)
        r.load_state_dict(st)
        runs[prec] = r
    out = {k: [] for k in ("dE_per_electron", "dE_err_per_electron", "dvar_rel", "dtheta_rel",
                           "walkers_differing", "E_mixed", "E_fp64")}
    for _ in range(n_iter):
        for r in runs.values():
            r.step()
        m, f = runs["mixed"], runs["fp64"]
        sm, sf = m.stats.cpu().tolist(), f.stats.cpu().tolist()
        out["E_mixed"].append(sm[0])
        out["E_fp64"].append(sf[0])
        out["dE_per_electron"].append(abs(sm[0] - sf[0]) / su.N)
        out["dE_err_per_electron"].append(math.sqrt(sm[1] ** 2 + sf[1] ** 2) / su.N)
        out["dvar_rel"].append(abs(sm[2] - sf[2]) / sf[2])
        out["dtheta_rel"].append(float((m.theta - f.theta).norm() / f.theta.norm()))
        diff = ((m.R - f.R).abs().amax(dim=(1, 2)) > 1e-9) | (m.S != f.S).any(dim=1)
        out["walkers_differing"].append(int(diff.sum()))
    del runs
    out.update(iterations=n_iter, max_dE_per_electron=max(out["dE_per_electron"]),
               max_dvar_rel=max(out["dvar_rel"]))
    return out


def traffic_ratio():
    """DRAM bytes per algorithmic byte of the row-GEMM launches from an ncu capture of one timed
    step (profiles/rowgemm_traffic.json, key dram_bytes_per_algorithmic_byte), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "rowgemm_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_algorithmic_byte"])
    except (OSError, ValueError, KeyError):
        return None


# ---------------------------------------------------------------------------------------------
# CPU baseline: whole iterations of the float64 oracle port, measured at a few walker counts
# ---------------------------------------------------------------------------------------------
def workload_config(su, P):
    """The `config` object both arms print (same workload, same keys)."""
    return {"workload": f"{su.name}: N={su.N}, W={su.n_walkers}, P={P}; {su.n_sweeps} sweeps + "
                        "local energies with Ewald + per-sample Jacobian + median-MAD clip + "
                        "MinSR update",
            "walkers": su.n_walkers, "electrons": su.N, "params": P}


class CpuIteration:
    """The reference algorithm on the host (oracle port: float64 torch on the CPU, all host
    threads): whole VMC iterations (sweeps with log psi recomputed per proposal, dense-Hessian
    local energies, Ewald, reverse-mode per-sample Jacobian, clip, explicit Gram + LU solve,
    update) at a small walker count, and the explicit Gram / LU rates at the full size."""

    def __init__(self, cfg, walkers=None):
        sys.path.insert(0, ROOT)
        import numpy as np
        from oracle import nqs_oracle as O
        from nqs.configs import config
        torch.set_num_threads(os.cpu_count() or 1)
        self.O, self.np = O, np
        self.model, self.params, self.su = config(cfg, walkers)
        self.theta, self.unravel = O.real_ravel(self.params["params"])
        self.P = int(self.theta.shape[0])
        self.ew = O.Ewald(self.su.L, 1.0, self.su.ewald_eta, self.su.n_real, self.su.n_recip)
        self.rng = np.random.default_rng(0)

    def iteration(self, W):
        """Seconds of one whole oracle iteration over W walkers."""
        su = self.su
        R = torch.as_tensor(self.rng.uniform(0, su.L, (W, su.N, 2)))
        S = torch.as_tensor(self.rng.integers(0, 2, (W, su.N)))
        t0 = time.perf_counter()
        self.O.vmc_iteration(self.model, self.theta, self.unravel, R, S, A=su.L, step=su.step,
                             n_sweeps=su.n_sweeps, n_spin_flips=2, rng=self.rng, m_star=1.0,
                             lambda_r=su.lambda_r, h_z=su.h_z, ewald=self.ew, lam=su.lam,
                             lr=su.lr, clip_k=5.0)
        return time.perf_counter() - t0

    def rates(self):
        """FLOP/s of the explicit Gram (2 n^2 P, sampled at 512 rows) and the LU solve
        ((2/3) n^3, sampled at n = 2048), the two steps whose cost grows faster than W."""
        n_full = 2 * self.su.n_walkers
        m = min(n_full, 512)
        A = torch.randn(m, self.P, dtype=torch.float64)
        A @ A.T
        t0 = time.perf_counter()
        A @ A.T
        gemm = 2.0 * m * m * self.P / (time.perf_counter() - t0)
        n = min(n_full, 2048)
        T = torch.randn(n, n, dtype=torch.float64)
        T = T @ T.T + n * torch.eye(n, dtype=torch.float64)
        rhs = torch.randn(n, dtype=torch.float64)
        torch.linalg.solve(T, rhs)
        t0 = time.perf_counter()
        torch.linalg.solve(T, rhs)
        lu = (2.0 / 3.0) * n ** 3 / (time.perf_counter() - t0)
        return gemm, lu

    def model_full(self, samples, gemm, lu):
        """Seconds per full iteration: the mean measured time when the samples ran at the full
        walker count; otherwise t(W) = a + b W fitted to the measured whole iterations (least
        squares) plus the Gram and LU of the full 2W system at the measured rates."""
        Ws = [w for w, _ in samples]
        ts = [t for _, t in samples]
        W = self.su.n_walkers
        if set(Ws) == {W}:
            t = sum(ts) / len(ts)
            return t, 0.0, t / W
        if len(set(Ws)) > 1:
            n = len(Ws)
            mw, mt = sum(Ws) / n, sum(ts) / n
            b = sum((w - mw) * (t - mt) for w, t in samples) / sum((w - mw) ** 2 for w in Ws)
            a = mt - b * mw
        else:
            a, b = 0.0, ts[0] / Ws[0]
        n2 = 2 * W
        t = a + b * W + 2.0 * n2 * n2 * self.P / gemm + (2.0 / 3.0) * n2 ** 3 / lu
        return t, a, b

    def describe(self, samples, a, b, gemm, lu, t_full):
        Ws = sorted({w for w, _ in samples})
        if Ws == [self.su.n_walkers]:
            return (f"float64 oracle port (torch CPU, {torch.get_num_threads()} threads), whole "
                    f"iterations at the configuration's W = {Ws[0]} measured end to end "
                    f"({len(samples)} runs): {t_full:.1f} s per iteration")
        return (f"float64 oracle port (torch CPU, {torch.get_num_threads()} threads), whole "
                f"iterations measured at W = {Ws} ({len(samples)} runs, "
                f"{1e3 * sum(t for _, t in samples) / len(samples):.0f} ms mean), fitted "
                f"t = a + b W (a = {a:.3f} s, b = {b:.4f} s/walker); plus the explicit Gram "
                f"2(2W)^2 P at {gemm / 1e9:.0f} GFLOP/s and the LU (2/3)(2W)^3 at {lu / 1e9:.0f} "
                f"GFLOP/s measured here: {t_full:.0f} s per iteration at W = {self.su.n_walkers}")


def sample_walkers(cpu, budget_s):
    """Walker counts for the timed whole iterations: the configuration's own W when one whole
    iteration fits in budget_s, else 1, 2, 4, ... while one iteration stays within about
    budget_s / 4 (at least two distinct counts)."""
    cpu.iteration(1)  # builds the torch.func transforms
    t1 = cpu.iteration(1)
    if cpu.su.n_walkers * t1 <= budget_s:
        return [cpu.su.n_walkers]
    Ws, w = [1], 2
    while (len(Ws) < 2 or w * t1 <= budget_s / 4) and w <= cpu.su.n_walkers:
        Ws.append(w)
        w *= 2
    return Ws


def cpu_baseline(cfg, budget_s, walkers=None):
    """(iter/s, description, threads) of the reference algorithm on the host cores."""
    cpu = CpuIteration(cfg, walkers)
    Ws = sample_walkers(cpu, budget_s)
    samples = [(w, cpu.iteration(w)) for w in Ws]
    gemm, lu = cpu.rates()
    t_full, a, b = cpu.model_full(samples, gemm, lu)
    return 1.0 / t_full, cpu.describe(samples, a, b, gemm, lu, t_full), torch.get_num_threads()


def run_reference(a):
    """The reference arm: the reference algorithm (the float64 oracle port: the reference's own
    JAX code cannot be installed on this image) on the host cores. Each step is one whole
    iteration at a small walker count (cycling through the sample counts), so ms_per_step is a
    measured time; value is the full configuration's iterations/s from the fit."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    cpu = CpuIteration(a.config, a.walkers)
    Ws = sample_walkers(cpu, a.cpu_budget)
    samples = []
    for i in range(a.warmup + a.steps):
        w = Ws[i % len(Ws)]
        t = cpu.iteration(w)
        if i >= a.warmup:
            samples.append((w, t))
    gemm, lu = cpu.rates()
    t_full, ca, cb = cpu.model_full(samples, gemm, lu)
    v = 1.0 / t_full
    ms = 1e3 * sum(t for _, t in samples) / max(len(samples), 1)
    desc = cpu.describe(samples, ca, cb, gemm, lu, t_full)
    line = {"impl": "reference", "metric": "VMC iter/s", "value": v, "unit": "VMC iter/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "ms_per_step_note": "measured whole oracle iterations at the sample walker counts",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(cpu.su, cpu.P),
            "cpu_baseline": {"value": v, "unit": "VMC iter/s", "cores": torch.get_num_threads(),
                             "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": "VMC iter/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_multi(a, rank, world):
    """Configuration 4: 64 independent VMC instances (electron counts 6..26, walkers 512..4096,
    their own r_s, Rashba and Zeeman) advanced together; one step = one VMC iteration of every
    instance, captured once as a CUDA graph (knobs per (N, W) bucket from the autotuner)."""
    from nqs import _lib
    from nqs.batched import MultiVMC, tuning_table, walker_steps
    from nqs.configs import config4_instances
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    inst = config4_instances(64, seed=rank)
    t0 = time.perf_counter()
    mv = MultiVMC(inst, precision="mixed", use_graph=True)
    for it in mv.its:
        it.sample(20)  # thermalise once
    rep = mv.autotune()
    t_tune = time.perf_counter() - t0
    L = _lib.lib()
    c0 = L.nqs_kernel_launches()
    mv.capture(warmup=1)  # one eager step + the captured one: the kernels of a step, twice
    per_step_kernels = (L.nqs_kernel_launches() - c0) // 2
    clocks = Clocks(dev.index)
    clocks.start()  # before the warm-up steps: its start-up stays out of the timed steps
    for _ in range(max(0, a.warmup - 1)):
        mv.step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        mv.step()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / a.steps, dev)
    # end to end: every instance's walkers and theta from pinned host memory before the step,
    # and back (with the energy statistics) after it
    hs = [(it.R.cpu().pin_memory(), it.S.cpu().pin_memory(), it.theta.cpu().pin_memory(),
           torch.empty(5, dtype=torch.float64).pin_memory()) for it in mv.its]
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(a.steps):
        for it, (Rh, Sh, Th, _) in zip(mv.its, hs):
            it.R.copy_(Rh, non_blocking=True)
            it.S.copy_(Sh, non_blocking=True)
            it.theta.copy_(Th, non_blocking=True)
        mv.step()
        for it, (Rh, Sh, Th, sth) in zip(mv.its, hs):
            Rh.copy_(it.R, non_blocking=True)
            Sh.copy_(it.S, non_blocking=True)
            Th.copy_(it.theta, non_blocking=True)
            sth.copy_(it.stats, non_blocking=True)
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1) / a.steps, dev)
    h2d = sum(Rh.numel() * 8 + Sh.numel() * 4 + Th.numel() * 8 for Rh, Sh, Th, _ in hs)
    wsteps = walker_steps(mv.its)
    line = {
        "metric": "VMC iter/s", "value": job_throughput(ms, world), "unit": "VMC iter/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/bf16+f64",
        "data": "synthetic (seeded uniform walkers, N(0,0.02^2) weights)",
        "config": {"workload": "config4: 64 independent VMC instances, N in {6..26}, W in "
                               "{512..4096}, width 64, 3 blocks, K=2; one step = one iteration "
                               "of every instance (one CUDA graph launch)",
                   "instances": len(mv.its), "walkers": sum(it.W for it in mv.its),
                   "electrons": [it.N for it in mv.its]},
        "walker_steps_per_s": world * wsteps / (ms * 1e-3),
        "instances": [{"N": it.N, "W": it.W, "E": float(it.stats[0])} for it in mv.its],
        "autotune": {"table": tuning_table(rep), "seconds": t_tune},
        "e2e": {"value": job_throughput(e2e_ms, world), "unit": "VMC iter/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d + 40 * len(hs),
                "ms_per_step": e2e_ms},
        "clocks": clk, "gpu_launches": int(per_step_kernels),
        "gpu_launches_note": "kernels of one step (counted while it was enqueued for capture); "
                             "each timed step replays them as one CUDA graph launch",
    }
    return line


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    world = int(os.environ.get("WORLD_SIZE", 1))
    rank = int(os.environ.get("RANK", 0))
    if world > 1:
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if a.config == 4:
        line = run_multi(a, rank, world)
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    r = run_ours(a, rank, world)
    su = r["su"]
    cpu = None
    if rank == 0 and not a.no_cpu:
        try:
            v, desc, cores = cpu_baseline(a.config, a.cpu_budget, a.walkers)
            cpu = {"value": v, "unit": "VMC iter/s", "cores": cores, "kind": "port", "sample": desc}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "VMC iter/s", "cores": None, "kind": "port",
                   "sample": f"failed: {e}"}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    ms = r["ms"]
    ph = r["phases"]
    W = su.n_walkers
    line = {
        "metric": "VMC iter/s", "value": job_throughput(ms, world), "unit": "VMC iter/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/bf16+f64",
        "data": "synthetic (seeded uniform walkers, N(0,0.02^2) weights)",
        "config": workload_config(su, r["P"]),
        "precision": {"network": "float32, Dense GEMMs tcgen05 TF32", "gram": "bf16 tcgen05",
                      "determinants / Cholesky / energies": "float64"},
        "l2": f"working set (O: 2W x P f32 = {2 * W * r['P'] * 4 / 1e9:.1f} GB) exceeds L2 "
              "every step",
        "parallelism": f"{world} independent replicas",
        "walker_steps_per_s": world * W * su.n_sweeps / (ph["sample_ms"] * 1e-3),
        "eloc_evals_per_s": world * W / (ph["local_energy_ms"] * 1e-3),
        "phases_ms": ph, "energy": {"mean": r["stats"][0], "err": r["stats"][1],
                                    "var": r["stats"][2]},
        "fp64_plain": r["fp64"], "accuracy_vs_fp64": r["acc"], "bf16_network": r["bf16net"],
        "trajectory_vs_fp64": r["traj"],
        "roofline": r["roofline"],
        "roofline_second": r["roofline_second"], "roofline_gram": r["roofline_gram"],
        "cpu_baseline": cpu,
        "e2e": r["e2e"], "clocks": r["clocks"], "gpu_launches": int(r["launches"]),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
