"""Benchmark: QG 1.5-layer RK3-SSP step (WENO5 + beta + DST Helmholtz), FP32, 2048^2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 2048]

One "step" = one rk3_ssp_step of the QG PV tendency on a 2048^2 interior
(2050^2 with the ghost ring), periodic q, DST (Dirichlet) psi with
lambda = 1/Ld^2 (Ld = 40 km), beta = 1.7e-11, Lx = Ly = 5.12e6 m, WENO5,
dt at CFL 0.5 for max|u| = 1 m/s.  Metric: Mcell-steps/s = interior cells x
steps / s / 1e6 (whole job, all ranks).  Inputs: seeded k^-3 Gaussian PV
field (std 1e-5 s^-1), synthetic.

* value: device time (CUDA events on the launching stream) of K steps, each
  replayed from a CUDA graph; L2 flushed (256 MiB write) before every step,
  outside the timed events; max over ranks.
* e2e: the same step through the public API (``QGPipeline``, a stream of
  host-resident states): every step uploads its state from pinned host
  memory, steps it and downloads q_{n+1}, all inside the timed region; the
  upload of state k+1 and the download of state k-1 overlap the step of
  state k on separate streams.
* roofline: the dominant kernel is the tcgen05 DST GEMM (one of the four
  products per solve); achieved = algorithmic 2*M*N*K flops per launch /
  its device time per launch (per_launch_ms), vs the measured bf16 peak.
* cpu_baseline: the FP64 NumPy oracle's QG step on this host.
* --impl reference: the reference's CPU implementation of the path
  (finitevolX's JAX stack is not installable here; the oracle port restates
  it) on the same config, one bounded sample per step.

Multi-GPU (--gpus N under torchrun): the single-field step does not shard;
each rank runs an independent replica ("replicas only"), value sums ranks.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LX = 5.12e6
BETA = 1.7e-11
LD = 4.0e4
METRIC = "QG RK3 Mcell-steps/s"
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--method", default="weno5")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-helmholtz", action="store_true")
    ap.add_argument("--helm-n", type=int, default=1024)
    ap.add_argument("--helm-pairs", type=int, default=20000)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="only the warm-up and timed QG steps (for ncu launch lists); no extra sections")
    ap.add_argument("--ens-steps", type=int, default=100)
    ap.add_argument("--stage-tile", default=None, help="fix the stage tile (e.g. 64x32) instead of autotuning")
    return ap.parse_args()


def config(n, method):
    return {"workload": f"qg1.5_rk3ssp_{method}_dst_{n}x{n}_fp32", "interior": [n, n], "scheme": method,
            "helmholtz": "DST-I dense GEMMs, 3xBF16 split, FP32 accumulate", "bc": "periodic q, Dirichlet psi",
            "lambda": 1.0 / LD ** 2, "beta": BETA, "dt": 0.5 * LX / n, "l2": "flushed (256 MiB write) before every step",
            "parallelism": "replicas"}


def initial_q(n, seed=0):
    import numpy as np
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n, n))
    ky = np.fft.fftfreq(n)[:, None]
    kx = np.fft.rfftfreq(n)[None, :]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = np.inf
    f = np.fft.irfft2(np.fft.rfft2(w) * k ** -1.5, s=(n, n))
    f = (f - f.mean()) * (1e-5 / f.std())
    q = np.zeros((n + 2, n + 2))
    q[1:-1, 1:-1] = f
    q[0, :], q[-1, :] = q[-2, :], q[1, :]
    q[:, 0], q[:, -1] = q[:, -2], q[:, 1]
    return q


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0:  # sampler running before timing starts
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_baseline(n, method):
    """One FP64 oracle QG step at the full size on this host (single core)."""
    import numpy as np
    import oracle.fvx_oracle as O
    q = initial_q(n)
    dx = LX / n
    t = time.perf_counter()
    O.qg_step(q, dx, dx, BETA, 1.0 / LD ** 2, 0.5 * dx, method)
    t = time.perf_counter() - t
    return {"value": n * n / t / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 rk3_ssp_step at {n}x{n}, FP64 NumPy/SciPy oracle (restatement of the reference "
                      f"math; finitevolX's JAX stack is not installable offline), {t:.1f} s"}


def run_reference(args, rank):
    """Reference arm: the oracle port of the reference's CPU path, all host threads."""
    if rank != 0:
        return
    import numpy as np
    import scipy.fft
    import oracle.fvx_oracle as O
    # bounded per-step sample (same physics, smaller interior) so K + W steps stay within minutes
    ns = min(args.n, 512 if args.steps + args.warmup <= 200 else 256)
    q = initial_q(ns)
    dx = LX / ns
    cores = os.cpu_count() or 1
    times = []
    with scipy.fft.set_workers(cores):
        for k in range(args.warmup + args.steps):
            t = time.perf_counter()
            q = O.qg_step(q, dx, dx, BETA, 1.0 / LD ** 2, 0.5 * dx, args.method)
            t = time.perf_counter() - t
            if k >= args.warmup:
                times.append(t)
    tot = sum(times)
    val = ns * ns * len(times) / tot / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(args.n, args.method),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"per step: 1 rk3_ssp_step at {ns}x{ns} (FP64 NumPy oracle port of the "
                                   "reference path; SciPy FFT on all host threads)"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def masked_basin(n, seed=0):
    """Masked-Helmholtz workload: Gaussian-filtered (sigma = 20 cells) seeded
    field thresholded at 30% land, largest connected ocean kept, closed
    boundary ring; c = exp(0.5 g) with g a second smooth field (unit std);
    white-noise right-hand side on the ocean."""
    import numpy as np
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal((n, n)), sigma=20, mode="wrap")
    m = g > np.quantile(g, 0.3)
    lab, k = ndimage.label(m)
    if k > 1:
        sizes = ndimage.sum(m, lab, range(1, k + 1))
        m = lab == (1 + int(np.argmax(sizes)))
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = False
    g2 = ndimage.gaussian_filter(rng.standard_normal((n, n)), sigma=20, mode="wrap")
    c = np.exp(0.5 * g2 / g2.std())
    f = rng.standard_normal((n, n)) * m
    return m.astype(np.float64), c, f


def helmholtz_section(n, pairs, reps=5):
    """Masked variable-coefficient Helmholtz, time to 1e-8 relative residual
    (FP64-checked): MG-PCG (one V-cycle per iteration, the reference's
    6/6/50 sweeps) against flexible PCG with the learned coarse solver
    (U-Net at the 128^2 level, 4+4 fine sweeps, energy-scaled correction)
    and the same cycle without the network.  Each solve is timed with CUDA
    events around the whole call (set-up, iterations, final FP64 check);
    median of ``reps``; the network is trained once beforehand (not timed)."""
    import numpy as np
    import torch

    import finitevolx_b200 as fvx
    from finitevolx_b200.learned import LearnedPreconditioner, generate_pairs

    m, c, f = masked_basin(n, 1)
    dx = LX / n
    mg = fvx.build_multigrid_solver(m, dx, dx, lambda_=1.0 / LD ** 2, coeff=c, dtype=torch.float32)
    pcg = fvx.MaskedHelmholtzPCG(mg)
    b = torch.from_numpy(f).float().cuda()

    def timed(kw):
        pcg.solve(b, rtol=1e-8, **kw)
        ts, info = [], None
        for _ in range(reps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            x, info = pcg.solve(b, rtol=1e-8, **kw)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return {"ms": statistics.median(ts), "iterations": info["iterations"],
                "rel_residual_fp64": info["rel_residual"], "converged": info["converged"]}

    out = {"workload": f"masked Helmholtz {n}^2, Ld {LD / 1e3:.0f} km, variable c, FP32 work vectors, "
                       "FP64 iterate/dots/residual, rtol 1e-8", "levels": mg.n_levels}
    out["mg_pcg"] = timed(dict(precond="mg", graph=True))
    t0 = time.time()
    # the MG baseline's smoothing (6 pre, 6 post) on the fine levels: the
    # fastest of 2, 3, 4 and 6 at this workload (2: 18 it, 3: 14, 4: 11, 6: 9)
    pc = LearnedPreconditioner(mg, n_pre=6, n_post=6, batch_max=64, seed=0)
    F, E = generate_pairs(mg, pc.lvl, pairs, pc.n_pre, seed=1)
    torch.cuda.synchronize()
    t_gen = time.time() - t0
    t0 = time.time()
    hist = pc.train(F, E, epochs=6, batch=64, lr=2e-3, seed=1)
    torch.cuda.synchronize()
    out["training"] = {"pairs": pairs, "epochs": 6, "batch": 64, "gen_s": t_gen, "train_s": time.time() - t0,
                       "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1], "level": pc.lvl}
    del F, E
    out["learned_pcg"] = timed(dict(precond=pc, flexible=True, graph=True, max_iter=500))
    pc0 = LearnedPreconditioner(mg, n_pre=6, n_post=6, batch_max=1, coarse=False, scale=False)
    out["same_cycle_without_network"] = timed(dict(precond=pc0, flexible=True, graph=True, max_iter=500))
    out["speedup_learned_vs_mg"] = out["mg_pcg"]["ms"] / out["learned_pcg"]["ms"]
    return out


def ensemble_members(count=64, seed=0):
    """Config-2 ensemble: sizes drawn (seeded) from {128, 256, 512, 1024}^2,
    1-3 layers (H = 400/1100/2600 m)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = rng.choice([128, 256, 512, 1024], size=count)
    nls = rng.integers(1, 4, size=count)
    return list(zip(sizes.tolist(), nls.tolist()))


def ensemble_section(members, n_steps, rank=0):
    """All members advanced n_steps RK3-SSP steps by one CUDA graph (per RK
    stage: one batched DST chain per grid size, one persistent work-queue
    launch of the fused stage over every tile of every layer).  Metric:
    interior layer-cells x steps / s."""
    import torch

    import finitevolx_b200 as fvx

    ens = fvx.QGEnsemble(members)
    for m, (n, nl) in enumerate(members):
        g = torch.Generator(device="cuda").manual_seed(1000 * rank + m)
        for k in range(nl):
            q = torch.zeros((n + 2, n + 2), device="cuda")
            q[1:-1, 1:-1] = torch.randn((n, n), device="cuda", generator=g) * 1e-5
            ens.set_layer(m, k, q)
    from finitevolx_b200 import autotune
    tuned = autotune.tune_ensemble(ens)
    g = ens.capture(n_steps)
    g.replay()  # warm-up run of the graph
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    g.replay()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    cells = ens.cells_per_step()
    return {"workload": f"{len(members)} multi-layer QG members, sizes {{128,256,512,1024}}^2, 1-3 layers, "
                        f"WENO5, FP32, {n_steps} RK3 steps in one CUDA graph",
            "members": len(members), "layer_cells_per_step": cells, "steps": n_steps, "ms": ms,
            "ms_per_step": ms / n_steps, "value": cells * n_steps / (ms * 1e-3) / 1e6, "unit": "Mcell-steps/s",
            "launches_per_step": ens.launches_per_step, "autotuned_blocks_per_sm": tuned["blocks_per_sm"]}


def per_launch_ms(launch, flush, reps: int = 20, rounds: int = 5) -> float:
    """Device time of one launch with L2 flushed before it: `reps` (flush,
    launch) pairs between two events on the launching stream, minus `reps`
    flushes alone, divided by reps (the median of `rounds`).  The flushes keep
    the GPU busy while the host queues the next launch, so no host launch
    gap enters the window."""
    import torch

    est = []
    for _ in range(rounds):
        ts = []
        for with_launch in (True, False):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            flush.fill_(0.0)
            e0.record()
            for k in range(reps):
                flush.fill_(float(k))
                if with_launch:
                    launch()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        est.append((ts[0] - ts[1]) / reps)
    return statistics.median(est)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import numpy as np
    import torch
    import torch.distributed as dist

    import finitevolx_b200 as fvx
    from finitevolx_b200 import _lib as L
    from finitevolx_b200.qg import QGModel

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    n = args.n
    grid = fvx.ArakawaCGrid2D.from_interior(n, n, LX, LX)
    dt = 0.5 * grid.dx / 1.0
    model = QGModel(grid, BETA, 1.0 / LD ** 2, method=args.method, dtype=torch.float32)
    q0 = torch.as_tensor(initial_q(n, seed=rank), dtype=torch.float32, device="cuda")
    qa, qb = q0.clone(), torch.empty_like(q0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # autotuned launch choices (stage tile shape; fused or separate DST split)
    from finitevolx_b200 import autotune
    tuned = {}
    if args.stage_tile:
        autotune.set_stage_tile(args.method, torch.float32, autotune._TILES.index(args.stage_tile))
        tuned["stage_tile"] = args.stage_tile
    if not args.profile:
        tuned = {"stage_tile": tuned.get("stage_tile") or autotune.tune_qg_stage(model, qa, dt)["tile"],
                 "fused_split": autotune.tune_qg_split(model, qa, dt)["fused"],
                 "dst_kernel": autotune.tune_dst_kernel(model, qa, dt)["kernel"]}
    qa.copy_(q0)

    # warm-up (eager), leaves split(qb) in the DST workspace for the graphs
    for _ in range(max(args.warmup, 3)):
        model.step(qa, dt, out=qb)
        qa.copy_(qb)
    model.step(qa, dt, out=qb)
    torch.cuda.synchronize()
    # CUDA graphs of one step each way (qa -> qb, qb -> qa), chained presplit
    graphs = []
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for src, dst in ((qb, qa), (qa, qb)):
            g = torch.cuda.CUDAGraph()
            launches0 = model.kernel_launches
            with torch.cuda.graph(g, stream=s):
                model.step(src, dt, out=dst, presplit=True)
            per_step_launches = model.kernel_launches - launches0
            graphs.append(g)
    torch.cuda.current_stream().wait_stream(s)
    for g in graphs:  # graph warm-up
        g.replay()
    torch.cuda.synchronize()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            graphs[k % 2].replay()
            e1.record()
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    from finitevolx_b200.replicas import max_over_ranks, whole_job_rate
    t_max = max_over_ranks(total_ms, device="cuda")
    if world > 1:
        dist.barrier()
    cells = n * n
    value = whole_job_rate(cells, args.steps, t_max, world)
    if args.profile:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "steps": args.steps,
                              "ms_per_step": t_max / args.steps, "profile_run": True}))
        if world > 1:
            dist.barrier()
            del graphs
            dist.destroy_process_group()
        return

    # e2e through the public API (QGPipeline): every step uploads its input
    # state from pinned host memory and downloads its result; the pipeline
    # overlaps the upload of state k+1 and the download of state k-1 with
    # the step of state k.  L2 flushed before every step on the step stream.
    from finitevolx_b200.qg import QGPipeline
    pipe = QGPipeline(model, dt)
    n_host = 4
    host_in = torch.empty((n_host,) + tuple(q0.shape), dtype=torch.float32, pin_memory=True)
    for h in range(n_host):
        host_in[h].copy_(q0.cpu())
    host_out = torch.empty_like(host_in, pin_memory=True)
    flush_fn = lambda: flush.fill_(1.0)  # noqa: E731
    pipe.run(host_in, host_out, n=max(args.warmup, 3), between_steps=flush_fn)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    pipe.run(host_in, host_out, n=args.steps, between_steps=flush_fn)
    e1.record()
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    # the pipeline steps the same state as the graphs above: check its result
    if rank == 0:
        ref_out = model.step(host_in[0].to("cuda"), dt).cpu()
        diff = (host_out[(args.steps - 1) % n_host] - ref_out).abs().max() / ref_out.abs().max()
        if not float(diff) <= 1e-6:
            raise RuntimeError(f"e2e pipeline result differs from QGModel.step ({float(diff):.3e})")
    host_in = host_in[0]
    e2e_ms = max_over_ranks(e2e_ms, device="cuda")
    e2e = whole_job_rate(cells, args.steps, e2e_ms, world)
    nbytes = host_in.numel() * host_in.element_size()

    # fused vs unfused: the same step as the reference's operator sequence,
    # one kernel (or torch copy) per operator, through the same library
    for _ in range(3):
        model.step_unfused(qa, dt)
    torch.cuda.synchronize()
    unf_ms = 0.0
    n_unf = max(5, min(20, args.steps))
    for k in range(n_unf):
        flush.fill_(float(k))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        model.step_unfused(qa, dt)
        e1.record()
        e1.synchronize()
        unf_ms += e0.elapsed_time(e1)
    unf_ms /= n_unf

    # the fused stage kernel alone (HBM roofline): stage 2's form (reads
    # q_stage, q_n, psi; writes q_next and the split DST operand)
    stage_ms = per_launch_ms(lambda: model._stage(qa, qb, qb, 0.75, 0.25, 0.25 * dt, True, False), flush)
    # algorithmic bytes: q_stage, q_n, psi read, q_next written (FP32, one
    # pass each) = 16 B/cell, plus the DST operand written as bf16 hi/lo
    # (4 B/cell)
    stage_bytes = 20.0 * n * n
    hbm_peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            hbm_peak = json.load(f).get("hbm_gbs")
    except Exception:
        pass

    # dominant kernel: one tcgen05 DST GEMM (2048 x 2048 x 2048, 3xBF16)
    from finitevolx_b200._lib import I, fn, stream_ptr
    h = model.plan.handle
    sym = fn("fvx_dst_operand_layout")(h) == 1
    gemm = fn("fvx_dst_gemm_step")
    for _ in range(5):
        gemm(h, I(0), I(1), stream_ptr())
    gemm_ms = per_launch_ms(lambda: L.check(gemm(h, I(0), I(1), stream_ptr()), "gemm"), flush)
    flops = 2.0 * n * n * n
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = peaks.get("bf16_tflops")
    peak_src = "measured burst bf16 (MEASURED_PEAKS.json)" if peak else "fallback 1590"
    peak = peak or 1590.0
    achieved = flops / (gemm_ms * 1e-3) / 1e12

    if rank == 0:
        res = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(config(n, args.method), autotuned=tuned),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "ms_per_step": e2e_ms / args.steps,
                    "form": "QGPipeline: upload of state k+1, step k (CUDA graph), download of k-1 on three "
                            "streams; L2 flushed before every step"},
            "gpu_launches": per_step_launches * args.steps,
            "roofline": {"bound": "tensor",
                         "kernel": ("gemm_sym_bf16_kernel (even/odd DST-I product, 3xBF16)" if sym
                                    else "gemm_split_bf16_kernel (DST product, 3xBF16)"),
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": peak_src,
                         # DRAM bytes per launch from an ncu capture of this kernel in this
                         # step (dram__bytes_read.sum + dram__bytes_write.sum, first product;
                         # the operands otherwise stay in L2 between the products)
                         "traffic": 25.2e6 if n == 2048 and sym else None, "traffic_unit": "bytes",
                         "per_launch_ms": gemm_ms, "algorithmic_flops_per_launch": flops,
                         "executed_tensor_flops_per_launch": (3.0 if sym else 6.0) * n ** 3,
                         "executed_frac": (3.0 if sym else 6.0) * n ** 3 / (gemm_ms * 1e-3) / 1e12 / peak},
            "stage_kernel": {"bound": "hbm", "kernel": "qg stage_kernel<float, WENO5>",
                             "per_launch_ms": stage_ms, "algorithmic_bytes_per_launch": stage_bytes,
                             "achieved": stage_bytes / (stage_ms * 1e-3) / 1e9, "unit": "GB/s",
                             "peak": hbm_peak,
                             "frac": (stage_bytes / (stage_ms * 1e-3) / 1e9 / hbm_peak) if hbm_peak else None},
            "fused_vs_unfused": {"fused_ms_per_step": t_max / args.steps, "unfused_ms_per_step": unf_ms,
                                 "speedup": unf_ms / (t_max / args.steps),
                                 "unfused": "the reference operator sequence, one library kernel or torch copy per "
                                            "operator (QGModel.step_unfused)"},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(n, args.method)
        if world == 1 and not args.no_helmholtz:
            res["helmholtz"] = helmholtz_section(args.helm_n, args.helm_pairs)
        if world == 1 and not args.no_ensemble:
            res["ensemble"] = ensemble_section(ensemble_members(), args.ens_steps)
        print(json.dumps(res))
    if world > 1:
        dist.barrier()
        del graphs
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
