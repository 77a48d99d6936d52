"""Benchmark: timesteps/s of the meeuuw hot path at 512x512 Q2xQ1 (FK viscosity, 4.2M particles).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 512]

One step = one full timestep of the box path on the GPU (particle interpolation + material,
projections, Stokes right-hand side + device Uzawa solve to an FP64 relative residual of 1e-8,
pressure normalisation, dt, energy assembly + solve, heat flux / Nu, strain rate, vrms,
RK4 advection, locate).  The product path is the mixed-precision solver (FP32 multigrid-PCG
inner solves, FP64 refinement) warm-started from the previous step; the plain FP64 path is
measured beside it.  With N > 1 each rank advances its own independent model (replicas: a
single model does not shard), so `value` is the sum over ranks of timesteps/s ("weak").

`--impl reference` times the CPU oracle (a restatement of the reference's Numba/SciPy path, pinned
to the reference's own functions and driver) on a bounded sample: one full timestep of the same
model at 256x256 (and 128x128), measured, reported at 512x512 scaled by the element count.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
if "--ensemble" in sys.argv:
    # one stream per model: with CUDA's default 8 hardware work queues, 64 models' streams share
    # queues and serialise; 32 queues (read when CUDA initialises, before torch does) took the
    # 64-model ensemble from 88 to 129 model-steps/s (measured)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "timesteps/s at 512x512 Q2xQ1, learned+mixed vs plain GPU at 1e-8 Stokes residual"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-profile", action="store_true", help="skip the torch-profiler launch count")
    ap.add_argument("--roofline-only", action="store_true", help="set up the model, time the operator apply, exit")
    ap.add_argument("--kernels-only", action="store_true",
                    help="set up the model, run the warm-up steps, time the particle and energy kernels, the FP32 "
                         "assembly and the U-Net convolutions, exit")
    ap.add_argument("--host-loops", action="store_true",
                    help="solver loops driven from the host (same kernels; lets a kernel profiler list every launch)")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="instead of the 512x512 model: an uneven ensemble of this many models (64..192 squared)")
    ap.add_argument("--ensemble-batched-only", action="store_true",
                    help="with --ensemble: time only the mode with every Stokes solve in one cluster launch, skip "
                         "the other modes and the accuracy runs (for kernel profiles)")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.stop_ = index, [], threading.Event()

    def _run(self):
        while not self.stop_.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self.stop_.wait(0.2)

    def __enter__(self):
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop_.set()
        self.th.join(timeout=10)

    def summary(self):
        import statistics
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for nm, v in zip(names, r[4:8]):
                if "Active" in v and "Not" not in v:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------------------------------- ours
def run_ours(args):
    import torch
    import torch.distributed as dist

    from meeuuw_b200 import _lib, configs, ops
    from meeuuw_b200.timestep import GPUModel

    from meeuuw_b200 import replicas
    world, rank, local = replicas.world()
    torch.cuda.set_device(local)
    replicas.init("nccl")            # replicas only: collectives for timing, none on the data path

    def barrier():
        replicas.barrier(device="cuda")

    def max_over_ranks(v):
        return replicas.max_over_ranks(v, device="cuda")

    n = args.n
    cfg = configs.fk_convection(n, seed=1000 + rank)
    host = configs.build_host_model(cfg)

    def timed(model, K, W):
        for _ in range(W):
            model.step()
        model.check()
        if not args.host_loops:
            # the whole step as one CUDA graph (solver loops as conditional nodes); the learned
            # guess is consulted at the cold start among the warm-up steps and idle afterwards
            model.capture_step()
        barrier()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.cuda.nvtx.range_push("timed")     # lets a profiler select exactly the timed steps
        for _ in range(K):
            model.step()
        torch.cuda.nvtx.range_pop()
        e.record()
        barrier()
        ms = s.elapsed_time(e)
        model.check()
        return ms

    # ---- product path: mixed precision, learned warm start (gated; previous-step fallback) ----
    model = GPUModel(cfg, host, stokes="mixed", tol=1e-8)
    if args.host_loops:
        model.solve_kw = dict(model.solve_kw, host_loops=1)
    learned = None
    wpath = os.path.join(ROOT, "meeuuw_b200", "weights", "unet_fk128.npz")
    if os.path.exists(wpath):
        from meeuuw_b200.unet import LearnedGuess, UNet
        learned = LearnedGuess(model, UNet.load(wpath), judge="cold")
        model.guess = learned
    if args.roofline_only:
        from meeuuw_b200 import fe_tables
        model.solver.set_viscosity(torch.ones(model.nel, 9, dtype=torch.float64, device="cuda"), None)
        print(json.dumps({"roofline": roofline_apply(model, torch)}), flush=True)
        return
    if args.kernels_only:
        for _ in range(args.warmup):
            model.step()
        model.check()
        roof = roofline_apply(model, torch)
        print(json.dumps({"roofline": roof, "kernel_rooflines": kernel_rooflines(model, torch, roof["peak"]),
                          "unet_tensor_cores": unet_throughput(torch)}), flush=True)
        return
    dev_index = torch.cuda.current_device()
    with ClockSampler(dev_index) as clk:
        ms = timed(model, args.steps, args.warmup)
    ms = max_over_ranks(ms)
    diag = model.diagnostics()
    ms_per_step = ms / args.steps
    value = world * args.steps / (ms / 1000.0)

    # ---- launches per step (profiled step, untimed) ----
    launches = None
    kernel_mix = {}
    try:
        if args.no_profile:
            raise RuntimeError("launch count skipped (--no-profile)")
        from torch.profiler import ProfilerActivity, profile
        graph, model.graph = model.graph, None          # an eager step: the recorded one's kernels
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            model.step()
            torch.cuda.synchronize()
        model.graph = graph
        names = [evt.name for evt in prof.events() if evt.device_type.name == "CUDA"]
        ours = [nm for nm in names if "mw::" in nm]
        launches = int(len(ours) * args.steps)
        kernel_mix = {}
        for nm in ours:
            k = nm.split("(")[0].replace("void ", "")
            kernel_mix[k] = kernel_mix.get(k, 0) + 1
    except Exception as ex:  # profiler unavailable: leave the claim empty
        kernel_mix = {"error": str(ex)}

    # ---- where a step's time goes (two more steps with CUDA events between the phases) ----
    def phases(m, k=2):
        graph, m.graph = m.graph, None                  # eager steps, events between the phases
        m.enable_phase_timing(True)
        for _ in range(k):
            m.step()
        out = {p: v / k for p, v in m.phase_times().items()}
        m.enable_phase_timing(False)
        m.graph = graph
        return out

    phase_ms = phases(model)

    # ---- roofline of the dominant kernel: fine-level operator apply (FP32), CUDA events ----
    roof = roofline_apply(model, torch)
    kroof = kernel_rooflines(model, torch, roof["peak"])
    unet_tc = unet_throughput(torch)

    # ---- plain FP64 path (same problem, same warm start) ----
    plain = None
    if not args.no_plain:
        pmodel = GPUModel(cfg, host, stokes="f64", tol=1e-8)
        Kp = max(2, args.steps // 2)
        pms = max_over_ranks(timed(pmodel, Kp, args.warmup))
        pdiag = pmodel.diagnostics()
        plain = {"value": world * Kp / (pms / 1000.0), "ms_per_step": pms / Kp, "steps": Kp,
                 "stokes": pdiag["stokes"], "vrms": pdiag["vrms"], "Nu": pdiag["Nu"],
                 "phases_ms_per_step": phases(pmodel)}
        del pmodel

    # ---- accuracy: both arms advanced the same steps from the same state ----
    accuracy = None
    if not args.no_plain:
        ma, mb = GPUModel(cfg, host, stokes="mixed", tol=1e-8), GPUModel(cfg, host, stokes="f64", tol=1e-8)
        na = 5
        for _ in range(na):
            ma.step()
            mb.step()
        da, db = ma.diagnostics(), mb.diagnostics()
        accuracy = {"steps": na, "vrms_rel_diff": abs(da["vrms"] - db["vrms"]) / abs(db["vrms"]),
                    "Nu_rel_diff": abs(da["Nu"] - db["Nu"]) / abs(db["Nu"]),
                    "T_max_abs_diff": float((ma.T - mb.T).abs().max().item())}
        del ma, mb

    # ---- both arms' first step against the FP64 oracle's first step (512x512, stored) ----
    vs_oracle = None
    if rank == 0 and not args.no_plain:
        vs_oracle = step1_vs_oracle(torch, wpath if learned else None)

    # ---- end to end through host buffers ----
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(model, torch, max(2, args.steps // 2), world, barrier, max_over_ranks)

    # ---- CPU baseline (rank 0, N = 1 only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(n)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32 (FP32 inner multigrid-PCG, FP64 refinement/reductions)",
            "data": "synthetic (seeded FK convection: T0 + N(0,1e-3), 16 random particles/element)",
            "config": {"workload": f"fk_convection {n}x{n} Q2xQ1, Ra=1e6, eta=exp(-ln(1e5) T), geometric "
                                   f"averaging, RK4, 16 particles/element, Crank-Nicolson energy",
                       "nel": cfg.nel, "nparticle": cfg.nparticle, "stokes_tol": 1e-8,
                       "stokes_solver": "device Uzawa (cd_u_eta recurrence) + multigrid-PCG K solves, mixed",
                       "warm_start": ("learned U-Net (gated on the Uzawa residual, consulted at cold starts), "
                                      "previous-step fallback") if learned else "previous step",
                       "stokes_loops": "device (conditional nodes)" if model.solver.device_loops()
                       else "host",
                       "step_execution": "host-driven loops (profiling)" if args.host_loops else
                       "one CUDA graph per time step, recorded after the warm-up (both arms)",
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (swarm state ~0.5 GB, fields ~0.2 GB)"},
            "clocks": clk.summary(), "gpu_launches": launches, "kernel_mix_per_step": kernel_mix,
            "roofline": roof, "kernel_rooflines": kroof, "unet_tensor_cores": unet_tc, "e2e": e2e, "plain_fp64": plain,
            "speedup_vs_plain_fp64": (value / plain["value"]) if plain else None,
            "last_step": {"vrms": diag["vrms"], "Nu": diag["Nu"], "dt": diag["dt"], "stokes": diag["stokes"],
                          "energy_iters_relres": list(getattr(model, "energy_info", (None, None)))},
            "phases_ms_per_step": phase_ms,
            "mixed_vs_fp64": accuracy,
            "step1_vs_fp64_oracle": vs_oracle,
            "warm_start_picks": dict(learned.picks) if learned else None,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    replicas.finalize()


def kernel_rooflines(model, torch, peak_gbs):
    """The particle kernels and the FP32 Stokes assembly on the bench's model, each timed alone with
    CUDA events on its stream (mean of `reps` launches after a warm-up), against HBM: algorithmic
    bytes per launch / duration.  Algorithmic bytes count each per-particle or per-element array once
    and each nodal array the kernel gathers from once.  The particle kernels run in FP64 (the
    reference's arithmetic), so their FP64 issue rate, not HBM, is what bounds them; the FP32
    assembly also reports FLOP/s against the FP32 non-tensor peak (148 SMs x 128 lanes x 2 x the
    maximum SM clock)."""
    from meeuuw_b200 import ops
    m, b = model, model.box
    n, nel, nn, npp = m.npart, m.nel, m.nn, m.np_
    nact = int(m.active.sum().item())
    P = m.props
    reps = 10

    def timed(fn, prep=None):
        for _ in range(2):
            if prep:
                prep()
            fn()
        tot = 0.0
        for _ in range(reps):
            if prep:
                prep()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            tot += s.elapsed_time(e)
        return tot * 1000.0 / reps

    out = {}

    def add(name, us, algo, **kw):
        gbs = algo / (us * 1e-6) / 1e9
        out[name] = dict(us_per_launch=us, algorithmic_bytes=int(algo), achieved_gbs=gbs, frac_hbm=gbs / peak_gbs, **kw)

    r, t, iel = torch.empty_like(m.r), torch.empty_like(m.t), torch.empty_like(m.iel)
    add("k_locate", timed(lambda: ops.locate(b, m.active, m.x, m.z, r, t, iel, m.err)), 37 * nact + (n - nact) * 13)
    nodal = dict(exx=m.exx_n, ezz=m.ezz_n, exz=m.exz_n, q=m.q, T=m.T)
    props = {k: torch.empty_like(v) for k, v in P.items()}
    add("k_interp_material", timed(lambda: ops.interp_material(b, m.active, m.r, m.t, m.iel, m.mat, nodal,
                                                               m.material, props)),
        109 * n + 5 * 8 * nn)
    x, z, act = m.x.clone(), m.z.clone(), m.active.clone()
    up, wp = torch.empty_like(m.x), torch.empty_like(m.x)

    def prep_adv():
        x.copy_(m.x)
        z.copy_(m.z)
        act.copy_(m.active)
    dtv = float(m.dt_out[0].item()) or 1e-6
    add("k_advect (RK%d)" % m.cfg.RKorder, timed(lambda: ops.advect(b, m.cfg.RKorder, dtv, x, z, act, m.u, m.w, up, wp,
                                                                   m.err), prep_adv),
        50 * n + 2 * 8 * nn, bound_note="FP64 issue (4 stages: element index, reduced coordinates, Q2 basis, 18 gathers)")
    # the matrix-free energy operator of the last step: y = A x (5 coefficient planes x 9 Gauss
    # points per element, x and y, the Dirichlet flags) and its set-up (8 Gauss-point input arrays
    # read, the planes written; per node T, flags and values read, diagonal, flags and rhs written)
    if m.cfg.solve_T and getattr(m, "energy_op", None) is not None:
        y = torch.empty_like(m.T)
        add("k_energy_op_apply", timed(lambda: ops.energy_op_apply(b, m.energy_op, m.T, y)), nel * 360 + nn * 17)
        qf = m.qf
        qe = {k: qf[k] for k in ("rhoq", "etaq", "Tq", "uq", "wq", "hcondq", "hcapaq", "alphaq", "hprodq")}
        qe.update(m.geo)
        op2, rhs2 = torch.empty_like(m.energy_op), torch.empty_like(m.rhs_T)
        add("k_energy_op_setup", timed(lambda: ops.energy_op_setup(b, m.T, qe, m.tables, m.bc_fix_T, m.bc_val_T, 0.0,
                                                                   m.cfg.rho0, m.cfg.formulation, op2, rhs2,
                                                                   dt_dev=m.dt_out)),
            nel * (576 + 360) + nn * 34)
        del op2, rhs2, y
    # FP32 Stokes assembly, the full layout (the drop-in's build_matrix_stokes; the time step's solve
    # is matrix-free and does not assemble)
    q = m.stokes_inputs()
    res = ops.assemble_stokes(b, False, 1, q, m.tables, m.bc_fix_V, m.bc_val_V, m.cfg.eta_ref, m.L_ref)
    us = timed(lambda: ops.assemble_stokes(b, False, 1, q, m.tables, m.bc_fix_V, m.bc_val_V, m.cfg.eta_ref, m.L_ref,
                                           out=res))
    algo = nel * (9 * 9 * 8 + 8 + 468 * 4) + 2 * nn * 9 + 2 * nn * 8 + npp * 8
    flops = 1.7e4 * nel
    sm_mhz = None
    try:
        sm_mhz = float(subprocess.run(["nvidia-smi", "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits",
                                       f"--id={torch.cuda.current_device()}"], capture_output=True, text=True,
                                      timeout=5).stdout.strip())
    except Exception:
        pass
    fp32_peak = 148 * 128 * 2 * (sm_mhz or 1965.0) * 1e6 / 1e12
    add("k_assemble_stokes<float> (full VV)", us, algo, gflop=flops / 1e9, tflops=flops / (us * 1e-6) / 1e12,
        frac_fp32_peak=flops / (us * 1e-6) / 1e12 / fp32_peak, fp32_peak_tflops=fp32_peak)
    del res
    torch.cuda.empty_cache()
    return out


def unet_throughput(torch):
    """The learned warm start's network on the tensor cores: the U-Net forward at 128x128 (batch 1,
    the cold-start inference; batch 16, the training batch) and its largest implicit convolutions,
    timed with CUDA events (mean of 20 after 3 warm-ups), against MEASURED_PEAKS.json bf16_tflops.
    FLOPs: 2 M Cout 9 Cin per convolution (M = batch x pixels of the layer's grid)."""
    from meeuuw_b200 import ops
    import meeuuw_b200.unet as U
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("bf16_tflops", 1590.0)
    wpath = os.path.join(ROOT, "meeuuw_b200", "weights", "unet_fk128.npz")
    net = U.UNet.load(wpath) if os.path.exists(wpath) else U.UNet(seed=0)

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    def net_flops(B, n):
        tot, h = 0, n
        for lvl, (c1, c2) in enumerate(net.enc):
            tot += 2 * B * h * h * 9 * (c1.cin * c1.cout + c2.cin * c2.cout)
            if lvl < len(net.enc) - 1:
                h //= 2
        for c1, c2 in net.dec:
            h *= 2
            tot += 2 * B * h * h * 9 * (c1.cin * c1.cout + c2.cin * c2.cout)
        return tot + 2 * B * h * h * 9 * net.head.cin * net.head.cout

    out = {"peak_tflops": peak, "peak_source": "MEASURED_PEAKS.json bf16_tflops (of measured)" if "bf16_tflops" in peaks
           else "fallback 1590"}
    g = torch.Generator(device="cuda").manual_seed(0)
    for B in (1, 16):
        X = torch.randn(B, 128, 128, 2, device="cuda", generator=g).to(torch.bfloat16)
        ms = timed(lambda: net.forward(X, B, 128, 128))
        fl = net_flops(B, 128)
        out[f"forward_b{B}"] = {"ms": ms, "gflop": fl / 1e9, "tflops": fl / (ms * 1e-3) / 1e12,
                                "frac_bf16_peak": fl / (ms * 1e-3) / 1e12 / peak}
    # single implicit convolutions at the training batch: (B, H, W, Cin, Cout)
    for B, H, C, N in ((16, 128, 96, 32), (16, 32, 384, 128), (16, 16, 256, 256), (64, 64, 128, 64)):
        X = torch.randn(B * H * H, C, device="cuda", generator=g).to(torch.bfloat16)
        Wt = (torch.randn(N, U._kp(C), device="cuda", generator=g) * 0.05).to(torch.bfloat16)
        y = torch.empty(B * H * H, N, dtype=torch.bfloat16, device="cuda")
        ms = timed(lambda: ops.conv3x3_bf16(X, B, H, H, C, Wt, out=y, relu=True, out_bf16=True))
        fl = 2 * B * H * H * N * 9 * C
        out[f"conv_b{B}_{H}x{H}_{C}to{N}"] = {"ms": ms, "gflop": fl / 1e9, "tflops": fl / (ms * 1e-3) / 1e12,
                                               "frac_bf16_peak": fl / (ms * 1e-3) / 1e12 / peak}
    return out


def step1_vs_oracle(torch, weights):
    """Both arms' first step of the 512x512 model (seed 1000) against the FP64 oracle's first step
    (tests/golden/oracle_fk512_step1.npz: the oracle restating the reference, cd_u_eta with SuperLU):
    relative vrms, Nu and dt errors and the largest T error on the stored nodes.  The first step is
    a cold start, so the product path's learned guess (the U-Net on the pooled 128x128 fields) is
    measured here against the same path started from zero (Schur / multigrid-PCG iterations, time)."""
    import numpy as np

    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    path = os.path.join(ROOT, "tests", "golden", "oracle_fk512_step1.npz")
    if not os.path.exists(path):
        return None
    d = np.load(path)
    meta = json.loads(str(d["meta"]))
    cfg = configs.fk_convection(meta["n"], seed=meta["seed"])
    host = configs.build_host_model(cfg)
    out = {"oracle": {"vrms": float(d["vrms"]), "Nu": float(d["Nu"]), "solver": meta["solver"],
                      "stokes_relative_residual": float(d["stokes_residual"])}}
    for arm in ("product", "product_zero_guess", "plain_fp64"):
        m = GPUModel(cfg, host, stokes="f64" if arm == "plain_fp64" else "mixed", tol=1e-8)
        if arm == "product" and weights:
            from meeuuw_b200.unet import LearnedGuess, UNet
            m.guess = LearnedGuess(m, UNet.load(weights), judge="cold")
        if arm == "product_zero_guess":
            m.warm_start = "zero"
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        m.step()
        e1.record()
        dd = m.diagnostics()
        T = m.T.cpu().numpy()[d["nodes"]]
        out[arm] = {"vrms_rel_err": abs(dd["vrms"] / float(d["vrms"]) - 1),
                    "Nu_rel_err": abs(dd["Nu"] / float(d["Nu"]) - 1),
                    "dt_rel_err": abs(dd["dt"] / float(d["dt"]) - 1), "T_max_abs_err": float(np.abs(T - d["T"]).max()),
                    "stokes_outer_iters": dd["stokes"].get("outer_iters"),
                    "stokes_inner_iters": dd["stokes"].get("inner_iters"),
                    "first_step_ms": e0.elapsed_time(e1)}
        if arm == "product" and weights:
            out[arm]["warm_start_pick"] = dict(m.guess.picks)
        del m
        torch.cuda.empty_cache()
    return out


def roofline_apply(model, torch):
    """Average duration of the fine-level FP32 operator apply (k_apply), CUDA events on its stream."""
    from meeuuw_b200 import _lib
    S = model.solver
    nv, npp = S.nv, S.np
    u = torch.randn(nv, dtype=torch.float32, device="cuda")
    p = torch.randn(npp, dtype=torch.float32, device="cuda")
    yV = torch.empty_like(u)
    yP = torch.empty_like(p)
    for _ in range(5):
        S.apply(u, p, yV, yP, precision="f32")
    reps = 50
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        S.apply(u, p, yV, yP, precision="f32")
    e.record()
    torch.cuda.synchronize()
    us = s.elapsed_time(e) * 1000.0 / reps
    nel, nn = model.nel, model.nn
    # algorithmic bytes per apply: read u (2nn f32), p (np f32), eta (9 nel f32), Dirichlet mask (2nn u8);
    # write yV (2nn f32), yP (np f32)
    algo = 4 * 2 * nn + 4 * npp + 4 * 9 * nel + 2 * nn + 4 * 2 * nn + 4 * npp
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = algo / (us * 1e-6) / 1e9
    # DRAM bytes (read + write) of one launch at 512x512 from an ncu capture of this kernel
    # (profiles/k_apply_fp32_fk512.txt); other sizes scale with the element count
    traffic = int(20162560 * nel / 262144)
    # the Chebyshev smoothing step (mode CHEB, the kernel the V-cycle launches most): reads x, b,
    # diag, d (2nn f32 each), eta, mask; writes d and x_out (2nn f32 each); no pressure
    b = torch.randn(nv, dtype=torch.float32, device="cuda")
    d = torch.zeros_like(b)
    xo = torch.empty_like(b)
    for _ in range(5):
        S.cheb_step_f32(b, u, xo, d, 1)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        S.cheb_step_f32(b, u, xo, d, 1)
    e.record()
    torch.cuda.synchronize()
    us_c = s.elapsed_time(e) * 1000.0 / reps
    algo_c = 4 * 2 * nn * 4 + 4 * 9 * nel + 2 * nn + 4 * 2 * nn * 2
    cheb = {"kernel": "mw::k_apply<float, AM_CHEB> (fine level)", "us_per_launch": us_c, "algorithmic_bytes": algo_c,
            "achieved": algo_c / (us_c * 1e-6) / 1e9, "frac": algo_c / (us_c * 1e-6) / 1e9 / peak}
    return {"kernel": "mw::k_apply<float, AM_APPLY> (fine level, 512x512)", "bound": "hbm", "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "us_per_launch": us,
            "algorithmic_bytes": algo, "cheb_mode": cheb,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else "fallback 6650"}


def run_e2e(model, torch, K, world, barrier, max_over_ranks):
    """Same metric through host buffers: each step uploads the swarm and T from pinned host memory
    and reads back the step's state (x, z, active, T) and scalars."""
    names = ("x", "z", "T")
    host = {k: torch.empty(getattr(model, k).shape, dtype=getattr(model, k).dtype, pin_memory=True) for k in names}
    host_act = torch.empty(model.active.shape, dtype=torch.bool, pin_memory=True)
    for k in names:
        host[k].copy_(getattr(model, k))
    host_act.copy_(model.active)
    sc = torch.empty(3, dtype=torch.float64, pin_memory=True)
    h2d = sum(host[k].numel() * host[k].element_size() for k in names) + host_act.numel()
    d2h = h2d + 3 * 8

    def one():
        for k in names:
            getattr(model, k).copy_(host[k], non_blocking=True)
        model.active.copy_(host_act, non_blocking=True)
        from meeuuw_b200 import ops
        ops.locate(model.box, model.active, model.x, model.z, model.r, model.t, model.iel, model.err)
        model.step()
        for k in names:
            host[k].copy_(getattr(model, k), non_blocking=True)
        host_act.copy_(model.active, non_blocking=True)
        sc.copy_(model.gq_out, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    one()
    barrier()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(K):
        one()
    e.record()
    barrier()
    ms = max_over_ranks(s.elapsed_time(e))
    return {"value": world * K / (ms / 1000.0), "unit": "timesteps/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": K}


# ---------------------------------------------------------------------------------------- CPU
def cpu_step(n, seed=1000):
    """One full oracle timestep (the first) of the FK workload at n x n, measured: wall time (s),
    per-phase times (s), the Stokes iteration count and the element count.  The oracle restates
    the reference's numpy/Numba/SciPy path (SuperLU inner solves of cd_u_eta; K factorised under a
    symmetric minimum-degree ordering, which only reorders the factorisation -- SuperLU's default
    COLAMD ordering runs out of memory at 512x512)."""
    from meeuuw_b200 import configs
    from oracle.model import OracleModel
    cfg = configs.fk_convection(n, seed=seed)
    host = configs.build_host_model(cfg)
    om = OracleModel(cfg, host)
    om.stokes_kw = dict(permc_spec="MMD_AT_PLUS_A")
    om.energy_kw = dict(permc_spec="MMD_AT_PLUS_A")
    t0 = time.perf_counter()
    out = om.step(solver="cd_u_eta")
    t = time.perf_counter() - t0
    return t, dict(om.phase_seconds), int(out["stokes_iterations"]), cfg.nel


def cpu_sample(n_target, n_sample, repeats=1):
    """Measured oracle timesteps at n_sample x n_sample (median of `repeats`), reported in
    timesteps/s of the n_target x n_target workload by scaling with the element count (linear).
    Linear scaling is a lower bound on the CPU's time at n_target: the sparse factorisation and the
    Schur iteration grow faster than the element count (one full 512x512 oracle step took 423 s on
    one core where a 128x128 step took 11.7 s), so the reported value favours the CPU."""
    runs = [cpu_step(n_sample) for _ in range(max(1, repeats))]
    runs.sort(key=lambda r: r[0])
    t, phases, its, nel = runs[len(runs) // 2]
    scale = (n_target / n_sample) ** 2
    return {"value": 1.0 / (t * scale), "unit": "timesteps/s", "cores": 1, "kind": "port",
            "sample": (f"one full oracle timestep of the FK model at {n_sample}x{n_sample} (numpy/SciPy; cd_u_eta "
                       f"with SuperLU, {its} Schur iterations), measured {t:.2f} s (median of {len(runs)}); "
                       f"scaled to {n_target}x{n_target} by the element count (x{scale:g}, linear: a lower "
                       f"bound on the CPU's time there)"),
            "measured": {"n": n_sample, "seconds_per_step": t, "timesteps_per_s": 1.0 / t,
                         "phases_s": {k: round(v, 4) for k, v in phases.items()}},
            "cores_note": "single-threaded: the reference's Numba kernels are serial and SuperLU is serial"}


def cpu_baseline_sample(n_target):
    return cpu_sample(n_target, 128)


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # a bounded sample of the workload: the full oracle step at 256x256, measured; 128x128 beside it
    # shows how the step grows with the element count
    small = cpu_sample(args.n, 128)
    nrep = max(1, min(args.steps, 2))
    big = cpu_sample(args.n, 256, repeats=nrep)
    v = big["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "timesteps/s", "n_gpus": world,
            "steps": nrep, "warmup": 0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded FK convection)",
            "config": {"workload": f"fk_convection {args.n}x{args.n} Q2xQ1, Ra=1e6, eta=exp(-ln(1e5) T), geometric "
                                   f"averaging, RK4, 16 particles/element, Crank-Nicolson energy (CPU oracle: "
                                   f"measured at 256x256, scaled by element count)"},
            "cpu_baseline": {k: big[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "measured": {"256": big["measured"], "128": small["measured"]},
            "e2e": {"value": v, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _ensemble_state(ens):
    """(vrms per model, active flags, models converged, retired) of an ensemble after its steps."""
    diag = ens.diagnostics()
    conv = sum(1 for i, d in enumerate(diag) if ens.active[i] and d["stokes"]["converged"] == 1)
    return [d["vrms"] for d in diag], list(ens.active), conv, dict(ens.retired)


def run_ensemble(args):
    """Uneven ensemble (n ~ U[64,192], Ra ~ logU[1e4,1e7], contrast ~ logU[1,1e4], 16 particles per
    element): aggregate model-timesteps/s of the mixed-precision ensemble in its three modes -- the
    thread pool with autotuned concurrency, every model's step recorded as one CUDA graph (one launch
    per model per step), and every model's Stokes solve in one shared launch (one thread-block
    cluster per model) inside one recorded ensemble step -- each timed with CUDA events; `value` is
    the fastest mode.  Each model's vrms is compared with the same model run with the FP64 solver."""
    import torch
    from meeuuw_b200 import replicas
    from meeuuw_b200.ensemble import Autotuner, BatchedEnsemble, Ensemble, sample_configs
    world, rank, local = replicas.world()
    torch.cuda.set_device(local)
    replicas.init("nccl")
    all_cfgs = sample_configs(args.ensemble, seed=7)
    # the models are dealt to the GPUs balanced by element count; no data-path collective
    cfgs = [all_cfgs[i] for i in replicas.partition([c.nel for c in all_cfgs], world)[rank]]
    dev = torch.cuda.current_device()

    def timed(ens):
        for _ in range(args.warmup):
            ens.step()
        ens.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        replicas.barrier(device="cuda")
        done0 = ens.steps_done
        s.record()
        for _ in range(args.steps):
            ens.step()
        for st in ens.streams:               # the end event waits for every model's stream
            torch.cuda.current_stream().wait_stream(st)
        e.record()
        replicas.barrier(device="cuda")
        ms = replicas.max_over_ranks(s.elapsed_time(e), device="cuda")
        return ms, replicas.sum_over_ranks(ens.steps_done - done0, device="cuda")

    if args.ensemble_batched_only:       # the cluster-solve mode alone, no accuracy runs (kernel profiles)
        ens = BatchedEnsemble(cfgs)
        ms, n = timed(ens)
        if rank == 0:
            print(json.dumps({"mode": "batched", "models": len(all_cfgs), "model_steps_per_s": n / (ms / 1000.0),
                              "ms_per_step": ms / args.steps}), flush=True)
        replicas.finalize()
        return
    modes = {}
    with ClockSampler(dev) as clk:
        ens = Ensemble(cfgs, stokes="mixed")
        tune = Autotuner().tune(ens, steps=1, use_cache=False)        # tuned afresh; the cache only records it
        ms, n = timed(ens)
        modes["threads"] = {"model_steps_per_s": n / (ms / 1000.0), "ms_per_step": ms / args.steps,
                            "threads": tune["threads"], "autotune_seconds_per_step": tune["seconds_per_step"]}
        ens.close()
        del ens
        torch.cuda.empty_cache()
        # recorded steps; every model's cold first step runs eagerly with its learned guess (the network
        # runs on the model's grid padded to multiples of 8; a mesh its pooling factor does not divide
        # starts from zero), then the step is recorded
        guess, nguess = None, [0]
        wpath = os.path.join(ROOT, "meeuuw_b200", "weights", "unet_fk128.npz")
        if os.path.exists(wpath):
            from meeuuw_b200.unet import LearnedGuess, UNet
            net = UNet.load(wpath)

            def guess(m):
                try:
                    g = LearnedGuess(m, net, judge="cold")
                except ValueError:
                    return None
                nguess[0] += 1
                return g
        ens = Ensemble(cfgs, stokes="mixed", graphs=True, guess=guess)
        cold_learned = ens.first_step_info
        ms, n = timed(ens)
        modes["graphs"] = {"model_steps_per_s": n / (ms / 1000.0), "ms_per_step": ms / args.steps}
        states = {"graphs": _ensemble_state(ens)}
        have_guess = [m.guess is not None for m in ens.models]
        ens.close()
        del ens
        torch.cuda.empty_cache()
        # every model's Stokes solve in one launch (one thread-block cluster per model), the whole
        # ensemble step recorded as one graph; the cold first steps as in the graphs mode
        ens = BatchedEnsemble(cfgs, guess=guess)
        ms, n = timed(ens)
        modes["batched"] = {"model_steps_per_s": n / (ms / 1000.0), "ms_per_step": ms / args.steps}
        states["batched"] = _ensemble_state(ens)
        del ens
        torch.cuda.empty_cache()
    nsteps_done = 1 + args.warmup + args.steps
    # FP64 runs of the same models for the same number of steps: at the benchmark's 1e-8 and at 1e-10
    # (the reference both are measured against; FP64 at 1e-8 against it is the floor the tolerance
    # itself sets)
    def fp64_run(tol, stokes="f64"):
        ref = Ensemble(cfgs, stokes=stokes, graphs=True, tol=tol)
        for _ in range(nsteps_done - 1):
            ref.step()
        ref.synchronize()
        out = ([d["vrms"] for d in ref.diagnostics()], list(ref.active))
        ref.close()
        torch.cuda.empty_cache()
        return out
    # the same models' cold starts from zero (mixed), for the learned guess's gain
    ens0 = Ensemble(cfgs, stokes="mixed", graphs=True)
    cold_zero = ens0.first_step_info
    ens0.close()
    del ens0
    torch.cuda.empty_cache()
    sel = [i for i in range(len(cfgs)) if have_guess[i]]
    cold = {"models_with_learned_guess": len(sel), "models": len(cfgs),
            "schur_iters_learned": sum(cold_learned[i]["outer_iters"] for i in sel),
            "schur_iters_zero": sum(cold_zero[i]["outer_iters"] for i in sel),
            "pcg_iters_learned": sum(cold_learned[i]["inner_iters"] for i in sel),
            "pcg_iters_zero": sum(cold_zero[i]["inner_iters"] for i in sel)}
    fp64, act64 = fp64_run(1e-8)
    tight, act_t = fp64_run(1e-10)
    # the mixed arm at the reference's own tolerance: what the mixed precision alone costs
    mixed_tight, act_mt = fp64_run(1e-10, stokes="mixed")
    err_matched = [abs(mixed_tight[i] - tight[i]) / abs(tight[i]) for i in range(len(cfgs)) if act_mt[i] and act_t[i]]
    best = max(modes, key=lambda k: modes[k]["model_steps_per_s"])
    # the accuracy figures below are the fastest recorded mode's (the thread pool's models are
    # the graphs mode's, stepped from host threads)
    mixed, active, converged, retired = states[best if best in states else "graphs"]
    both = [i for i in range(len(cfgs)) if active[i] and act64[i] and act_t[i]]
    err = [abs(mixed[i] - tight[i]) / abs(tight[i]) for i in both]
    floor = sorted(abs(fp64[i] - tight[i]) / abs(tight[i]) for i in both)
    err_modes = {}
    for k, (mx, ac, _, _) in states.items():
        e = sorted(abs(mx[i] - tight[i]) / abs(tight[i]) for i in range(len(cfgs)) if ac[i] and act64[i] and act_t[i])
        err_modes[k] = {"max": e[-1] if e else None, "median": e[len(e) // 2] if e else None}
    retired = {cfgs[i].name: why for i, why in retired.items()}
    if world > 1:                            # gather the per-model figures on rank 0
        import torch.distributed as dist
        got = [None] * world
        dist.all_gather_object(got, (err, retired, converged, floor, err_matched))
        err = [x for g in got for x in g[0]]
        retired = {k: v for g in got for k, v in g[1].items()}
        converged = sum(g[2] for g in got)
        floor = sorted(x for g in got for x in g[3])
        err_matched = [x for g in got for x in g[4]]
    err = sorted(err)
    em = sorted(err_matched)
    matched = {"models": len(em), "max": em[-1] if em else None, "median": em[len(em) // 2] if em else None}
    line = {"metric": "aggregate model-timesteps/s, uneven ensemble (64..192 squared, 16 particles/element)",
            "value": modes[best]["model_steps_per_s"], "unit": "model-timesteps/s",
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": modes[best]["ms_per_step"],
            "higher_is_better": True, "dtype": "f64+f32", "data": "synthetic (seeded per model)",
            "n_gpus": world, "scaling": "weak" if world > 1 else None,
            "config": {"workload": f"ensemble of {len(all_cfgs)} FK convection models", "models": len(all_cfgs),
                       "elements_total": int(sum(c.nel for c in all_cfgs)), "mode": best,
                       "parallelism": f"models dealt to {world} GPU(s) by element count"},
            "modes": modes,
            "models_retired": retired,
            "stokes_converged_models": converged,
            "cold_start_first_step": cold,
            "vrms_rel_err_vs_fp64_1e-10": {"models": len(err), "max": err[-1] if err else None,
                                           "median": err[len(err) // 2] if err else None,
                                           "p90": err[int(0.9 * (len(err) - 1))] if err else None},
            "vrms_rel_err_by_mode": err_modes,
            "vrms_rel_err_mixed_1e-10_vs_fp64_1e-10": matched,
            "vrms_floor_fp64_1e-8_vs_1e-10": {"max": floor[-1] if floor else None,
                                              "median": floor[len(floor) // 2] if floor else None,
                                              "p90": floor[int(0.9 * (len(floor) - 1))] if floor else None},
            "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    replicas.finalize()


if __name__ == "__main__":
    a = parse()
    if a.ensemble:
        # more hardware work queues for the many model streams (read when CUDA initialises)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    if a.impl == "reference":
        run_reference(a)
    elif a.ensemble:
        run_ensemble(a)
    else:
        run_ours(a)
