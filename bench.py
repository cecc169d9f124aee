#!/usr/bin/env python
"""Throughput of the SPH hot path on B200 (particle-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl uph|reference]

Workload (the hydrostatic-tank configuration): still water 2.0 m wide x 1.0 m
deep at dx = 0.002 m -- 500,000 fluid particles on a lattice, density set
hydrostatically -- in an open tank with 3 wall layers, h = 1.3 dx,
rho0 = 1000, gamma = 7, c0 = 10 sqrt(2 g), dt = 0.2 h / c0.  Synthetic data
built from those numbers; no dataset is involved.

A step is one leapfrog step of the hot path (neighbour search, the rate pass,
kick-drift) over all particles, advanced on the device through the C ABI.
The headline is the reference's own formulation (the drop-in "REF"
profile) in FP64; `variants` adds the textbook WCSPH profile of the same
configuration (cubic spline, algebraic Tait, Monaghan viscosity) in FP64 and
with FP32 pair arithmetic.

One process per GPU; with N > 1 every rank advances its own tank (replicas,
no collective on the data path) and value = all ranks' particle-steps / the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200: plain SPH vs batched+surrogate at ≤1% ρ error"
UNIT = "particle-steps/s"
WORKLOAD = ("hydrostatic tank 2.0 x 1.0 m, dx=0.002 m (500,000 fluid particles) + 3 wall layers, h=1.3dx, "
            "rho0=1000, gamma=7, c0=10*sqrt(2g), dt=0.2h/c0; REF (drop-in) physics, FP64")

# Algorithmic bytes of one rate pass (the dominant kernel), which applies
# the leapfrog step in its epilogue: every interacting particle's 13 FP64
# fields (x y u v ut vt rho rhot p pt m 1/rho 1/rhot) + orig index + itype +
# its cell-list entry read once (120 B); every fluid particle's *_min state
# read (4 x 8 B), its candidate list read (24 record indices of 2 B and a
# 1 B count) and its post-step state written once (x y, the four *_min,
# u v ut vt rho rhot p pt 1/rho 1/rhot: 16 x 8 B), 209 B.  (The rates and
# the Tait pressure are written by a call's last step only; the first pass
# after a cell-list build writes the candidate lists instead of reading
# them.)  Neighbour re-reads are served on chip.
PASS_BYTES_PER_SLOT = 13 * 8 + 4 + 4 + 8
PASS_BYTES_PER_FLUID = 4 * 8 + 24 * 2 + 1 + 16 * 8
# with --separate-corrector the pass writes the 12 rates + Tait pressure and
# reads the sponge factor instead (112 B); the corrector is its own launch
PASS_BYTES_PER_FLUID_RATES = 13 * 8 + 8


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_deck():
    from uph_b200 import deck as D
    return D.hydrostatic_tank(width=2.0, depth=1.0, dx=0.002, layers=3)


# ---------------------------------------------------------------- clocks ----

class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    QUERY = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 10:
                    continue
                if self.uuid and parts[1] != self.uuid:
                    continue
                rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].lower().startswith("active")})
        pw = [float(r[4]) for r in rows if r[4].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


# ------------------------------------------------------------ CPU baseline ---

def cpu_reference_run(deck, budget_s: float, max_steps: int, warmup: int = 1):
    """The reference's own solver (oracle/_ref, compiled from its sources) on
    the host cores: returns (particle-steps/s, steps timed, threads, kind)."""
    from oracle import oracle as O
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        if os.path.exists(os.path.join(O.REF_DIR, "libuph_ref.so")):
            run = O.RefRun(tmp, eta_override=deck.eta_override, fluid_capacity_pct=16)
            kind = "reference"
            step = run.step
        else:
            o = O.Oracle(deck.uph_params(), deck.initial_state())
            kind = "port"
            threads = 1
            step = o.step
        for _ in range(warmup):
            step(1)
        t0 = time.perf_counter()
        step(1)
        first = time.perf_counter() - t0
        n = int(max(1, min(max_steps - 1, budget_s / max(first, 1e-9) - 1)))
        t1 = time.perf_counter()
        step(n)
        total = first + (time.perf_counter() - t1)
        inputbp_share = None
        if kind == "reference":
            # the per-step re-read of the boundary decks inside derivatives()
            inputbp_share = run.time_inputbp(3) / (total / (n + 1))
            run.close()
    steps = n + 1
    return deck.n_fluid * steps / total, steps, threads, kind, inputbp_share


# ---------------------------------------------------------------- ranks ---

class Ranks:
    """Barrier and max-over-ranks of a replicated run over torch.distributed
    (NCCL on the GPUs; any backend works, the tests use gloo on the CPU).
    Every rank makes the same calls in the same order."""

    def __init__(self, world: int, device):
        self.world = world
        self.device = device

    def barrier(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())


def whole_job_rate(units_per_rank: float, slowest_seconds: float, world: int) -> float:
    """Weak scaling of replicas: every rank's units over the slowest rank's time."""
    return world * units_per_rank / slowest_seconds


# ---------------------------------------------------------------- GPU arm ---

def gpu_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from uph_b200._capi import PREC_FP32_PAIR, PROFILE_REF, PROFILE_WCSPH
    from uph_b200.sim import Simulation

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    deck = workload_deck()
    nf, n_all = deck.n_fluid, deck.n_all

    ranks = Ranks(world, dev)
    barrier, max_over_ranks = ranks.barrier, ranks.max

    def timed_steps(sim, k, sampler=None):
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = sim.launch_count()
        e0.record(stream)
        sim.step(k)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        return e0.elapsed_time(e1), sim.launch_count() - l0, clocks

    # --- headline: REF profile, FP64
    sim = Simulation.from_deck(deck, profile=PROFILE_REF)
    sim.set_fused_step(not args.separate_corrector)
    sim.set_stream(stream.cuda_stream)
    sim.step(args.warmup)
    sim.profile(True)
    try:
        uuid = torch.cuda.get_device_properties(dev).uuid
        uuid = "GPU-" + str(uuid) if uuid else None
    except Exception:
        uuid = None
    builds0 = sim.stats()["list_builds"]
    ms, launches, clocks = timed_steps(sim, args.steps, ClockSampler(uuid) if rank == 0 else None)
    ktimes = sim.kernel_times()
    stats = sim.stats()
    stats["list_builds_per_step"] = (stats["list_builds"] - builds0) / args.steps
    sim.profile(False)
    ms_max = max_over_ranks(ms)
    value = whole_job_rate(nf * args.steps, ms_max / 1e3, world)

    pass_ms, pass_n = ktimes.get("rate_pass", (0.0, 0))
    pass_avg_s = pass_ms / max(pass_n, 1) / 1e3
    pass_bytes = n_all * PASS_BYTES_PER_SLOT + nf * (PASS_BYTES_PER_FLUID_RATES if args.separate_corrector
                                                     else PASS_BYTES_PER_FLUID)
    peak, peak_kind = load_peaks()
    achieved = pass_bytes / pass_avg_s / 1e9 if pass_avg_s > 0 else 0.0
    # DRAM read + write bytes of one launch from the committed ncu capture
    # (profiles/rate_pass_ref_fp64_hydrostatic500k.md)
    # and its FP64-pipe activity, the compute roof this kernel is held by
    traffic = None
    fp64_active = None
    tpath = os.path.join(ROOT, "profiles", "rate_pass_traffic.txt")
    # the capture is of the pass that applies the step
    if os.path.exists(tpath) and not args.separate_corrector:
        with open(tpath) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 2 and parts[0] == "ref_fp64_bytes_per_launch":
                    traffic = int(parts[1])
                if len(parts) == 2 and parts[0] == "ref_fp64_pipe_active":
                    fp64_active = float(parts[1])

    # --- e2e: every step through the C ABI with pinned host buffers: upload
    # the state the step reads (sim.STEP_INPUT_FIELDS), one step, download
    # the state it hands to the next step (sim.STEP_OUTPUT_FIELDS)
    from uph_b200._capi import empty_state
    from uph_b200.sim import STEP_INPUT_FIELDS, STEP_OUTPUT_FIELDS

    def pinned_like(a):
        t = torch.empty(a.shape, dtype=torch.int32 if a.dtype == np.int32 else torch.float64, pin_memory=True)
        return t.numpy()

    st_host = {}
    for name, a in deck.initial_state().items():
        st_host[name] = pinned_like(a)
        st_host[name][...] = a
    out_host = {name: pinned_like(a) for name, a in empty_state(nf, n_all).items() if name in STEP_OUTPUT_FIELDS}
    in_host = {name: (out_host[name] if name in out_host else st_host[name]) for name in STEP_INPUT_FIELDS}
    h2d = sum(a.nbytes for a in in_host.values())
    d2h = sum(a.nbytes for a in out_host.values())
    k_e2e = max(1, min(args.steps, args.e2e_steps))
    sim.upload(st_host, 0)
    sim.step(1)
    sim.download(out_host)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    itime = 1
    for _ in range(k_e2e):
        sim.upload(in_host, itime)
        sim.step(1)
        sim.download(out_host)
        itime += 1
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = whole_job_rate(nf * k_e2e, e2e_s, world)
    niac = int(stats["niac"])
    sim.close()

    # --- e2e through the reference-facing call: derivatives(System*, t) of
    # libuph_sph.so once per step, the leapfrog on the host (libuph_driver.so
    # restates src/bin/sph.cc:90-168), host System arrays in and out every step
    e2e_dropin = {}
    if not args.no_dropin_e2e:
        from uph_b200.dropin import DropInRun
        k_dr = max(1, min(args.steps, args.e2e_steps))
        for level in (2, 0):
            run = DropInRun(deck.uph_params(), deck.initial_state(), pair_export=level)
            run.step(1)  # first call: device state, page-locking of the System's arrays
            barrier()
            t0 = time.perf_counter()
            run.step(k_dr)
            dt_s = max_over_ranks(time.perf_counter() - t0)
            run.close()
            bi, bo = DropInRun.bytes_per_step(nf, n_all, niac, level)
            e2e_dropin[f"pair_export_{level}"] = {
                "value": whole_job_rate(nf * k_dr, dt_s, world), "unit": UNIT, "steps": k_dr,
                "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo}

    # --- variants: the WCSPH profile of the same configuration, FP64 and
    # FP32 pair arithmetic, from the same state for the same steps; the FP32
    # path's per-field error against the FP64 one is reported with it
    variants = {}
    k_var = max(1, min(args.steps, args.variant_steps))
    finals = {}
    for label, prof, prec in [("wcsph_fp64", PROFILE_WCSPH, 0), ("wcsph_fp32_pair", PROFILE_WCSPH, PREC_FP32_PAIR)]:
        v = Simulation.from_deck(deck, profile=prof, precision=prec)
        v.set_fused_step(not args.separate_corrector)
        v.set_stream(stream.cuda_stream)
        v.step(args.warmup)
        v.profile(True)
        vms, _, _ = timed_steps(v, k_var)
        kt = v.kernel_times()
        finals[label] = v.download()
        v.close()
        vms = max_over_ranks(vms)
        p_ms, p_n = kt.get("rate_pass", (0.0, 0))
        variants[label] = {"value": whole_job_rate(nf * k_var, vms / 1e3, world), "steps": k_var,
                           "ms_per_step": vms / k_var, "rate_pass_ms": p_ms / max(p_n, 1),
                           "state_after_steps": args.warmup + k_var}
    variants["wcsph_fp32_pair"]["error_vs_fp64"] = field_errors(finals["wcsph_fp32_pair"], finals["wcsph_fp64"], nf)
    if not args.no_batched:
        variants["batched_tanks"] = batched_arm(args, stream.cuda_stream)
    if not args.no_dambreak:
        variants.update(dambreak_arm(args, stream))
    if not args.no_surrogate:
        variants["flume_surrogate"] = surrogate_arm(args, stream)

    return dict(value=value, ms=ms_max, launches=launches, clocks=clocks, ktimes=ktimes, stats=stats,
                pass_avg_s=pass_avg_s, pass_bytes=pass_bytes, achieved=achieved, peak=peak, peak_kind=peak_kind,
                traffic=traffic, fp64_active=fp64_active, e2e_value=e2e_value, h2d=h2d, d2h=d2h, k_e2e=k_e2e, variants=variants,
                deck=deck, e2e_dropin=e2e_dropin)


ERROR_FIELDS = ["density", "DynamicPressure", "Velocity", "dvdt", "Position"]


def field_errors(got, want, nf):
    """Per-field error of one state against another over the fluid:
    max |got - want| / max |want| (norm-wise), and for Position the largest
    displacement difference in metres."""
    out = {}
    for f in ERROR_FIELDS:
        g = np.asarray(got[f])[:nf]
        w = np.asarray(want[f])[:nf]
        if f == "Position":
            out["Position_max_abs_m"] = float(np.abs(g - w).max())
        else:
            scale = float(np.abs(w).max())
            out[f] = float(np.abs(g - w).max() / scale) if scale > 0 else float(np.abs(g - w).max())
    return out


def dambreak_arm(args, stream):
    """The dam-break configurations, WCSPH physics (cubic spline, Tait,
    Monaghan alpha = 0.01), hydrostatic initial pressure in the column:
    - dambreak_5k: tank 4.0 x 3.0 m, column 1.0 x 2.0 m, dx = 0.02 m, 2 wall
      layers, FP64, 1,000 steps as one CUDA-graph replay (the case is small
      enough that launches, not kernels, would otherwise dominate);
    - dambreak_2M: tank 8.0 x 4.0 m, column 2.0 x 4.0 m, dx = 0.002 m,
      FP32 pair arithmetic with FP64 integration, 500 steps."""
    import torch
    from uph_b200 import deck as D
    from uph_b200.sim import Simulation

    out = {}
    big = D.dam_break(tank=(8.0, 4.0), column=(2.0, 4.0), dx=0.002, layers=2, hydrostatic=True, local_depth=4.0)
    cases = [("dambreak_5k_fp64_graph", D.dam_break(tank=(4.0, 3.0), column=(1.0, 2.0), dx=0.02, layers=2,
                                                    hydrostatic=True), 0, 1000, True),
             # c0 = 10 sqrt(g H) with H = 4 m, the column height (the 5k case's
             # 10 sqrt(2 g) belongs to its own 2 m column); FP32 pair
             # arithmetic (the configuration) and FP64 (what FP32 buys)
             ("dambreak_2M_fp32_pair", big, 1, 500, False),
             ("dambreak_2M_fp64", big, 0, 500, False)]
    finals = {}
    for label, deck, prec, steps, graph in cases:
        s = Simulation.from_deck(deck, profile=1, precision=prec)
        s.set_stream(stream.cuda_stream)
        s.step(1)
        if graph:
            s.set_graph(steps)
            s.step(steps)  # records the graph and runs it once
        else:
            s.step(args.warmup)
        s.profile(not graph)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        entry = {"value": deck.n_fluid * steps / sec, "n_fluid": deck.n_fluid, "steps": steps,
                 "ms_per_step": sec / steps * 1e3}
        if not graph:
            ms, n = s.kernel_times().get("rate_pass", (0.0, 0))
            entry["rate_pass_ms"] = ms / max(n, 1)
        st = s.stats()
        # largest |rho - rho0| / rho0 over the fluid: the weak compressibility
        # the configuration allows (about 1 %), not an error against a reference
        entry["max_density_deviation_from_rho0"] = st["max_abs_density_error"]
        if deck is big:
            finals[label] = s.download()
        s.close()
        out[label] = entry
    out["dambreak_2M_fp32_pair"]["error_vs_fp64"] = field_errors(finals["dambreak_2M_fp32_pair"],
                                                                 finals["dambreak_2M_fp64"], big.n_fluid)
    out["dambreak_2M_fp32_pair"]["speedup_vs_fp64"] = (out["dambreak_2M_fp32_pair"]["value"] /
                                                       out["dambreak_2M_fp64"]["value"])
    return out


SURROGATE_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "uph_b200", "weights", "flume_mpnn.npz")


def surrogate_arm(args, stream):
    """The wave-flume configuration with the learned surrogate: flume
    10.0 x 1.0 m (`--sur-length`), depth 0.5 m, dx = 0.005 m (200k fluid particles), piston
    A = 0.04 m, T = 1.3 s, 3-column piston and hydrostatic walls, WCSPH.
    After a warm-up of `--sur-warm` s from rest (plain FP32 pair), the same
    state is advanced `--sur-steps` SPH steps
    - plain: the plain FP64 path (one uph_sim_step per macro step's length);
    - surrogate: uph_sur_advance with the trained network (fused BF16
      tcgen05 kernels) on an FP64 simulation, whose plain solver is the judge
      every 10th macro step and takes over after a failed check.
    Both are timed with CUDA events on the simulations' stream.  Errors
    compare the surrogate's final state with the plain one: RMS and largest
    relative density error, largest free-surface height difference per
    5 cm bin as a fraction of the depth."""
    import torch
    from uph_b200 import deck as D
    from uph_b200 import surrogate as SG
    from uph_b200._capi import PREC_FP32_PAIR, PROFILE_WCSPH
    from uph_b200.sim import Simulation
    weights = args.sur_weights or SURROGATE_WEIGHTS
    if not os.path.exists(weights):
        return {"unavailable": f"no trained weights at {os.path.relpath(weights)}"}
    cfg, params = SG.Surrogate.load_file(weights)
    L, depth = args.sur_length, 0.5
    deck = D.wave_flume(L, depth, 0.005, amplitude=0.04, period=1.3, piston_layers=3, hydrostatic_walls=True)
    K = cfg.macro_steps
    nmacro = max(1, args.sur_steps // K)
    steps = nmacro * K
    warm = int(round(args.sur_warm / cfg.dt))
    w = Simulation.from_deck(deck, PROFILE_WCSPH, PREC_FP32_PAIR)
    w.set_stream(stream.cuda_stream)
    w.step(warm)
    st0 = w.download()
    w.close()
    nf = deck.n_fluid
    judge = SG.Judge(depth=depth, surface_x0=0.0, surface_x1=L, surface_bins=int(L / 0.05))

    def new_sim(prec):
        sim = Simulation(deck.uph_params(PROFILE_WCSPH, prec))
        sim.set_stream(stream.cuda_stream)
        sim.upload(st0, warm)
        sim.set_wall_motion(*deck.wall_table)
        return sim

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, out

    plain = new_sim(0)
    plain.step(K)  # first-call allocations, untimed
    plain.upload(st0, warm)
    t_plain, _ = timed(lambda: [plain.step(K) for _ in range(nmacro)])
    ref = plain.download()
    plain.close()
    sur = SG.Surrogate(cfg, deck.n_all + 128, params)
    sur.set_stream(stream.cuda_stream)
    s = new_sim(0)
    sur.advance(s, 1, judge)  # first-call allocations and weight images, untimed, then start over
    s.close()
    s = new_sim(0)
    t_sur, rep = timed(lambda: sur.advance(s, nmacro, judge))
    out = s.download()
    s.close()
    err = SG.state_errors(out, ref, nf, depth, 0.0, L, judge.surface_bins)
    # the network alone (no judge) over the same span, for its own drift
    s = new_sim(0)
    t_net, rep_net = timed(lambda: sur.advance(s, nmacro, SG.Judge(depth=depth, surface_x0=0.0, surface_x1=L,
                                                                      surface_bins=judge.surface_bins,
                                                                      judge_every=1 << 30)))
    net_err = SG.state_errors(s.download(), ref, nf, depth, 0.0, L, judge.surface_bins)
    s.close()
    sur.close()
    # tensor work of one network evaluation: multiply-adds per node of the
    # encoder (E1, E2, W_pq), each round (W2, N1, N2 and W_pq or Dec1, Dec2)
    macs = 128 * 128 * 2 + 256 * 128 + cfg.rounds * (128 * 128 + 128 * 256 + 128 * 128 + 256 * 128)
    flops_eval = 2.0 * macs * deck.n_all
    r = rep.to_dict()
    return {"value": nf * steps / t_sur, "plain_fp64_value": nf * steps / t_plain, "speedup_vs_plain": t_plain / t_sur,
            "n_fluid": nf, "steps": steps, "macro_steps": K, "judge_every": judge.judge_every,
            "errors_vs_plain": err, "network_only": {"value": nf * steps / t_net, "errors_vs_plain": net_err, "report": rep_net.to_dict()},
            "report": r, "network_tflops_per_eval": flops_eval / 1e12,
            "warm_s": args.sur_warm, "weights": os.path.relpath(weights)}


def batched_arm(args, stream_ptr):
    """The batched-tank configuration: 256 dam-break and sloshing tanks from
    seed 0 (1.5k-30k particles each, ~2.9 M in all), WCSPH physics.
    - plain: every tank its own simulation in FP64, advanced one after the
      other, 1 + graph_steps steps each (the plain GPU path);
    - batched: all tanks as one simulation, FP32 pair arithmetic with FP64
      integration, autotuned, graph_steps steps per CUDA-graph replay.
    Errors compare the batched state with the plain one after the same
    1 + graph_steps steps: density relative to rho0, free-surface height
    relative to the tank's column height."""
    import torch
    from uph_b200 import batch as B
    from uph_b200.sim import Simulation

    gsteps = args.graph_steps
    tanks = B.draw_tanks(seed=0, count=args.tanks)
    batch = B.build_batch(tanks)
    nf_total = batch.deck.n_fluid
    stream = torch.cuda.current_stream()

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    # plain: one FP64 simulation per tank
    sims = []
    for k in range(len(tanks)):
        d, table = B.tank_deck(batch, k)
        s = Simulation.from_deck(d, profile=1, precision=0)
        s.set_stream(stream.cuda_stream)
        if table is not None:
            s.set_wall_motion(*table)
        sims.append((d, s))
    plain_s = timed(lambda: [s.step(1 + gsteps) for _, s in sims])
    plain_value = nf_total * (1 + gsteps) / plain_s
    plain_states = []
    for d, s in sims:
        plain_states.append((d.n_fluid, s.download()))
        s.close()

    # tuning for this size class (trials on a throw-away copy)
    tuner = Simulation.from_deck(batch.deck, profile=1, precision=1)
    tuner.set_wall_motion(batch.wall_x0, batch.wall_hs, batch.wall_om)
    choice, _ = tuner.autotune(trial_steps=5)
    tuner.close()

    sim = Simulation.from_deck(batch.deck, profile=1, precision=1)
    sim.set_stream(stream.cuda_stream)
    sim.set_wall_motion(batch.wall_x0, batch.wall_hs, batch.wall_om)
    sim.set_tuning(*choice)
    sim.set_graph(gsteps)
    sim.step(1)
    sim.step(gsteps)  # records the graph and runs it once
    st = sim.download()
    rho0, dx = batch.deck.params["density0"], batch.deck.params["dx"]
    max_drho = max_fs = 0.0
    for k, spec in enumerate(tanks):
        f0, f1 = batch.fluid_ranges[k]
        n, pst = plain_states[k]
        max_drho = max(max_drho, float(np.abs(st["density"][f0:f1] - pst["density"][:n]).max() / rho0))
        length = 2.5 * spec.width if spec.kind == "dambreak" else spec.width
        x0 = batch.offsets[k][0]
        hb = B.free_surface_heights(st["Position"][f0:f1], x0, length, dx)
        hp = B.free_surface_heights(pst["Position"][:n], x0, length, dx)
        max_fs = max(max_fs, float(np.abs(hb - hp).max() / spec.height))
    reps = args.graph_replays
    l0 = sim.launch_count()
    batched_s = timed(lambda: [sim.step(gsteps) for _ in range(reps)])
    launches = sim.launch_count() - l0
    sim.close()
    batched_value = nf_total * gsteps * reps / batched_s
    return {
        "tanks": len(tanks), "n_fluid": nf_total, "steps_per_graph": gsteps,
        "batched_fp32_graph": {"value": batched_value, "ms_per_step": batched_s / (gsteps * reps) * 1e3,
                               "replays": reps, "kernels_per_replay": launches // max(reps, 1),
                               "tuning": {"cell_reach": choice[0], "tile": choice[1], "resort_interval": choice[2]}},
        "plain_per_tank_fp64": {"value": plain_value, "steps": 1 + gsteps},
        "speedup": batched_value / plain_value,
        "max_density_error": max_drho, "max_free_surface_error": max_fs,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["uph", "reference"], default="uph")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--variant-steps", type=int, default=500)
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for the CPU baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tanks", type=int, default=256, help="batched-tank configuration: number of tanks")
    ap.add_argument("--graph-steps", type=int, default=200, help="steps per CUDA-graph replay of the batch")
    ap.add_argument("--graph-replays", type=int, default=3)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-dambreak", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-dropin-e2e", action="store_true")
    ap.add_argument("--separate-corrector", action="store_true",
                    help="run the leapfrog corrector as its own launch after each rate pass "
                         "(uph_sim_set_fused_step(0)) instead of in the pass's epilogue")
    ap.add_argument("--sur-steps", type=int, default=2000, help="wave-flume surrogate configuration: SPH steps")
    ap.add_argument("--sur-warm", type=float, default=1.0, help="wave-flume warm-up from rest (s)")
    ap.add_argument("--sur-length", type=float, default=10.0, help="wave-flume length (m); 10 m is the workload")
    ap.add_argument("--sur-weights", default=None, help="trained surrogate file (default uph_b200/weights/flume_mpnn.npz)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "uph":
        args.warmup = 3
    # the reference's per-thread scratch has 64 rows (System.c:209)
    os.environ.setdefault("OMP_NUM_THREADS", str(min(64, os.cpu_count() or 1)))

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference's own CPU solver on rank 0's host cores; other ranks idle
        if rank != 0:
            return
        deck = workload_deck()
        value, steps, threads, kind, share = cpu_reference_run(deck, budget_s=60.0, max_steps=max(2, args.steps),
                                                               warmup=min(args.warmup, 1))
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": deck.n_fluid / value * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": WORKLOAD, "parallelism": "host OpenMP"},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                                 "sample": f"{steps} leapfrog steps of the full 500k-particle tank (bounded to ~60 s)",
                                 "inputbp_share_of_step": share},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    try:
        r = gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if rank != 0:
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        v, steps, threads, kind, share = cpu_reference_run(r["deck"], budget_s=args.cpu_budget, max_steps=1000)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": kind, "inputbp_share_of_step": share,
               "sample": f"{steps} leapfrog steps of the same 500k-particle tank on the host "
                         f"(reference solver compiled from its sources; search stand-in for libnabo)"}
    kt = {k: {"ms_total": round(v[0], 4), "launches": v[1]} for k, v in r["ktimes"].items() if v[1]}
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_fluid": r["deck"].n_fluid, "n_particles": r["deck"].n_all,
                   "l2": "state 0.2 GB per GPU > 126 MB L2; no flush between steps",
                   "leapfrog": "separate corrector launch" if args.separate_corrector
                               else "in the rate pass's epilogue",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": r["achieved"], "peak": r["peak"], "unit": "GB/s",
                     "frac": r["achieved"] / r["peak"], "traffic": r["traffic"],
                     "kernel": "rate pass (k_ref_pass)", "bytes_per_launch": r["pass_bytes"],
                     "avg_launch_ms": r["pass_avg_s"] * 1e3, "peak_source": r["peak_kind"],
                     "fp64_pipe_active_ncu": r["fp64_active"]},
        "cpu_baseline": cpu,
        "e2e": {"value": r["e2e_value"], "unit": UNIT, "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"], "steps": r["k_e2e"],
                "how": "per step: uph_sim_upload from pinned host memory of the state a step reads (positions, "
                       "velocities, density and pressure of every particle, mass, type, sponge, the fluid's "
                       "predictor rates and fluctuations), uph_sim_step(1), uph_sim_download of the state it hands "
                       "to the next step"},
        "e2e_dropin": dict(r["e2e_dropin"], how="per step: the host leapfrog of src/bin/sph.cc:90-168 "
                           "(libuph_driver.so) around derivatives(System*, t) of libuph_sph.so, the reference's own "
                           "entry point: the fields it reads copied in and its rates, fluctuations, Tait pressure and "
                           "(pair_export_2) the full pair list copied out"),
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
        "kernel_ms": kt,
        "variants": r["variants"],
        "stats": {"niac": r["stats"]["niac"], "max_neighbors": r["stats"]["max_neighbors"],
                  "list_builds_per_step": r["stats"]["list_builds_per_step"]},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
