"""Benchmark: Brunel-12.5k real-time factor & synaptic events/s on one B200.

Workload (the reference's full-scale Brunel on its kernel path, per-edge
delays): NE=10000, NI=2500 iaf_psc_alpha, CE=1000, CI=250, g=5, eta=2, J=0.1 mV
PSP, recurrent delays Uniform(1.0 ms, 3.0 ms) rounded to the 0.1 ms grid
(kernel ring timing), one Poisson unit per neuron (delay 1.5 ms), dt=0.1 ms,
separate 'ex' / 'in_' receptor ports.  Connectivity, delays, initial V_m and
the Poisson counts come from the reference kernel path's random streams for
seed 1234 (brunel.build_kernel_network).  One bench step = one simulated
second (10 000 time steps) of the resident network.  Synthetic, seeded
inputs; no dataset is involved.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  ``value`` is the whole-job real-time factor
(simulated seconds per wall second, summed over ranks; each rank runs an
independent replica); ``e2e`` is the same metric through the public
``Simulator.simulate`` call with host buffers.
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

STEPS_PER_SIM_S = 10_000  # dt = 0.1 ms
STEPS_PER_BENCH_STEP = STEPS_PER_SIM_S  # --sim-ms changes the simulated time per bench step
METRIC = "Brunel-12.5k real-time factor & synaptic events/s, FP32 vs FP64 path, 1 B200"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].isdigit():
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [int(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


def headline_program(precision=32, seed=1234):
    """The headline network compiled for `precision` (32 or 64); the plan
    records every spike (the synaptic-event count needs them all)."""
    from brainpy.state_b200 import brunel
    net, p, _ = brunel.build_kernel_network(order=2500, seed=seed)
    prog = net.compile("float64" if precision == 64 else "float32", spike_capacity=1 << 23)
    prog.plan._deg = brunel.kernel_out_degree(prog)
    return prog, p


def time_runs(pl, n_runs, stream, flush):
    import torch
    times, spikes, events = [], 0, 0
    for _ in range(n_runs):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pl.run(STEPS_PER_BENCH_STEP, stream=stream.cuda_stream)
        e1.record(stream)
        flush.zero_()  # write 256 MiB > L2 between timed iterations
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        st, g = pl.spikes()
        spikes += st.size
        events += int(pl._deg[g].sum())
    return times, spikes, events


def _cv_isi(steps, gids, min_spikes=3):
    """Mean over neurons with at least min_spikes spikes of the coefficient of
    variation of their inter-spike intervals (_kernel/validation/stats.py:44-59)."""
    import numpy as np
    if steps.size == 0:
        return None
    order = np.lexsort((steps, gids))
    s, g = steps[order], gids[order]
    cuts = np.nonzero(np.diff(g))[0] + 1
    cvs = []
    for a, b in zip(np.concatenate([[0], cuts]), np.concatenate([cuts, [g.size]])):
        if b - a >= min_spikes:
            isi = np.diff(s[a:b]).astype(np.float64)
            if isi.mean() > 0:
                cvs.append(isi.std() / isi.mean())
    return round(float(np.mean(cvs)), 4) if cvs else None


def run_ours(args):
    import torch
    import torch.distributed as dist
    from brainpy.state_b200 import brunel

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    from brainpy.state_b200 import dist as D
    prog, p = headline_program(32, seed=D.replica_seed(1234, rank))
    pl = prog.plan
    N = p["NE"] + p["NI"]
    time_runs(pl, args.warmup, stream, flush)
    # the tiled path's shape from pilot runs on the warmed-up network (its
    # state restored after each pilot), then one more warm-up run
    tuned = None
    if pl.engine == "tiled":
        g, pz, pms = pl.tune_tiled(pilot_steps=2000)
        tuned = {"grid": g, "poll_pause_ns": pz, "pilot_ms": round(pms, 3)}
        time_runs(pl, 1, stream, flush)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        times, nspk, nev = time_runs(pl, args.steps, stream, flush)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    ms_step = D.max_over_ranks(sum(times) / len(times))  # the slowest replica's time
    sim_ms = STEPS_PER_BENCH_STEP * 0.1
    rtf = world * sim_ms / ms_step
    syn_ev_s = world * (nev / args.steps) / (ms_step / 1000.0)
    rate_hz = nspk / args.steps / N
    drive_ev_s = world * N * p["rate"] * (sim_ms / 1000.0) / (ms_step / 1000.0)
    kms, launches = pl.kernel_time()
    cv_isi = _cv_isi(*pl.spikes())  # the last timed launch's spikes (outside the timed region)

    # roofline of the persistent kernel: algorithmic bytes per launch
    # (64 B/neuron/time step: 7 FP32 state words read+written and the ring
    # slot read+clear; 16 B per synaptic event: packed edge + weight read and
    # the 4 B red.add read-modify-write; 8 B per spiking row: indptr pair)
    ev_launch = nev / args.steps
    spk_launch = nspk / args.steps
    alg_bytes = 64.0 * N * STEPS_PER_BENCH_STEP + 16.0 * ev_launch + 8.0 * spk_launch
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (ms_step / 1000.0) / 1e9
    traffic, traffic_source = None, None
    prof = os.path.join(ROOT, "profiles", "k_lif_tiled_brunel12500_ncu_full.md")
    if os.path.exists(prof):
        with open(prof) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch ="):
                    # an ncu capture of one launch of this kernel, given per
                    # 10 000 time steps and scaled to this launch's steps (not
                    # measured in this run)
                    traffic = int(line.split("=")[1]) * STEPS_PER_BENCH_STEP // 10000
                    traffic_source = ("ncu capture summarised in profiles/"
                                      "k_lif_tiled_brunel12500_ncu_full.md, scaled")
    kbits = pl.ring_fraction_bits
    engine = pl.engine

    result = {
        "metric": METRIC, "value": round(rtf, 3), "unit": "x real time (simulated s / wall s)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "numerics": f"f32 state, weights and propagators; arrivals summed exactly in an int32 "
                    f"fixed-point ring of 2^-{kbits} pA resolution (weights rounded once)",
        "data": "synthetic (seeded Brunel network, the reference kernel path's streams)",
        "config": CONFIG_HEADLINE(N, p, int(pl._deg.sum()), sim_ms, world),
        "tiled_shape": tuned,
        "syn_events_per_s": round(syn_ev_s, 1), "drive_events_per_s": round(drive_ev_s, 1),
        "rate_hz": round(rate_hz / (sim_ms / 1000.0), 3),
        "cv_isi": cv_isi,
        "ms_per_time_step": round(ms_step / STEPS_PER_BENCH_STEP, 6),
        "wall_s_timed": round(wall, 4),
        "gpu_launches": int(args.steps) * int(launches),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "traffic_source": traffic_source, "peak_kind": peak_kind,
                     "kernel": "bspk::k_lif_tiled<float, 0, true, 512, 112>", "engine": engine},
        "clocks": clk.summary(),
    }
    pl.close()
    del prog, pl
    # the secondary sections run on a single GPU only: with N > 1 the other ranks
    # would wait on rank 0 for minutes at the final barrier
    if rank == 0 and not args.quick and world == 1:
        result["fp64"] = fp64_numbers(args, stream, flush)
        result["e2e"] = e2e_numbers(args)
        par, cpu = parity_numbers(args)
        result["parity"] = par
        result["cpu_baseline"] = cpu
        if not args.no_extras:
            result["sweep_batch"] = sweep_numbers(args)
            result["bptt"] = bptt_numbers(args)
            result["adex_stdp"] = adex_numbers(args)
    if world > 1 and not args.quick and not args.no_extras:
        # every rank takes part (same collectives in the same order on all ranks)
        sw = sweep_sharded(rank, world)
        if rank == 0:
            result["sweep_batch_sharded"] = sw
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def CONFIG_HEADLINE(N, p, edges, sim_ms, world):
    return {"workload": "brunel_order2500_kernel_path_per_edge_delay_U(1.0,3.0)ms", "N": N,
            "CE": p["CE"], "CI": p["CI"], "edges": edges, "delays_steps": [10, 30],
            "dt_ms": 0.1, "seed": 1234,
            "step": f"{sim_ms:.0f} ms simulated ({int(round(sim_ms / 0.1))} time steps)",
            "l2": "flushed between timed iterations (256 MiB write)",
            "parallelism": f"replicas{world}"}


def fp64_numbers(args, stream, flush):
    prog, p = headline_program(64)
    pl = prog.plan
    time_runs(pl, 1, stream, flush)
    k = max(2, args.steps // 3)
    times, nspk, nev = time_runs(pl, k, stream, flush)
    ms = sum(times) / len(times)
    sim_ms = STEPS_PER_BENCH_STEP * 0.1
    kbits = pl.ring_fraction_bits
    pl.close()
    return {"path": f"FP64 state and weights, arrivals in an int64 fixed-point ring of "
                    f"2^-{kbits} pA resolution",
            "rtf": round(sim_ms / ms, 3), "ms_per_step": round(ms, 4),
            "syn_events_per_s": round(nev / k / (ms / 1000.0), 1),
            "rate_hz": round(nspk / k / (p["NE"] + p["NI"]) / (sim_ms / 1000.0), 3),
            "network": "the headline network with its delays drawn in float64 (the reference's "
                       "x64 streams)"}


def e2e_numbers(args):
    """The same metric through the kernel front end's public call,
    ``Runner.simulate(1000 ms)``, with host buffers in the loop: every call
    restores the initial state from the host checkpoint (h2d), runs 10 000
    steps, and reads back the spikes of 50 E + 50 I neurons and the V_m
    traces of 100 E neurons (d2h), as the reference's build_brunel observers
    record them (_kernel/validation/brunel.py:130-139)."""
    import torch
    from brainpy.state_b200 import brunel
    net, p, _ = brunel.build_kernel_network(order=2500, seed=1234)
    E, I = net.populations[0], net.populations[1]
    from brainpy.state_b200.kernel import PopulationView
    rec_e = net.observe(PopulationView(net, E.gids[:50]), "spike", name="rec_E")
    rec_i = net.observe(PopulationView(net, I.gids[:50]), "spike", name="rec_I")
    rec_v = net.observe(PopulationView(net, E.gids[::100][:100]), "V_m", name="rec_V")
    prog = net.compile("float32")
    runner = prog.runner()
    runner.simulate(1000.0)  # warm-up
    k = max(2, args.steps // 2)
    torch.cuda.synchronize()
    h2d = d2h = 0
    t0 = time.perf_counter()
    for _ in range(k):
        res = runner.simulate(1000.0)
        h2d += runner.h2d_bytes
        d2h += runner.d2h_bytes
    wall = (time.perf_counter() - t0) / k
    rate_e = float(res[rec_e]["spike"].sum()) / 50.0
    prog.plan.close()
    return {"value": round(1.0 / wall, 3), "unit": "x real time (simulated s / wall s)",
            "h2d_bytes_per_step": int(h2d // k), "d2h_bytes_per_step": int(d2h // k),
            "api": "kernel Runner.simulate(1000 ms) (state restored from host, spikes of 100 "
                   "and V_m of 100 neurons read back)", "rate_hz_E": round(rate_e, 3)}


def parity_numbers(args, seconds=3):
    """FP32 and FP64 forms against the float64 oracle on the same networks,
    each realised independently by the oracle (oracle/kernel_net.py): the
    population-rate relative error over `seconds` s (FP32) and 1 s (FP64), and
    the max / RMS V_m error of 100 sampled neurons over the first 30 steps.
    The oracle's first simulated second, on all host threads, is the
    cpu_baseline."""
    import numpy as np
    import torch
    from brainpy.state_b200 import brunel
    from brainpy.state_b200.kernel import PopulationView
    from oracle import kernel_net as KN
    cores = _host_threads()
    out, cpu = {}, None
    rec = np.arange(0, 12500, 125)  # 100 sampled neurons (E and I)
    for bits, secs in ((32, seconds), (64, 1)):
        net, p, _ = brunel.build_kernel_network(order=2500, seed=1234)
        obs = net.observe(PopulationView(net, rec), "V_m", name="taps")
        prog = net.compile("float64" if bits == 64 else "float32", spike_capacity=1 << 23)
        sim, _ = KN.build(p, seed=1234, order=2500, bits=bits)
        sim.set_threads(cores)
        sim.record_v(rec)
        runner = prog.runner()
        v_gpu = runner.simulate(3.0)[obs]["V_m"]            # the first 30 steps
        prog.plan.restore(prog._ck0)
        count = 0
        for _ in range(secs):
            prog.plan.run(10000)
            count += prog.plan.spikes()[0].size
        torch.cuda.synchronize()
        prog.plan.close()
        ref = 0
        v_ref = None
        for s_ in range(secs):
            t0 = time.perf_counter()
            st, _, vv = sim.run(10000, cap=1 << 21)
            wall = time.perf_counter() - t0
            if s_ == 0:
                v_ref = vv[:30]
                if bits == 32:
                    cpu = {"value": round(1.0 / wall, 5), "unit": "x real time", "cores": cores,
                           "kind": "port",
                           "sample": "1000 ms simulated (10 000 steps) of the headline network, "
                                     "float64 oracle, %d threads (per-neuron phases parallel, "
                                     "delivery serial)" % cores}
            ref += st.size
        dv = np.abs(v_gpu - v_ref)
        n = p["NE"] + p["NI"]
        out[f"fp{bits}"] = {"seconds": secs, "rate_hz": round(count / n / secs, 4),
                            "oracle_rate_hz": round(ref / n / secs, 4),
                            "rate_rel_err": round(abs(count - ref) / ref, 5),
                            "v_max_abs_err_mV_30steps": float(dv.max()),
                            "v_rms_err_mV_30steps": float(np.sqrt(np.mean(dv ** 2))),
                            "v_neurons": int(rec.size)}
    out["oracle"] = "float64 C restatement (oracle/), same network realised independently"
    return out, cpu


def sweep_numbers(args):
    """Batched parameter sweep: 256 Brunel instances of uneven sizes in one
    persistent launch, 1 s simulated, FP32, against the FP64 batch of the same
    instances (same connectivity and drives) for the per-instance rate error."""
    import numpy as np
    import torch
    from brainpy.state_b200 import brunel
    specs = brunel.sweep_instances()
    steps = 10000
    out = {}
    for prec in (32, 64):
        t0 = time.perf_counter()
        b, params = brunel.build_batch(specs, precision=prec)
        build_s = time.perf_counter() - t0
        tile, cps, _ = b.tune(pilot_steps=300)
        b.run(steps)
        ms, _ = b.kernel_time()
        cnt = [b.spike_counts(k) for k in range(len(specs))]
        out[prec] = dict(ms=ms, build_s=build_s, shape=b.shape(), cnt=cnt, params=params)
        b.close()
        torch.cuda.synchronize()
    N = sum(s["NE"] + s["NI"] for s in specs)
    edges = sum((s["NE"] + s["NI"]) * (p["CE"] + p["CI"]) for s, p in zip(specs, out[32]["params"]))
    r32, r64, ev = [], [], 0.0
    for k, (s, p) in enumerate(zip(specs, out[32]["params"])):
        n = s["NE"] + s["NI"]
        c32, c64 = out[32]["cnt"][k], out[64]["cnt"][k]
        r32.append(c32.sum() / n)
        r64.append(c64.sum() / n)
        # out-degree of an E (I) neuron: n * CE / NE (n * CI / NI)
        ev += c32[:s["NE"]].sum() * n * p["CE"] / s["NE"] + c32[s["NE"]:].sum() * n * p["CI"] / s["NI"]
    r32, r64 = np.array(r32), np.array(r64)
    err = np.abs(r32 - r64) / np.maximum(r64, 1e-12)
    ms32 = out[32]["ms"]
    # per-instance rate error of the FP32 batch against the float64 oracle on
    # the same instance (connectivity, drive stream and V_m), for instances
    # spread over the size range (the oracle cannot run all 256 in minutes)
    from oracle import sweep_net
    order = np.argsort([s["NE"] for s in specs])
    pick = order[np.linspace(0, len(specs) - 1, 8).astype(int)]
    orc = []
    for k in pick:
        osim, _ = sweep_net.build(specs[k], threads=_host_threads())
        ref = osim.run(steps, cap=1 << 23)[0].size
        n = specs[k]["NE"] + specs[k]["NI"]
        orc.append({"instance": int(k), "N": int(n), "rate_hz_fp32": round(float(r32[k]), 4),
                    "rate_hz_oracle": round(ref / n, 4),
                    "rel_err": round(abs(float(r32[k]) * n - ref) / max(ref, 1), 5)})
    orc_err = np.array([o["rel_err"] for o in orc])
    return {"workload": "256 Brunel instances, NE~U[500,8000], NI=NE/4, eps=0.1, g~U[3,8], "
                        "eta~U[0.9,4], delay 1.5 ms, 1000 ms each, one persistent launch",
            "neurons": int(N), "edges": int(edges),
            "neuron_updates_per_s": round(N * steps / (ms32 / 1000.0), 1),
            "syn_events_per_s": round(ev / (ms32 / 1000.0), 1),
            "ms_per_simulated_s": round(ms32, 3), "ms_fp64": round(out[64]["ms"], 3),
            "shape_fp32": out[32]["shape"], "build_s": round(out[32]["build_s"], 3),
            "rate_hz_median": round(float(np.median(r64)), 3),
            "rate_rel_err_median": round(float(np.median(err)), 5),
            "rate_rel_err_max": round(float(err.max()), 5),
            "within_1pct": int((err <= 0.01).sum()), "within_5pct": int((err <= 0.05).sum()),
            "vs_oracle": {"instances": orc, "rel_err_median": round(float(np.median(orc_err)), 5),
                          "rel_err_max": round(float(orc_err.max()), 5),
                          "oracle": "float64 oracle, same instance realised independently, "
                                    "1000 ms"},
            "vs_fp64_note": "rate_rel_err_* compare the FP32 batch with the FP64 batch of the "
                            "same 256 instances"}


def sweep_sharded(rank, world):
    """The sweep batch sharded by instance over the ranks: each rank runs its
    longest-processing-time share of the 256 instances (cost ~ n^2, the edge
    count at fixed connection probability) in one persistent launch, with no
    collective on the data path; the job's time is the slowest rank's."""
    from brainpy.state_b200 import brunel
    from brainpy.state_b200 import dist as D
    specs = brunel.sweep_instances()
    costs = [float(s["NE"] + s["NI"]) ** 2 for s in specs]
    mine = D.shard_instances(costs, rank, world)
    steps = 10000
    b, _ = brunel.build_batch([specs[i] for i in mine], precision=32)
    b.tune(pilot_steps=300)
    b.run(steps)
    ms, _ = b.kernel_time()
    b.close()
    n_local = sum(specs[i]["NE"] + specs[i]["NI"] for i in mine)
    ms_max = D.max_over_ranks(ms)
    n_all = D.sum_over_ranks(n_local)
    inst_all = D.sum_over_ranks(len(mine))
    return {"workload": "the 256-instance sweep of sweep_batch, sharded by instance over "
                        f"{world} GPUs (LPT on n^2), 1000 ms each, FP32",
            "instances": int(inst_all), "instances_rank0": len(mine),
            "ms_per_simulated_s": round(ms_max, 3),
            "neuron_updates_per_s": round(n_all * steps / (ms_max / 1000.0), 1),
            "scaling": "strong", "collectives": "timing reductions only"}


def adex_numbers(args):
    """The AdEx conductance network with plasticity (16 000 E + 4 000 I
    aeif_cond_alpha, RKF45 tolerance 1e-6, 40 M lognormal conductance edges of
    which 25.6 M are plastic E->E stdp_synapse, 5 kHz drive), 2000 ms in FP32
    through Simulator.simulate, timed on the device (all kernels of the run)."""
    from brainpy.state_b200 import adex_net
    from brainpy.state_b200.units import ms
    t0 = time.perf_counter()
    sim, h = adex_net.build(scale=1.0, precision=32, n_record=200)
    res = sim.simulate(2000.0 * ms)
    wall = time.perf_counter() - t0
    kms, launches = sim._plan.kernel_time()
    spk = res.spikes(h["rec"])
    par = adex_parity()
    return {"workload": "16000E+4000I aeif_cond_alpha, in-degree 1600 E + 400 I, lognormal "
                        "weights (ln 1 nS, 0.5), E->E stdp_synapse (25.6 M edges), 5 kHz drive "
                        "of 6 nS, RKF45 tol 1e-6, 2000 ms, FP32 state and stages / FP64 error control",
            "parity": par,
            "ms_per_simulated_s": round(kms / 2.0, 2),
            "rtf": round(2000.0 / kms, 4),
            "rate_hz_sampled": round(float(spk.sum()) / spk.shape[1] / 2.0, 3),
            "rk_substeps_per_neuron_step": round(
                sim._plan.rk_substeps() / float((h["NE"] + h["NI"]) * 20000), 3),
            "build_and_run_wall_s": round(wall, 2)}


def adex_parity(scale=0.1, seconds=1):
    """The same AdEx + STDP network at `scale` (NE = 16000 scale, in-degrees
    10 %), FP32 on the GPU against the float64 oracle on the same realised
    network (oracle/mirror.py): population rate over `seconds` s and the mean
    E->E weight at the end."""
    from brainpy.state_b200 import adex_net
    from brainpy.state_b200.units import ms
    from oracle import mirror
    sim, h = adex_net.build(scale=scale, precision=32)
    sim.simulate(0.0 * ms)
    osim, pids = mirror.from_simulator(sim, threads=_host_threads())
    n = h["NE"] + h["NI"]
    res = sim.cont(seconds * 1000.0 * ms)
    count = float(res.spikes(h["rec"]).sum())
    w_gpu = sim._plan.weights(h["ee"].proj_id)
    t0 = time.perf_counter()
    ref = 0
    for _ in range(seconds):
        ref += osim.run(10000, cap=1 << 22)[0].size
    wall = time.perf_counter() - t0
    w_ref = osim.weights(pids[0], w_gpu.size)
    return {"scale": scale, "neurons": n, "seconds": seconds,
            "rate_hz": round(count / n / seconds, 4), "oracle_rate_hz": round(ref / n / seconds, 4),
            "rate_rel_err": round(abs(count - ref) / max(ref, 1), 5),
            "mean_ee_weight_nS": float(w_gpu.mean()),
            "oracle_mean_ee_weight_nS": float(w_ref.mean()), "oracle_wall_s": round(wall, 2)}


def bptt_numbers(args):
    """Gradient training workload: loss + gradient through the hand-written
    adjoint (800 E + 200 I iaf_psc_exp, batch 64, 1000 steps, checkpoint 50),
    and its finite-difference agreement on 64 random weights (FP64, relaxed
    forward, 200 steps)."""
    import numpy as np
    import torch
    from brainpy.state_b200.autograd import LifAdjoint
    from brainpy.state_b200.lif_task import make_task
    T = make_task()
    res = {"workload": "800E+200I iaf_psc_exp, 10% recurrent, 100 Poisson inputs, batch 64, "
                       "1000 steps dt=1 ms, 10 readouts, fast-sigmoid slope 25/mV, checkpoint 50"}
    for prec in (32, 64):
        dt = torch.float64 if prec == 64 else torch.float32
        adj = LifAdjoint(T["cfg"], T["row_ptr"], T["col"], precision=prec, ckpt_every=50)
        w = torch.tensor(T["w"], dtype=dt, device="cuda")
        wi = torch.tensor(T["w_in"], dtype=dt, device="cuda")
        inp = torch.tensor(T["inputs"], dtype=torch.uint8, device="cuda")
        tg = torch.tensor(T["targets"], dtype=dt, device="cuda")
        def timed():
            for _ in range(2):
                adj.forward(w, wi, inp, tg)
                adj.backward()
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            k = 3
            fw = bw = 0.0
            for _ in range(k):
                ev[0].record()
                adj.forward(w, wi, inp, tg)
                ev[1].record()
                adj.backward()
                ev[2].record()
                torch.cuda.synchronize()
                fw += ev[0].elapsed_time(ev[1])
                bw += ev[1].elapsed_time(ev[2])
            return fw / k, bw / k

        fw, bw = timed()
        res[f"fp{prec}"] = {"forward_ms": round(fw, 3), "backward_ms": round(bw, 3),
                            "grads_per_s": round(1000.0 / (fw + bw), 3),
                            "trial_steps_per_s": round(64 * 1000 * 1000.0 / (fw + bw), 1),
                            "weight_gradients": "contraction" if adj.contraction
                            else "read-modify-write"}
        if adj.contraction:
            # the same backward with per-trial read-modify-writes of the gradients
            adj.contraction = False
            res[f"fp{prec}"]["backward_ms_read_modify_write"] = round(timed()[1], 3)
            adj.contraction = True
        adj.close()
    # finite differences on 64 random weights (32 recurrent, 32 input) at the
    # configured 1000 steps, FP64, relaxed forward with t_ref = 0 (smooth in
    # the weights): central differences with the configuration's h = 1e-3 and
    # with h = 1e-5 (inside the linear range of the relaxed soft reset)
    params = list(T["cfg"]["params"])
    params[3] = 0.0
    Tf = make_task(relaxed=True, params=params, n_steps=1000)
    adj = LifAdjoint(Tf["cfg"], Tf["row_ptr"], Tf["col"], precision=64, ckpt_every=50)
    w = torch.tensor(Tf["w"], dtype=torch.float64, device="cuda")
    wi = torch.tensor(Tf["w_in"], dtype=torch.float64, device="cuda")
    inp = torch.tensor(Tf["inputs"], dtype=torch.uint8, device="cuda")
    tg = torch.tensor(Tf["targets"], dtype=torch.float64, device="cuda")
    adj.forward(w, wi, inp, tg)
    dw, dwi = adj.backward()
    dw, dwi = dw.cpu().numpy(), dwi.cpu().numpy().reshape(-1)
    rng = np.random.default_rng(7)
    picks = [(w, dw, q) for q in rng.choice(w.numel(), 32, replace=False)] + \
            [(wi.reshape(-1), dwi, q) for q in rng.choice(wi.numel(), 32, replace=False)]
    fd = {}
    for h in (1e-3, 1e-5):
        a_, f_ = [], []
        for arr, grad, q in picks:
            wp = arr.clone()
            wp[q] += h
            lp = float(adj.forward(*((wp, wi) if arr is w else (w, wp.reshape(wi.shape))), inp, tg))
            wp[q] -= 2 * h
            lm = float(adj.forward(*((wp, wi) if arr is w else (w, wp.reshape(wi.shape))), inp, tg))
            a_.append(grad[q])
            f_.append((lp - lm) / (2 * h))
        a_, f_ = np.array(a_), np.array(f_)
        rel = np.abs(a_ - f_) / np.maximum(np.abs(f_), 1e-3 * np.abs(f_).max())
        fd[f"h={h:g}"] = {"max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
                          "within_1e-3": int((rel <= 1e-3).sum())}
    res["fd_check"] = {"weights": 64, "steps": 1000, "batch": 64, "precision": "fp64",
                       "forward": "relaxed, t_ref = 0", **fd}
    adj.close()
    return res


def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    """CPU reference arm: the float64 restatement of the reference's step
    (the oracle; the reference itself is JAX, which is not installed) on the
    headline network realised by the oracle alone (no product code is
    imported), timed on all host threads; rank 0 only.  Each step is a
    bounded sample of `--ref-sample-ms` of simulated time (the repo arm's step
    is 1000 ms); the metric is the same real-time factor."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import kernel_net as KN
    p = KN.brunel_params(2500)
    sim, _ = KN.build(p, seed=1234, order=2500, bits=32)
    cores = _host_threads()
    sim.set_threads(cores)
    sample_ms = float(args.ref_sample_ms)
    n = int(round(sample_ms / 0.1))
    for _ in range(args.warmup):
        sim.run(min(n, 1000), cap=5_000_000)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sim.run(n, cap=5_000_000)
        times.append(time.perf_counter() - t0)
    wall = sum(times) / len(times)
    rtf = (sample_ms / 1000.0) / wall
    N = p["NE"] + p["NI"]
    edges = N * (p["CE"] + p["CI"])
    res = {"impl": "reference", "metric": METRIC, "value": round(rtf, 5),
           "unit": "x real time (simulated s / wall s)", "n_gpus": int(args.gpus),
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(wall * 1000, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded Brunel network, the reference kernel path's streams)",
           "config": CONFIG_HEADLINE(N, p, edges, 1000.0, int(args.gpus)),
           "reference_sample": f"each step times {sample_ms:.0f} ms simulated "
                               f"({n} time steps) of the same network",
           "cpu_baseline": {"value": round(rtf, 5), "unit": "x real time", "cores": cores,
                            "kind": "port",
                            "sample": f"{sample_ms:.0f} ms simulated per step, float64 "
                                      f"oracle restatement, {cores} threads (the reference is "
                                      "JAX, not installable here)"},
           "e2e": {"value": round(rtf, 5), "unit": "x real time (simulated s / wall s)",
                   "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(res), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quick", action="store_true", help="FP32 headline only")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the sweep-batch and gradient sections")
    ap.add_argument("--sim-ms", type=float, default=1000.0,
                    help="simulated time per bench step (default one second)")
    ap.add_argument("--ref-sample-ms", type=float, default=250.0,
                    help="reference arm: simulated time per timed step")
    args = ap.parse_args()
    global STEPS_PER_BENCH_STEP
    STEPS_PER_BENCH_STEP = int(round(args.sim_ms / 0.1))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
