"""Benchmark of the B200-native RK3 dycore step (cell-substeps/s).

Default workload (N=1): the real-like moist synthetic case at 433 x 433 x 50
(dx 1 km, top 20 km, seeded k^-2 terrain 0-3 km, theta 295 K + N=0.011,
5->20 m/s shear + noise, qv/qc/qr, specified lateral boundaries,
moist_adv_opt 1, dt 6 s, 6 acoustic substeps = 10 substeps per RK3 step).
Each timed step is one full RK3 step of that workload from the same resident
input carry (every input array is ~75 MB, far larger than the 126 MB L2 in
aggregate, so no L2 flush is needed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``e2e`` is the same step through the C ABI with host buffers: every step
copies its whole input state (and the boundary strips) from pinned host
memory to the device and reads the advanced state and mudf -- everything the
next step reads -- back, inside the timed region (the variant that also reads
back the carry's diagnostic leaves is reported beside it as
``e2e.full_carry``); the device input and output
sets are double-buffered so that step n+1's input copy and step n's output
copy overlap step n's compute on their own streams, as a caller streaming
cases through the GPU would run it; it runs as many steps as the device-timed
region, with the first input copy and the last output copy (the pipeline's
fill and drain) inside the timed region.  The one-stream serial figure (copy
in, step, copy out) is reported beside it.

Prints ONE JSON line (rank 0).  Beside the float64 step it also times the
mixed-precision variant (FP32 advective fluxes, float64 accumulation) on the
same input and reports it under "mixed" (skip with --no-mixed), and the
cost of the two hand-written adjoints against their forwards at the same grid
under "adjoint" (skip with --no-adjoint), and the step epilogue (guards and
the end-of-step lateral boundary pass) under "epilogue" (skip with
--no-epilogue).  ``--impl reference`` times the reference
algorithm's CPU implementation available here -- the NumPy restatement in
``oracle/`` (JAX, the reference's own runtime, is not installed) -- on the
host cores, on bounded 64 x 64 x 50 samples of the same workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "cell-substeps/s"
NX, NY, NZ = 433, 433, 50
SAMPLE = (64, 64, 50)


def _workload_name(nx, ny, nz, precision):
    return f"real_like_moist_{nx}x{ny}x{nz}_specified_lbc_moist_adv_opt1_dt6_ns6_{precision}"


# ---------------------------------------------------------------------------
# CPU reference arm: the oracle restatement on bounded samples
# ---------------------------------------------------------------------------

def _cpu_worker(args):
    """Run W warm-up + K oracle steps on a bounded sample; return step seconds."""
    nx, ny, nz, steps, warmup, seed = args
    sys.path.insert(0, HERE)
    from types import SimpleNamespace
    from oracle import dycore as D
    from wrf_gpu_b200 import cases
    case = cases.real_like_moist(nx, ny, nz, seed=seed)
    nl = D.Namelist(metrics=case.metrics, **case.controls)
    carry0 = SimpleNamespace(state=case.state, mudf=case.mudf)
    with np.errstate(all="ignore"):
        for _ in range(warmup):
            D.rk_scan_step(carry0, nl, lead_seconds=0.0)
        t0 = time.perf_counter()
        for _ in range(steps):
            D.rk_scan_step(carry0, nl, lead_seconds=0.0)
        t1 = time.perf_counter()
    return t1 - t0


def cpu_reference(steps, warmup, procs):
    import multiprocessing as mp
    nx, ny, nz = SAMPLE
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        times = pool.map(_cpu_worker, [(nx, ny, nz, steps, warmup, i) for i in range(procs)])
    tmax = max(times)
    units = procs * steps * nx * ny * nz * 10
    return units / tmax, tmax


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def _measured_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    import glob
    import re
    for path in glob.glob(os.path.join(HERE, "profiles", "dram_*.md")):
        with open(path) as f:
            m = re.search(r"traffic_bytes_per_launch %s(?:_tiled)?: (\d+)" % re.escape(kernel), f.read())
        if m:
            return float(m.group(1)), os.path.relpath(path, HERE)
    return None, None


def _peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def max_over_ranks(ms, dist=None, device="cpu"):
    """The largest of each rank's duration, returned on every rank (ranks
    are replicas: the job takes as long as its slowest rank)."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(ms, world, cells, nsub, steps):
    """Whole-job cell-substeps/s of `world` replicas each advancing `cells`
    cells through `steps` RK3 steps of `nsub` substeps in `ms` (the max over
    ranks)."""
    return world * cells * nsub * steps / (ms / 1000.0)


def run_gpu(args, rank, world, local_rank):
    import torch
    from wrf_gpu_b200 import build, cases, dycore, perfmodel, _capi
    build.build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nx, ny, nz = args.nx, args.ny, args.nz
    case = cases.real_like_moist(nx, ny, nz, seed=rank)
    nl = dycore.OperationalNamelist.from_case(case, device=dev, precision=args.precision)
    carry = dycore.carry_from_case(case, device=dev)
    stp = dycore.Stepper(nl, device=dev)
    out = stp.alloc_carry(carry)
    stream = torch.cuda.current_stream(dev)
    tuned = stp.autotune(carry, out) if not args.no_tune else (0, 0, 0)
    ns = nl.acoustic_substeps
    nsub = perfmodel.substeps_per_step(ns)
    cells = nx * ny * nz

    def step():
        stp.step_into(carry, out, lead_seconds=0.0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    # capture one step in a CUDA graph (launch-bound overhead removed)
    graph = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream(dev)
    s.wait_stream(stream)
    with torch.cuda.stream(s):
        step()
    stream.wait_stream(s)
    torch.cuda.synchronize(dev)
    with torch.cuda.graph(graph):
        step()
    graph.replay()
    torch.cuda.synchronize(dev)

    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local_rank)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    if dist is not None:
        dist.barrier()
    ms_per_step = ms / args.steps
    value = replica_throughput(ms, world, cells, nsub, args.steps)

    # per-kernel timing over a second, instrumented region of the same steps
    _capi.profile_enable(True, max_records=stp.launches_per_step * args.steps + 16)
    for _ in range(args.steps):
        step()
    prof = _capi.profile_read()
    _capi.profile_enable(False)
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_n) = dom
    hbm, peak_src = _peaks()
    bpl = perfmodel.kernel_bytes_per_launch(dom_name, nx, ny, nz, damp_opt=nl.damp_opt)
    roof = None
    if bpl is not None and dom_n:
        achieved = bpl / (dom_ms / dom_n / 1000.0) / 1e9
        roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1), "peak": hbm,
                "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "bytes_per_launch": bpl, "avg_launch_ms": round(dom_ms / dom_n, 4),
                "traffic": None, "kernel_share": round(dom_ms / sum(v[0] for v in prof.values()), 4)}
        traffic, src = _measured_traffic(dom_name)
        if traffic is not None:
            roof["traffic"] = traffic
            roof["traffic_source"] = f"ncu dram__bytes_read.sum + dram__bytes_write.sum, {src}"
    step_bytes = perfmodel.step_bytes(nx, ny, nz, ns, moist=True)
    whole = {"bytes_per_step": step_bytes, "achieved_gbs": round(step_bytes / (ms_per_step / 1000.0) / 1e9, 1),
             "frac": round(step_bytes / (ms_per_step / 1000.0) / 1e9 / hbm, 4)}
    kernels = {k: {"ms_per_step": round(v[0] / args.steps, 4), "launches_per_step": v[1] // args.steps}
               for k, v in prof.items() if v[1]}

    # end to end through the C ABI with host buffers (pinned), copies timed
    host_in = {}
    for f in ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation", "mu_total",
              "mu_perturbation", "qv", "qc", "qr", "qi", "qs", "qg", "u_bdy", "v_bdy"):
        host_in[f] = getattr(carry.state, f).cpu().pin_memory()
    host_in["mudf"] = carry.mudf.cpu().pin_memory()
    state_fields = ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation", "mu_total",
                    "mu_perturbation", "qv", "qc", "qr", "qi", "qs", "qg")
    # read back every step: the advanced state and mudf -- what the next step
    # reads; the carry's diagnostic leaves (t_2ave, ww, muave, muts, ph_tend,
    # the saves) are read back too in the full-carry variant reported beside it
    diag_fields = tuple(f for f in _capi.CARRY_OUT_FIELDS if f != "mudf")
    out_tensors = [getattr(out.state, f) for f in state_fields] + [out.mudf]
    out_full = out_tensors + [getattr(out, f) for f in diag_fields]
    host_full = [torch.empty(t.shape, dtype=t.dtype).pin_memory() for t in out_full]
    host_out = host_full[:len(out_tensors)]
    h2d = sum(t.numel() * 8 for t in host_in.values())
    d2h = sum(t.numel() * 8 for t in host_out)
    d2h_full = sum(t.numel() * 8 for t in host_full)

    def e2e_step():
        for f, h in host_in.items():
            dst = carry.mudf if f == "mudf" else getattr(carry.state, f)
            dst.copy_(h, non_blocking=True)
        step()
        for h, t in zip(host_out, out_tensors):
            h.copy_(t, non_blocking=True)

    def _max_over_ranks(ms):
        return max_over_ranks(ms, dist, dev)

    # (a) serial: copy in, step, copy out on one stream
    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    torch.cuda.synchronize(dev)
    # as many steps as the device-timed region (at least 3): the first
    # step's input copy and the last step's output copy are not overlapped
    # with any compute, and stay inside the timed region
    k_e2e = max(3, args.steps)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(k_e2e):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize(dev)
    serial_ms = _max_over_ranks(f0.elapsed_time(f1))

    # (b) streaming: the same per-step copies (every step copies its whole
    # input state in and its whole output state out), double-buffered on the
    # device so that step n+1's input copy and step n's output copy overlap
    # step compute on their own streams (PCIe is full duplex)
    carry_b = dycore.carry_from_case(case, device=dev)
    out_b = stp.alloc_carry(carry_b)
    graph_b = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph_b):
        stp.step_into(carry_b, out_b, lead_seconds=0.0)
    torch.cuda.synchronize(dev)
    out_full_b = [getattr(out_b.state, f) for f in state_fields] + [out_b.mudf] + [getattr(out_b, f)
                                                                                 for f in diag_fields]
    bufs = [(carry, out_full, graph), (carry_b, out_full_b, graph_b)]
    s_in = torch.cuda.Stream(dev)
    s_out = torch.cuda.Stream(dev)

    def streamed(nsteps, t0=None, t1=None, full=False):
        nout = len(host_full) if full else len(host_out)
        torch.cuda.synchronize(dev)
        if t0 is not None:
            t0.record(s_in)
        done = []
        for n in range(nsteps):
            cb, ob, gb = bufs[n % 2]
            with torch.cuda.stream(s_in):
                if n >= 2:
                    s_in.wait_event(done[n - 2][0])  # step n-2 has read this input set
                for f, h in host_in.items():
                    dst = cb.mudf if f == "mudf" else getattr(cb.state, f)
                    dst.copy_(h, non_blocking=True)
                in_ev = torch.cuda.Event()
                in_ev.record(s_in)
            stream.wait_event(in_ev)
            if n >= 2:
                stream.wait_event(done[n - 2][1])  # step n-2's outputs are copied out
            gb.replay()
            st_ev = torch.cuda.Event()
            st_ev.record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(st_ev)
                for h, t in zip(host_full[:nout], ob[:nout]):
                    h.copy_(t, non_blocking=True)
                out_ev = torch.cuda.Event()
                out_ev.record(s_out)
            done.append((st_ev, out_ev))
        if t1 is not None:
            t1.record(s_out)
        torch.cuda.synchronize(dev)

    streamed(2)
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    streamed(k_e2e, g0, g1)
    e2e_ms = _max_over_ranks(g0.elapsed_time(g1))
    e2e_value = replica_throughput(e2e_ms, world, cells, nsub, k_e2e)
    streamed(k_e2e, g0, g1, full=True)
    full_ms = _max_over_ranks(g0.elapsed_time(g1))
    del graph_b, bufs
    out_ok = bool(torch.isfinite(out.state.w).all().item() and torch.isfinite(out.state.theta).all().item())
    del graph

    # the mixed-precision variant (FP32 advective fluxes, float64 accumulation)
    # on the same input, timed the same way, beside the float64 line
    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        nl_m = dycore.OperationalNamelist.from_case(case, device=dev, precision="mixed")
        stp_m = dycore.Stepper(nl_m, device=dev)
        out_m = stp_m.alloc_carry(carry)
        stp_m.params.march_levels, stp_m.params.column_lanes = stp.params.march_levels, stp.params.column_lanes
        stp_m.params.column_width = stp.params.column_width

        def step_m():
            stp_m.step_into(carry, out_m, lead_seconds=0.0)

        for _ in range(args.warmup):
            step_m()
        torch.cuda.synchronize(dev)
        graph_m = torch.cuda.CUDAGraph()
        s2 = torch.cuda.Stream(dev)
        s2.wait_stream(stream)
        with torch.cuda.stream(s2):
            step_m()
        stream.wait_stream(s2)
        torch.cuda.synchronize(dev)
        with torch.cuda.graph(graph_m):
            step_m()
        graph_m.replay()
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            graph_m.replay()
        g1.record(stream)
        torch.cuda.synchronize(dev)
        ms_m = max_over_ranks(g0.elapsed_time(g1), dist, dev)
        # one-step difference from the float64 step on this workload
        diff = {}
        for f in ("u", "v", "w", "theta"):
            a, b = getattr(out_m.state, f), getattr(out.state, f)
            diff[f] = float((a - b).abs().max().item() / max(b.abs().max().item(), 1e-300))
        mixed = {"value": replica_throughput(ms_m, world, cells, nsub, args.steps), "unit": METRIC,
                 "ms_per_step": ms_m / args.steps, "dtype": "f32 fluxes / f64 accumulation",
                 "rel_diff_vs_fp64_one_step": diff,
                 "error_60_steps": (mixed_sixty_step_error(args.nx, args.ny, args.nz, dev)
                                    if rank == 0 and world == 1 and not args.no_mixed60 else None),
                 "stated_error": "60 forecast steps of this workload (specified-boundary cadence, step + "
                                 "end-of-step boundary pass): within 2x the float64 trajectory's own one-ulp "
                                 "spread per field, max-abs and rms (tests/test_gpu_mixed.py); <= 1e-5 on "
                                 "u, v, w, theta after 60 steps of the smooth 3-D warm bubble vs the oracle"}
        del graph_m
    return dict(value=value, ms_per_step=ms_per_step, clocks=clk, roofline=roof, whole_step_roofline=whole,
                kernels=kernels, e2e={"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                                      "d2h_bytes_per_step": d2h, "steps": k_e2e, "ms_per_step": e2e_ms / k_e2e,
                                      "copies": "every step copies its whole input state and strips "
                                                "host->device and reads back the advanced state and mudf (the "
                                                "next step's inputs) device->host, pinned; double-buffered so "
                                                "copies overlap compute on separate streams; the timed "
                                                "region includes the pipeline's fill (the first step's input "
                                                "copy) and drain (the last step's output copy)",
                                      "full_carry": {"d2h_bytes_per_step": d2h_full,
                                                     "ms_per_step": full_ms / k_e2e,
                                                     "value": replica_throughput(full_ms, world, cells, nsub,
                                                                                 k_e2e),
                                                     "what": "the same with the carry's diagnostic leaves "
                                                             "(t_2ave, ww, muave, muts, ph_tend, saves) read "
                                                             "back too"},
                                      "serial_ms_per_step": serial_ms / k_e2e,
                                      "serial_value": replica_throughput(serial_ms, world, cells, nsub, k_e2e)},
                launches=stp.launches_per_step * args.steps, finite=out_ok, mixed=mixed,
                adjoint=adjoint_ratios(case, dev) if not args.no_adjoint else None,
                epilogue=epilogue_cost(case, dev) if not args.no_epilogue else None,
                tuned={"march_levels": tuned[0], "column_lanes": tuned[1], "column_width": tuned[2]})


def mixed_sixty_step_error(nx, ny, nz, dev, nsteps=60):
    """The mixed variant's difference from the float64 trajectory after 60
    forecast steps of the workload under the WRF specified-boundary cadence
    (RK3 step + guards + end-of-step boundary pass each step), with the
    float64 trajectory's own spread when its initial theta moves by one ulp
    (this moist flow amplifies any rounding difference), relative max-abs and
    rms on u, v, w, theta."""
    import torch
    from wrf_gpu_b200 import cases, dycore

    def run(precision, ulp=False):
        case = cases.with_full_leaves(cases.real_like_moist(nx, ny, nz))
        case.controls["specified_bdy_cadence"] = True
        if ulp:
            case.state.theta = np.nextafter(case.state.theta, np.inf)
        nl = dycore.OperationalNamelist.from_case(case, device=dev, precision=precision)
        c = dycore.carry_from_case(case, device=dev)
        for n in range(nsteps):
            c, _ = dycore.forecast_step(c, nl, n)
        torch.cuda.synchronize(dev)
        return {f: getattr(c.state, f).cpu().numpy() for f in ("u", "v", "w", "theta")}

    ref, mix, ulp = run("fp64"), run("mixed"), run("fp64", ulp=True)
    mx = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    rms = lambda a, b: float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b * b)), 1e-300))
    return {"steps": nsteps, "max_abs": {f: mx(mix[f], ref[f]) for f in ref},
            "rms": {f: rms(mix[f], ref[f]) for f in ref},
            "fp64_one_ulp_spread_max_abs": {f: mx(ulp[f], ref[f]) for f in ref},
            "fp64_one_ulp_spread_rms": {f: rms(ulp[f], ref[f]) for f in ref},
            "finite": bool(all(np.isfinite(v).all() for v in ref.values()))}


def adjoint_ratios(case, dev, reps=10):
    """Adjoint / forward cost of the two hand-written adjoints at the workload's
    grid (doubly periodic operators): the acoustic substep's VJP against one
    forward substep, and the scalar-advection adjoint against its forward.
    Operator inputs are synthesised from the workload state (timing does not
    depend on the values): the stage's transport velocities, masses, pressure
    and geopotential, unit moisture factors and a uniform tridiagonal
    factorisation."""
    import ctypes

    import torch
    from wrf_gpu_b200 import _capi, adjoint, dycore
    nl = dycore.OperationalNamelist.from_case(case, device=dev, run_boundary=False, bc_source="ideal")
    st = dycore.State.from_host(case.state, device=dev)
    nz, ny, nx = st.theta.shape
    z = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)
    full = lambda v, *s: torch.full(s, v, dtype=torch.float64, device=dev)
    mu = st.mu_total
    muu = torch.cat([mu[:, :1], 0.5 * (mu[:, 1:] + mu[:, :-1]), mu[:, -1:]], dim=1).contiguous()
    muv = torch.cat([mu[:1], 0.5 * (mu[1:] + mu[:-1]), mu[-1:]], dim=0).contiguous()
    ph = st.ph_total
    consts = {"u_tend": z(nz, ny, nx + 1), "v_tend": z(nz, ny + 1, nx), "t_tend": z(nz, ny, nx),
              "rw_tend": z(nz + 1, ny, nx), "ph_tend": z(nz + 1, ny, nx), "alt": full(1.1, nz, ny, nx),
              "pb": (st.p_total - st.p_perturbation).contiguous(), "c2a": full(1.3e5, nz, ny, nx),
              "cqu": full(1.0, nz, ny, nx + 1), "cqv": full(1.0, nz, ny + 1, nx), "cqw": full(1.0, nz + 1, ny, nx),
              "php": (0.5 * (ph[1:] + ph[:-1])).contiguous(), "pt1": ph.contiguous(),
              "a": full(-0.1, nz + 1, ny, nx), "alpha": full(0.9, nz + 1, ny, nx), "gamma": full(-0.1, nz + 1, ny, nx),
              "ww_1": z(nz + 1, ny, nx), "mut": mu.contiguous(), "muu": muu, "muv": muv,
              "u_1": st.u, "v_1": st.v, "w_save": st.w, "theta": st.theta,
              "phb0": (st.ph_total[0] - st.ph_perturbation[0]).contiguous()}
    op = adjoint.AcousticOp(nl, consts, float(nl.dt_s) / float(nl.acoustic_substeps), device=dev)
    x = [z(nz, ny, nx + 1), z(nz, ny + 1, nx), z(nz + 1, ny, nx), z(nz + 1, ny, nx), z(nz, ny, nx), z(nz, ny, nx),
         st.p_perturbation.clone(), st.p_perturbation.clone(), z(nz, ny, nx), z(nz + 1, ny, nx),
         st.mu_perturbation.clone(), mu.clone(), z(ny, nx), z(ny, nx)]
    co = [torch.randn_like(t) for t in x]
    xo = [t.clone() for t in x]
    op.forward_(xo)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    xs = [t.clone() for t in x]
    f_ms = timed(lambda: op.forward_(xs))
    vs_ms = timed(lambda: op.vjp(x, co, xo))
    vr_ms = timed(lambda: op.vjp(x, co))
    aop = adjoint._Op(nl)
    q = st.theta.clone()
    ru, rv = torch.randn_like(q) * 5.0e4, torch.randn_like(q) * 5.0e4
    rom = torch.randn(nz + 1, ny, nx, dtype=torch.float64, device=dev) * 1.0e3
    tend = torch.empty_like(q)
    af = timed(lambda: aop.apply("wrfgpu_scalar_advection", q, ru, rv, rom, tend))
    ab = timed(lambda: aop.apply("wrfgpu_scalar_advection_adjoint", q, ru, rv, rom, tend))
    ru_bar, rv_bar, rom_bar = torch.empty_like(ru), torch.empty_like(rv), torch.empty_like(rom)
    lib = _capi.load()
    sp = torch.cuda.current_stream(dev).cuda_stream
    P = lambda t: ctypes.c_void_p(t.data_ptr())

    q_bar = torch.empty_like(q)

    def full_vjp():
        _capi.check(lib.wrfgpu_scalar_advection_vjp(
            ctypes.byref(aop.params), ctypes.byref(aop.metrics), P(q), P(tend), P(ru), P(rv), P(rom), P(q_bar),
            P(ru_bar), P(rv_bar), P(rom_bar), ctypes.c_void_p(sp)))

    av = timed(full_vjp)
    del op, aop
    return {"acoustic_substep": {"forward_ms": f_ms, "vjp_stored_ms": vs_ms, "vjp_recompute_ms": vr_ms,
                                 "ratio_stored": vs_ms / f_ms, "ratio_recompute": vr_ms / f_ms,
                                 "note": "VJP from a stored checkpoint of the substep output / recomputing it"},
            "scalar_advection": {"forward_ms": af, "adjoint_ms": ab, "ratio": ab / af,
                                 "full_vjp_ms": av, "full_vjp_ratio": av / af,
                                 "note": "adjoint_ms: the cotangent of the advected field alone; full_vjp_ms: "
                                         "those of the field and of ru, rv, rom in one launch"},
            "data": "operator inputs synthesised from the workload state"}


def epilogue_cost(case, dev, reps=20):
    """The step epilogue (guards, full end-of-step boundary pass, guards of the
    bounded state; ``wrfgpu_step_epilogue``) on the workload's state, timed
    with CUDA events over ``reps`` calls.  The strips the workload does not
    carry (p, pb, mub, phb, qv) are synthesised from its own (timing does not
    depend on the values).  Algorithmic bytes: every state field (u, v, w,
    theta, p and p', ph and ph', mu and mu', six species) read once and
    written once, plus the limiter's reduction pass (theta, origin theta and
    mu_total) and the origin theta read again where theta is written; the
    guards' origin reads on offending cells and the strips (0.2 % of it) are
    not counted."""
    import ctypes

    import torch
    from wrf_gpu_b200 import _capi, dycore
    st = dycore.State.from_host(case.state, device=dev)
    nz, ny, nx = st.theta.shape
    tb = st.theta_bdy
    st.p_bdy, st.pb_bdy, st.qv_bdy = torch.zeros_like(tb), torch.full_like(tb, 5.0e4), torch.full_like(tb, 1.0e-3)
    st.mub_bdy, st.phb_bdy = torch.full_like(st.mu_bdy, 9.0e4), torch.full_like(st.ph_bdy, 2.0e4)
    nl = dycore.OperationalNamelist.from_case(case, device=dev, run_boundary=True, bc_source="wrfbdy",
                                              specified_bdy_cadence=False)
    lib = _capi.load()
    p = dycore.step_params(nl)
    n = ctypes.c_size_t(0)
    _capi.check(lib.wrfgpu_step_epilogue_workspace_size(ctypes.byref(p), ctypes.byref(n)))
    ws = torch.empty(n.value + 256, dtype=torch.uint8, device=dev)
    wsp = ctypes.c_void_p((ws.data_ptr() + 255) // 256 * 256)
    raw = torch.empty(_capi.THETA_DIAG_BYTES, dtype=torch.uint8, device=dev)
    ins, out, outs = dycore._state_structs(st)
    org = dycore._inputs_struct(st)
    lv = dycore._leaves_struct(st)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    call = lambda: _capi.check(lib.wrfgpu_step_epilogue(ctypes.byref(p), ctypes.byref(org), ctypes.byref(ins),
                                                        ctypes.byref(lv), ctypes.byref(outs), 1800.0, 0,
                                                        ctypes.c_void_p(raw.data_ptr()), wsp, n.value, sp))
    for _ in range(3):
        call()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        call()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / reps
    m = nz * ny * nx
    sizes = (nz * ny * (nx + 1) + nz * (ny + 1) * nx + (nz + 1) * ny * nx + m + 2 * m + 2 * ny * nx
             + 2 * (nz + 1) * ny * nx + 6 * m)
    nbytes = 8 * (2 * sizes + 3 * m + 2 * ny * nx)
    peak, src = _peaks()
    gbs = nbytes / (ms * 1e-3) / 1e9
    diag = dycore.theta_limiter_diagnostics(raw)
    # launches: the limiter's reduction and scalars, every field's elementwise part, every ring band, the record
    return {"ms": ms, "algorithmic_bytes": nbytes, "achieved_gbs": gbs, "peak_gbs": peak, "peak_source": src,
            "frac": gbs / peak, "launches": 5, "limited_cells": int(diag["theta_limited_cell_count"]),
            "what": "guards + full end-of-step lateral boundary pass + guards of the bounded state "
                    "(operational_mode.py:4950-4983 without physics), one call per rep, inputs larger than L2"}


def run_batched(args):
    """Batched-domains workload (nests and ensemble members in one call):
    a 3-level nest 150x150x45 (dx 9 km, dt 54 s), 301x301x45 (3 km, 18 s),
    433x433x45 (1 km, 6 s) and 16 members of 129x129x45 (1 km, seeded), each
    advanced one RK3 step per call by wrfgpu_rk3_step_batched, captured in
    one CUDA graph; compared with the same members stepped one after another.
    Parent-child nest coupling is not part of the step, so the nest levels are
    independent members here (the 3:1 time-step ratio is not sub-cycled)."""
    import torch
    from wrf_gpu_b200 import build, cases, dycore, perfmodel
    build.build()
    dev = torch.device("cuda", 0)
    specs = [(150, 150, 45, 9000.0, 54.0, 0), (301, 301, 45, 3000.0, 18.0, 1), (433, 433, 45, 1000.0, 6.0, 2)]
    specs += [(129, 129, 45, 1000.0, 6.0, 10 + m) for m in range(16)]
    members = [cases.real_like_moist(nx, ny, nz, dx=dx, dt=dt, seed=sd) for nx, ny, nz, dx, dt, sd in specs]
    nls = [dycore.OperationalNamelist.from_case(c, device=dev) for c in members]
    carries = [dycore.carry_from_case(c, device=dev) for c in members]
    bs = dycore.BatchStepper(nls, device=dev)
    outs = bs.alloc_carries(carries)
    stream = torch.cuda.current_stream(dev)
    cell_substeps = sum(c.nx * c.ny * c.nz * perfmodel.substeps_per_step(nl.acoustic_substeps)
                        for c, nl in zip(members, nls))
    for _ in range(args.warmup):
        bs.step_into(carries, outs, lead_seconds=0.0)
    torch.cuda.synchronize(dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        bs.step_into(carries, outs, lead_seconds=0.0)
    graph.replay()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_b = e0.elapsed_time(e1) / args.steps
    e0.record(stream)
    for _ in range(args.steps):
        for st, c, o in zip(bs.steppers, carries, outs):
            st.step_into(c, o, lead_seconds=0.0)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_s = e0.elapsed_time(e1) / args.steps
    del graph
    line = {"metric": METRIC, "value": cell_substeps / (ms_b / 1000.0), "unit": METRIC, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched_nest3_ens16_nz45", "members": len(members),
                       "cells": sum(c.nx * c.ny * c.nz for c in members), "cuda_graph": True},
            "sequential": {"value": cell_substeps / (ms_s / 1000.0), "ms_per_step": ms_s}}
    print(json.dumps(line))
    return 0


def run_sharded(args, rank, world, local_rank):
    """The workload split into y slabs (``wrf_gpu_b200.sharding``): with
    ``--shard`` under torchrun one slab per rank, halo blocks swapped over
    NCCL after each step (strong scaling of the one domain); with
    ``--slabs K`` on one GPU, K slabs driven from one process (the halo
    hand-over is a pack / unpack on the device), which measures what a
    slab step and the exchange's packing cost.  Timed: whole RK3 steps of
    every slab plus the exchange; the exchange alone is timed beside it."""
    import torch
    from wrf_gpu_b200 import build, cases, dycore, perfmodel, sharding
    build.build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nx, ny, nz = args.nx, args.ny, args.nz
    # every strip of the end-of-step boundary pass, from the initial edge rows
    case = cases.with_full_leaves(cases.real_like_moist(nx, ny, nz, seed=0))
    # a forecast over several steps runs with WRF's specified-boundary cadence
    case.controls["specified_bdy_cadence"] = True
    nl = dycore.OperationalNamelist.from_case(case, device=dev)
    carry = dycore.carry_from_case(case, device=dev)
    stream = torch.cuda.current_stream(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        drv = sharding.DistributedSlab(nl, boundary_pass=True)
        slabs = [drv.slab]
        nslab = world
    else:
        drv = sharding.SlabRing(nl, max(1, args.slabs), boundary_pass=True)
        slabs = drv.slabs
        nslab = len(slabs)
    drv.load(carry)
    nsub = perfmodel.substeps_per_step(nl.acoustic_substeps)
    dt = nl.dt_s
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the same forecast steps on the whole domain (RK3 step + end-of-step boundary pass), for the
    # cost of the halo rows
    whole_ms, whole_finite = None, None
    if world == 1:
        from dataclasses import replace as _replace
        nl_pass = _replace(nl, disable_guards=True)
        c = carry
        for i in range(args.warmup + args.steps):
            if i == args.warmup:
                e0.record(stream)
            nxt = dycore.rk_scan_step(c, nl, lead_seconds=(i + 1) * dt)
            st, _ = dycore.step_epilogue(nxt.state, c.state, (i + 1) * dt, nl_pass)
            c = nxt.replace(state=st)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        whole_ms = e0.elapsed_time(e1) / args.steps
        whole_finite = bool(torch.isfinite(c.state.w).all().item())
        del c, nxt
    del carry
    for i in range(args.warmup):
        drv.step((i + 1) * dt)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    e0.record(stream)
    for i in range(args.steps):
        drv.step((args.warmup + i + 1) * dt)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    # the exchange alone: pack every slab's send blocks and unpack them into its neighbours
    e0.record(stream)
    for i in range(args.steps):
        drv.exchange()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ex_ms = max_over_ranks(e0.elapsed_time(e1), dist, dev) / args.steps
    L = slabs[0].layout
    send_bytes = sum(b.numel() * 8 for b in slabs[0].pack())
    finite = bool(all(torch.isfinite(s.carry.state.w).all().item() for s in slabs))
    if dist is not None:
        dist.barrier()
    line = {"metric": METRIC, "value": nx * ny * nz * nsub * args.steps / (ms / 1000.0), "unit": METRIC,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong" if world > 1 else "none", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": _workload_name(nx, ny, nz, "fp64"), "nx": nx, "ny": ny, "nz": nz,
                       "parallelism": f"y-slabs x{nslab}" + (" over NCCL" if world > 1 else " in one process"),
                       "halo_rows": L.halo, "rows_per_slab": L.n_local, "owned_rows": L.own,
                       "stepped_over_owned": round(L.n_local * nslab / ny, 3)},
            "exchange": {"ms_per_step": ex_ms, "bytes_sent_per_slab_step": send_bytes,
                         "what": "pack + unpack" + (" + NCCL send/recv" if world > 1 else " (no transfer)")},
            "step": "RK3 step + end-of-step lateral boundary pass per slab, forecast leads",
            "whole_domain_ms_per_step": whole_ms, "whole_domain_finite": whole_finite, "finite": finite}
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_profile_target(args):
    """A few plain RK3 steps of the workload (the target of ncu captures)."""
    import torch
    from wrf_gpu_b200 import build, cases, dycore
    build.build()
    case = cases.real_like_moist(args.nx, args.ny, args.nz, specified=not args.periodic)
    case.controls["diff_6th_opt"] = args.diff_6th
    nl = dycore.OperationalNamelist.from_case(case, precision=args.precision)
    stp = dycore.Stepper(nl)
    stp.params.column_width = args.column_width
    carry = dycore.carry_from_case(case)
    out = stp.alloc_carry(carry)
    for _ in range(args.profile_steps):
        stp.step_into(carry, out, lead_seconds=0.0)
    torch.cuda.synchronize()
    print("ok", float(out.state.w.abs().max().item()))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--nz", type=int, default=NZ)
    ap.add_argument("--cpu-procs", type=int, default=0)
    ap.add_argument("--no-mixed", action="store_true", help="skip timing the mixed-precision variant")
    ap.add_argument("--no-mixed60", action="store_true",
                    help="skip the mixed variant's 60-step error against the float64 trajectory")
    ap.add_argument("--no-adjoint", action="store_true", help="skip timing the adjoints against their forwards")
    ap.add_argument("--no-epilogue", action="store_true", help="skip timing the step epilogue (guards + boundary pass)")
    ap.add_argument("--no-tune", action="store_true", help="skip the tile-shape tuner (built-in defaults)")
    ap.add_argument("--workload", choices=("moist433", "batched"), default="moist433",
                    help="batched: the nest + ensemble set advanced by the batched call (1 GPU)")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="profiling target: run this many plain steps of the workload (no timing, no JSON) and exit")
    ap.add_argument("--periodic", action="store_true", help="with --profile-steps: doubly periodic boundaries")
    ap.add_argument("--diff-6th", type=int, default=0, help="with --profile-steps: diff_6th_opt of the step")
    ap.add_argument("--column-width", type=int, default=0,
                    help="with --profile-steps: column kernel (0 default, 1 one thread per column, 16 / 32 tiled)")
    ap.add_argument("--shard", action="store_true",
                    help="under torchrun: one y slab of the workload per rank, halos swapped over NCCL")
    ap.add_argument("--slabs", type=int, default=0,
                    help="one GPU: the workload as this many y slabs driven from one process")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    workload = _workload_name(args.nx, args.ny, args.nz, args.precision)

    if args.workload == "batched" and args.impl == "ours":
        return run_batched(args)
    if args.profile_steps > 0:
        return run_profile_target(args)

    if args.impl == "reference":
        if rank != 0:
            return 0
        procs = args.cpu_procs or max(1, min(os.cpu_count() or 1, 32))
        value, tmax = cpu_reference(args.steps, args.warmup, procs)
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tmax * 1000.0 / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": workload, "sample": f"{SAMPLE[0]}x{SAMPLE[1]}x{SAMPLE[2]} crops x {procs} procs"},
                "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "port",
                                 "sample": f"{procs} processes x {args.steps} RK3 steps of a "
                                           f"{SAMPLE[0]}x{SAMPLE[1]}x{SAMPLE[2]} real-like moist sample (NumPy oracle; "
                                           "JAX is not installed, so the reference's own JAX-CPU step cannot run)"},
                "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    if args.shard or args.slabs > 0:
        rc = run_sharded(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return rc
    r = run_gpu(args, rank, world, local_rank)
    cpu = None
    if rank == 0:
        # bounded CPU baseline sample: 1 process, 2 steps of the 64x64x50 sample
        v, tmax = cpu_reference(2, 0, 1)
        cpu = {"value": v, "unit": METRIC, "cores": 1, "kind": "port",
               "sample": f"2 RK3 steps of a {SAMPLE[0]}x{SAMPLE[1]}x{SAMPLE[2]} crop of the same workload "
                         f"on 1 core (NumPy oracle), {tmax:.1f} s"}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32/f64",
                "data": "synthetic",
                "config": {"workload": workload, "nx": args.nx, "ny": args.ny, "nz": args.nz,
                           "substeps_per_step": 10, "l2": "inputs larger than L2 (no flush)",
                           "parallelism": f"replicas x{world}", "cuda_graph": True, "tile_shapes": r["tuned"]},
                "e2e": r["e2e"], "roofline": r["roofline"], "whole_step_roofline": r["whole_step_roofline"],
                "cpu_baseline": cpu, "clocks": r["clocks"], "gpu_launches": r["launches"],
                "kernels": r["kernels"], "finite": r["finite"], "mixed": r["mixed"], "adjoint": r["adjoint"],
                "epilogue": r["epilogue"]}
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
