#!/usr/bin/env python
"""Benchmark of the B200 APT step on the throughput configuration.

Workload (one GPU): 3D multi-grain directional solidification, line (frozen
gradient) temperature, 256 x 256 x 512 interior cells, 600 seeded Voronoi grains,
NUM_PF = 8 slots, FP32 storage, periodic x/y and no-flux z; synthetic seeded
inputs of the reference's shapes (the reference ships no dataset).

A "step" is one explicit time step of the whole grid (one launch of the fused
step kernel).  `value` = interior cells x K / device time of K steps (CUDA events
on the solver's stream, inputs resident in HBM; the 4.4 GB of pair buffers are
far larger than L2, so no flush is needed).  `e2e` = the same metric through the
C ABI with host buffers: initial fields host->device, all steps of the
configuration (2000), argmax map and grain volumes device->host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cupf|reference]
Under torchrun each rank runs an independent replica (the step does not shard:
no collective on the data path); value sums the replicas' cells over the max
of the ranks' times.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

INTERIOR = (256, 256, 512)
NUM_PF = 8
GRAINS = 600
SEED = 0
CONFIG_STEPS = 2000
SERVE_STEPS = 1000  # steps of each served request (the served-stream configuration)
METRIC = "3D APT Mcell-upd/s"
UNIT = "Mcell-upd/s"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "apt_step_c2_ncu.md")


def workload_config(extra=None):
    c = {"workload": "3D APT line step %dx%dx%d interior, NUM_PF=%d, %d grains"
                     % (*INTERIOR, NUM_PF, GRAINS),
         "interior": list(INTERIOR), "num_pf": NUM_PF, "grains": GRAINS, "seed": SEED,
         "bc": "110", "thermal": "line G=1 K/um R=0.05 m/s", "config_steps": CONFIG_STEPS,
         "l2": "inputs larger than L2 (2 x 2.2 GB pair buffers), no flush"}
    if extra:
        c.update(extra)
    return c


from cupf_b200.replicas import dist_env, max_over_ranks, replica_throughput  # noqa: E402


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", "cupf_clocks_%d_%d.csv" % (os.getpid(), device))

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        load = [v for v in sm if mx and v > 0.3 * max(mx)] or sm
        return {"sm_mhz": float(np.median(load)) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def measured_peak():
    try:
        d = json.load(open(PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the step kernel from the committed ncu summary."""
    try:
        for line in open(TRAFFIC_PROFILE):
            if line.startswith("traffic_bytes_per_launch_c2:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


def make_case():
    from cupf_b200 import cases
    return cases.line_case(*INTERIOR, num_pf=NUM_PF, num_grains=GRAINS, seed=SEED, bc="110")


def cpu_baseline(case, budget_s=15.0, max_steps=4):
    """FP64 oracle (OpenMP, all host threads) on the same workload: bounded number of steps."""
    from oracle import CpuOracle
    o = CpuOracle()
    ph32, ids = case.initial_slots()
    ph = ph32.astype(np.float64)
    ph_b, ids_b = ph.copy(), ids.copy()
    p = case.params
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)
    steps, t_total = 0, 0.0
    while steps < max_steps and t_total < budget_s:
        t = float(np.float32(np.float32(steps + 1) * np.float32(p.dt)) * np.float32(p.tau0))
        t0 = time.perf_counter()
        o.set_bc(p, ph, ids)
        o.rhs_psi_f64(case, t, ph, ids, ph_b, ids_b)
        t_total += time.perf_counter() - t0
        ph, ph_b = ph_b, ph
        ids, ids_b = ids_b, ids
        steps += 1
    cores = os.cpu_count()
    return {"value": cells * steps / t_total / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d FP64 steps of the full %dx%dx%d grid (%.1f s)" % (steps, *INTERIOR, t_total)}


def run_reference(args, ws, rank):
    """Reference arm: the reference's algorithm on the host cores (the oracle
    port in double precision, OpenMP), each step a bounded slab of the workload."""
    if rank != 0:
        return 0
    from cupf_b200 import cases
    from oracle import CpuOracle
    slab = (INTERIOR[0], INTERIOR[1], 64)
    c = cases.line_case(*slab, num_pf=NUM_PF, num_grains=GRAINS, seed=SEED, bc="110")
    o = CpuOracle()
    ph32, ids = c.initial_slots()
    ph = ph32.astype(np.float64)
    ph_b, ids_b = ph.copy(), ids.copy()
    p = c.params
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)

    def one(n):
        nonlocal ph, ph_b, ids, ids_b
        t = float(np.float32(np.float32(n) * np.float32(p.dt)) * np.float32(p.tau0))
        o.set_bc(p, ph, ids)
        o.rhs_psi_f64(c, t, ph, ids, ph_b, ids_b)
        ph, ph_b = ph_b, ph
        ids, ids_b = ids_b, ids

    for n in range(args.warmup):
        one(n + 1)
    t0 = time.perf_counter()
    for n in range(args.steps):
        one(args.warmup + n + 1)
    dt = time.perf_counter() - t0
    v = cells * args.steps / dt / 1e6
    sample = "each step: one FP64 step of a %dx%dx%d slab of the workload" % slab
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config({"reference_sample": sample}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


SERVE_GRIDS = [(48, 48, 48), (96, 96, 96), (128, 128, 256), (192, 192, 192)]


def serve_requests(n, seed=0):
    """Seeded config-4 stream: grid uniform from SERVE_GRIDS, 10-300 grains,
    seed 0-9999, G 0.1-10 K/um (1e5-1e7 K/m), R 0.01-0.5 m/s, 1000 steps,
    Poisson arrivals at 4 per second."""
    from cupf_b200 import cases
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += rng.exponential(1.0 / 4.0)
        g = SERVE_GRIDS[rng.integers(len(SERVE_GRIDS))]
        c = cases.line_case(*g, num_pf=NUM_PF, num_grains=int(rng.integers(10, 301)),
                            seed=int(rng.integers(0, 10000)), G=float(rng.uniform(0.1, 10.0)),
                            R=float(rng.uniform(0.01, 0.5)), bc="110")
        out.append((t, c))
    return out


def run_serve(args):
    """Continuous-batching benchmark: submit each request at its arrival time,
    pump the server meanwhile; report sims/hr and p50/p99 time-to-result."""
    import torch
    from cupf_b200.server import Server
    torch.cuda.set_device(0)
    reqs = serve_requests(args.serve_requests)
    lines = []
    for prec in args.serve_precisions.split(","):
        with Server(precision=prec, num_pf=NUM_PF, max_active=64, steps_per_round=25,
                    autotune=True) as srv:
            # warm the autotuner and the kernels on one request of every grid shape
            warm = [srv.submit(c, 5) for c in
                    [next(c for _, c in reqs if c.meta["interior"] == g) for g in SERVE_GRIDS
                     if any(c.meta["interior"] == g for _, c in reqs)]]
            srv.run_until_done(warm)
            for w in warm:
                srv.release(w)
            t0 = time.perf_counter()
            ids = []
            cells = 0
            k = 0
            with ClockSampler(0) as clk:
                while k < len(reqs) or any(srv.status(r) < 2 for r in ids):
                    now = time.perf_counter() - t0
                    while k < len(reqs) and reqs[k][0] <= now:
                        c = reqs[k][1]
                        ids.append(srv.submit(c, SERVE_STEPS))
                        p = c.params
                        cells += (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2) * SERVE_STEPS
                        k += 1
                    running, pending, _ = srv.pump()
                    if running == 0 and pending == 0 and k < len(reqs):
                        time.sleep(max(0.0, reqs[k][0] - (time.perf_counter() - t0)))
            res = [srv.result(r) for r in ids]
            ttr = np.array([r["times"][2] - r["times"][0] for r in res])
            span = max(r["times"][2] for r in res) - min(r["times"][0] for r in res)
            for r in ids:
                srv.release(r)
            # capacity: the same requests all submitted at once (the stream above is
            # paced by its arrivals: 4/s x 1000 steps x 3.1 M cells on average, about
            # 12 G cell-updates/s of offered load)
            busy0, _ = srv.stats()
            with ClockSampler(0) as clk_sat:
                t1 = time.perf_counter()
                sat = [srv.submit(c, SERVE_STEPS) for _, c in reqs]
                srv.run_until_done(sat)
                sat_span = time.perf_counter() - t1
            busy = (srv.stats()[0] - busy0) / 1e3
            for r in sat:
                srv.release(r)
            lines.append({"metric": "served sims/hr", "impl": "cupf-serve", "precision": prec,
                          "value": len(res) / span * 3600.0, "unit": "sims/hr",
                          "p50_s": float(np.percentile(ttr, 50)),
                          "p99_s": float(np.percentile(ttr, 99)),
                          "mcell_upd_per_s": cells / span / 1e6, "requests": len(res),
                          "arrival_rate_per_s": 4.0, "steps_per_request": SERVE_STEPS,
                          "saturated": {"sims_per_hr": len(sat) / sat_span * 3600.0,
                                        "mcell_upd_per_s": cells / sat_span / 1e6,
                                        "seconds": sat_span, "device_busy_s": busy,
                                        "clocks": clk_sat.summary(),
                                        "note": "all requests submitted at once"},
                          "grids": [list(g) for g in SERVE_GRIDS], "clocks": clk.summary(),
                          "data": "synthetic Poisson stream, seed 0"})
            print(json.dumps(lines[-1]), flush=True)
    return 0


EK2D_GRID = (2048, 8192)
EK2D_STEPS = 50000
EK2D_BYTES = {"fp64": 48, "fp32": 24, "fp16": 12, "bf16": 12}  # psi, U, dpsi read + written


def ek2d_cpu_baseline(budget_s=15.0):
    """FP64 oracle (OpenMP, all host threads) on a 512x2048 slab of the 2D case."""
    from cupf_b200 import ek2d
    from oracle import Ek2dOracle
    c = ek2d.directional_case(512, 2048, 200, sites=8, amp=0.01)
    o = Ek2dOracle()
    s = o.new_state(c, np.float64)
    o.run(c, s, 0, prestep=True)
    steps, t_total = 0, 0.0
    while t_total < budget_s and steps < 200:
        t0 = time.perf_counter()
        o.run(c, s, 5)
        t_total += time.perf_counter() - t0
        steps += 5
    cells = 512 * 2049
    return {"value": cells * steps / t_total / 1e6, "unit": "Mcell-upd/s", "cores": os.cpu_count(),
            "kind": "port", "sample": "%d FP64 oracle steps of a 512x2048 slab (%.1f s)" % (steps, t_total)}


def run_ek2d(args):
    """Split-precision 2D Echebarria-Karma directional solidification: the full
    run in FP64 (the error reference), FP32, FP16 and BF16 storage, each timed on
    the device after `warmup` untimed steps; QoI errors against the FP64 run."""
    from cupf_b200 import ek2d
    nx, ny = EK2D_GRID if not args.ek2d_grid else tuple(args.ek2d_grid)
    steps = args.ek2d_steps
    warm = min(args.warmup, steps // 2)
    case = ek2d.directional_case(nx, ny, steps, sites=32, amp=0.01)
    p = case.params
    dxd = float(p.dx) * float(p.W0)
    q0 = ek2d.qois(case.phi, case.y64(), dxd)
    cells = nx * (ny + 1)
    res = {}
    for prec in ("fp64", "fp32", "fp16", "bf16"):
        with ek2d.EK2DSolver(case, precision=prec) as sv:
            sv.set_state(case.psi, case.U)
            sv.prestep()
            sv.time_steps(warm)
            with ClockSampler(0) as clk:
                ms = sv.time_steps(steps - warm)
            st = sv.get_state()
            y = sv.get_y()
            info = sv.info()
        q = ek2d.qois(st["phi"], y, dxd)
        per = ms / (steps - warm)
        res[prec] = {"ms_per_step": per, "mcell_upd_per_s": cells / per / 1e3, "qois": q,
                     "frame_shifts": info["shifts"], "clocks": clk.summary(),
                     "hbm_gbs": EK2D_BYTES[prec] * cells / (per * 1e-3) / 1e9}
    ref = res["fp64"]["qois"]
    adv = ref["tip_y"] - q0["tip_y"]
    for prec, r in res.items():
        q = r["qois"]
        r["tip_advance_rel_err"] = abs(q["tip_y"] - ref["tip_y"]) / abs(adv) if adv else None
        r["tip_err_cells"] = abs(q["tip_y"] - ref["tip_y"]) / dxd
        r["spacing_rel_err"] = (abs(q["spacing"] - ref["spacing"]) / ref["spacing"]
                                if ref["spacing"] else None)
    # end to end through the C ABI with host buffers: create, H2D of psi/U, the
    # pre-step and all steps, D2H of the final fields
    t0 = time.perf_counter()
    with ek2d.EK2DSolver(case, precision="fp16") as sv:
        sv.set_state(case.psi, case.U)
        sv.prestep()
        sv.step(steps)
        st = sv.get_state()
    e2e_s = time.perf_counter() - t0
    head = res["fp16"]
    # the reference's own step pair (set_BC + merge_PF, 2DdendriteMPI/line_model/PF.cu,
    # compiled for sm_100a) on the same grid and initial state, device time per step
    ref = None
    try:
        from oracle import RefEK2D
        intR = float(case.Rt[0]) * float(p.tau0) / float(p.W0) * float(p.dt)
        lT = (float(p.c_infm) * (1.0 / float(p.k) - 1.0) / float(case.Gt[0])) / float(p.W0)
        rsteps = min(200, steps)
        rms = RefEK2D().time_steps(p, case.psi, case.phi, case.U, np.zeros_like(case.psi), case.y,
                                   intR, lT, rsteps)
        ref = {"ms_per_step": rms / rsteps, "speedup_fp32": rms / rsteps / res["fp32"]["ms_per_step"],
               "speedup_fp16": rms / rsteps / res["fp16"]["ms_per_step"],
               "what": "reference set_BC + merge_PF (line_model/PF.cu) compiled for sm_100a, same grid"}
    except FileNotFoundError as e:
        ref = {"unavailable": str(e)}
    peak, src = measured_peak()
    out = {"metric": "2D EK Mcell-upd/s (split precision)", "value": head["mcell_upd_per_s"],
           "unit": "Mcell-upd/s", "n_gpus": 1, "steps": steps - warm, "warmup": warm,
           "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "fp16 storage, fp32 compute", "data": "synthetic",
           "config": {"workload": "2D Echebarria-Karma directional solidification %dx%d, k=0.14, "
                                  "G=0.1 K/um, R=1e4 um/s, 32 seeded sites +-0.01 W0, %d steps"
                                  % (nx, ny, steps),
                      "grid": [nx, ny], "dx_W0": float(p.dx), "W0_um": float(p.W0),
                      "dt": float(p.dt), "l2": "fields 2x%.0f MB (fp16) per step" % (
                          6 * (nx + 2) * (ny + 3) / 1e6)},
           "roofline": {"bound": "hbm", "achieved": head["hbm_gbs"], "peak": peak, "unit": "GB/s",
                        "frac": head["hbm_gbs"] / peak, "traffic": None, "peak_source": src,
                        "algorithmic_bytes_per_cell": EK2D_BYTES["fp16"]},
           "precisions": res,
           "reference_kernels": ref,
           "e2e": {"value": cells * steps / e2e_s / 1e6, "unit": "Mcell-upd/s",
                   "h2d_bytes_per_step": 2 * 4 * case.fnx * case.fny / steps,
                   "d2h_bytes_per_step": 4 * 4 * case.fnx * case.fny / steps, "seconds": e2e_s},
           "cpu_baseline": None if args.no_cpu_baseline else ek2d_cpu_baseline(),
           "clocks": head["clocks"], "gpu_launches": steps - warm}
    print(json.dumps(out))
    return 0


DENSE_INTERIOR = (128, 128, 128)
DENSE_GRAINS = 80   # the line case's grain density of 600 grains on 256x256


def dense_cpu_baseline(case, budget_s=15.0):
    """The full-PF oracle (FP32, OpenMP over all host threads) on the same case."""
    from oracle import DenseOracle
    o = DenseOracle()
    p = case.params
    ph = o.ini(p, case.phi, case.alpha)
    steps, t_total = 0, 0.0
    a = ph
    while t_total < budget_s and steps < 40:
        t0 = time.perf_counter()
        a, _ = o.run(case, case.meta["R"], a, 2, step0=steps)
        t_total += time.perf_counter() - t0
        steps += 2
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)
    return {"value": cells * steps / t_total / 1e6, "unit": "Mcell-upd/s", "cores": os.cpu_count(),
            "kind": "port", "sample": "%d full-PF oracle steps of the same case from the initial "
                                      "state (%.1f s)" % (steps, t_total)}


def run_dense(args):
    """The full (non-APT, -a) mode: one phi field per grain.  The library's step
    (one launch that evaluates the grains present near each cell and writes the
    next step's per-cell lists), the reference's own set_BC_3D + rhs_psi pair on
    the same state, and the APT step on the same case (the speed-up the -a
    comparison is for), each timed on the device after warm-up steps from the
    initial state.

    Roofline bytes of the library's step: per interior cell its list count read
    and written (8 B), and per grain that is not -1 at the cell its list entry read
    and written (2 x 6 B), its value written and its previous value reset (2 x 4 B)
    -- 20 B per present (cell, grain) pair, counted from the state.  The reference
    reads and writes every grain of every cell (8 B x grains per cell)."""
    import ctypes as C
    import torch
    from cupf_b200 import cases
    from cupf_b200.dense import DenseSolver
    from cupf_b200.solver import APTSolver
    nx, ny, nz = DENSE_INTERIOR if not args.interior else tuple(args.interior)
    ng = max(4, int(DENSE_GRAINS * nx * ny / (DENSE_INTERIOR[0] * DENSE_INTERIOR[1])))
    case = cases.line_case(nx, ny, nz, num_pf=NUM_PF, num_grains=ng, seed=SEED, bc="110")
    p = case.params
    cells = nx * ny * nz
    R = case.meta["R"]
    steps, warm = args.steps, max(args.warmup, 3)
    def present_pairs(ph):
        a = ph.reshape(ng, p.fnz, p.fny, p.fnx)[:, 1:-1, 1:-1, 1:-1]
        return int(np.count_nonzero(a != -1.0))

    with DenseSolver(case) as s:
        s.init_from_argmax(case.phi, case.alpha)
        s.prestep()
        s.step(warm)
        s.sync()
        pairs0 = present_pairs(s.get_slots())
        with ClockSampler(0) as clk:
            ms = s.time_steps(steps)
        over = s.overflow_cells()
        pairs1 = present_pairs(s.get_slots())
        torch.cuda.synchronize()
    per = ms / steps
    pairs = 0.5 * (pairs0 + pairs1)
    # end to end through the C ABI with host buffers
    t0 = time.perf_counter()
    with DenseSolver(case) as s:
        s.init_from_argmax(case.phi, case.alpha)
        s.prestep()
        s.step(warm + steps)
        phi, alpha = s.collect(clear=True)
    e2e_s = time.perf_counter() - t0
    # the reference's kernels on the same initial state
    ref = None
    try:
        from oracle import DenseOracle, RefDenseGPU
        rg = RefDenseGPU()
        rg.check(rg.L.refd_set_params(p, R))
        ph0 = DenseOracle().ini(p, case.phi, case.alpha)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        a, b = dev(ph0), dev(ph0)
        x, y, z = (dev(np.asarray(v, np.float32)) for v in (case.x, case.y, case.z))
        si, co = dev(np.asarray(case.sint, np.float32)), dev(np.asarray(case.cost, np.float32))
        rms = C.c_float()
        argv = (x.data_ptr(), y.data_ptr(), z.data_ptr(), a.data_ptr(), b.data_ptr(), si.data_ptr(),
                co.data_ptr(), C.byref(rms))
        rg.check(rg.L.refd_run_steps(warm + (warm % 2), 0, *argv))
        rg.check(rg.L.refd_run_steps(steps, warm + (warm % 2), *argv))
        ref = {"ms_per_step": rms.value / steps, "what": "reference set_BC_3D + rhs_psi "
               "(3DgrainMPI/PhaseField.cu) compiled for sm_100a, same case"}
        del a, b
        torch.cuda.empty_cache()
    except FileNotFoundError as e:
        ref = {"unavailable": str(e)}
    with APTSolver(case, precision="fp32") as s:
        s.init_from_argmax(case.phi, case.alpha)
        s.step(warm)
        s.sync()
        apt_ms = s.time_steps(steps) / steps
    nbytes = 8 + 20 * pairs / cells  # per cell-update, see the docstring
    peak, src = measured_peak()
    achieved = cells * nbytes / (per * 1e-3) / 1e9
    out = {"metric": "3D full-PF (-a) Mcell-upd/s", "value": cells / per / 1e3, "unit": "Mcell-upd/s",
           "n_gpus": 1, "steps": steps, "warmup": warm, "ms_per_step": per,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
           "data": "synthetic",
           "config": {"workload": "3D full-PF line step %dx%dx%d interior, NUM_PF = %d grains"
                                  % (nx, ny, nz, ng),
                      "interior": [nx, ny, nz], "grains": ng, "seed": SEED,
                      "l2": "phi buffers 2x%.0f MB" % (4 * ng * case.length / 1e6)},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "traffic": None, "peak_source": src,
                        "algorithmic_bytes_per_cell": nbytes,
                        "present_grains_per_cell": pairs / cells,
                        "full_pf_bytes_per_cell": 8 * ng},
           "reference_kernels": ref,
           "speedup_vs_reference_kernels": (ref["ms_per_step"] / per) if "ms_per_step" in ref else None,
           "apt_same_case": {"ms_per_step": apt_ms, "num_pf": NUM_PF,
                             "speedup_apt_over_full_pf": per / apt_ms},
           "overflow_cells_last_step": over,
           "e2e": {"value": cells * (warm + steps) / e2e_s / 1e6, "unit": "Mcell-upd/s",
                   "h2d_bytes_per_step": 8 * case.length / (warm + steps),
                   "d2h_bytes_per_step": 8 * case.length / (warm + steps), "seconds": e2e_s},
           "cpu_baseline": None if args.no_cpu_baseline else dense_cpu_baseline(case),
           "clocks": clk.summary(), "gpu_launches": steps}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cupf", choices=["cupf", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--serve", action="store_true", help="served-batch benchmark (config 4)")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--serve-precisions", default="fp32,fp16")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "bf16", "fp16"])
    ap.add_argument("--interior", type=int, nargs=3, metavar=("NX", "NY", "NZ"),
                    help="smaller line case for profiling (grains scale with the xy area)")
    ap.add_argument("--workload", default="apt3d", choices=["apt3d", "ek2d", "dense"],
                    help="ek2d: the split-precision 2D dendrite benchmark; dense: the full-PF "
                         "(-a) mode against the reference kernels and the APT step")
    ap.add_argument("--ek2d-grid", type=int, nargs=2, metavar=("NX", "NY"))
    ap.add_argument("--ek2d-steps", type=int, default=EK2D_STEPS)
    args = ap.parse_args()
    if args.interior:
        global INTERIOR, GRAINS
        GRAINS = max(10, int(GRAINS * args.interior[0] * args.interior[1] / (INTERIOR[0] * INTERIOR[1])))
        INTERIOR = tuple(args.interior)
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    if args.serve:
        return run_serve(args)
    if args.workload == "ek2d":
        return run_ek2d(args)
    if args.workload == "dense":
        return run_dense(args)

    import torch
    from cupf_b200.solver import APTSolver
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)

    case = make_case()
    p = case.params
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)
    solver = APTSolver(case, precision=args.precision, device=device)
    solver.init_from_argmax(case.phi, case.alpha)
    solver.step(args.warmup)
    solver.sync()

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize(device)

    barrier()
    solver.active_cells()  # restart the counter of computed cells
    with ClockSampler(device) as clk:
        ms = solver.time_steps(args.steps)
    barrier()
    active = solver.active_cells() / args.steps  # cells of the computed items per launch
    ms = max_over_ranks(pg, ms, "cuda")
    value = replica_throughput(ws, cells, args.steps, ms)

    # The same number of steps with every work item computed (the reference's full
    # sweep, no quiet items left alone), continuing from the state reached above.
    solver.set_skip_quiet(False)
    solver.step(2)
    barrier()
    ms_full = max_over_ranks(pg, solver.time_steps(args.steps), "cuda")
    solver.set_skip_quiet(True)

    # roofline of the step kernel (the only kernel in the timed region): the
    # algorithmic bytes are the slot pairs of the cells it computes, each read
    # once and written once; the cells of quiet items are neither read nor written
    bytes_per_cell = 2 * NUM_PF * (8 if args.precision == "fp32" else 4)
    launch_s = ms / 1e3 / args.steps
    achieved = active * bytes_per_cell / launch_s / 1e9
    peak, peak_kind = measured_peak()
    traffic = profile_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic_bytes_per_launch": active * bytes_per_cell,
                "computed_cells_per_launch": active, "interior_cells": cells}
    full_sweep = {"value": replica_throughput(ws, cells, args.steps, ms_full), "unit": UNIT,
                  "ms_per_step": ms_full / args.steps,
                  "hbm_gbs": cells * bytes_per_cell / (ms_full / 1e3 / args.steps) / 1e9,
                  "note": "every work item computed, steps %d-%d" % (
                      args.warmup + args.steps + 3, args.warmup + 2 * args.steps + 2)}

    # end to end through the C ABI with host buffers: a whole C2 simulation
    e2e = None
    if not args.no_e2e:
        def through_abi(nsteps):
            """create + H2D of phi/alpha + nsteps + argmax D2H + volumes, host wall time
            (max over ranks)."""
            barrier()
            t0 = time.perf_counter()
            with APTSolver(case, precision=args.precision, device=device) as s2:
                s2.init_from_argmax(case.phi, case.alpha)
                s2.step(nsteps)
                phi, alpha = s2.collect(clear=True)
                vols = s2.grain_volumes(GRAINS)
            torch.cuda.synchronize(device)
            sec = max_over_ranks(pg, time.perf_counter() - t0, "cuda")
            assert vols.sum() == cells
            return sec

        L = case.length
        # a whole C2 simulation (2000 steps) through the C ABI: the configuration's
        # own workload, and the headline end-to-end number
        full_s = through_abi(CONFIG_STEPS)
        # and the same steps as the device-timed region (warm-up + timed steps from
        # the same initial state): the state is young there, with more active slots
        # per cell than the simulation's average, and the fixed costs weigh more
        nwin = args.warmup + args.steps
        win_s = through_abi(nwin)
        e2e = {"value": ws * cells * CONFIG_STEPS / full_s / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": (8 * L) / CONFIG_STEPS,  # phi + alpha, float32/int32
               "d2h_bytes_per_step": (8 * L + 8 * (GRAINS + 1)) / CONFIG_STEPS,
               "steps": CONFIG_STEPS, "seconds": full_s,
               "includes": "handle create + H2D phi/alpha + 2000 steps + argmax D2H + volumes",
               "same_steps_as_timed_region": {"value": ws * cells * nwin / win_s / 1e6,
                                              "steps": nwin, "seconds": win_s}}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(case)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "fp32" if args.precision == "fp32" else args.precision + " storage, fp32 compute",
                "data": "synthetic",
                "config": workload_config({"parallelism": "replicas x%d" % ws,
                                           "storage": args.precision,
                                           "quiet_items": "work items whose cells stay exact "
                                           "empty pairs are left alone (results bit-identical "
                                           "to the full sweep, which full_sweep times); "
                                           "computed cells per launch %d of %d" % (active, cells)}),
                "hbm_gbs": achieved, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "full_sweep": full_sweep,
                "clocks": clk.summary(), "gpu_launches": args.steps,
                "baseline_metric": "3D APT Mcell-upd/s & HBM GB/s, mixed vs FP32; served sims/hr,"
                                   " p50/p99 at <=1e-3 err"}
        print(json.dumps(line), flush=True)
    solver.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
