#!/usr/bin/env python
"""Benchmark of the B200 APT step on the throughput configuration.

Workload (one GPU): 3D multi-grain directional solidification, line (frozen
gradient) temperature, 256 x 256 x 512 interior cells, 600 seeded Voronoi grains,
NUM_PF = 8 slots, FP32 storage, periodic x/y and no-flux z; synthetic seeded
inputs of the reference's shapes (the reference ships no dataset).

A "step" is one explicit time step of the whole grid (one launch of the fused
step kernel) with every work item computed, as the reference sweeps every cell.
`value` = interior cells x K / device time of K steps (CUDA events on the
solver's stream, inputs resident in HBM; the 4.4 GB of pair buffers are far
larger than L2, so no flush is needed).  `quiet_skip` times the same K steps from
the same state with the library's default of leaving alone work items whose
cells stay exact empty pairs (bit-identical results).  `e2e` = the same metric
through the C ABI with host buffers: initial fields host->device, all steps of
the configuration (2000), argmax map and grain volumes device->host.

The same line also carries, on one GPU: the FP16- and BF16-storage steps on the
same workload ("mixed vs FP32"), the errors of FP32/FP16/BF16 storage against
the FP64 oracle (64^3 case, 1000 steps, fixture tests/golden/fp64/qoi.npz), the
served stream (sims/hr, p50/p99 time-to-result, capacity, per-result errors of
the 48^3 and 96^3 requests against FP64-oracle fixtures), the reference's own
APTsetBC3D + APTrhs_psi kernels compiled for sm_100a timed on the same state,
and the host-CPU baseline.

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
FP64_QOI = os.path.join(ROOT, "tests", "golden", "fp64", "qoi.npz")
ERROR_TOL = 1e-3  # relative error bound on volume fractions and interface position


def workload_config(extra=None, pair_bytes=8):
    """The workload's description; `pair_bytes` is the size of one stored
    (phi, id) slot (8 for FP32 storage, 4 for the 16-bit forms)."""
    nx, ny, nz = INTERIOR
    buf = (nx + 2) * (ny + 2) * (nz + 2) * NUM_PF * pair_bytes
    c = {"workload": "3D APT line step %dx%dx%d interior, NUM_PF=%d, %d grains"
                     % (*INTERIOR, NUM_PF, GRAINS),
         "interior": list(INTERIOR), "num_pf": NUM_PF, "grains": GRAINS, "seed": SEED,
         "bc": "110", "thermal": "line G=1 K/um R=0.05 m/s", "config_steps": CONFIG_STEPS,
         "sweep": "every work item computed",
         "l2": "inputs %s L2 (2 x %.1f MB pair buffers against 126 MB), no flush"
               % ("larger than" if buf > 126e6 else "NOT larger than", buf / 1e6)}
    if extra:
        c.update(extra)
    return c


from cupf_b200.replicas import dist_env, max_over_ranks, replica_throughput  # noqa: E402


def physical_gpu(device):
    """nvidia-smi's name for CUDA device `device`: its UUID (nvidia-smi numbers
    GPUs in its own order and ignores CUDA_VISIBLE_DEVICES, so an ordinal would
    name another GPU when the job is pinned to a subset)."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(device).uuid)
        if u:
            return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        pass
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if vis:
        ent = [v.strip() for v in vis.split(",") if v.strip()]
        if device < len(ent):
            return ent[device]
    return str(device)


class ClockSampler:
    """nvidia-smi clock/throttle sampling of one GPU during the timed region.
    `device` is a CUDA ordinal; the sampler resolves it to the physical GPU."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.gpu = physical_gpu(device)
        self.proc = None
        self.path = os.path.join("/tmp", "cupf_clocks_%d_%d_%d.csv" % (os.getpid(), device,
                                                                     time.monotonic_ns()))

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, "--query-gpu=" + self.Q,
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
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"],
                    "gpu": self.gpu}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "gpu": self.gpu}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        load = [v for v in sm if mx and v > 0.3 * max(mx)] or sm
        return {"sm_mhz": float(np.median(load)) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "gpu": self.gpu, "nvidia_smi_index": rows[0][0]}


def measured_peak():
    try:
        d = json.load(open(PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_case():
    from cupf_b200 import cases
    return cases.line_case(*INTERIOR, num_pf=NUM_PF, num_grains=GRAINS, seed=SEED, bc="110")


class _Fp64Stepper:
    """The FP64 oracle (the reference's step in double precision, OpenMP over all
    host threads) advancing one state of a case: the CPU side of the comparison."""

    def __init__(self, case):
        from oracle import CpuOracle
        self.o = CpuOracle()
        self.case = case
        ph32, ids = case.initial_slots()
        self.ph = ph32.astype(np.float64)
        del ph32
        self.ids = ids
        self.ph_b, self.ids_b = self.ph.copy(), ids.copy()
        self.n = 0

    def step(self):
        p = self.case.params
        self.n += 1
        t = float(self.n) * float(p.dt) * float(p.tau0)  # FP64 time
        self.o.set_bc(p, self.ph, self.ids)
        self.o.rhs_psi_f64(self.case, t, self.ph, self.ids, self.ph_b, self.ids_b)
        self.ph, self.ph_b = self.ph_b, self.ph
        self.ids, self.ids_b = self.ids_b, self.ids


def cpu_baseline(case, budget_s=15.0, max_steps=4):
    """FP64 oracle (OpenMP, all host threads) on the same workload: a bounded
    number of whole-grid steps from the initial state."""
    st = _Fp64Stepper(case)
    p = case.params
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)
    steps, t_total = 0, 0.0
    while steps < max_steps and t_total < budget_s:
        t0 = time.perf_counter()
        st.step()
        t_total += time.perf_counter() - t0
        steps += 1
    return {"value": cells * steps / t_total / 1e6, "unit": UNIT, "cores": os.cpu_count(),
            "kind": "port",
            "sample": "%d FP64 steps of the full %dx%dx%d grid (%.1f s)" % (steps, *INTERIOR, t_total)}


def run_reference(args, ws, rank):
    """Reference arm: the reference's algorithm on the host cores (the oracle
    port in double precision, OpenMP over all host threads; the reference ships
    its step only as CUDA) on the same 256x256x512 grid as the library's arm:
    `warmup` untimed whole-grid steps, then `steps` timed whole-grid steps from
    the same initial state."""
    if rank != 0:
        return 0
    case = make_case()
    st = _Fp64Stepper(case)
    p = case.params
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)
    for _ in range(args.warmup):
        st.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st.step()
    dt = time.perf_counter() - t0
    v = cells * args.steps / dt / 1e6
    sample = ("steps %d-%d of the whole %dx%dx%d grid in FP64 (the library arm's grid, state "
              "and steps)" % (args.warmup + 1, args.warmup + args.steps, *INTERIOR))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "same_config": True,
            "config": workload_config({"reference_sample": sample}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def load_fp64_fixture():
    try:
        return dict(np.load(FP64_QOI))
    except Exception:
        return None


def qoi_errors(volumes, qoi, ref_volumes, ref_qoi):
    """Errors of a result against the FP64 oracle: volume-weighted L1 relative
    error of the grain volume fractions, relative error of the mean interface
    height (interface position) and of the interface area."""
    v = np.asarray(volumes, np.float64)
    r = np.asarray(ref_volumes, np.float64)
    return {"volume_fraction_l1_rel_err": float(np.abs(v - r).sum() / r.sum()),
            "interface_height_rel_err": float(abs(qoi[2] - ref_qoi[2]) / ref_qoi[2]),
            "interface_area_rel_err": float(abs(qoi[1] - ref_qoi[1]) / ref_qoi[1])}


def within_tol(e):
    return bool(e["volume_fraction_l1_rel_err"] <= ERROR_TOL and
                e["interface_height_rel_err"] <= ERROR_TOL)


def storage_errors(fix, precisions=("fp32", "fp16", "bf16")):
    """Each storage on the 64^3 line case (20 grains, NUM_PF = 5, 1000 steps,
    from init_from_argmax like every production path) against the FP64 oracle's
    QoIs of the same case (tests/golden/fp64/qoi.npz)."""
    from cupf_b200 import cases
    from cupf_b200.solver import APTSolver
    if fix is None:
        return {"unavailable": "fixture %s missing" % FP64_QOI}
    c = cases.line_case(64, 64, 64, num_pf=5, num_grains=20, seed=0, bc="110")
    steps = int(fix["steps"])
    out = {"case": "64^3 line, 20 grains, NUM_PF=5, %d steps" % steps, "tolerance": ERROR_TOL}
    for prec in precisions:
        with APTSolver(c, precision=prec) as s:
            s.init_from_argmax(c.phi, c.alpha)
            s.step(steps)
            s.collect(clear=True)
            vols = s.grain_volumes(c.params.num_theta)[1:]
            q = s.qoi_sums()
        e = qoi_errors(vols, q, fix["c1_volumes"], fix["c1_qoi"])
        if "c1_f32_volumes" in fix:
            e["fp32_oracle"] = qoi_errors(fix["c1_f32_volumes"], fix["c1_f32_qoi"],
                                          fix["c1_volumes"], fix["c1_qoi"])
        if "c1_p64_volumes" in fix:
            e["fp64_perturbed"] = qoi_errors(fix["c1_p64_volumes"], fix["c1_p64_qoi"],
                                             fix["c1_volumes"], fix["c1_qoi"])
        e["within_tolerance"] = within_tol(e)
        out[prec] = e
    return out


def serve_stream(prec, nreq, fix=None, device=0):
    """Continuous-batching run of the seeded Poisson stream: submit each request
    at its arrival time, pump the server meanwhile; then the same requests all
    submitted at once (capacity).  Returns sims/hr, p50/p99 time-to-result,
    cell-update rates and, for the requests the FP64-oracle fixture covers
    (the 48^3 and 96^3 grids), each result's error against it."""
    from cupf_b200.server import SERVE_GRIDS, Server, poisson_stream
    reqs = poisson_stream(nreq, seed=0, num_pf=NUM_PF)
    fix_idx = set(int(i) for i in fix["served_index"]) if fix is not None else set()
    with Server(device=device, precision=prec, num_pf=NUM_PF, max_active=64, steps_per_round=25,
                autotune=True) as srv:
        # warm the autotuner and the kernels on one request of every grid shape
        shapes = [g for g in SERVE_GRIDS if any(c.meta["interior"] == g for _, c in reqs)]
        warm = [srv.submit(next(c for _, c in reqs if c.meta["interior"] == g), 5) for g in shapes]
        srv.run_until_done(warm)
        # the autotuner's tile shape per grid shape: (column-tile height, z chunk)
        tiles = {"x".join(map(str, g)): list(srv.tile(w)) for g, w in zip(shapes, warm)}
        for w in warm:
            srv.release(w)
        t0 = time.perf_counter()
        ids = []
        cells = 0
        k = 0
        with ClockSampler(device) as clk:
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
        errors = []
        for i, r in enumerate(res):
            if i in fix_idx:
                e = qoi_errors(r["volumes"][1:], r["qoi"], fix["srv%d_volumes" % i],
                               fix["srv%d_qoi" % i])
                e["request"] = i
                e["grid"] = list(reqs[i][1].meta["interior"])
                e["grains"] = reqs[i][1].meta["num_grains"]
                if "srv%d_f32_volumes" % i in fix:
                    # what single precision itself (the oracle's FP32 restatement of
                    # the reference) makes of the same request against FP64
                    e["fp32_oracle"] = qoi_errors(fix["srv%d_f32_volumes" % i],
                                                  fix["srv%d_f32_qoi" % i],
                                                  fix["srv%d_volumes" % i], fix["srv%d_qoi" % i])
                if "srv%d_p64_volumes" % i in fix:
                    # how far the request's own dynamics carry one float ulp of
                    # noise on the initial state, all in FP64
                    e["fp64_perturbed"] = qoi_errors(fix["srv%d_p64_volumes" % i],
                                                     fix["srv%d_p64_qoi" % i],
                                                     fix["srv%d_volumes" % i], fix["srv%d_qoi" % i])
                errors.append(e)
        for r in ids:
            srv.release(r)
        # capacity: the same requests all submitted at once (the paced stream
        # offers about 12 G cell-updates/s, below what one GPU serves), after an
        # untimed burst of the same requests for one round each, which leaves the
        # server's recycled host and device buffers as a server running steadily
        # holds them
        warm = [srv.submit(c, 25) for _, c in reqs]
        srv.run_until_done(warm)
        for r in warm:
            srv.release(r)
        busy0, _ = srv.stats()
        with ClockSampler(device) as clk_sat:
            t1 = time.perf_counter()
            sat = [srv.submit(c, SERVE_STEPS) for _, c in reqs]
            srv.run_until_done(sat)
            sat_span = time.perf_counter() - t1
        busy = (srv.stats()[0] - busy0) / 1e3
        for r in sat:
            srv.release(r)
    worst = {}
    if errors:
        for key in ("volume_fraction_l1_rel_err", "interface_height_rel_err"):
            worst[key] = max(e[key] for e in errors)
        worst["within_tolerance"] = bool(all(within_tol(e) for e in errors))
        worst["results_within_tolerance"] = sum(within_tol(e) for e in errors)
        # requests whose FP64 run from a one-ulp-perturbed start already differs
        # from the FP64 run by more than the tolerance (the bound is below what
        # the request's dynamics resolve)
        worst["results_fp64_perturbed_beyond_tolerance"] = sum(
            1 for e in errors if "fp64_perturbed" in e and not within_tol(e["fp64_perturbed"]))
    return {"precision": prec, "tiles_autotuned": tiles, "sims_per_hr": len(res) / span * 3600.0,
            "p50_s": float(np.percentile(ttr, 50)), "p99_s": float(np.percentile(ttr, 99)),
            "mcell_upd_per_s": cells / span / 1e6, "requests": len(res),
            "arrival_rate_per_s": 4.0, "steps_per_request": SERVE_STEPS,
            "capacity": {"sims_per_hr": len(sat) / sat_span * 3600.0,
                         "mcell_upd_per_s": cells / sat_span / 1e6, "seconds": sat_span,
                         "device_busy_s": busy,
                         "device_mcell_upd_per_s": cells / busy / 1e6 if busy > 0 else None,
                         "clocks": clk_sat.summary(),
                         "note": "the same requests all submitted at once; the device rate "
                                 "counts the rounds' device time only (the span also holds "
                                 "admission, retirement and host time)"},
            "errors_vs_fp64": {"results": errors, "worst": worst, "tolerance": ERROR_TOL,
                               "which": "every request of the stream with a %s grid (%d of %d; "
                                        "the oracle's cost bounds the rest)"
                                        % (" or ".join(sorted({"x".join(map(str, e["grid"]))
                                                               for e in errors})) or "no",
                                           len(errors), len(res))},
            "clocks": clk.summary()}


def run_serve(args):
    """Continuous-batching benchmark alone: one JSON line per storage."""
    import torch
    from cupf_b200.server import SERVE_GRIDS
    torch.cuda.set_device(0)
    fix = load_fp64_fixture()
    for prec in args.serve_precisions.split(","):
        r = serve_stream(prec, args.serve_requests, fix)
        line = {"metric": "served sims/hr", "impl": "cupf-serve", "value": r["sims_per_hr"],
                "unit": "sims/hr", **r, "grids": [list(g) for g in SERVE_GRIDS],
                "data": "synthetic Poisson stream, seed 0"}
        print(json.dumps(line), flush=True)
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
    import torch
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
    # how far the front's own dynamics carry a rounding-sized perturbation: FP64
    # again from the initial state with psi moved by one float ulp, up or down at
    # random, on a seeded half of the cells
    rng = np.random.default_rng(7)
    psi0 = np.ascontiguousarray(case.psi, np.float32)
    move = rng.random(psi0.shape) < 0.5
    up = rng.random(psi0.shape) < 0.5
    psi_p = psi0.copy()
    psi_p[move & up] = np.nextafter(psi0[move & up], np.float32(np.inf))
    psi_p[move & ~up] = np.nextafter(psi0[move & ~up], np.float32(-np.inf))
    with ek2d.EK2DSolver(case, precision="fp64") as sv:
        sv.set_state(psi_p, case.U)
        sv.prestep()
        sv.step(steps)
        st = sv.get_state()
        y = sv.get_y()
    q = ek2d.qois(st["phi"], y, dxd)
    res["fp64_perturbed"] = {
        "what": "FP64 from the initial psi with one float ulp of noise on half the cells",
        "qois": q, "tip_err_cells": abs(q["tip_y"] - ref["tip_y"]) / dxd,
        "tip_advance_rel_err": abs(q["tip_y"] - ref["tip_y"]) / abs(adv) if adv else None,
        "spacing_rel_err": (abs(q["spacing"] - ref["spacing"]) / ref["spacing"]
                            if ref["spacing"] else None)}
    # end to end through the C ABI with host buffers: create, H2D of psi/U, the
    # pre-step and all steps, D2H of the final fields
    # (inputs and read-back fields in page-locked host memory, filled beforehand)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory().numpy()
    in_psi, in_U = pin(case.psi), pin(case.U)
    out_st = [torch.empty(case.fny * case.fnx, dtype=torch.float32, pin_memory=True).numpy()
              for _ in range(4)]
    t0 = time.perf_counter()
    with ek2d.EK2DSolver(case, precision="fp16") as sv:
        sv.set_state(in_psi, in_U)
        sv.prestep()
        sv.step(steps)
        st = sv.get_state(out=out_st)
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


MELT_INTERIOR = (256, 256, 768)
MELT_GRAINS = 400
TIPP = 20  # moving-domain check interval of the reference's line runs (APTPhaseField.cu:29)


def run_meltpool(args):
    """Moving-domain melt-pool configuration at its stated size: a 256 x 256 x 768
    window, 400 substrate grains, NUM_PF = 8, the analytic paraboloid pool
    (radius 60 um, length 120 um, 0.5 m/s scan, G = 1 K/um; thermalType 5),
    Philox nucleation at undercooling N(10 K, 2 K) from the same field's 4-D
    table, the frame check every 20 steps, in FP32 and FP16 storage.  Per
    storage: `steps` steps of the reference's loop order (step, nucleation pass,
    frame check, step) timed on the host clock around synchronised work, and the
    step kernel alone over the same state with CUDA events."""
    import torch
    from cupf_b200 import cases
    from cupf_b200.solver import APTSolver
    torch.cuda.set_device(0)
    nx, ny, nz = MELT_INTERIOR if not args.interior else tuple(args.interior)
    grains = max(10, int(MELT_GRAINS * nx * ny / (MELT_INTERIOR[0] * MELT_INTERIOR[1])))
    cells = nx * ny * nz
    steps = args.steps - (args.steps % 2)
    warm = args.warmup + (args.warmup % 2)
    peak, src = measured_peak()
    res = {}
    for prec in ("fp32", "fp16"):
        d = cases.derive_params({**cases.LINE_CONSTANTS, "R": 0.5})
        t_end = (warm + steps + 2 * TIPP) * float(d["dt"]) * float(d["tau0"])
        case = cases.meltpool_case(nx, ny, nz, num_pf=NUM_PF, num_grains=grains, seed=SEED,
                                   t_end=t_end)
        p = case.params
        thres = int(0.8 * p.fnz)
        with APTSolver(case, precision=prec) as s:
            s.set_skip_quiet(False)  # every work item computed, as the reference sweeps
            s.init_from_argmax(case.phi, case.alpha)
            s.nucl_init()
            state = {"tip": 1, "mc": 0, "moved": 0, "nuclei": 0}

            def pair(it, last=False):
                s.step(1)
                # the running count of nuclei (a read that waits) only at the end
                n = s.nucleate(False, count=last)
                if last:
                    state["nuclei"] = n
                if (2 * it + 2) % TIPP == 0:
                    state["tip"], state["mc"], m = s.move_domain(state["tip"], thres, state["mc"])
                    state["moved"] += m
                s.step(1)

            for it in range(warm // 2):
                pair(it)
            s.sync()
            with ClockSampler(0) as clk:
                t0 = time.perf_counter()
                for it in range(warm // 2, (warm + steps) // 2):
                    pair(it, last=it == (warm + steps) // 2 - 1)
                s.sync()
                wall = time.perf_counter() - t0
            kern_ms = s.time_steps(max(steps, 20)) / max(steps, 20)
        bpc = NUM_PF * (16 if prec == "fp32" else 8)
        res[prec] = {"mcell_upd_per_s": cells * steps / wall / 1e6, "ms_per_step": wall * 1e3 / steps,
                     "step_kernel_ms": kern_ms,
                     "step_kernel_mcell_upd_per_s": cells / kern_ms / 1e3,
                     "hbm_gbs": cells * bpc / (kern_ms * 1e-3) / 1e9,
                     "roofline_frac": cells * bpc / (kern_ms * 1e-3) / 1e9 / peak,
                     "frame_shifts": state["moved"], "nuclei": state["nuclei"],
                     "clocks": clk.summary()}
    head = res["fp32"]
    out = {"metric": "3D APT melt-pool Mcell-upd/s", "value": head["mcell_upd_per_s"],
           "unit": "Mcell-upd/s", "n_gpus": 1, "steps": steps, "warmup": warm,
           "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
           "config": {"workload": "melt pool %dx%dx%d window, %d grains, NUM_PF=%d, analytic "
                                  "paraboloid r0=60 um V=0.5 m/s, Philox nucleation N(10 K, 2 K), "
                                  "moving domain" % (nx, ny, nz, grains, NUM_PF),
                      "loop": "step, nucleation pass, frame check every 20 steps, step (the "
                              "reference's evolve order); every work item computed"},
           "roofline": {"bound": "hbm", "achieved": head["hbm_gbs"], "peak": peak, "unit": "GB/s",
                        "frac": head["roofline_frac"], "traffic": None, "peak_source": src,
                        "of": "step kernel alone, window cells x 128 B"},
           "precisions": res, "clocks": head["clocks"], "gpu_launches": steps}
    print(json.dumps(out), flush=True)
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
    # end to end through the C ABI with host buffers (page-locked, filled beforehand)
    in_phi = torch.from_numpy(np.ascontiguousarray(case.phi, np.float32)).pin_memory().numpy()
    in_alpha = torch.from_numpy(np.ascontiguousarray(case.alpha, np.int32)).pin_memory().numpy()
    out_f = (torch.empty(case.length, dtype=torch.float32, pin_memory=True).numpy(),
             torch.empty(case.length, dtype=torch.int32, pin_memory=True).numpy())
    t0 = time.perf_counter()
    with DenseSolver(case) as s:
        s.init_from_argmax(in_phi, in_alpha)
        s.prestep()
        s.step(warm + steps)
        phi, alpha = s.collect(clear=True, out=out_f)
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
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cupf", choices=["cupf", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--serve", action="store_true", help="served-batch benchmark (config 4)")
    ap.add_argument("--serve-requests", type=int, default=40,
                    help="requests of the served stream (0: no served run in the default line)")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: no other storages, errors, served stream or reference "
                         "kernels")
    ap.add_argument("--serve-precisions", default="fp32,fp16")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "bf16", "fp16"])
    ap.add_argument("--interior", type=int, nargs=3, metavar=("NX", "NY", "NZ"),
                    help="smaller line case for profiling (grains scale with the xy area)")
    ap.add_argument("--workload", default="apt3d", choices=["apt3d", "ek2d", "dense", "meltpool"],
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
    if args.workload == "meltpool":
        return run_meltpool(args)

    return run_apt3d(args, ws, rank, local)


def reference_kernels(case, steps, warmup):
    """The reference's own APTsetBC3D + APTrhs_psi pair (3DgrainMPI/APTPhaseField.cu,
    compiled unmodified for sm_100a; block 32x4 as its evolve loop launches it),
    timed on the device over the same steps from the same initial state."""
    import ctypes as C
    import torch
    try:
        from oracle import RefGPU
        ref = RefGPU(NUM_PF)
    except (FileNotFoundError, OSError) as e:
        return {"unavailable": str(e)}
    p = case.params
    ref.check(ref.L.ref_set_params(p))
    ph0, id0 = case.initial_slots()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    x, y, z, sint, cost = (dev(a) for a in (case.x, case.y, case.z, case.sint, case.cost))
    a_ph, a_id, b_ph, b_id = dev(ph0), dev(id0), dev(ph0), dev(id0)
    del ph0, id0
    ms = C.c_float()
    args = [x.data_ptr(), y.data_ptr(), z.data_ptr(), a_ph.data_ptr(), b_ph.data_ptr(),
            a_id.data_ptr(), b_id.data_ptr(), sint.data_ptr(), cost.data_ptr()]
    w = warmup + (warmup % 2)  # the harness runs step pairs; an even warm-up keeps the buffers
    ref.check(ref.L.ref_run_steps(w, 0, *args, C.byref(ms)))
    ref.check(ref.L.ref_run_steps(steps, w, *args, C.byref(ms)))
    del a_ph, a_id, b_ph, b_id
    torch.cuda.empty_cache()
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)
    return {"ms_per_step": ms.value / steps, "value": cells * steps / ms.value / 1e3,
            "unit": UNIT, "steps": steps, "warmup": w,
            "what": "reference APTsetBC3D + APTrhs_psi (3DgrainMPI/APTPhaseField.cu) compiled "
                    "for sm_100a, same grid and initial state, device time"}


def run_apt3d(args, ws, rank, local):
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
    extras = ws == 1 and not args.no_extras

    case = make_case()
    p = case.params
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize(device)

    def window(solver, skip_quiet, clocks=False):
        """From the initial state: `warmup` untimed steps, then `steps` timed steps
        (CUDA events on the solver's stream, max over ranks)."""
        solver.init_from_argmax(case.phi, case.alpha)
        solver.set_skip_quiet(skip_quiet)
        solver.step(args.warmup)
        barrier()
        solver.active_cells()  # restart the counters of computed cells and merge overflows
        solver.merge_overflows()
        clk = ClockSampler(device) if clocks else None
        if clk:
            clk.__enter__()
        ms = solver.time_steps(args.steps)
        ovf = solver.merge_overflows()
        if clk:
            # keep the GPU under the same load for about half a second more, so the
            # sampler (100 ms period) sees the clocks of this kernel even when the
            # timed region itself is shorter than its period
            t_end = time.perf_counter() + 0.5
            while time.perf_counter() < t_end:
                solver.step(max(1, args.steps))
                solver.sync()
            clk.__exit__(None, None, None)
        barrier()
        active = solver.active_cells() / args.steps  # cells of the computed items per launch
        ms = max_over_ranks(pg, ms, "cuda")
        window.overflows = {"aliased_per_step": ovf[0] / args.steps,
                            "dropped_per_step": ovf[1] / args.steps}
        return ms, active, clk.summary() if clk else None

    bytes_per_cell = {"fp32": 16, "fp16": 8, "bf16": 8}
    with APTSolver(case, precision=args.precision, device=device) as solver:
        ms, active, clocks = window(solver, False, clocks=True)
        overflows = window.overflows
        ms_q, active_q, _ = window(solver, True)
    value = replica_throughput(ws, cells, args.steps, ms)
    bpc = NUM_PF * bytes_per_cell[args.precision]
    launch_s = ms / 1e3 / args.steps
    achieved = cells * bpc / launch_s / 1e9
    peak, peak_kind = measured_peak()
    # roofline of the step kernel (the only kernel in the timed region): every
    # interior cell's slot pairs read once and written once.  DRAM traffic is not
    # measured by this run (a profiler capture is needed): null here.
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic_bytes_per_launch": cells * bpc,
                "algorithmic_bytes_per_cell": bpc, "interior_cells": cells}
    quiet = {"value": replica_throughput(ws, cells, args.steps, ms_q), "unit": UNIT,
             "ms_per_step": ms_q / args.steps, "computed_cells_per_launch": active_q,
             "computed_hbm_gbs": active_q * bpc / (ms_q / 1e3 / args.steps) / 1e9,
             "note": "same state and steps; work items whose cells stay exact empty pairs are "
                     "left alone (results bit-identical); value counts every interior cell"}

    # the other storages on the same workload (mixed vs FP32)
    precisions = None
    if extras:
        precisions = {args.precision: {"value": value, "ms_per_step": ms / args.steps,
                                       "hbm_gbs": achieved, "quiet_skip_value": quiet["value"]}}
        for prec in ("fp16", "bf16"):
            if prec == args.precision:
                continue
            with APTSolver(case, precision=prec, device=device) as s2:
                m2, _, _ = window(s2, False)
                m2q, _, _ = window(s2, True)
            bpc2 = NUM_PF * bytes_per_cell[prec]
            precisions[prec] = {"value": cells * args.steps / m2 / 1e3,
                                "ms_per_step": m2 / args.steps,
                                "hbm_gbs": cells * bpc2 / (m2 / 1e3 / args.steps) / 1e9,
                                "quiet_skip_value": cells * args.steps / m2q / 1e3,
                                "speedup_vs_fp32_full_sweep": ms / m2}
        fix = load_fp64_fixture()
        precisions["errors_vs_fp64"] = storage_errors(fix)

    # end to end through the C ABI with host buffers: a whole C2 simulation
    e2e = None
    if not args.no_e2e:
        # the inputs and the read-back fields in page-locked host memory, filled
        # before the timed region
        def pinned(n, dt):
            return torch.empty(n, dtype=dt, pin_memory=True).numpy()
        in_phi, in_alpha = pinned(case.length, torch.float32), pinned(case.length, torch.int32)
        in_phi[:] = np.asarray(case.phi, np.float32).ravel()
        in_alpha[:] = np.asarray(case.alpha, np.int32).ravel()
        out_fields = (pinned(case.length, torch.float32), pinned(case.length, torch.int32))

        def through_abi(nsteps, skip_quiet):
            """create + H2D of phi/alpha + nsteps + argmax D2H + volumes, host wall time
            (max over ranks)."""
            barrier()
            t0 = time.perf_counter()
            with APTSolver(case, precision=args.precision, device=device) as s2:
                s2.set_skip_quiet(skip_quiet)
                s2.init_from_argmax(in_phi, in_alpha)
                s2.step(nsteps)
                phi, alpha = s2.collect(clear=True, out=out_fields)
                vols = s2.grain_volumes(GRAINS)
            torch.cuda.synchronize(device)
            sec = max_over_ranks(pg, time.perf_counter() - t0, "cuda")
            assert vols.sum() == cells
            return sec

        L = case.length
        full_s = through_abi(CONFIG_STEPS, False)
        quiet_s = through_abi(CONFIG_STEPS, True)
        e2e = {"value": ws * cells * CONFIG_STEPS / full_s / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": (8 * L) / CONFIG_STEPS,  # phi + alpha, float32/int32
               "d2h_bytes_per_step": (8 * L + 8 * (GRAINS + 1)) / CONFIG_STEPS,
               "steps": CONFIG_STEPS, "seconds": full_s,
               "includes": "handle create + H2D phi/alpha + 2000 steps (every work item "
                           "computed) + argmax D2H + volumes",
               "host_memory": "page-locked inputs and read-back fields",
               "quiet_skip": {"value": ws * cells * CONFIG_STEPS / quiet_s / 1e6,
                              "seconds": quiet_s}}

    served = None
    ref_k = None
    if extras:
        ref_k = reference_kernels(case, args.steps, args.warmup)
        if "ms_per_step" in ref_k:
            ref_k["speedup_full_sweep"] = ref_k["ms_per_step"] / (ms / args.steps)
        if args.serve_requests > 0:
            fix = load_fp64_fixture()
            served = {}
            for prec in args.serve_precisions.split(","):
                served[prec] = serve_stream(prec, args.serve_requests, fix, device)
            if "fp32" in served:
                fp32_single = cells * args.steps / (ms if args.precision == "fp32" else
                                                    precisions["fp32"]["ms_per_step"] * args.steps) / 1e3
                for prec, r in served.items():
                    r["capacity_vs_fp32_single_full_sweep"] = (r["capacity"]["mcell_upd_per_s"] /
                                                               fp32_single)

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
                                           "storage": args.precision},
                                          8 if args.precision == "fp32" else 4),
                "hbm_gbs": achieved, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "quiet_skip": quiet, "precisions": precisions, "served": served,
                "reference_kernels": ref_k, "merge_overflows": overflows,
                "clocks": clocks, "gpu_launches": args.steps,
                "baseline_metric": "3D APT Mcell-upd/s & HBM GB/s, mixed vs FP32; served sims/hr,"
                                   " p50/p99 at <=1e-3 err"}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
