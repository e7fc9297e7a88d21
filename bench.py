#!/usr/bin/env python3
"""Benchmark of the FALL3D ADS time step on B200 (cell*bin*steps/s).

python bench.py --gpus N --steps K --warmup W [--impl reference] [--workload ...]

One process per GPU (torchrun for N > 1).  Ensemble members are independent
replicas, so each rank advances its own members with no data-path
collective ("scaling": "weak"); torch.distributed only provides the barrier
around the timed region and the max-over-ranks of the device time.

Workloads (seeded synthetic inputs standing in for a meteo database):
  ensemble  (default, the headline) the 64-member ensemble on uneven grids,
            12 bins (fall3d_b200.ensemble): FP32 + batched ensemble + learned
            settling velocity timed; the plain FP64 form (one domain per
            member, iterative settling velocity) timed on the first member of
            each grid class and weighted by the class member counts; errors
            of those members against their FP64 runs after the same steps
  c2        400x300x60 grid, 20 bins, random-phase winds, log-normal K, two
            Suzuki sources (one domain per GPU), FP32 precision form timed,
            FP64 form timed on the same inputs for the ratio
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell·bin·steps/s on 1 B200: FP32+ensemble+MLP vs plain FP64, ≤1e-5 rel L2"
# precision forms of the timed ensemble: FP32 stencil on the compensated
# hi + lo state (conservative, the default), or on a plain FP32 state
PRECISIONS = {"fp32c": 2, "fp32": 1}
FORMS = {"fp32c": "FP32 stencils on a compensated FP32 hi + lo state with a conservative FP64 "
                  "final update per cell (FP64 deposit, flux sums, CFL)",
         "fp32": "FP32 state and stencils (FP64 deposit, flux sums, CFL)"}
UNIT = "cell*bin*steps/s"
L2_BYTES = 126 * 2**20


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ---------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return ws, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def cuda_events(stream_ptr: int, device: int):
    import torch
    s = torch.cuda.ExternalStream(stream_ptr, device=torch.device("cuda", device))
    return s, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


# ---------------------------------------------------------------------------
def run_aux(args, local):
    """The kernels around the step on the 400x300x60x20 domain (FP32 form):
    the meteo term from corner fields with CMAQ horizontal and similarity
    vertical K, wet deposition, radioactive decay, the gravity current,
    kept boundary halos, the output reductions and the mass sink.  Prints
    event-timed costs (ms) per call or per step; the per-kernel launch list
    comes from ncu on this workload."""
    import torch
    from fall3d_b200 import workloads as W
    from fall3d_b200.ads import PREC_FP32, Domain, set_zsweep_epilogue
    torch.cuda.set_device(local)
    wl = W.random_c2(seed=0)
    g = wl.grid
    nb = wl.nbins
    rng = np.random.default_rng(7)
    shp = (g.nx + 1, g.ny + 1, g.nz + 1)
    zz = (np.arange(g.nz + 1) / g.nz)[None, None, :]
    uc = [np.asfortranarray(rng.uniform(-20.0, 20.0, shp)) for _ in range(2)]
    vc = [np.asfortranarray(rng.uniform(-20.0, 20.0, shp)) for _ in range(2)]
    wc = [np.asfortranarray(rng.uniform(-0.3, 0.3, shp)) for _ in range(2)]
    tvc = [np.asfortranarray(290.0 - 40.0 * zz + rng.uniform(-2.0, 2.0, shp)) for _ in range(2)]
    n2 = (g.nx, g.ny)
    pblh = np.asfortranarray(rng.uniform(300.0, 2500.0, n2))
    mon = np.asfortranarray(rng.choice([-1.0, 1.0], n2) * rng.uniform(10.0, 500.0, n2))
    ust = np.asfortranarray(rng.uniform(0.05, 0.8, n2))
    pre = np.asfortranarray(rng.uniform(0.0, 20.0, n2))
    cat = np.ones(nb, np.int32)
    spe = np.ones(nb, np.int32)
    cat[-4:], spe[-4:] = 3, [8, 9, 6, 7]  # Sr90, Y90, Cs137, I131
    dom = Domain(g, nb, wl.limiter, wl.time_marching, PREC_FP32, device=local)
    st, e0, e1 = cuda_events(dom.stream_ptr, local)
    ms = {}

    def timed(name, fn, reps=1):
        torch.cuda.synchronize(local)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(local)
        ms[name] = round(e0.elapsed_time(e1) / reps, 4)

    dom.set_terrain()
    timed("meteo_term_cmaq_similarity_incl_h2d", lambda: dom.set_meteo_corners_kdiffu(
        uc, vc, wc, 2, 3, 0.5, tvc_pair=tvc, pblh=pblh, mon=mon, ust=ust, t_its=0.0, t_ite=3600.0))
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    dom.set_source(wl.src_ijk, wl.src_vals)
    _, dt = dom.grid_get_time_step(0.5, wl.criterion, wl.cfl, wl.run_end)
    c0, a0 = W.random_state(wl, seed=3)
    dom.upload_state(c0, a0)
    K = max(args.steps, 1)
    t = [0.0]

    def steps():
        for _ in range(K):
            dom.step_async(dt, t[0], 0)
            t[0] += dt
    for _ in range(args.warmup):
        dom.step_async(dt, t[0], 0)
    timed("step_plain", steps)
    ms["step_plain"] = round(ms["step_plain"] / K, 4)
    dom.phys_wet_deposition(8.4e-5, 0.79, pre, pblh, cat, wl.diam)
    dom.phys_radionuclides(cat, spe)
    set_zsweep_epilogue(True)  # inside the z sweep
    timed("step_wet_decay_zsweep_epilogue", steps)
    ms["step_wet_decay_zsweep_epilogue"] = round(ms["step_wet_decay_zsweep_epilogue"] / K, 4)
    set_zsweep_epilogue(False)  # the default: separate passes after the z sweep
    timed("step_wet_decay", steps)
    ms["step_wet_decay"] = round(ms["step_wet_decay"] / K, 4)
    dom.set_gravity_current(g.lon_p[g.nx // 2], g.lat_p[g.ny // 2], -3600.0, 1e9, 430.0, 0.1, 0.02, 0.2, 1e6,
                            0.8 * g.z_c.max(), 0.0)
    timed("step_wet_decay_gravity_current", steps)
    ms["step_wet_decay_gravity_current"] = round(ms["step_wet_decay_gravity_current"] / K, 4)
    dom.keep_boundary_halo()
    timed("step_all_kept_halo", steps)
    ms["step_all_kept_halo"] = round(ms["step_all_kept_halo"] / K, 4)
    dom.nc_IO_out_res(range(nb - 4))  # first call: scratch allocation
    dom.grid_get_mass_sink()
    timed("output_species_incl_d2h", lambda: dom.nc_IO_out_res(range(nb - 4)), reps=3)
    timed("mass_sink_incl_d2h", lambda: dom.grid_get_mass_sink(), reps=3)
    dom.close()
    print(json.dumps({"workload": f"aux: {g.nx}x{g.ny}x{g.nz} grid, {nb} bins, FP32 form",
                      "ms": ms, "steps": K}), flush=True)


# ---------------------------------------------------------------------------
def sweep_bytes(wl, prec_bytes: int, d: str) -> float:
    """Algorithmic HBM bytes of one sweep launch (per the roofline model):
    c read+write per cell*bin, the per-face fields once, and for z the
    per-bin settling velocity."""
    g = wl.grid
    nx, ny, nz, nb = g.nx, g.ny, g.nz, wl.nbins
    cells = nx * ny * nz
    c_rw = 2.0 * prec_bytes * cells * nb
    # FP32: one float4 per face {two wind snapshots, face diffusion, 1/dxb};
    # FP64: current wind + face diffusion
    face = 16.0
    if d == "x":
        return c_rw + face * (nx + 1) * ny * nz
    if d == "y":
        return c_rw + face * (ny + 1) * nx * nz
    return c_rw + face * (nz + 1) * nx * ny + prec_bytes * (nz + 1) * nx * ny * nb


def load_traffic(kernel: str, workload: str, algorithmic: float = None):
    """DRAM bytes per launch from an ncu capture (profiles/traffic.json).
    Workloads too large to capture use the measured/algorithmic ratio of
    the same kernel on the 400x300x60x20 case, scaled to their algorithmic
    bytes."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d.get(workload, {}).get(kernel)
        if e is not None:
            return float(e)
        ratio = d.get("ratio_measured_to_algorithmic", {})
        if algorithmic is not None and kernel in ratio:
            return float(ratio[kernel]) * algorithmic
        if algorithmic is not None and kernel == "fused32" and ratio:
            return float(sum(ratio.values()) / len(ratio)) * algorithmic
        return None
    except Exception:
        return None


def traffic_source(kernel: str, workload: str) -> str:
    """Where load_traffic's figure for this kernel and workload comes from."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            direct = kernel in json.load(f).get(workload, {})
    except Exception:
        direct = False
    if direct:
        return ("ncu DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum, one pass) of this "
                "kernel on the same workload")
    return ("ncu DRAM bytes of the same kernel on the 400x300x60x20 case, as a ratio to its "
            "algorithmic bytes, times this launch's algorithmic bytes")


def setup_domain(wl, prec, device):
    from fall3d_b200.ads import Domain
    dom = Domain(wl.grid, wl.nbins, wl.limiter, wl.time_marching, prec, device=device)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    dom.set_source(wl.src_ijk, wl.src_vals)
    s_mid = 0.5
    _, dt = dom.grid_get_time_step(s_mid, wl.criterion, wl.cfl, wl.run_end)
    return dom, dt


def time_steps(dom, dt, K, W, device, pg, t0=0.0):
    """W warm-up steps then K timed steps; device time by CUDA events."""
    import torch
    t = t0
    for it in range(W):
        dom.step_async(dt, t, it)
        t += dt
    dom.synchronize()
    s, e0, e1 = cuda_events(dom.stream_ptr, device)
    torch.cuda.synchronize(device)
    barrier(pg)
    n0 = dom.launch_count()
    e0.record(s)
    for it in range(W, W + K):
        dom.step_async(dt, t, it)
        t += dt
    e1.record(s)
    dom.synchronize()
    torch.cuda.synchronize(device)
    barrier(pg)
    launches = dom.launch_count() - n0
    return e0.elapsed_time(e1), launches, t


def run_c2(args, ws, rank, local, pg):
    import torch
    from fall3d_b200 import workloads as W
    from fall3d_b200.ads import PREC_FP64
    torch.cuda.set_device(local)
    wl = W.random_c2(seed=rank)
    g = wl.grid
    cbs = float(g.nx * g.ny * g.nz * wl.nbins)
    K, Wu = args.steps, args.warmup
    out = {}
    # ---- FP64 plain form (ratio denominator), same steps from the same state
    dom64, dt = setup_domain(wl, PREC_FP64, local)
    ms64, _, _ = time_steps(dom64, dt, K, Wu, local, pg)
    ms64 = max_over_ranks(pg, ms64)
    fp64_value = ws * cbs * K / (ms64 / 1e3)
    c64 = dom64.download_state()[0] if rank == 0 else None
    dom64.close()
    # ---- the precision form (headline on this workload)
    prec = PRECISIONS[args.precision]
    dom, dt32 = setup_domain(wl, prec, local)
    with ClockSampler(local) as clk:
        ms, launches, t_end = time_steps(dom, dt32, K, Wu, local, pg)
    ms = max_over_ranks(pg, ms)
    value = ws * cbs * K / (ms / 1e3)
    out.update(value=value, ms_per_step=ms / K, fp64_value=fp64_value, launches=launches,
               clocks=clk.summary(), fp64_ms_per_step=ms64 / K)
    out["fp64_roofline"] = fp64_roofline(fp64_value / ws, out["clocks"].get("sm_mhz"))
    if c64 is not None:
        # FP32 form against the FP64 form after the same W+K steps (dt of the
        # FP64 CFL reduction in both)
        c32 = dom.download_state()[0]
        a, b = c64[2:-2, 2:-2, 2:-2, :], c32[2:-2, 2:-2, 2:-2, :]
        out["fp32_rel_l2_vs_fp64"] = float(np.linalg.norm(b - a) / np.linalg.norm(a))
        out["fp32_rel_l2_vs_fp64_worst_bin"] = float(max(
            np.linalg.norm(b[..., q] - a[..., q]) / max(np.linalg.norm(a[..., q]), 1e-300)
            for q in range(a.shape[-1])))
        del c32
    # ---- per-kernel profile (event-timed phases) for the roofline
    dom.set_profiling(True)
    t = t_end
    for it in range(3):
        dom.step_async(dt32, t, K + Wu + it)
        t += dt32
    prof, n = dom.get_profile()
    dom.set_profiling(False)
    per = {"x": prof[1] / n, "y": prof[2] / n, "z": prof[3] / n}
    dom_k = max(per, key=per.get)
    # the compensated form also reads and writes the low part (4 B each)
    byts = sweep_bytes(wl, 4, dom_k) + (2.0 * 4 * cbs if prec == 2 else 0.0)
    peak, kind = hbm_peak()
    achieved = byts / (per[dom_k] / 1e3) / 1e9
    out["roofline"] = {"bound": "hbm",
                       "kernel": f"k_sweep32<{'xyz'.index(dom_k)},2,2,{int(prec == 2)}> ({dom_k} sweep)",
                       "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                       "frac": round(achieved / peak, 4), "peak_kind": kind,
                       "traffic": load_traffic(f"sweep32{'c' if prec == 2 else ''}_{dom_k}", "c2"),
                       "algorithmic_bytes": byts, "launch_ms": round(per[dom_k], 4),
                       "sweep_ms": {k: round(v, 4) for k, v in per.items()}}
    # ---- e2e through the C ABI with host buffers
    out["e2e"] = e2e_c2(dom, wl, dt32, K, local, pg, ws, cbs)
    dom.close()
    out["workload"] = wl
    return out


def e2e_c2(dom, wl, dt, K, device, pg, ws, cbs):
    """Same metric end to end through the public API: every step crosses the
    C ABI from host scalars and reads the boundary fluxes back (48 B); the
    meteo term is uploaded from pinned host memory and charged per step at
    the FALL3D coupling interval (3600 s of model time / dt steps)."""
    from fall3d_b200.ads import Domain  # noqa: F401  (API in use)
    pinned = [np.asfortranarray(a) for a in (wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3)]
    meteo_bytes = sum(a.nbytes for a in pinned)
    barrier(pg)
    t0 = time.perf_counter()
    dom.set_meteo(*pinned, None, wl.t_its, wl.t_ite)
    t1 = time.perf_counter()
    f = np.zeros(6)
    t = 0.0
    for it in range(K):
        dom.F3D_time_step(dt, t, it, f)
        t += dt
    t2 = time.perf_counter()
    steps_per_meteo = max(1.0, 3600.0 / dt)
    t_meteo = t1 - t0
    t_steps = t2 - t1
    t_tot = max_over_ranks(pg, t_steps + t_meteo * K / steps_per_meteo)
    return {"value": ws * cbs * K / t_tot, "unit": UNIT,
            "h2d_bytes_per_step": int(meteo_bytes / steps_per_meteo + 20),
            "d2h_bytes_per_step": 48,
            "meteo_upload_s": round(t_meteo, 4), "steps_per_meteo_interval": round(steps_per_meteo, 1)}


def cpu_baseline_c2(wl, steps=2):
    """The CPU FP64 oracle (restatement of the reference path) with all host
    threads, on a bounded sample of the same workload."""
    from oracle import oracle as O
    from fall3d_b200.source import dense_source
    g = wl.grid
    threads = os.cpu_count() or 1
    orc = O.Oracle(g, wl.nbins, wl.limiter, wl.time_marching, threads=threads)
    vs = column_vset(O, wl)
    c = np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, wl.nbins), order="F")
    a = np.zeros((g.nx + 4, g.ny + 4, wl.nbins), order="F")
    s = dense_source(g, wl.src_ijk, wl.src_vals, wl.nbins)
    f = np.zeros(6)
    t0 = time.perf_counter()
    t = 0.0
    for it in range(steps):
        orc.time_step(6.5, t, wl.t_its, wl.t_ite, it, c, a, s, wl.u12, wl.v12, wl.w12, wl.k1,
                      wl.k2, wl.k3, vs, f)
        t += 6.5
    el = time.perf_counter() - t0
    return {"value": g.nx * g.ny * g.nz * wl.nbins * steps / el, "unit": UNIT, "cores": threads,
            "kind": "port", "sample": f"{steps} steps of the full {g.nx}x{g.ny}x{g.nz}x{wl.nbins} "
                                      f"case, CPU FP64 oracle, OpenMP over pencils"}


def column_vset(O, wl):
    """Settling velocity from the oracle per level (air properties of these
    synthetic workloads vary with height only), broadcast over the columns."""
    g = wl.grid
    vs = np.zeros((g.nx, g.ny, g.nz + 3, wl.nbins), order="F")
    T = wl.tc[0, 0, :]
    rho = wl.rhoc[0, 0, :]
    for k in range(g.nz + 1):
        visa = 1.827e-5 * ((291.15 + 120.0) / (T[k] + 120.0)) * (T[k] / 291.15) ** 1.5
        for b in range(wl.nbins):
            v, _, _ = O.vset_point(wl.diam[b], wl.rhop[b], wl.psi[b], rho[k], visa, wl.vset_model)
            vs[:, :, k + 1, b] = v
    vs[:, :, 0, :] = vs[:, :, 1, :]
    vs[:, :, g.nz + 2, :] = vs[:, :, g.nz + 1, :]
    return vs


def run_reference_c2(args, ws, rank):
    """Reference arm on the single-domain c2 workload."""
    if rank != 0:
        return
    from fall3d_b200 import workloads as W
    wl = W.random_c2(seed=0)
    from oracle import oracle as O
    from fall3d_b200.source import dense_source
    g = wl.grid
    threads = os.cpu_count() or 1
    orc = O.Oracle(g, wl.nbins, wl.limiter, wl.time_marching, threads=threads)
    vs = column_vset(O, wl)
    c = np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, wl.nbins), order="F")
    a = np.zeros((g.nx + 4, g.ny + 4, wl.nbins), order="F")
    s = dense_source(g, wl.src_ijk, wl.src_vals, wl.nbins)
    f = np.zeros(6)
    t = 0.0
    for it in range(args.warmup):
        orc.time_step(6.5, t, wl.t_its, wl.t_ite, it, c, a, s, wl.u12, wl.v12, wl.w12, wl.k1,
                      wl.k2, wl.k3, vs, f)
        t += 6.5
    t0 = time.perf_counter()
    for it in range(args.steps):
        orc.time_step(6.5, t, wl.t_its, wl.t_ite, args.warmup + it, c, a, s, wl.u12, wl.v12,
                      wl.w12, wl.k1, wl.k2, wl.k3, vs, f)
        t += 6.5
    el = time.perf_counter() - t0
    cbs = g.nx * g.ny * g.nz * wl.nbins
    v = cbs * args.steps / el
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "c2: 400x300x60 grid, 20 bins, 2 Suzuki sources",
                       "parallelism": "cpu-openmp"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full steps of the 400x300x60x20 case"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# The 64-member ensemble: FP32 + batched ensemble + learned settling velocity
# against the plain FP64 form (one domain per member, iterative settling
# velocity) on the same members.
ENS_CONFIG = ("64 members on uneven grids: 16x(200x150x40) + 32x(400x300x60) + 16x(600x450x80), "
              "12 bins (phi -2..6), winds x(1+-20%), source height +-2 km, mass rate x[0.5,2] "
              "log-uniform")
METEO_INTERVAL_S = 3600.0   # meteo coupling interval: settling velocity recomputed once per hour


def class_reps(ew):
    """First member (unperturbed winds) of every grid class."""
    return [ew.member_class.index(c) for c in range(len(ew.classes))]


def fp64_member_domain(ew, m, device):
    """The plain FP64 form of member m: its own domain, iterative settling
    velocity, the member's perturbed winds and source."""
    from fall3d_b200.ads import PREC_FP64, Domain
    wl = ew.classes[ew.member_class[m]]
    f = ew.wind_factor[m]
    dom = Domain(wl.grid, wl.nbins, wl.limiter, wl.time_marching, PREC_FP64, device=device)
    dom.set_meteo(np.asfortranarray(f * wl.u12), np.asfortranarray(f * wl.v12), wl.w12, wl.k1, wl.k2,
                  wl.k3, None, wl.t_its, wl.t_ite)
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    ijk, vals = ew.src[m]
    dom.set_source(ijk, vals)
    return dom


def deposit_mass(g, acum):
    area = g.dX1_p[2:-2][:, None] * (g.Hm1_p * g.dX2_p[2:-2])[None, :]
    return float((acum[2:-2, 2:-2, :] * area[:, :, None]).sum())


def run_ensemble(args, ws, rank, local, pg):
    import torch
    from fall3d_b200.ensemble import Ensemble, autotune, ensemble_workload
    from fall3d_b200.mlp import trained_surrogate
    torch.cuda.set_device(local)
    K, Wu = args.steps, args.warmup
    ew = ensemble_workload(seed=rank)
    nm, nb = len(ew.member_class), ew.nbins
    cbs = float(ew.cell_bins())
    out = {"workload": ew, "state_bytes": 8 if args.precision == "fp32c" else 4}
    # ---- learned settling velocity (trained once, outside the timed region)
    t0 = time.perf_counter()
    sur = trained_surrogate(device=local)
    out["mlp_train_s"] = round(time.perf_counter() - t0, 2)
    out["mlp_train_ms_device"] = round(sur.train_ms, 1)
    # ---- FP32 batched ensemble; class settling velocity by the iteration
    # (timed, for the plain arm) and then by the surrogate (kept)
    ens = Ensemble([c.grid for c in ew.classes], nb, ew.member_class, ew.wind_factor, 2, 2,
                   PRECISIONS[args.precision], local)
    vinfo = {"iter_ms": [], "mlp_ms": [], "fallback_faces": [], "faces": []}
    for ci, wl in enumerate(ew.classes):
        ens.set_class_meteo(ci, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
        for rep in range(2):  # second pass timed (warm)
            ens.compute_class_vset(ci, wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
            it_ms = ens.vset_ms()
            nfb = ens.compute_class_vset_mlp(ci, sur, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat, 1)
            ml_ms = ens.vset_ms()
        vinfo["iter_ms"].append(round(it_ms, 3))
        vinfo["mlp_ms"].append(round(ml_ms, 3))
        vinfo["fallback_faces"].append(int(nfb))
        vinfo["faces"].append(int((wl.grid.nz + 1) * wl.grid.ny * wl.grid.nx * nb))
    for m, (ijk, vals) in enumerate(ew.src):
        ens.set_member_source(m, ijk, vals)
    run_end = ew.classes[0].run_end
    dts = ens.compute_time_steps(0.5, 2, 0.9, run_end)
    reps = class_reps(ew)
    steps_per_meteo = [max(1.0, METEO_INTERVAL_S / dts[m]) for m in reps]
    # ---- autotune (tile shapes / mode), then a fresh start
    key = f"ens64-{nb}-{args.precision}-{torch.cuda.get_device_name(local)}"
    tune = autotune(ens, key, steps=2)
    out["tuning"] = {"mode": ["kernels+graphs", "persistent"][tune["tuning"][0]],
                     "bins_per_block": tune["tuning"][1], "ctas_per_sm": tune["tuning"][2],
                     "candidates": [{"tuning": r["tuning"], "ms_per_step": round(r.get("ms_per_step", -1), 3)}
                                    for r in tune.get("all", [])]}
    ens.reset_state()
    ens.set_clock(np.zeros(nm), 0)
    ens.run(Wu)
    ens.synchronize()
    s = torch.cuda.ExternalStream(ens.stream_ptr, device=torch.device("cuda", local))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(local)
    barrier(pg)
    n0 = ens.launch_count()
    with ClockSampler(local) as clk:
        e0.record(s)
        ens.run(K)
        e1.record(s)
        ens.synchronize()
    torch.cuda.synchronize(local)
    barrier(pg)
    ms_steps = max_over_ranks(pg, e0.elapsed_time(e1))
    if ens.status() != 0:
        raise RuntimeError("device barrier timeout in the timed region")
    # settling velocity once per meteo interval, per class, amortised per step
    vset_amort = sum(vinfo["mlp_ms"][c] / steps_per_meteo[c] for c in range(len(ew.classes)))
    ms_tot = ms_steps + K * vset_amort
    out.update(value=ws * cbs * K / (ms_tot / 1e3), ms_per_step=ms_tot / K,
               steps_only_value=ws * cbs * K / (ms_steps / 1e3), launches=ens.launch_count() - n0,
               clocks=clk.summary(), vset=vinfo, vset_amortised_ms_per_step=round(vset_amort, 4),
               steps_per_meteo_interval=[round(x, 1) for x in steps_per_meteo])
    # ---- plain FP64 arm: each class's first member as its own domain, the
    # same W + K steps with the same dt; error of the FP32+MLP members
    fp64_ms = []
    errs = []
    iter_amort = 0.0
    flux_tot = ens.get_fluxes()  # boundary-flux totals of the W + K steps
    for ci, m in enumerate(reps):
        dom = fp64_member_domain(ew, m, local)
        g = ew.classes[ci].grid
        ms64, _, _ = time_steps(dom, float(dts[m]), K, Wu, local, pg)
        fp64_ms.append(max_over_ranks(pg, ms64))
        c64, a64 = dom.download_state()
        mv64 = dom.grid_get_mass_volume()
        out64 = float(np.abs(dom.get_fluxes(np.zeros(6))[:5]).sum())
        dom.close()
        c32, a32 = ens.download_member_state(m)
        mv32 = ens.mass_volume(m)
        out32 = float(np.abs(flux_tot[m, :5]).sum())
        i64, i32 = c64[2:-2, 2:-2, 2:-2, :], c32[2:-2, 2:-2, 2:-2, :]
        d64, d32 = deposit_mass(g, a64), deposit_mass(g, a32)
        errs.append({"member": m, "grid": f"{g.nx}x{g.ny}x{g.nz}",
                     "conc_rel_l2": float(np.linalg.norm(i32 - i64) / np.linalg.norm(i64)),
                     "conc_rel_l2_worst_bin": float(max(np.linalg.norm(i32[..., q] - i64[..., q]) /
                                                        max(np.linalg.norm(i64[..., q]), 1e-300)
                                                        for q in range(nb))),
                     "deposit_rel": abs(d32 / d64 - 1.0) if d64 else 0.0,
                     # mass budget: in the volume + ground deposit + out through
                     # the lateral and top boundaries (mod_Grid.F90:1340-1511)
                     "mass_rel": abs((mv32 + d32 + out32) / (mv64 + d64 + out64) - 1.0),
                     # grid_get_mass_volume alone (mod_Grid.F90:1340-1389)
                     "mass_volume_rel": abs(mv32 / mv64 - 1.0)})
        del c64, a64, c32, a32, i64, i32
        n_c = ew.member_class.count(ci)
        # every plain member job recomputes its own settling velocity by the iteration
        iter_amort += sum(vinfo["iter_ms"][ci] / max(1.0, METEO_INTERVAL_S / dts[q])
                          for q in range(nm) if ew.member_class[q] == ci)
    fp64_step_ms = sum(ew.member_class.count(ci) * fp64_ms[ci] / K for ci in range(len(reps)))
    fp64_tot = fp64_step_ms + iter_amort
    out.update(fp64_value=ws * cbs / (fp64_tot / 1e3), fp64_ms_per_step=fp64_tot,
               fp64_steps_value=ws * cbs / (fp64_step_ms / 1e3),
               fp64_class_ms_per_step=[round(x / K, 3) for x in fp64_ms], errors=errs)
    out["ens"], out["sur"], out["dts"], out["reps"] = ens, sur, dts, reps
    out["steps_per_meteo"] = steps_per_meteo
    return out


# FP64 operations (DFMA + DADD + DMUL, thread level) per cell*bin*step of the
# plain FP64 sweeps, from ncu on the 400x300x60x20 case
# (profiles/k_sweep64_c2.md); FP64 pipe of the B200: 64 operations per clock
# per SM on 148 SMs.
FP64_OPS_PER_CELLBIN_STEP = 1066


def fp64_roofline(steps_value, sm_mhz):
    if not FP64_OPS_PER_CELLBIN_STEP or not sm_mhz:
        return None
    peak = 148 * 64 * sm_mhz * 1e6
    achieved = FP64_OPS_PER_CELLBIN_STEP * steps_value
    return {"bound": "fp64 pipe", "ops_per_cellbin_step": FP64_OPS_PER_CELLBIN_STEP,
            "achieved_tops": round(achieved / 1e12, 3), "peak_tops": round(peak / 1e12, 3),
            "frac": round(achieved / peak, 4),
            "note": "step kernels of the plain FP64 form (settling velocity excluded); "
                    "peak = 148 SMs x 64 FP64 ops/clock at the sampled SM clock"}


def time_plain_fp32(args, ew, ws, local, pg, tuning):
    """The plain FP32 form (no compensated state) on the same ensemble, for
    reference: W + K steps from rest, device time of the K."""
    import torch
    from fall3d_b200.ensemble import Ensemble
    nb = ew.nbins
    ens = Ensemble([c.grid for c in ew.classes], nb, ew.member_class, ew.wind_factor, 2, 2, 1, local)
    for ci, wl in enumerate(ew.classes):
        ens.set_class_meteo(ci, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
        ens.compute_class_vset(ci, wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    for m, (ijk, vals) in enumerate(ew.src):
        ens.set_member_source(m, ijk, vals)
    ens.compute_time_steps(0.5, 2, 0.9, ew.classes[0].run_end)
    ens.set_tuning(*tuning)
    ens.set_clock(np.zeros(len(ew.member_class)), 0)
    ens.run(args.warmup)
    ens.synchronize()
    s = torch.cuda.ExternalStream(ens.stream_ptr, device=torch.device("cuda", local))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(pg)
    e0.record(s)
    ens.run(args.steps)
    e1.record(s)
    ens.synchronize()
    ms = max_over_ranks(pg, e0.elapsed_time(e1)) / args.steps
    ens.close()
    return {"value": ws * float(ew.cell_bins()) / (ms / 1e3), "ms_per_step": round(ms, 3),
            "note": "plain FP32 state, same workload and tuning, step kernels only"}


def ens_roofline(r, K):
    """Dominant kernel of the ensemble step, from event-timed profiled steps
    in the tuned mode; algorithmic bytes: every member's concentration (the
    compensated form: its hi and lo parts) read and written once per sweep,
    the class fields (shared by the members of a class) once."""
    ens, ew = r["ens"], r["workload"]
    ens.set_profiling(True)
    ens.run(3)
    ens.synchronize()
    ms, n = ens.get_profile()
    ens.set_profiling(False)
    per = ms / max(n, 1)
    nb = ew.nbins

    def bytes_dir(d):
        tot = 0.0
        for ci, wl in enumerate(ew.classes):
            g = wl.grid
            nmem = ew.member_class.count(ci)
            cells = g.nx * g.ny * g.nz
            # c read + write: FP32 (4 B), or the compensated pair hi + lo (8 B)
            tot += nmem * 2.0 * r["state_bytes"] * cells * nb
            tot += sweep_bytes(wl, 4, d) - 2.0 * 4 * cells * nb  # class fields once
        return tot

    peak, kind = hbm_peak()
    if r["tuning"]["mode"] == "persistent":
        byts = sum(bytes_dir(d) for d in "xyz")
        t = per[1]
        name = "k_fused32 (persistent step: x, y, z sweeps of all 64 members)"
        tkey = "fused32"
    else:
        sw = {"x": per[1], "y": per[2], "z": per[3]}
        dk = max(sw, key=sw.get)
        byts = bytes_dir(dk)
        t = sw[dk]
        cmp = int(r["state_bytes"] == 8)
        name = f"k_sweep32<{'xyz'.index(dk)},2,2,{cmp}> ({dk} sweep of all 64 members)"
        tkey = f"sweep32{'c' if cmp else ''}_{dk}"
    achieved = byts / (t / 1e3) / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": kind,
            "traffic": load_traffic(tkey, "ensemble", byts), "algorithmic_bytes": byts,
            "traffic_source": traffic_source(tkey, "ensemble"),
            "launch_ms": round(t, 3),
            "phase_ms": {k: round(float(v), 3) for k, v in zip(("prep", "x", "y", "z", "flux"), per)}}


def pinned_copy(a):
    """A Fortran-ordered copy of a in page-locked host memory (f3d_host_alloc)."""
    import ctypes as C
    from fall3d_b200._lib import check, lib
    p = C.c_void_p()
    check(lib().f3d_host_alloc(max(a.nbytes, 1), C.byref(p)), "f3d_host_alloc")
    buf = (C.c_char * a.nbytes).from_address(p.value)
    arr = np.ndarray(a.shape, a.dtype, buffer=buf, order="F")
    arr[...] = a
    return arr, p


def e2e_ensemble(r, K, pg, ws):
    """The same metric through the public API with host buffers: every step is
    f3d_ens_step with host dt/time arrays and the boundary fluxes of all
    members read back; the meteo term (from pinned host memory) and the
    surrogate settling velocity (corner air fields uploaded) are charged per
    step at the meteo coupling interval of the most frequently updated class."""
    from fall3d_b200._lib import lib
    ens, ew, sur, dts = r["ens"], r["workload"], r["sur"], r["dts"]
    nm = len(ew.member_class)
    cbs = float(ew.cell_bins())
    held = []
    pin = []
    for wl in ew.classes:
        arrs = []
        for a in (wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, wl.rhoc, wl.tc):
            x, h = pinned_copy(np.asfortranarray(a))
            arrs.append(x)
            held.append(h)
        pin.append(arrs)
    meteo_bytes = sum(x.nbytes for arrs in pin for x in arrs)
    ens.reset_state()
    barrier(pg)
    t0 = time.perf_counter()
    for ci, wl in enumerate(ew.classes):
        u, v, w, k1, k2, k3, rc, tc = pin[ci]
        ens.set_class_meteo(ci, u, v, w, k1, k2, k3, None, wl.t_its, wl.t_ite)
        ens.compute_class_vset_mlp(ci, sur, rc, tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat, 1)
    t1 = time.perf_counter()
    fl = np.zeros(6 * nm)
    times = np.zeros(nm)
    for it in range(K):
        ens.step(dts, times, it, fl)
        times = times + dts
    t2 = time.perf_counter()
    for h in held:
        lib().f3d_host_free(h)
    spm = min(r["steps_per_meteo"])
    t_tot = max_over_ranks(pg, (t2 - t1) + (t1 - t0) * K / spm)
    return {"value": ws * cbs * K / t_tot, "unit": UNIT,
            "h2d_bytes_per_step": int(meteo_bytes / spm + 16 * nm + 8),
            "d2h_bytes_per_step": 48 * nm,
            "meteo_and_vset_upload_s": round(t1 - t0, 3), "steps_per_meteo_interval": round(spm, 1)}


def oracle_member_steps(O, ew, m, dt, steps, threads, warm=0):
    """Seconds for `steps` FP64 oracle steps of member m (after `warm`)."""
    from fall3d_b200.source import dense_source
    wl = ew.classes[ew.member_class[m]]
    g = wl.grid
    orc = O.Oracle(g, wl.nbins, wl.limiter, wl.time_marching, threads=threads)
    vs = column_vset(O, wl)
    f = ew.wind_factor[m]
    u12, v12 = np.asfortranarray(f * wl.u12), np.asfortranarray(f * wl.v12)
    c = np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, wl.nbins), order="F")
    a = np.zeros((g.nx + 4, g.ny + 4, wl.nbins), order="F")
    ijk, vals = ew.src[m]
    src = dense_source(g, ijk, vals, wl.nbins)
    fl = np.zeros(6)
    t = 0.0
    for it in range(warm):
        orc.time_step(dt, t, wl.t_its, wl.t_ite, it, c, a, src, u12, v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, fl)
        t += dt
    t0 = time.perf_counter()
    for it in range(warm, warm + steps):
        orc.time_step(dt, t, wl.t_its, wl.t_ite, it, c, a, src, u12, v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, fl)
        t += dt
    return time.perf_counter() - t0


def cpu_baseline_ensemble(ew, dts, steps=1, warm=0):
    """The CPU FP64 oracle (restatement of the reference path), all host
    threads, on a bounded sample: `steps` steps (after `warm` untimed ones)
    of the first member of each grid class, weighted by the number of
    members of the class."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    reps = class_reps(ew)
    secs = [oracle_member_steps(O, ew, m, float(dts[m]), steps, threads, warm) for m in reps]
    tot = sum(ew.member_class.count(ci) * secs[ci] for ci in range(len(reps)))
    return {"value": float(ew.cell_bins()) * steps / tot, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} step(s) of the first member of each grid class (200x150x40, 400x300x60, "
                      f"600x450x80; 12 bins) after {warm} untimed, FP64 oracle with OpenMP over "
                      f"pencils; rate = sample cell*bin*steps / measured seconds, classes weighted by "
                      f"their member counts (16, 32, 16)",
            "class_seconds": [round(x, 3) for x in secs]}


def run_reference_ensemble(args, ws, rank):
    """Reference arm: the CPU restatement of the reference path (the Fortran
    reference cannot be built here) on the host cores, on the same ensemble
    workload and metric.  Each step is a bounded sample of the 64-member
    step: one time step of the first member of each grid class.  The rate is
    the sample's cell*bin*steps over its measured seconds, with the classes
    weighted by their member counts; ms_per_step is the measured wall time
    of one sampled step (what this process actually ran)."""
    if rank != 0:
        return
    from fall3d_b200.ensemble import ensemble_workload
    ew = ensemble_workload(seed=0)
    dts = [6.0] * len(ew.member_class)
    base = cpu_baseline_ensemble(ew, dts, steps=args.steps, warm=args.warmup)
    v = base["value"]
    sample_s = sum(base["class_seconds"])
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sample_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "ensemble: " + ENS_CONFIG,
                       "sample": "each step: one step of the first member of each grid class "
                                 "(3 of the 64 members), class rates weighted by member counts",
                       "parallelism": "cpu-openmp"},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def line_ensemble(args, ws, res):
    ew = res["workload"]
    e = res["errors"]
    line = {
        "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "ensemble: " + ENS_CONFIG,
                   "form": FORMS[args.precision] + ", batched ensemble step, learned settling "
                           "velocity (surrogate + one Steffensen correction; iteration outside the "
                           "envelope), once per 1 h meteo interval",
                   "parallelism": f"replicas x{ws} (one 64-member ensemble per GPU)",
                   "l2": f"inputs larger than L2: member concentrations total "
                         f"{ew.cell_bins() * 4 / 2**30:.1f} GiB vs {L2_BYTES / 2**20:.0f} MiB L2"},
        "fp64_plain_value": res["fp64_value"],
        "fp64_ms_per_step": res["fp64_ms_per_step"],
        "speedup_vs_fp64_plain": res["value"] / res["fp64_value"],
        "fp64_roofline": fp64_roofline(res["fp64_steps_value"], res["clocks"].get("sm_mhz")),
        "steps_only_value": res["steps_only_value"],
        "gpu_launches": res["launches"],
        "clocks": res["clocks"],
        "roofline": res["roofline"],
        "e2e": res["e2e"],
        "errors_vs_fp64": {
            "conc_rel_l2_max": max(x["conc_rel_l2"] for x in e),
            "deposit_rel_max": max(x["deposit_rel"] for x in e),
            "mass_rel_max": max(x["mass_rel"] for x in e),
            "mass_volume_rel_max": max(x["mass_volume_rel"] for x in e),
            "members": e},
        "tuning": res["tuning"],
        "vset": dict(res["vset"], amortised_ms_per_step=res["vset_amortised_ms_per_step"],
                     steps_per_meteo_interval=res["steps_per_meteo_interval"],
                     mlp_train_s=res["mlp_train_s"], mlp_train_ms_device=res["mlp_train_ms_device"]),
        "fp64_class_ms_per_step": res["fp64_class_ms_per_step"],
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ensemble", choices=["ensemble", "c2", "aux"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp32c", choices=sorted(PRECISIONS))
    ap.add_argument("--no-plain-fp32", action="store_true",
                    help="skip timing the plain FP32 form beside the compensated headline")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        # CPU only: rank 0 runs the reference path on the host cores, the other
        # ranks exit at once; no process group (nor GPU) is needed
        ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
        if args.workload == "ensemble":
            run_reference_ensemble(args, ws, rank)
        else:
            run_reference_c2(args, ws, rank)
        return
    ws, rank, local, pg = dist_setup()
    if args.workload == "aux":
        run_aux(args, local)
        return
    if args.workload == "ensemble":
        res = run_ensemble(args, ws, rank, local, pg)
        res["roofline"] = ens_roofline(res, args.steps)
        res["e2e"] = e2e_ensemble(res, args.steps, pg, ws)
        if rank == 0:
            line = line_ensemble(args, ws, res)
            if ws == 1 and not args.no_cpu_baseline:
                # the reference arm's sample, with up to 10 of its steps (about 45 s)
                line["cpu_baseline"] = cpu_baseline_ensemble(res["workload"], res["dts"],
                                                             steps=min(args.steps, 10), warm=1)
        tuning = res["ens"].tuning
        res["ens"].close()
        res["sur"].close()
        if args.precision == "fp32c" and not args.no_plain_fp32:
            plain = time_plain_fp32(args, res["workload"], ws, local, pg, tuning)
            if rank == 0:
                line["fp32_plain"] = plain
        if rank == 0:
            print(json.dumps(line), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return
    res = run_c2(args, ws, rank, local, pg)
    wl = res.pop("workload")
    if rank == 0:
        g = wl.grid
        line = {
            "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"c2: {g.nx}x{g.ny}x{g.nz} grid, {wl.nbins} bins, one domain per GPU",
                       "form": FORMS[args.precision],
                       "parallelism": f"replicas x{ws}",
                       "l2": f"inputs larger than L2: c is {g.nx*g.ny*g.nz*wl.nbins*4/2**20:.0f} MiB "
                             f"vs {L2_BYTES/2**20:.0f} MiB L2"},
            "fp64_plain_value": res["fp64_value"],
            "fp64_ms_per_step": res["fp64_ms_per_step"],
            "fp64_roofline": res["fp64_roofline"],
            "speedup_vs_fp64": res["value"] / res["fp64_value"],
            "gpu_launches": res["launches"],
            "clocks": res["clocks"],
            "roofline": res["roofline"],
            "e2e": res["e2e"],
        }
        for k in ("fp32_rel_l2_vs_fp64", "fp32_rel_l2_vs_fp64_worst_bin"):
            if k in res:
                line[k] = res[k]
        if ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_c2(wl)
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
