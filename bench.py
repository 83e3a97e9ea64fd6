#!/usr/bin/env python
"""Benchmark of the HERCULES time step on B200: gridpoint-steps/s, mixed vs FP64.

Workload: neutral closed channel, 4th-order FD horizontally, RK3, constant
flow-rate forcing, tanh-stretched wall-normal grid, 512x384x256, seeded laminar
Poiseuille + 10% uniform noise (synthetic: no dataset is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A "step" is one full time step (3 RK sub-steps with 15 Helmholtz/Poisson column
solves, 5 forward + 5 inverse 2-D FFT pairs, statistics). `value` is the
FP32-mixed throughput summed over all ranks; the FP64 run of the same workload
is reported beside it with the mixed-vs-FP64 error. N>1 runs independent
replicas, one per GPU (the north star keeps one domain on one GPU), so the
scaling is weak. --impl reference times the CPU restatement of the reference's
step (the Fortran/MPI reference cannot be built in this image) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "channel_fd4_512x384x256": (512, 384, 256),
    # the same channel with temperature (stable stratification, Ri_b = 0.1)
    "channel_fd4_512x384x256_ri0.1": (512, 384, 256),
    "channel_fd4_256x256x128": (256, 256, 128),
    "channel_fd4_96x64x64": (96, 64, 64),
    # profiling size: production nz with a few GB on the device
    "channel_fd4_256x192x256": (256, 192, 256),
    # stratified open channel, pseudo-spectral horizontal derivatives (cds=3, issk=1)
    "open_spectral_256x256x128": (256, 256, 128),
    "open_spectral_128x128x128": (128, 128, 128),
    # 64 independent stratified closed channels of uneven grids, one CUDA graph per
    # step (grids from {32x32x33, 48x32x49, 64x48x65, 96x64x65}; size = total points)
    "ensemble64": (0, 0, 0),
}
DEFAULT_WORKLOAD = "channel_fd4_512x384x256"
# CPU samples of the same physics, sized for 10-30 s of host work
# (a 16-level slab of the configured 512 x 384 plane: the same transform lengths and
# per-column work as the full grid, whose oracle step would take about a minute)
CPU_SAMPLE_GRID = (512, 384, 16)
REF_STEP_GRID = (512, 384, 16)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="run one precision only (profiling); the headline needs both")
    ap.add_argument("--graph", action="store_true", help="replay each step from a captured CUDA graph")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing leg")
    ap.add_argument("--no-tune", action="store_true", help="ensemble: default tile shapes, no autotuner")
    ap.add_argument("--tile", type=int, nargs=4, default=None,
                    help="single-channel workloads: the tile shapes (hc_params.tile), default automatic")
    ap.add_argument("--stats-gate", choices=["config3", "config2"], default=None,
                    help="run the mixed-vs-FP64 statistics gate (long runs) and print its lines")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint/forward timing leg (Ekman 64x64x65) and print it")
    return ap.parse_args()


def is_spectral(workload: str) -> bool:
    return workload.startswith("open_spectral")


def make_case(workload: str, prec: int, tile=None):
    """Parameters and seeded initial fields of a workload (tile: hc_params.tile)."""
    from hercules_b200 import inputs
    from hercules_b200.params import config_channel_fd, config_open_channel_spectral
    nx, ny, nz = WORKLOADS[workload]
    if is_spectral(workload):
        p = config_open_channel_spectral(nx, ny, nz, got=0.1, precision=prec)
        f = inputs.loglaw_stratified(p, seed=10)
    else:
        p = config_channel_fd(nx, ny, nz, precision=prec)
        if workload.endswith("_ri0.1"):
            p = p.replace(isscalar=1, got=0.1, tbot=0.0, ttop=1.0)
        f = inputs.poiseuille_noise(p, seed=3)
        if p.isscalar:
            from hercules_b200.params import mesh, t_line
            import numpy as np
            f["t"] = np.broadcast_to(t_line(p, mesh(p)["zc"])[:, None, None], (p.nz, p.ny, p.nx)).copy()
    return (p.replace(tile=list(tile)) if tile else p), f


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, lrank


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, idx: int):
        self.idx = idx
        self.p = None
        self.path = os.path.join("/tmp", f"hc_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        seen = set()
        for r in rows:
            for nm, v in zip(names, r[2]):
                if v.lower().startswith("active"):
                    seen.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(seen), "samples": len(rows)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# Algorithmic words per grid point per RK sub-step of each kernel category
# (physical fields and half spectra both count one word per point; every input
# read once, every output written once).
ALG_WORDS_SUB = {
    # FD path, neutral: RHS reads u,v,w,p,ff,gg,hh, writes qu,qv,qw,ff,gg,hh; the
    # column kernel reads 3 spectra, writes u,v,w,psi; the x inverse also reads p (+=)
    "fd": {"rhs_momentum": 13, "fft_x_r2c": 6, "fft_y_fwd": 6, "column_fd": 7, "fft_y_inv": 8,
           "fft_x_c2r": 9, "div_check": 3,
           # the fused 2-D transforms: forward 3 physical fields in, 3 half spectra
           # out; inverse 4 spectra and p in, u, v, w, p out
           "fft2d_fwd": 6, "fft2d_inv": 9},
    # spectral path (issk=1, scalar): products read u,v,w,t + 6 derivative images,
    # write 8 (+ 7 for T); assembly reads 4 spectra, 8 product spectra, 3 histories,
    # writes 3 histories + 3 RHS (+ 7 for T); the column kernel reads 3 RHS + p,
    # writes u,v,w,p,phi,div; transforms: 6 derivative + 4 state + 1 T inverse,
    # 8 + 3 forward, each pass reads and writes every field
    "sp": {"spec_products": 25, "fft_x_r2c": 22, "fft_y_fwd": 22, "spec_assemble": 28, "column_fd": 10,
           "column_t": 2, "fft_y_inv": 22, "fft_x_c2r": 22, "div_check": 4, "aux": 9,
           # fused 2-D transforms: 11 fields each way, one word in and one out
           "fft2d_fwd": 22, "fft2d_inv": 22},
}
# spectral path with the products fused with their x transform: the momentum
# kernel reads the products' 10 inputs and writes 8 x half spectra; the
# temperature kernel reads 4 and writes 3 (fused too unless a separate temperature
# products kernel shows in the profile, which then keeps 7 words and the x
# forward kernel 3 + 3)
ALG_WORDS_SP_FUSED = {"spec_products_fx": 25, "spec_products": 0, "fft_x_r2c": 0}
ALG_WORDS_SP_FUSED_MOM = {"spec_products_fx": 18, "spec_products": 7, "fft_x_r2c": 6}


# DRAM bytes (read + write) of one launch per kernel category, FP32-mixed, measured
# by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the 256x192x256 case
# and scaled by the point ratio to the grids below (every kernel streams its
# fields once, so traffic grows in proportion to the points).
TRAFFIC_CAPTURE = {"case": "channel_fd4_256x192x256 mixed", "metrics": "dram__bytes_read.sum + dram__bytes_write.sum",
                   "scaled_by_points": True}
_TRAFFIC_256x192x256 = {"rhs_momentum": 618.6e6, "column_fd": 295.2e6, "fft_x_r2c": 254.8e6, "fft_y_fwd": 244.5e6,
                        "fft_y_inv": 344.1e6, "fft_x_c2r": 406.9e6, "div_check": 154.9e6, "stats": 1020.2e6}
TRAFFIC = {(w, k): v * (WORKLOADS[w][0] * WORKLOADS[w][1] * WORKLOADS[w][2]) / (256 * 192 * 256)
           for w in ("channel_fd4_512x384x256", "channel_fd4_256x192x256") for k, v in _TRAFFIC_256x192x256.items()}

# FP32 storage: the statistics kernel sums each window of this many steps in FP32
# and folds the window into the FP64 accumulators on its last step
STATS_WINDOW = 16


def stats_bytes_per_point(kind: str, wbytes: int, with_t: bool = True) -> float:
    """Bytes per point and step the statistics kernel must move: u, v, w, t (and the
    uhx, vhy snapshots on the FD path) in the storage type, and the 11 accumulators
    read and written -- FP64 sums with FP64 storage; with FP32 storage FP32 window
    sums, plus once a window the fold (window read, FP64 sum read and written,
    window cleared). Without a temperature equation T is frozen: its three terms
    are added on request from T and mean_w, and a step moves 8 accumulators and
    no T."""
    nacc = 11 if with_t else 8
    reads = ((6 if kind == "fd" else 4) - (0 if with_t else 1)) * wbytes
    if wbytes == 8:
        return reads + nacc * 2 * 8
    return reads + nacc * 2 * 4 + nacc * (4 + 16 + 4) / STATS_WINDOW


def fused_mode(prof) -> str:
    """Which spectral products ran fused with their x transform, from the kernel
    categories of a profile."""
    if "spec_products_fx" not in prof:
        return ""
    return "mom" if "spec_products" in prof else "all"


def alg_bytes_step(kernel: str, npts: int, wbytes: int, kind: str, nsub: int = 3, fused: str = "") -> float:
    """Algorithmic bytes of one time step in one kernel category (the FD workloads
    are neutral, the spectral ones carry temperature; fused: "all" when the
    spectral products ran fused with their x transform, "mom" when only the
    momentum ones did)."""
    if kernel == "stats":
        return npts * stats_bytes_per_point(kind, wbytes, with_t=kind != "fd")
    if kind == "fd" and kernel == "div_check":
        # sub-steps 1 and 2 check the divergence inside the next momentum RHS; the
        # separate check runs once a step, after the last sub-step
        nsub = 1
    words = ALG_WORDS_SUB[kind].get(kernel, 0)
    if kind == "sp" and fused:
        words = (ALG_WORDS_SP_FUSED if fused == "all" else ALG_WORDS_SP_FUSED_MOM).get(kernel, words)
    return words * nsub * npts * wbytes


def run_gpu(args, ws, rank, hbm):
    import numpy as np
    import torch
    import torch.distributed as dist
    from hercules_b200 import engine, inputs
    from hercules_b200.params import config_channel_fd, PREC_FP64, PREC_MIXED

    nx, ny, nz = WORKLOADS[args.workload]
    npts = nx * ny * nz
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    results = {}
    chans = {}
    precs = {"both": (PREC_FP64, PREC_MIXED), "fp64": (PREC_FP64,), "mixed": (PREC_MIXED,)}[args.precision]
    for prec in precs:
        p, fields = make_case(args.workload, prec, args.tile)
        c = engine.Channel(p)
        c.load(fields)
        c.initialize()
        if args.graph:
            c.set_graph(True)
        rc = c.step_nodiag(args.warmup)
        assert rc == 0, rc
        barrier()
        clk = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
        with clk:
            barrier()
            rc = c.step_nodiag(args.steps)
            barrier()
        assert rc == 0, rc
        ms = max_over_ranks(c.last_ms)
        results[prec] = {"ms_per_step": ms / args.steps, "launches": c.last_launches,
                         "value": ws * npts * args.steps / (ms * 1e-3), "clocks": clk.summary()}
        chans[prec] = c

    if len(precs) == 1:
        for c in chans.values():
            c.close()
        return results, None, {}, None
    # mixed-vs-FP64 error after the same warmup+steps from the same seed
    err = {}
    for f in ("u", "v", "w"):
        a = chans[PREC_MIXED].download(f)
        b = chans[PREC_FP64].download(f)
        err[f] = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    pm = chans[PREC_MIXED].download("p")
    pf = chans[PREC_FP64].download("p")
    err["p"] = float(np.max(np.abs((pm - pm.mean()) - (pf - pf.mean()))) / np.max(np.abs(pf - pf.mean())))
    if chans[PREC_FP64].p.isscalar:
        a, b = chans[PREC_MIXED].download("t"), chans[PREC_FP64].download("t")
        err["t"] = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    # the running statistics (sums over the same steps), each relative to its own max
    for f in ("mean_u", "mean_v", "mean_w", "mean_uu", "mean_vv", "mean_ww", "mean_uw", "mean_vw") + \
            (("mean_t", "mean_tt", "mean_tw") if chans[PREC_FP64].p.isscalar else ()):
        a, b = chans[PREC_MIXED].download(f), chans[PREC_FP64].download(f)
        den = float(np.max(np.abs(b)))
        err[f] = float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a)))

    # per-kernel CUDA-event profile of 2 steps of each run
    kern = {}
    kind = "sp" if is_spectral(args.workload) else "fd"
    nprof = 2
    for prec, tag in ((PREC_MIXED, "mixed"), (PREC_FP64, "fp64")):
        c = chans[prec]
        c.set_profiling(True)
        c.step_nodiag(nprof)
        prof = c.kernel_profile()
        c.set_profiling(False)
        wb = 4 if prec == PREC_MIXED else 8
        kern[tag] = {}
        for k, v in prof.items():
            avg = v["total_ms"] / max(v["launches"], 1)
            b = alg_bytes_step(k, npts, wb, kind, fused=fused_mode(prof)) * nprof
            gbs = (b / (v["total_ms"] * 1e-3) / 1e9) if b and v["total_ms"] > 0 else None
            kern[tag][k] = {"launches": v["launches"], "avg_ms": avg, "total_ms": v["total_ms"],
                            "alg_bytes_per_launch": b / max(v["launches"], 1) if b else None,
                            "alg_gbs": gbs, "frac_of_hbm": gbs / hbm if gbs else None}
    for c in chans.values():
        c.close()

    # end-to-end through the public API with host buffers (mixed)
    e2e = None
    if not args.no_e2e:
        p, host = make_case(args.workload, PREC_MIXED, args.tile)
        host = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in host.items()}
        res = {f: torch.empty((p.nz, p.ny, p.nx), dtype=torch.float64).pin_memory().numpy()
               for f in ("u", "v", "w", "p", "t")}
        barrier()
        t0 = time.perf_counter()
        c = engine.Channel(p)
        ta = time.perf_counter()
        c.load(host)
        tb = time.perf_counter()
        c.initialize()
        tc = time.perf_counter()
        for _ in range(args.steps):
            c.step(1)
        td = time.perf_counter()
        outs = {f: c.download(f, out=res[f]) for f in ("u", "v", "w", "p", "t")}
        outs = None
        barrier()
        t1 = time.perf_counter()
        c.close()
        parts = {"create": ta - t0, "upload": tb - ta, "initialize": tc - tb, "steps": td - tc, "download": t1 - td}
        el = max_over_ranks(t1 - t0)
        from hercules_b200.params import HcDiag
        import ctypes
        e2e = {"value": ws * npts * args.steps / el, "unit": "gridpoint-steps/s",
               "h2d_bytes_per_step": int(5 * npts * 8 / args.steps),
               "d2h_bytes_per_step": int((5 * npts * 8) / args.steps + ctypes.sizeof(HcDiag)),
               "includes": "create + upload of 5 pinned host fields + initialize + K x (hc_step(1) with diag "
                           "copy-back) + download of 5 fields into pinned host buffers, wall clock",
               "parts_ms": {k: round(v * 1e3, 2) for k, v in parts.items()}}
        del outs

    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return results, err, kern, e2e


def run_adjoint(nsteps=50, ckpt=10):
    """The adjoint workload: Ekman layer 64x64x65 FP64, gradient of the mean wall
    shear stress at step 50 with respect to the starting velocity and a smooth
    body force, a checkpoint every 10 steps. Device time of the plain forward
    (hc_step, eager) against the checkpointed forward and the reverse sweep."""
    import numpy as np
    import torch
    from hercules_b200 import adjoint, engine, inputs
    from hercules_b200.params import config_ekman
    torch.cuda.set_device(0)
    p = config_ekman()
    f0 = inputs.small_random(p, seed=21)
    fields = {k: f0[k] for k in ("u", "v", "w")}
    for k in ("p", "ff", "gg", "hh"):          # reloaded before each timed run
        fields[k] = np.zeros_like(f0["u"])
    bf = inputs.gaussian_body_force(p, seed=22, ell=1.0, amp=0.01)
    seeds = {"u": adjoint.wall_shear_seed(p)}

    def fresh():
        c = engine.Channel(p)
        c.load(fields)
        c.set_body_force(*bf)
        c.initialize()
        return c
    c = fresh()
    c.step_nodiag(nsteps)          # warm-up of the plain path
    c.close()
    c = fresh()
    rc = c.step_nodiag(nsteps)
    assert rc == 0, rc
    eager_ms = c.last_ms
    c.close()
    c = fresh()                    # the faster forward: one CUDA graph per step
    c.set_graph(True)
    c.step_nodiag(2)
    c.load(fields)
    c.initialize()
    rc = c.step_nodiag(nsteps)
    assert rc == 0, rc
    fwd_ms, fwd_launch = c.last_ms, c.last_launches
    c.close()
    c = fresh()
    c.adjoint(nsteps, seeds, ckpt=ckpt)    # first call: allocates the checkpoints, captures the graphs
    c.load(fields)
    c.initialize()
    g = c.adjoint(nsteps, seeds, ckpt=ckpt)
    t = c.adjoint_timing()
    c.close()
    return {"workload": f"ekman {p.nx}x{p.ny}x{p.nz} FP64, mean wall shear at step {nsteps}, ckpt {ckpt}",
            "forward_ms": fwd_ms, "forward_launches": fwd_launch, "forward_eager_ms": eager_ms,
            "ckpt_forward_ms": t["forward_ms"], "reverse_ms": t["reverse_ms"],
            "reverse_launches": t["reverse_launches"],
            "reverse_over_forward": t["reverse_ms"] / fwd_ms,
            "gradient_over_forward": (t["forward_ms"] + t["reverse_ms"]) / fwd_ms,
            "grad_norm_u": float(np.sqrt(np.sum(g["u"] ** 2)))}


def run_ensemble(args):
    """All members of the seeded ensemble advanced through one graph per step,
    FP64 and mixed; value = total gridpoint-steps / device time."""
    import numpy as np
    import torch
    from hercules_b200 import engine, inputs
    from hercules_b200.params import PREC_FP64, PREC_MIXED
    torch.cuda.set_device(0)
    out = {}
    tiles = {}
    for prec in (PREC_FP64, PREC_MIXED):
        # tile shapes of each of the four member grids from the autotuner
        cases = inputs.ensemble_members(n=64, seed=1000, precision=prec, tune=not args.no_tune)
        for p, _ in cases:
            tiles[f"{p.nx}x{p.ny}x{p.nz}:{'mixed' if prec else 'fp64'}"] = list(p.tile)
        chans = []
        for p, fields in cases:
            c = engine.Channel(p)
            c.load(fields)
            c.initialize()
            chans.append(c)
        npts = sum(p.nx * p.ny * p.nz for p, _ in cases)
        e = engine.Ensemble(chans)
        e.step(args.warmup)
        clk = Clocks(0)
        with clk:
            e.step(args.steps)
        ms = e.last_ms
        out[prec] = {"value": npts * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps, "npts": npts,
                     "launches": e.launches_per_step * args.steps, "clocks": clk.summary(), "tiles": tiles}
        e.close()
        for c in chans:
            c.close()
    return out


def run_stats_gate(which: str):
    """The statistical gate of the mixed mode: the FP32-mixed and FP64 runs of the
    same seeded start, their running means turned into mean profiles, Reynolds
    stresses, wall friction and (with temperature) heat flux, compared as
    max |mixed - fp64| / max |fp64| per profile (gate: 1 %).

    config3: the 512x384x256 neutral closed channel (FD4, dp_opt=2), statistics of
    all 2000 steps; also with temperature (Ri_b = 0.1, Dirichlet walls) for the
    heat flux. config2: the 256x256x128 stratified open channel (pseudo-spectral,
    fixed bottom-cooling flux), 1000 steps at each Ri_b in {0, 0.1, 0.5, 1.0},
    statistics of the last 500."""
    import numpy as np
    import torch
    from hercules_b200 import engine, inputs, stats
    from hercules_b200.params import PREC_FP64, PREC_MIXED, config_channel_fd, config_open_channel_spectral, t_line
    torch.cuda.set_device(0)
    cases = []
    if which == "config3":
        for scal in (0, 1):
            cases.append((f"fd4_512x384x256{'_Ri0.1' if scal else ''}", 2000, 0,
                          lambda prec, scal=scal: config_channel_fd(512, 384, 256, precision=prec).replace(
                              **({"isscalar": 1, "got": 0.1, "tbot": 0.0, "ttop": 1.0} if scal else {}))))
    else:
        for ri in (0.0, 0.1, 0.5, 1.0):
            cases.append((f"spectral_256x256x128_Ri{ri}", 1000, 500,
                          lambda prec, ri=ri: config_open_channel_spectral(256, 256, 128, got=ri, precision=prec)))
    out = []
    for name, nsteps, skip, mk in cases:
        prof, fric, flux, ms = {}, {}, {}, {}
        for prec in (PREC_FP64, PREC_MIXED):
            p = mk(prec)
            fields = inputs.loglaw_stratified(p, seed=10) if p.cds == 3 else inputs.poiseuille_noise(p, seed=3)
            if p.isscalar and p.cds != 3:
                zc = __import__("hercules_b200.params", fromlist=["mesh"]).mesh(p)["zc"]
                fields["t"] = np.broadcast_to(t_line(p, zc)[:, None, None], (p.nz, p.ny, p.nx)).copy()
            c = engine.Channel(p)
            c.load(fields)
            c.initialize()
            base = None
            t_ms = 0.0
            if skip:
                rc = c.step_nodiag(skip)
                assert rc == 0, rc
                t_ms += c.last_ms
                base = {m: c.download(m) for m in stats.MEAN_FILES}
            rc = c.step_nodiag(nsteps - skip)
            assert rc == 0, rc
            t_ms += c.last_ms
            means = {}
            for m in stats.MEAN_FILES:
                a = c.download(m)
                means[m] = (a - base[m] if base else a) / float(nsteps - skip)
            c.close()
            pr = stats.profiles(means, p)
            prof[prec] = pr
            fric[prec] = stats.wall_friction(pr, p)
            flux[prec] = stats.heat_flux(pr, p) if p.isscalar else None
            ms[prec] = t_ms / nsteps
        keys = ("U", "uu", "vv", "ww", "uw") + (("T", "tt", "tw") if flux[PREC_FP64] is not None else ())
        d = stats.relative_difference(prof[PREC_MIXED], prof[PREC_FP64], keys=keys)
        d["tau_w"] = abs(fric[PREC_MIXED]["tau_w"] - fric[PREC_FP64]["tau_w"]) / abs(fric[PREC_FP64]["tau_w"])
        if flux[PREC_FP64] is not None:
            # the wall flux, or under a fixed bottom flux the wall temperature it sets
            # (relative to the temperature range across the channel)
            if p.tbc_bot:
                tb = flux[PREC_FP64]["t_wall_bottom"]
                d["t_wall_bottom"] = abs(flux[PREC_MIXED]["t_wall_bottom"] - tb) / max(abs(p.ttop - tb), 1e-300)
            else:
                qb = flux[PREC_FP64]["wall_bottom"]
                d["q_wall_bottom"] = abs(flux[PREC_MIXED]["wall_bottom"] - qb) / max(abs(qb), 1e-300)
        out.append({"case": name, "steps": nsteps, "statistics_over": nsteps - skip,
                    "rel_diff_mixed_vs_fp64": d, "max_rel_diff": max(d.values()),
                    "gate_1pct": max(d.values()) <= 0.01, "ms_per_step": {"fp64": ms[PREC_FP64], "mixed": ms[PREC_MIXED]},
                    "u_tau": {"fp64": fric[PREC_FP64]["u_tau"], "mixed": fric[PREC_MIXED]["u_tau"]}})
        print(json.dumps(out[-1]), flush=True)
    return out


def cpu_oracle_rate(grid, steps, warm=1):
    """Time the CPU restatement of the reference step (OpenMP, all host cores)."""
    from oracle import oracle as O
    from hercules_b200 import inputs
    from hercules_b200.params import config_channel_fd
    nx, ny, nz = grid
    p = config_channel_fd(nx, ny, nz)
    o = O.Oracle(p)
    o.load(inputs.poiseuille_noise(p, seed=3))
    o.initialize()
    o.step(warm)
    t0 = time.perf_counter()
    rc, _ = o.step(steps)
    el = time.perf_counter() - t0
    o.close()
    return nx * ny * nz * steps / el, el


def main():
    args = parse()
    ws, rank, lrank = dist_env()
    if ws > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(lrank)
    nx, ny, nz = WORKLOADS[args.workload]
    ncores = os.cpu_count() or 1
    hbm, peak_kind = peaks()
    base = {"metric": "gridpoint-steps/s mixed vs FP64 at stated err (1 B200)", "unit": "gridpoint-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded Poiseuille + 10% uniform noise)"}
    if is_spectral(args.workload):
        physics = ("stably stratified open channel, pseudo-spectral horizontal (2/3 rule, skew form), FD2 vertical, "
                   "RK3, dp_opt=1, nu=1/180, Pr=0.71, Ri_b=0.1, fixed bottom-cooling flux dT/dz=1, T=0 at the top, dt=1e-3")
        base["data"] = "synthetic (seeded log-law + 5% Gaussian noise, linear T + 1% noise)"
    else:
        physics = "neutral closed channel, FD4 horizontal, FD2 vertical, RK3, dp_opt=2, nu=1/2800, dt=1e-3, zstretch=1"
        if args.workload.endswith("_ri0.1"):
            physics = physics.replace("neutral", "stably stratified (Ri_b = 0.1, T from 0 to 1, Pr = 0.71)")
    fb = nx * ny * nz * 8
    cfg = {"workload": args.workload, "grid": [nx, ny, nz], "physics": physics, "parallelism": f"replicas x{args.gpus}",
           "l2": f"working set larger than L2 (one FP64 field {fb / 1e6:.0f} MB, FP32 {fb / 2e6:.0f} MB)"}
    if args.tile:
        cfg["tile"] = list(args.tile)

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        O.build()
        g = REF_STEP_GRID
        from hercules_b200.params import config_channel_fd
        rate_w, _ = cpu_oracle_rate(g, max(args.warmup, 1), warm=0) if args.warmup else (None, 0)
        rate, el = cpu_oracle_rate(g, args.steps, warm=0)
        line = dict(base)
        line.update({"impl": "reference", "value": rate, "ms_per_step": el / args.steps * 1e3,
                     "dtype": "f64", "config": dict(cfg, sample_grid=list(g)),
                     "cpu_baseline": {"value": rate, "unit": "gridpoint-steps/s", "cores": ncores, "kind": "port",
                                      "sample": f"{args.steps} steps of the same physics on a {g[0]}x{g[1]}x{g[2]} "
                                                f"slab of the {nx}x{ny}x{nz} grid (same plane and transform lengths; "
                                                "per-point rate; the reference's Fortran/MPI code cannot be built "
                                                "here: no gfortran/MPI)"},
                     "e2e": {"value": rate, "unit": "gridpoint-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        print(json.dumps(line), flush=True)
        return

    if args.stats_gate:
        if rank == 0:
            run_stats_gate(args.stats_gate)
        return

    if args.adjoint_only:
        if rank == 0:
            print(json.dumps({"adjoint": run_adjoint(), "note": "adjoint leg only, not a headline line"}), flush=True)
        return

    if args.workload == "ensemble64":
        if ws > 1:
            raise SystemExit("the ensemble workload runs on one GPU per process; launch replicas instead")
        r = run_ensemble(args)
        from hercules_b200.params import PREC_FP64, PREC_MIXED
        line = dict(base)
        line["data"] = "synthetic (64 seeded perturbed-Poiseuille members, Re_tau~U[100,300], Ri~U[0,1])"
        line.update({"value": r[PREC_MIXED]["value"], "ms_per_step": r[PREC_MIXED]["ms_per_step"],
                     "dtype": "f32 fields/FFT + f64 Thomas",
                     "config": {"workload": "ensemble64", "members": 64, "total_points": r[PREC_MIXED]["npts"],
                                "physics": "stratified closed channels, FD4, RK3, dp_opt=1, one CUDA graph per step",
                                "parallelism": "one GPU: each kernel of a stage launched once over all members "
                                               "(grouped launches), one CUDA graph per step"},
                     "fp64": {"value": r[PREC_FP64]["value"], "ms_per_step": r[PREC_FP64]["ms_per_step"]},
                     "mixed_speedup_vs_fp64": r[PREC_FP64]["ms_per_step"] / r[PREC_MIXED]["ms_per_step"],
                     "gpu_launches": int(r[PREC_MIXED]["launches"]), "clocks": r[PREC_MIXED]["clocks"],
                     "tiles": r[PREC_MIXED]["tiles"],
                     "roofline": None, "cpu_baseline": None, "e2e": None})
        print(json.dumps(line), flush=True)
        return
    results, err, kern, e2e = run_gpu(args, ws, rank, hbm)
    if rank != 0:
        return
    from hercules_b200.params import PREC_FP64, PREC_MIXED
    if args.precision != "both":
        # one precision only (profiling runs): no headline, no error or e2e legs
        r = next(iter(results.values()))
        line = dict(base)
        line.update({"value": r["value"], "ms_per_step": r["ms_per_step"], "precision": args.precision,
                     "config": cfg, "gpu_launches": int(r["launches"]), "clocks": r["clocks"],
                     "note": "single-precision profiling run, not a headline line"})
        print(json.dumps(line), flush=True)
        return
    mixed, fp64 = results[PREC_MIXED], results[PREC_FP64]
    # dominant kernel of the headline run and its roofline
    km = kern["mixed"]
    kind = "sp" if is_spectral(args.workload) else "fd"
    dom = max((k for k in km if km[k]["alg_gbs"]), key=lambda k: km[k]["total_ms"])
    ach = km[dom]["alg_gbs"]
    npts = nx * ny * nz
    roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm, "unit": "GB/s",
            "frac": ach / hbm if ach else None, "peak_kind": peak_kind, "traffic": TRAFFIC.get((args.workload, dom)),
            "traffic_capture": TRAFFIC_CAPTURE if (args.workload, dom) in TRAFFIC else None,
            "alg_bytes_per_launch": alg_bytes_step(dom, npts, 4, kind, fused=fused_mode(km))
            / max(km[dom]["launches"] / 2, 1)}
    # whole-step HBM fraction with the fixed per-point accounting of an ideally
    # fused step: FD neutral RK3 131 words (117 field words + 14 FP64 mean words);
    # spectral scalar RK3 3*49 field words + 4 stats reads + 22 FP64 mean words
    if kind == "fd":
        step_b = {PREC_FP64: 1048.0, PREC_MIXED: 117 * 4 + 14 * 8.0}
    else:
        step_b = {PREC_FP64: (3 * 49 + 4) * 8 + 22 * 8.0, PREC_MIXED: (3 * 49 + 4) * 4 + 22 * 8.0}
    roof["step_bytes_per_point"] = {"mixed": step_b[PREC_MIXED], "fp64": step_b[PREC_FP64]}
    roof["step_frac_of_hbm"] = step_b[PREC_MIXED] * mixed["value"] / args.gpus / (hbm * 1e9)
    roof["step_frac_fp64"] = step_b[PREC_FP64] * fp64["value"] / args.gpus / (hbm * 1e9)
    adj = None if args.no_adjoint or is_spectral(args.workload) else run_adjoint()
    cpu = None
    if not args.no_cpu_baseline and args.gpus == 1:
        rate, el = cpu_oracle_rate(CPU_SAMPLE_GRID, 2)
        cpu = {"value": rate, "unit": "gridpoint-steps/s", "cores": ncores, "kind": "port",
               "sample": f"2 steps of the same physics on a {CPU_SAMPLE_GRID[0]}x{CPU_SAMPLE_GRID[1]}x{CPU_SAMPLE_GRID[2]} "
                         f"slab of the {nx}x{ny}x{nz} grid ({el:.1f} s, OpenMP)"}
    line = dict(base)
    line.update({"value": mixed["value"], "ms_per_step": mixed["ms_per_step"], "dtype": "f32 fields/FFT + f64 Thomas",
                 "config": cfg, "fp64": {"value": fp64["value"], "ms_per_step": fp64["ms_per_step"]},
                 "mixed_speedup_vs_fp64": fp64["ms_per_step"] / mixed["ms_per_step"],
                 "err_vs_fp64": err, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                 "gpu_launches": int(mixed["launches"]), "clocks": mixed["clocks"], "clocks_fp64": fp64["clocks"],
                 "adjoint": adj, "kernels": kern})
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
