"""On-disk formats of the reference's output layer and the drive loop around it.

Restates, in Python on the host side of the C-ABI, the files `module_io`
writes and `read_init_fields` reads, so that a run of this engine leaves the
same `results/` directory a (single-rank) run of the reference leaves:

* raw records: interior-only float64 arrays in Fortran order (x fastest), no
  header, as 2DECOMP&FFT's `decomp_2d_write_one` / `decomp_2d_read_one` write and
  read them with one rank (src/module_io.f90:311-403, 546-598;
  src/module_tools.f90:260-316);
* planes of `decomp_2d_write_plane` (src/module_io.f90:408-542): the (nx, ny)
  x-y plane at interior level k, the (nx, nz) x-z plane at j, the (ny, nz) y-z
  plane at i, each Fortran order, file names without extension;
* text: the time series `tmsr_*.dat` (`2f14.8` then `f14.8` per level,
  src/module_io.f90:211-305) and `geo.info` (`4e14.6` per level,
  src/module_parameters.f90:495-504).

The velocity files carry u + u_mrf (the reference stores the relative velocity
and adds the frame speed on output, subtracting it again on input); mean fields
are the accumulators divided by the step count.
"""
from __future__ import annotations

import os
from typing import Dict, Iterable, Optional

import numpy as np

from .params import Params, mesh

FIELDS5 = ("u", "v", "w", "p", "t")
HIST4 = ("ff", "gg", "hh", "ss")
MEANS = ("mean_u", "mean_v", "mean_w", "mean_t", "mean_uu", "mean_vv", "mean_ww", "mean_uw",
         "mean_vw", "mean_tt", "mean_tw")


# ---------------------------------------------------------------------------
# Fortran edit descriptors used by the text files
# ---------------------------------------------------------------------------
def fortran_f(x: float, w: int = 14, d: int = 8) -> str:
    """Fw.d: fixed point, right-justified; a value that does not fit prints w stars."""
    s = f"{x:{w}.{d}f}"
    return s if len(s) <= w else "*" * w


def fortran_e(x: float, w: int = 14, d: int = 6) -> str:
    """Ew.d with the default two-digit exponent: 0.ddddddE+ee, mantissa in [0.1, 1)."""
    if x == 0.0 or not np.isfinite(x):
        body = "0." + "0" * d + "E+00" if x == 0.0 else str(x)
        return body.rjust(w)
    sign = "-" if x < 0 else ""
    a = abs(x)
    e = int(np.floor(np.log10(a))) + 1
    m = a / 10.0 ** e
    digits = round(m * 10 ** d)
    if digits >= 10 ** d:             # rounding carried into the next decade
        digits //= 10
        e += 1
    if digits < 10 ** (d - 1):        # log10 landed one decade high
        digits = round(a / 10.0 ** (e - 1) * 10 ** d)
        e -= 1
    exp = f"{'+' if e >= 0 else '-'}{abs(e):02d}"
    body = f"{sign}0.{digits:0{d}d}E{exp}"
    return body.rjust(w) if len(body) <= w else "*" * w


def fortran_i(n: int, w: int) -> str:
    """Iw.w: zero-padded to w digits; stars when it does not fit."""
    s = f"{n:0{w}d}"
    return s if len(s) <= w else "*" * w


# ---------------------------------------------------------------------------
# raw records
# ---------------------------------------------------------------------------
def write_raw(path: str, a: np.ndarray) -> None:
    """One interior field (nz, ny, nx) as raw float64, x fastest."""
    np.ascontiguousarray(a, dtype=np.float64).tofile(path)


def read_raw(path: str, p: Params) -> np.ndarray:
    a = np.fromfile(path, dtype=np.float64)
    if a.size != p.nx * p.ny * p.nz:
        raise ValueError(f"{path}: {a.size} values, expected {p.nx * p.ny * p.nz}")
    return a.reshape(p.nz, p.ny, p.nx)


def read_init_fields(results: str, p: Params) -> Dict[str, np.ndarray]:
    """read_init_fields (src/module_tools.f90:260-316): init_{u,v,w,p,t}.dat, u minus
    u_mrf; with dts != 2 (AB2) also init_{ff,gg,hh,ss}.dat."""
    out = {f: read_raw(os.path.join(results, f"init_{f}.dat"), p) for f in FIELDS5}
    out["u"] = out["u"] - p.u_mrf
    if p.dts != 2:
        for f in HIST4:
            out[f] = read_raw(os.path.join(results, f"init_{f}.dat"), p)
    return out


def write_init_fields(results: str, p: Params, fields: Dict[str, np.ndarray]) -> None:
    """The files read_init_fields reads (u given relative to the moving frame)."""
    os.makedirs(results, exist_ok=True)
    for f in FIELDS5:
        a = fields.get(f, np.zeros((p.nz, p.ny, p.nx)))
        write_raw(os.path.join(results, f"init_{f}.dat"), a + (p.u_mrf if f == "u" else 0.0))
    if p.dts != 2:
        for f in HIST4:
            write_raw(os.path.join(results, f"init_{f}.dat"), fields.get(f, np.zeros((p.nz, p.ny, p.nx))))


def output_backup(results: str, p: Params, fields: Dict[str, np.ndarray]) -> None:
    """output_backup (src/module_io.f90:311-360): bak_*.dat; histories only for AB2."""
    write_raw(os.path.join(results, "bak_u.dat"), fields["u"] + p.u_mrf)
    for f in ("v", "w", "p", "t"):
        write_raw(os.path.join(results, f"bak_{f}.dat"), fields[f])
    if p.dts != 2:
        for f in HIST4:
            write_raw(os.path.join(results, f"bak_{f}.dat"), fields[f])


def output_inst_fields(results: str, p: Params, fields: Dict[str, np.ndarray], time_step: int) -> None:
    """output_inst_fields (src/module_io.f90:366-403): inst_<f>NNN.dat, NNN = i3.3 of
    time_step / iinstfl."""
    tag = fortran_i(time_step // p.iinstfl, 3)
    write_raw(os.path.join(results, f"inst_u{tag}.dat"), fields["u"] + p.u_mrf)
    for f in ("v", "w", "p", "t"):
        write_raw(os.path.join(results, f"inst_{f}{tag}.dat"), fields[f])


def _ids(lst: Iterable[int]):
    """Slice indices up to the first 0 (the namelist arrays are zero-padded)."""
    out = []
    for n in lst:
        if n == 0:
            break
        out.append(int(n))
    return out


def output_2d_slices(results: str, p: Params, fields: Dict[str, np.ndarray], time_step: int) -> None:
    """output_2d_slices (src/module_io.f90:408-542): results/slices/xy2d_<f>_kIIII_tTTTTTT
    (k, j, i are 1-based interior indices, i4.4; TTTTTT = i6.6 of time_step / intv_2d)."""
    sdir = os.path.join(results, "slices")
    os.makedirs(sdir, exist_ok=True)
    tt = fortran_i(time_step // p.intv_2d, 6)
    vals = {f: fields[f] + (p.u_mrf if f == "u" else 0.0) for f in FIELDS5}
    if p.isxy2d == 1:
        for k in _ids(p.xy2d_id):
            for f in FIELDS5:
                write_raw(os.path.join(sdir, f"xy2d_{f}_k{fortran_i(k, 4)}_t{tt}"), vals[f][k - 1, :, :])
    if p.isxz2d == 1:
        for j in _ids(p.xz2d_id):
            for f in FIELDS5:
                write_raw(os.path.join(sdir, f"xz2d_{f}_j{fortran_i(j, 4)}_t{tt}"), vals[f][:, j - 1, :])
    if p.isyz2d == 1:
        for i in _ids(p.yz2d_id):
            for f in FIELDS5:
                write_raw(os.path.join(sdir, f"yz2d_{f}_i{fortran_i(i, 4)}_t{tt}"), vals[f][:, :, i - 1])


def output_mean_fields(results: str, means: Dict[str, np.ndarray], time_step: int) -> None:
    """output_mean_fields (src/module_io.f90:546-598): accumulators / time_step.
    The accumulators of the engine already include u_mrf where the reference's do."""
    for name in MEANS:
        write_raw(os.path.join(results, f"{name}.dat"), means[name] / time_step)


def start_time_series(results: str) -> None:
    """drive opens the five series files with status='replace' (src/module_navier_stokes.f90:81-93)."""
    os.makedirs(results, exist_ok=True)
    for f in ("u", "v", "w", "t", "p"):
        open(os.path.join(results, f"tmsr_{f}.dat"), "w").close()


def output_time_series(results: str, p: Params, fields: Dict[str, np.ndarray], time_sim: float) -> None:
    """output_time_series (src/module_io.f90:211-305): one line per call, time_sim and
    the column at the first interior point (single rank), each f14.8."""
    for f in ("u", "v", "w", "t", "p"):
        col = fields[f][:, 0, 0] + (p.u_mrf if f == "u" else 0.0)
        line = fortran_f(time_sim) + "".join(fortran_f(x) for x in col)
        with open(os.path.join(results, f"tmsr_{f}.dat"), "a") as fh:
            fh.write(line + "\n")


def write_geo_info(results: str, p: Params) -> None:
    """geo.info (src/module_parameters.f90:495-504): per level the cell centre, dz,
    l_t, l_b, each e14.6."""
    m = mesh(p)
    os.makedirs(results, exist_ok=True)
    with open(os.path.join(results, "geo.info"), "w") as fh:
        for kk in range(p.nz):
            vals = (m["zc"][kk], m["dz"][kk + 2], m["l_t"][kk + 2], m["l_b"][kk + 2])
            fh.write("".join(fortran_e(float(v)) for v in vals) + "\n")


def read_geo_info(path: str) -> np.ndarray:
    """(nz, 4) array: zc, dz, l_t, l_b."""
    rows = []
    for line in open(path):
        if line.strip():
            rows.append([float(line[q * 14:(q + 1) * 14]) for q in range(4)])
    return np.array(rows)


# ---------------------------------------------------------------------------
# the drive loop with its output schedule
# ---------------------------------------------------------------------------
def drive(channel, p: Params, nsteps: int, results: str = "results", fields0: Optional[dict] = None):
    """Set-up and time loop of drive (src/module_navier_stokes.f90:53-205) around a
    Channel: initial fields from `results/init_*.dat` when restart=1 (or `fields0`),
    geo.info, then every step the reference's outputs on its schedule (time series
    each step when istmsr=1; backups every ibackup, means every imeanfl,
    instantaneous fields every iinstfl, slices every intv_2d steps). Returns the
    per-step diagnostics."""
    os.makedirs(results, exist_ok=True)
    write_geo_info(results, p)
    if fields0 is None:
        if p.restart == 1:
            fields0 = read_init_fields(results, p)
        else:
            fields0 = {}
    channel.load(fields0)
    channel.initialize()
    if p.istmsr == 1:
        start_time_series(results)
    names = list(FIELDS5) + list(HIST4)
    indx_bk = indx_m = indx_ins = indx_slc = 1
    diags = []
    for _ in range(nsteps):
        d = channel.step(1)[0]
        diags.append(d)
        stps = d["step"]
        need_fields = (p.istmsr == 1 or indx_bk // p.ibackup == 1 or indx_ins // p.iinstfl == 1 or
                       ((p.isxy2d == 1 or p.isxz2d == 1 or p.isyz2d == 1) and indx_slc // p.intv_2d == 1))
        fields = {f: channel.download(f) for f in names} if need_fields else None
        if p.istmsr == 1:
            output_time_series(results, p, fields, d["time_sim"])
        if indx_bk // p.ibackup == 1:
            output_backup(results, p, fields)
            indx_bk = 0
        if indx_m // p.imeanfl == 1:
            output_mean_fields(results, {m: channel.download(m) for m in MEANS}, stps)
            indx_m = 0
        if indx_ins // p.iinstfl == 1:
            output_inst_fields(results, p, fields, stps)
            indx_ins = 0
        if p.isxy2d == 1 or p.isxz2d == 1 or p.isyz2d == 1:
            if indx_slc // p.intv_2d == 1:
                output_2d_slices(results, p, fields, stps)
                indx_slc = 0
        indx_bk += 1
        indx_m += 1
        indx_ins += 1
        indx_slc += 1
    return diags
