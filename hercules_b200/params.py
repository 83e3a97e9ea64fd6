"""Host-side mirror of the reference's parameter handling.

* ``HcParams`` / ``HcDiag`` are the ctypes images of ``hc_params`` / ``hc_diag``
  declared in ``include/hercules_b200.h``.
* ``read_parameters`` parses ``parameters.input`` Fortran namelists
  (&domain &modeling &constants &io), as ``initiate_parameters`` does in the
  reference (src/module_parameters.f90:145-157, 247-252).
* ``check_parameters`` repeats the reference's start-up checks
  (src/module_parameters.f90:254-270) and raises ``ValueError`` where the
  reference prints and stops.
"""
from __future__ import annotations

import ctypes
import re
from dataclasses import dataclass, field, asdict
from typing import Dict, List

PREC_FP64 = 0
PREC_MIXED = 1

FIELD_IDS = {
    "u": 0, "v": 1, "w": 2, "p": 3, "t": 4, "ff": 5, "gg": 6, "hh": 7, "ss": 8,
    "phi": 9, "mean_u": 10, "mean_v": 11, "mean_w": 12, "mean_t": 13,
    "mean_uu": 14, "mean_vv": 15, "mean_ww": 16, "mean_uw": 17, "mean_vw": 18,
    "mean_tt": 19, "mean_tw": 20,
}
MEAN_NAMES = ["mean_u", "mean_v", "mean_w", "mean_t", "mean_uu", "mean_vv",
              "mean_ww", "mean_uw", "mean_vw", "mean_tt", "mean_tw"]


class HcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("zstretch", ctypes.c_double),
        ("ochannel", ctypes.c_int), ("dp_opt", ctypes.c_int), ("cds", ctypes.c_int),
        ("issk", ctypes.c_int), ("dts", ctypes.c_int),
        ("isdamp", ctypes.c_int), ("nzdamp", ctypes.c_int),
        ("cdamp", ctypes.c_double),
        ("nu", ctypes.c_double), ("alpha", ctypes.c_double), ("got", ctypes.c_double),
        ("fc", ctypes.c_double), ("ug", ctypes.c_double), ("vg", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("imax", ctypes.c_int),
        ("u_mrf", ctypes.c_double),
        ("isscalar", ctypes.c_int),
        ("t_ref", ctypes.c_double), ("tbot", ctypes.c_double), ("ttop", ctypes.c_double),
        ("is_ri_var", ctypes.c_int),
        ("ri_str", ctypes.c_double), ("ri_end", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("tile", ctypes.c_int * 4),
        ("tbc_bot", ctypes.c_int),
        ("reserved", ctypes.c_int * 2),
    ]


class HcDiag(ctypes.Structure):
    _fields_ = [
        ("time_sim", ctypes.c_double), ("cfl", ctypes.c_double),
        ("div_avg", ctypes.c_double), ("div_max", ctypes.c_double),
        ("div_hist_max", ctypes.c_double), ("ubar", ctypes.c_double),
        ("dpx_drive", ctypes.c_double), ("got", ctypes.c_double),
        ("div_avg_sub", ctypes.c_double * 3), ("div_max_sub", ctypes.c_double * 3),
        ("nan_flag", ctypes.c_int), ("step", ctypes.c_int),
    ]

    def as_dict(self) -> Dict[str, float]:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if isinstance(v, ctypes.Array) else v
        return d


@dataclass
class Params:
    """All namelist entries of parameters.input (src/module_parameters.f90:40-142)."""
    # &domain
    p_row: int = 1
    p_col: int = 1
    lx: float = 12.56637061
    ly: float = 4.188790205
    lz: float = 2.0
    nx: int = 96
    ny: int = 64
    nz: int = 64
    zstretch: float = 1.0
    ochannel: int = 0
    # &modeling
    dp_opt: int = 1
    cds: int = 2
    issk: int = 1
    dts: int = 2
    isnoise: int = 0
    noise_mag: float = 0.1
    isdamp: int = 0
    nzdamp: int = 15
    cdamp: float = 0.01
    # &constants
    nu: float = 0.005555556
    alpha: float = 0.007936508
    got: float = 0.0
    fc: float = 0.0
    ug: float = 0.0
    vg: float = 0.0
    dt: float = 0.001
    imax: int = 200
    u_mrf: float = 0.0
    isscalar: int = 0
    t_ref: float = 0.0
    tbot: float = -0.5
    ttop: float = 0.5
    is_ri_var: int = 0
    ri_str: float = 0.0
    ri_end: float = 0.0
    # &io
    restart: int = 1
    istmsr: int = 0
    ibackup: int = 1000000
    iinstfl: int = 1000000
    imeanfl: int = 1000000
    isxy2d: int = 0
    xy2d_id: List[int] = field(default_factory=list)
    isxz2d: int = 0
    xz2d_id: List[int] = field(default_factory=list)
    isyz2d: int = 0
    yz2d_id: List[int] = field(default_factory=list)
    intv_2d: int = 1000
    # not namelist entries: storage/arithmetic precision of the GPU path and the
    # kernel tile shapes (0 = automatic)
    precision: int = PREC_FP64
    tile: List[int] = field(default_factory=lambda: [0, 0, 0, 0])
    # bottom temperature condition: 0 the wall temperature tbot (the reference's
    # only one), 1 the fixed wall gradient dT/dz = tbot (a fixed heat flux)
    tbc_bot: int = 0

    def to_c(self) -> HcParams:
        c = HcParams()
        for name, _ in HcParams._fields_:
            if name == "reserved":
                continue
            if name == "tile":
                for q, v in enumerate(self.tile[:4]):
                    c.tile[q] = int(v)
                continue
            setattr(c, name, getattr(self, name))
        return c

    def replace(self, **kw) -> "Params":
        d = asdict(self)
        d.update(kw)
        return Params(**d)

    @property
    def npoints(self) -> int:
        return self.nx * self.ny * self.nz


def check_parameters(p: Params) -> None:
    """Start-up checks of initiate_parameters (src/module_parameters.f90:254-270)."""
    if p.nx % p.p_row or p.ny % p.p_row:
        raise ValueError("nx and ny are not divisible by p_row! Quit!")
    if p.ny % p.p_col or p.nz % p.p_col:
        raise ValueError("ny and nz are not divisible by p_col! Quit!")
    if p.nx % 2 or p.ny % 2:
        raise ValueError("Please use even numbers for nx and ny! Quit!")
    if p.tbc_bot not in (0, 1):
        raise ValueError("tbc_bot must be 0 (fixed bottom temperature) or 1 (fixed bottom gradient)")


_NML_GROUP = re.compile(r"&(\w+)(.*?)/", re.S)


def _parse_value(text: str):
    text = text.strip().rstrip(",")
    items = [t.strip() for t in text.split(",") if t.strip()]
    vals = []
    for it in items:
        low = it.lower().replace("d", "e")
        try:
            if re.fullmatch(r"[+-]?\d+", low):
                vals.append(int(low))
            else:
                vals.append(float(low))
        except ValueError:
            vals.append(it.strip("'\""))
    return vals if len(vals) > 1 else (vals[0] if vals else None)


def read_parameters(path: str) -> Params:
    """Parse a Fortran namelist file with the four groups of the reference."""
    text = open(path).read()
    p = Params()
    names = {f for f in p.__dataclass_fields__}
    for group, body in _NML_GROUP.findall(text):
        # split "name = value" pairs; values may span commas (arrays)
        for m in re.finditer(r"(\w+)\s*=\s*([^=]*?)(?=\s+\w+\s*=|\s*$)", body, re.S):
            key, val = m.group(1).lower(), _parse_value(m.group(2))
            if key not in names:
                continue
            cur = getattr(p, key)
            if isinstance(cur, list):
                val = val if isinstance(val, list) else [val]
            elif isinstance(cur, int) and not isinstance(cur, bool):
                val = int(val)
            elif isinstance(cur, float):
                val = float(val)
            setattr(p, key, val)
    return p


# --------------------------------------------------------------------------
# The benchmark workloads (seeded synthetic inputs with the stated shapes).
# --------------------------------------------------------------------------
PI = 3.1415926535897932


def config_channel_fd(nx=96, ny=64, nz=64, precision=PREC_FP64) -> Params:
    """Neutral closed channel, Re_tau=180 nominal, 4th-order FD, RK3, constant
    flow-rate forcing (dp_opt=2, nu=1/2800), tanh stretching zstretch=1."""
    return Params(lx=4 * PI, ly=4 * PI / 3, lz=2.0, nx=nx, ny=ny, nz=nz, zstretch=1.0,
                  ochannel=0, dp_opt=2, cds=2, dts=2, nu=1.0 / 2800.0, alpha=1.0 / 2800.0 / 0.71,
                  dt=1e-3, imax=200, isscalar=0, precision=precision)


def config_open_channel_spectral(nx=256, ny=256, nz=128, got=0.1, precision=PREC_FP64) -> Params:
    """Stably stratified open channel, pseudo-spectral horizontal derivatives,
    Pr=0.71, a fixed bottom-cooling flux (dT/dz = 1 at the bottom wall,
    tbc_bot = 1) and T = 0 at the top."""
    nu = 1.0 / 180.0
    return Params(lx=4 * PI, ly=2 * PI, lz=1.0, nx=nx, ny=ny, nz=nz, zstretch=1.0,
                  ochannel=1, dp_opt=1, cds=3, issk=1, dts=2, nu=nu, alpha=nu / 0.71,
                  got=got, dt=1e-3, imax=1000, isscalar=1, tbc_bot=1, tbot=1.0, ttop=0.0,
                  precision=precision)


def config_ekman(nx=64, ny=64, nz=65, precision=PREC_FP64) -> Params:
    """Ekman layer in D units: G=ug=1, nu=1/Re_D=0.0025, fc=2 nu=0.005, dt=0.1."""
    return Params(lx=4 * PI, ly=4 * PI, lz=20.0, nx=nx, ny=ny, nz=nz, zstretch=1.1,
                  ochannel=1, dp_opt=3, cds=2, dts=2, nu=0.0025, alpha=0.0025 / 0.71,
                  fc=0.005, ug=1.0, vg=0.0, dt=0.1, imax=50, isscalar=0, isdamp=0,
                  precision=precision)


def t_line(p: Params, z):
    """The linear temperature between the walls that the bottom condition allows:
    from tbot at z = 0 to ttop at z = lz (fixed wall temperatures), or with the
    wall gradient dT/dz = tbot up to ttop at z = lz (tbc_bot = 1)."""
    if p.tbc_bot:
        return p.ttop - p.tbot * (p.lz - z)
    return p.tbot + (p.ttop - p.tbot) * z / p.lz


def mesh(p: Params):
    """Host copy of get_mesh_param (src/module_parameters.f90:432-508).

    Returns a dict of numpy arrays indexed by Fortran k-1 (length nz+4):
    dz, l_t, l_b, dz_t, dz_b, plus zc (cell centres, interior only, length nz)
    and zw (the nz+1 cell faces)."""
    import numpy as np
    nz = p.nz
    nka = nz + 4
    kstr3, kend3 = 3, nz + 2
    zmin, zmax = 0.0, p.lz
    if p.ochannel == 0:
        zmean = 0.5 * (zmin + zmax)
        coeff_a = (2.0 + nz) * 0.5
    else:
        zmean = zmin + zmax
        coeff_a = (1.0 + nz) * 1.0
    zz = np.zeros(nka + 2)
    for k in range(1, nz + 2):
        zz[k + 2] = zmean + (zmin - zmean) / np.tanh(2.0 * p.zstretch) * \
            np.tanh(2.0 * p.zstretch * (k - coeff_a) / (1.0 - coeff_a))
    dz = np.zeros(nka + 2)
    for k in range(kstr3, kend3 + 1):
        dz[k] = zz[k + 1] - zz[k]
    dz[kstr3 - 1] = dz[kstr3]
    dz[kend3 + 1] = dz[kend3]
    dz[kstr3 - 2] = dz[kstr3]
    dz[kend3 + 2] = dz[kend3]
    l_t = np.zeros(nka + 2)
    l_b = np.zeros(nka + 2)
    dz_t = np.zeros(nka + 2)
    dz_b = np.zeros(nka + 2)
    for k in range(kstr3 - 1, kend3 + 2):
        l_t[k] = dz[k] / (dz[k] + dz[k + 1])
        l_b[k] = dz[k] / (dz[k] + dz[k - 1])
        dz_t[k] = 0.5 * (dz[k] + dz[k + 1])
        dz_b[k] = 0.5 * (dz[k] + dz[k - 1])
    zw = zz[3:nz + 4].copy()
    zc = 0.5 * (zw[:-1] + zw[1:])
    return {"dz": dz[1:nka + 1].copy(), "l_t": l_t[1:nka + 1].copy(), "l_b": l_b[1:nka + 1].copy(),
            "dz_t": dz_t[1:nka + 1].copy(), "dz_b": dz_b[1:nka + 1].copy(), "zc": zc, "zw": zw}
