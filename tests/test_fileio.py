"""The reference's on-disk formats (module_io, read_init_fields, geo.info) and the
drive loop's output schedule. CPU tests drive the oracle through a small
adapter; the GPU test checks that the engine leaves the same files."""
import os

import numpy as np
import pytest

from hercules_b200 import fileio, inputs
from hercules_b200.params import Params, mesh


def small(**kw):
    base = dict(lx=4.0, ly=3.0, lz=2.0, nx=16, ny=12, nz=9, zstretch=1.1, ochannel=0, dp_opt=1,
                cds=2, dts=2, nu=1.0 / 300.0, alpha=1.0 / 300.0 / 0.71, dt=2e-3, imax=100, isscalar=1, got=0.2)
    base.update(kw)
    return Params(**base)


class OracleChannel:
    """The oracle behind the subset of the Channel interface drive() uses."""

    def __init__(self, oracle_lib, p):
        self.o = oracle_lib.Oracle(p)

    def load(self, fields):
        self.o.load(fields)

    def initialize(self):
        self.o.initialize()

    def step(self, n=1):
        rc, d = self.o.step(n)
        assert rc == 0
        return d

    def download(self, name):
        return self.o.get(name)


def test_fortran_edit_descriptors():
    assert fileio.fortran_e(1.0) == "  0.100000E+01"
    assert fileio.fortran_e(0.5) == "  0.500000E+00"
    assert fileio.fortran_e(-0.0123456789) == " -0.123457E-01"
    assert fileio.fortran_e(0.0) == "  0.000000E+00"
    assert fileio.fortran_e(0.9999999999) == "  0.100000E+01"
    assert fileio.fortran_f(1.5) == "    1.50000000"
    assert fileio.fortran_f(-0.25) == "   -0.25000000"
    assert fileio.fortran_f(1e9) == "*" * 14
    assert fileio.fortran_i(7, 3) == "007" and fileio.fortran_i(1234, 3) == "***"
    assert fileio.fortran_i(12, 6) == "000012"


def test_init_fields_round_trip_with_moving_frame(tmp_path):
    p = small(u_mrf=0.7, dts=1)
    f = inputs.small_random(p, seed=2)
    fileio.write_init_fields(str(tmp_path), p, f)
    raw = np.fromfile(str(tmp_path / "init_u.dat"), dtype=np.float64)
    assert raw.size == p.nx * p.ny * p.nz
    # Fortran order: x fastest, the file holds u + u_mrf
    assert raw[1] == pytest.approx(f["u"][0, 0, 1] + 0.7)
    assert raw[p.nx] == pytest.approx(f["u"][0, 1, 0] + 0.7)
    g = fileio.read_init_fields(str(tmp_path), p)
    for k in ("u", "v", "w", "p", "t", "ff", "gg", "hh", "ss"):
        assert np.allclose(g[k], f[k], rtol=0, atol=1e-15), k


def test_geo_info_matches_mesh(tmp_path):
    p = small(nz=17)
    fileio.write_geo_info(str(tmp_path), p)
    lines = open(tmp_path / "geo.info").read().splitlines()
    assert len(lines) == p.nz and all(len(l) == 56 for l in lines)
    g = fileio.read_geo_info(str(tmp_path / "geo.info"))
    m = mesh(p)
    ref = np.stack([m["zc"], m["dz"][2:p.nz + 2], m["l_t"][2:p.nz + 2], m["l_b"][2:p.nz + 2]], axis=1)
    # E14.6 keeps 6 digits of a mantissa in [0.1, 1): relative error <= 5e-6
    assert np.allclose(g, ref, rtol=5e-6, atol=1e-12)


def test_drive_writes_the_reference_results_layout(tmp_path, oracle_lib):
    p = small(istmsr=1, ibackup=3, imeanfl=2, iinstfl=4, isxy2d=1, xy2d_id=[2, 5, 0], isxz2d=1, xz2d_id=[3],
              isyz2d=1, yz2d_id=[1], intv_2d=2, u_mrf=0.2)
    res = str(tmp_path / "results")
    f0 = inputs.small_random(p, seed=4)
    ch = OracleChannel(oracle_lib, p)
    d = fileio.drive(ch, p, 8, results=res, fields0=f0)
    assert [x["step"] for x in d] == list(range(1, 9))
    files = set(os.listdir(res))
    for f in ("u", "v", "w", "p", "t"):
        assert f"bak_{f}.dat" in files and f"inst_{f}001.dat" in files and f"inst_{f}002.dat" in files
        assert f"tmsr_{f}.dat" in files
    assert "bak_ff.dat" not in files                      # RK3 keeps no histories
    for name in fileio.MEANS:
        assert f"{name}.dat" in files
    # backup at steps 3 and 6 (the last one stays): u + u_mrf of step 6 is not the final state
    u_final = ch.download("u")
    bak = np.fromfile(os.path.join(res, "bak_u.dat")).reshape(p.nz, p.ny, p.nx)
    assert not np.allclose(bak, u_final + p.u_mrf)
    # means written at step 8 = accumulators / 8
    mu = np.fromfile(os.path.join(res, "mean_u.dat")).reshape(p.nz, p.ny, p.nx)
    assert np.allclose(mu, ch.download("mean_u") / 8, rtol=1e-15, atol=0)
    # time series: 8 lines of (nz + 1) f14.8 values, time first
    lines = open(os.path.join(res, "tmsr_u.dat")).read().splitlines()
    assert len(lines) == 8 and all(len(l) == 14 * (p.nz + 1) for l in lines)
    assert float(lines[-1][:14]) == pytest.approx(d[-1]["time_sim"], abs=1e-8)
    assert float(lines[-1][14:28]) == pytest.approx(u_final[0, 0, 0] + p.u_mrf, abs=1e-8)
    # slices every 2 steps: xy at k = 2, 5, xz at j = 3, yz at i = 1
    sl = set(os.listdir(os.path.join(res, "slices")))
    assert "xy2d_u_k0002_t000004" in sl and "xy2d_t_k0005_t000001" in sl
    assert "xz2d_w_j0003_t000003" in sl and "yz2d_p_i0001_t000004" in sl
    xy = np.fromfile(os.path.join(res, "slices", "xy2d_v_k0005_t000004"))
    assert np.array_equal(xy, ch.download("v")[4].ravel())
    xz = np.fromfile(os.path.join(res, "slices", "xz2d_u_j0003_t000004"))
    assert np.allclose(xz, (u_final[:, 2, :] + p.u_mrf).ravel(), rtol=0, atol=1e-15)
    yz = np.fromfile(os.path.join(res, "slices", "yz2d_w_i0001_t000004"))
    assert np.array_equal(yz, ch.download("w")[:, :, 0].ravel())


def test_drive_restart_reads_init_files(tmp_path, oracle_lib):
    p = small(restart=1, dts=1, u_mrf=-0.3)
    res = str(tmp_path / "results")
    f0 = inputs.small_random(p, seed=6)
    fileio.write_init_fields(res, p, f0)
    a = OracleChannel(oracle_lib, p)
    fileio.drive(a, p, 2, results=res)
    b = OracleChannel(oracle_lib, p)
    b.load(f0)
    b.initialize()
    b.step(2)
    # the file holds u + u_mrf, so the restarted u differs from the original by an ulp
    for f in ("u", "v", "w", "p", "t", "ff"):
        x, y = a.download(f), b.download(f)
        assert np.max(np.abs(x - y)) <= 1e-10 * np.max(np.abs(y)), f


@pytest.mark.gpu
def test_engine_drive_files_match_oracle(tmp_path, oracle_lib, engine):
    p = small(istmsr=1, ibackup=2, imeanfl=2, iinstfl=2, isxy2d=1, xy2d_id=[3], intv_2d=2, nx=32, ny=24, nz=17)
    f0 = inputs.small_random(p, seed=8)
    ra, rb = str(tmp_path / "gpu"), str(tmp_path / "cpu")
    c = engine.Channel(p)
    fileio.drive(c, p, 4, results=ra, fields0=f0)
    fileio.drive(OracleChannel(oracle_lib, p), p, 4, results=rb, fields0=f0)
    for name in sorted(os.listdir(rb)):
        pa, pb = os.path.join(ra, name), os.path.join(rb, name)
        if name.endswith(".dat") and not name.startswith("tmsr"):
            a, b = np.fromfile(pa), np.fromfile(pb)
            assert a.shape == b.shape
            assert np.max(np.abs(a - b)) <= 1e-10 * max(np.max(np.abs(b)), 1e-30), name
        elif name.startswith("tmsr") or name == "geo.info":
            la, lb = open(pa).read().split(), open(pb).read().split()
            assert len(la) == len(lb)
            assert np.allclose([float(x) for x in la], [float(x) for x in lb], rtol=1e-7, atol=2e-8), name
    c.close()
