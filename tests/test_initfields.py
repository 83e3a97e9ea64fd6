"""Initial-field tooling (misc/Turb_Gen/Interpolate_Initial_Fields.m restated):
the not-a-knot spline against scipy's, exact reproduction of cubics, the
script's layout quirk, and the reference's own 32^3 coarse fields when present."""
import os

import numpy as np
import pytest

from hercules_b200 import fileio, initfields
from hercules_b200.params import Params

REF_TURB = "/root/reference/misc/Turb_Gen"


def test_get_z_walls_and_symmetry():
    z = initfields.get_z(0.0, 2.0, 32)
    assert z[0] == pytest.approx(0.0, abs=1e-15) and z[-1] == pytest.approx(2.0, abs=1e-15)
    assert np.allclose(z + z[::-1], 2.0, atol=1e-14)
    assert np.all(np.diff(z) > 0) and np.diff(z)[0] < np.diff(z)[15]     # clustered at the walls


@pytest.mark.parametrize("n", [4, 5, 9, 32])
def test_spline_matches_scipy_not_a_knot(n):
    scipy = pytest.importorskip("scipy.interpolate")
    rng = np.random.default_rng(n)
    x = np.sort(rng.uniform(0, 3, n))
    y = rng.standard_normal(n)
    xq = np.linspace(x[0], x[-1], 97)
    ref = scipy.CubicSpline(x, y, bc_type="not-a-knot")(xq)
    got = initfields.spline_matrix(x, xq) @ y
    assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_tensor_spline_reproduces_cubics():
    """A not-a-knot spline reproduces any cubic, so the tensor product reproduces
    any polynomial of degree <= 3 in each variable."""
    lx, ly, lz = 4 * np.pi, 4 * np.pi / 3, 2.0
    src = (np.linspace(0, lx, 12), np.linspace(0, ly, 10), initfields.get_z(0, lz, 9))
    dst = (np.linspace(0, lx, 31), np.linspace(0, ly, 17), initfields.get_z(0, lz, 23))
    f = lambda x, y, z: (1 + 0.3 * x - 0.02 * x ** 3) * (0.5 - y ** 2 + 0.1 * y ** 3) * (z ** 3 - 2 * z)
    Z, Y, X = np.meshgrid(src[2], src[1], src[0], indexing="ij")
    Z2, Y2, X2 = np.meshgrid(dst[2], dst[1], dst[0], indexing="ij")
    got = initfields.interpolate(f(X, Y, Z), src, dst)
    assert np.max(np.abs(got - f(X2, Y2, Z2))) <= 1e-10 * np.max(np.abs(f(X2, Y2, Z2)))


def test_same_grid_is_identity_and_layouts_agree_for_square_planes(tmp_path):
    rng = np.random.default_rng(3)
    n1 = (8, 8, 6)
    c = rng.standard_normal((n1[2], n1[1], n1[0]))
    for f in ("u", "v"):
        c.tofile(str(tmp_path / f"coarse_{f}_32_cubic.dat"))
    same = initfields.refine({"u": c}, 4.0, 3.0, 2.0, n1)["u"]
    assert np.allclose(same, c, atol=1e-13)
    a = initfields.write_init_files(str(tmp_path / "a"), 4.0, 3.0, 2.0, n1, (20, 20, 11), str(tmp_path), uscaling=1.5)
    b = initfields.write_init_files(str(tmp_path / "b"), 4.0, 3.0, 2.0, n1, (20, 20, 11), str(tmp_path), uscaling=1.5,
                                    layout="reference")
    assert sorted(a) == ["u", "v"]           # the loop ends at the first missing input (coarse_w)
    for f in ("u", "v"):
        fa = np.fromfile(str(tmp_path / "a" / f"init_{f}.dat"))
        fb = np.fromfile(str(tmp_path / "b" / f"init_{f}.dat"))
        assert np.allclose(fa, fb, rtol=0, atol=1e-12)
    # nx2 != ny2: the script's byte order differs from HERCULES's x-fastest one
    initfields.write_init_files(str(tmp_path / "c"), 4.0, 3.0, 2.0, n1, (24, 16, 11), str(tmp_path), layout="reference")
    initfields.write_init_files(str(tmp_path / "d"), 4.0, 3.0, 2.0, n1, (24, 16, 11), str(tmp_path))
    fc = np.fromfile(str(tmp_path / "c" / "init_v.dat"))
    fd = np.fromfile(str(tmp_path / "d" / "init_v.dat"))
    assert fc.size == fd.size and not np.allclose(fc, fd)


@pytest.mark.skipif(not os.path.isdir(REF_TURB), reason="reference coarse fields not present")
def test_reference_coarse_fields_refine_to_a_restart(tmp_path):
    """The reference's 32^3 turbulence (u, v, w, p; no t) refined to a 64x64x48
    closed channel and read back as a restart."""
    n2 = (64, 64, 48)
    out = initfields.write_init_files(str(tmp_path), 4 * np.pi, 4 * np.pi / 3, 2.0, (32, 32, 32), n2, REF_TURB)
    assert sorted(out) == ["p", "u", "v", "w"]
    c = initfields.read_coarse(os.path.join(REF_TURB, "coarse_u_32_cubic.dat"), (32, 32, 32))
    # the corner nodes coincide: values kept exactly
    for k, kk in ((0, 0), (-1, -1)):
        assert out["u"][kk, 0, 0] == pytest.approx(c[k, 0, 0], abs=1e-12)
        assert out["u"][kk, -1, -1] == pytest.approx(c[k, -1, -1], abs=1e-12)
    # bounded by the spline's overshoot
    assert np.max(np.abs(out["u"])) <= 1.5 * np.max(np.abs(c))
    np.zeros((n2[2], n2[1], n2[0])).tofile(str(tmp_path / "init_t.dat"))
    p = Params(lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, nx=n2[0], ny=n2[1], nz=n2[2], restart=1)
    f = fileio.read_init_fields(str(tmp_path), p)
    assert np.array_equal(f["u"], out["u"] - p.u_mrf) and f["w"].shape == (48, 64, 64)
