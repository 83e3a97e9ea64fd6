"""Statistics post-processing (Plot_Mean_Profiles.m restated, plus wall friction
and heat flux): known-answer checks on CPU, and the mixed-precision statistical
gate on the GPU."""
import numpy as np
import pytest

from hercules_b200 import fileio, inputs, stats
from hercules_b200.params import PREC_MIXED, Params, config_channel_fd, mesh


def small(**kw):
    base = dict(lx=4.0, ly=3.0, lz=2.0, nx=16, ny=12, nz=9, zstretch=1.1, ochannel=0, dp_opt=1,
                cds=2, dts=2, nu=1.0 / 300.0, alpha=1.0 / 300.0 / 0.71, dt=2e-3, imax=100)
    base.update(kw)
    return Params(**base)


def test_profiles_of_constructed_means():
    p = small()
    z = mesh(p)["zc"]
    shape = (p.nz, p.ny, p.nx)
    rng = np.random.default_rng(0)
    U = (z * (2 - z))[:, None, None] * np.ones(shape)
    a = rng.standard_normal(shape) * 0.01
    means = {"mean_u": U + a, "mean_v": np.zeros(shape), "mean_w": np.zeros(shape), "mean_t": np.zeros(shape),
             "mean_uu": (U + a) ** 2 + 0.04, "mean_vv": np.full(shape, 0.01), "mean_ww": np.full(shape, 0.02),
             "mean_uw": np.full(shape, -0.003), "mean_vw": np.zeros(shape), "mean_tt": np.zeros(shape),
             "mean_tw": np.zeros(shape)}
    pr = stats.profiles(means, p)
    assert np.allclose(pr["U"], (U + a).mean(axis=(1, 2)))
    assert np.allclose(pr["uu"], 0.04) and np.allclose(pr["vv"], 0.01) and np.allclose(pr["uw"], -0.003)
    wf = stats.wall_friction(pr, p)
    d = mesh(p)["dz"]
    assert wf["tau_bottom"] == pytest.approx(p.nu * pr["U"][0] / (0.5 * d[2]))
    assert wf["u_tau"] == pytest.approx(np.sqrt(abs(wf["tau_w"])))


def test_heat_flux_of_linear_conduction():
    """Pure conduction between tbot and ttop: the molecular flux is the same at the
    walls and at every face."""
    p = small(tbot=0.0, ttop=1.0, zstretch=1.0)
    z = mesh(p)["zc"]
    T = z / p.lz
    pr = {"T": T, "tw": np.zeros(p.nz)}
    hf = stats.heat_flux(pr, p)
    q = -p.alpha / p.lz
    assert np.allclose(hf["molecular_faces"], q, rtol=1e-12)
    assert hf["wall_bottom"] == pytest.approx(q, rel=1e-12) and hf["wall_top"] == pytest.approx(q, rel=1e-12)


def test_profiles_from_results_files(tmp_path, oracle_lib):
    p = small(imeanfl=5, isscalar=1, got=0.3)
    o = oracle_lib.Oracle(p)
    o.load(inputs.small_random(p, seed=3))
    o.initialize()
    o.step(5)
    means = {f"mean_{k}": o.get(f"mean_{k}") for k in ("u", "v", "w", "t", "uu", "vv", "ww", "uw", "vw", "tt", "tw")}
    fileio.output_mean_fields(str(tmp_path), means, 5)
    fileio.write_geo_info(str(tmp_path), p)
    pr = stats.profiles(stats.read_mean_fields(str(tmp_path), p), p)
    assert np.allclose(pr["U"], (means["mean_u"] / 5).mean(axis=(1, 2)), rtol=1e-14)
    geo = fileio.read_geo_info(str(tmp_path / "geo.info"))
    assert np.allclose(pr["z"], geo[:, 0], rtol=5e-6)


@pytest.mark.gpu
def test_mixed_precision_statistics_within_one_percent(engine):
    """The statistical gate of the mixed mode: mean profiles and Reynolds stresses
    accumulated over 300 steps agree with the FP64 run to 1% (max over z of the
    difference over the profile's maximum)."""
    res = {}
    for prec in (0, PREC_MIXED):
        p = config_channel_fd(nx=48, ny=32, nz=33, precision=prec)
        c = engine.Channel(p)
        c.load(inputs.poiseuille_noise(p, seed=1))
        c.initialize()
        c.step(300)
        means = {name: c.download(name) / 300.0 for name in stats.MEAN_FILES}
        res[prec] = stats.profiles(means, p)
        c.close()
    d = stats.relative_difference(res[PREC_MIXED], res[0])
    assert all(v <= 0.01 for v in d.values()), d
