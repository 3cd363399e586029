"""The mean.h5 / tke.h5 / stats.h5 profiles of SAVE_STATS_CHAN
(for/save_stats.f) on the CPU oracle against closed forms, and the file
layout of WriteStatH5 / WriteHDF5_real (for/hdf5.f:1345-1622)."""
import numpy as np
import pytest

from diablo_b200 import grid as G, h5, params as P, statsfile
from diablo_b200.channel import MEAN_NAMES, SCAL_NAMES
from oracle.oracle import Oracle


def modes_case(A=0.7, B=0.3, C=0.4):
    """u1 = A cos(3 kz0 z), u3 = C cos(2 kx0 x), th = B cos(2 kx0 x), uniform
    in y: closed forms for every vorticity, dissipation and scalar profile."""
    p = P.kelvin_helmholtz(24, 17, 20)
    g = G.channel_grid(G.create_grid(2, p.ny, 20.0, 1.5))
    nx, ny, nz = p.nx, p.ny, p.nz
    x = np.arange(nx) * p.lx / nx
    z = np.arange(nz) * p.lz / nz
    kx, kz = 2 * np.pi / p.lx * 2, 2 * np.pi / p.lz * 3
    u = np.zeros((3, ny + 2, nz + 2, nx + 2))
    th = np.zeros((1, ny + 2, nz + 2, nx + 2))
    u[0, :, :nz, :nx] = A * np.cos(kz * z)[None, :, None]
    u[2, :, :nz, :nx] = C * np.cos(kx * x)[None, None, :]
    th[0, :, :nz, :nx] = B * np.cos(kx * x)[None, None, :]
    o = Oracle(p, g, 0.01)
    o.init_from_physical(u, th)
    return p, g, o, kx, kz


def test_oracle_mean_profiles_closed_forms():
    A, B, C = 0.7, 0.3, 0.4
    p, g, o, kx, kz = modes_case(A, B, C)
    m = o.mean_stats()
    ny = p.ny
    J = slice(2, ny)                                 # rows whose y-neighbours are interior
    # omega_y = du/dz - dw/dx, two orthogonal modes
    assert np.allclose(m["omega_y"][1 : ny + 1], np.sqrt((A * kz) ** 2 + (C * kx) ** 2) / np.sqrt(2), rtol=1e-13)
    assert np.abs(m["omega_x"][1 : ny + 1]).max() < 1e-14
    assert np.abs(m["omega_z"][J]).max() < 1e-14
    # epsilon = NU <du/dz^2 + dw/dx^2>, both GYF quantities interpolated to GY
    w = (g.dyf[1 : ny - 1] + g.dyf[2:ny]) / (2 * g.dy[2:ny])
    eps = p.nu * ((A * kz) ** 2 + (C * kx) ** 2) / 2 * w
    assert np.allclose(m["epsilon"][J], eps, rtol=1e-13)
    assert m["epsilon"][1] == 0.0 and m["epsilon"][ny] == 0.0
    assert np.allclose(m["pe_diss01"][1 : ny + 1], (B * kx) ** 2 / 2, rtol=1e-13)
    assert np.allclose(m["thrms01"][1 : ny + 1], B / np.sqrt(2), rtol=1e-13)
    assert np.abs(m["thv01"]).max() < 1e-15
    # the 13 profiles shared with the plane statistics are orc_stats'
    base = o.stats()
    for k in range(13):
        assert np.array_equal(m[MEAN_NAMES[k]], base[k])


def test_statfile_layout(tmp_path):
    path = str(tmp_path / "mean.h5")
    f = statsfile.StatFile(path)
    assert f.write_real("time", 0.5) == 1
    assert f.write_stat("ume", np.arange(5.0), 0.5) == 1
    assert f.write_stat("ume", np.arange(5.0) + 1, 0.75) == 2
    f2 = statsfile.StatFile(path)                    # reopened: SAMPLES continues
    assert f2.samples("ume") == 2 and f2.samples("time") == 1 and f2.samples("vme") == 0
    f2.write_real("time", 0.75)
    raw = h5.read(path)                              # the HDF5 tree WriteStatH5 creates
    ume = raw.children["ume"]
    assert int(ume.attrs["SAMPLES"]) == 2 and ume.attrs["SAMPLES"].shape == ()
    assert np.array_equal(ume.children["0002"].data, np.arange(5.0) + 1)
    assert ume.children["0002"].data.dtype == np.dtype("<f8")
    assert float(ume.children["0002"].attrs["Time"]) == 0.75 and ume.children["0002"].attrs["Time"].shape == ()
    r = statsfile.read(path)
    assert r["ume"]["SAMPLES"] == 2 and r["ume"]["data"].shape == (2, 5)
    assert list(r["ume"]["Time"]) == [0.5, 0.75]
    assert r["time"]["Time"] is None and list(r["time"]["data"][:, 0]) == [0.5, 0.75]


class _OracleRun:
    """What StatsWriter reads from a Channel, on the oracle."""

    def __init__(self, o, t):
        self.o, self.p, self.grid, self.time = o, o.p, o.grid, t

    def mean_stats(self):
        return self.o.mean_stats()


@pytest.mark.parametrize("quirk", [True, False])
def test_stats_writer_files(tmp_path, quirk):
    p, g, o, _, _ = modes_case()
    w = statsfile.StatsWriter(str(tmp_path), omega_z_quirk=quirk)
    m1 = w.save(_OracleRun(o, 0.0))
    o.step(2)
    m2 = w.save(_OracleRun(o, 0.02))
    w.save(_OracleRun(o, 0.02), final=True)
    mean = statsfile.read(str(tmp_path / "mean.h5"))
    names = ["time", "gyf"] + MEAN_NAMES + [f"{s}01" for s in SCAL_NAMES]
    assert sorted(mean) == sorted(names)
    assert all(mean[k]["SAMPLES"] == 2 for k in names)
    rows = slice(1, p.ny + 1)
    assert np.array_equal(mean["ume"]["data"][1], m2["ume"][rows])
    assert np.array_equal(mean["gyf"]["data"][0], g.gyf[rows]) and list(mean["ume"]["Time"]) == [0.0, 0.02]
    oz = mean["omega_z"]["data"][1]
    assert np.array_equal(oz, (m2["omega_y"] if quirk else m2["omega_z"])[rows])
    tke = statsfile.read(str(tmp_path / "tke.h5"))
    assert sorted(tke) == ["epsilon", "gyf", "time"]
    assert np.array_equal(tke["epsilon"]["data"][0], m1["epsilon"][rows])
    stats = statsfile.read(str(tmp_path / "stats.h5"))
    assert sorted(stats) == ["GYF", "THBAR01", "UBAR", "VBAR", "WBAR"]
    # two samples: weights 1/2 and (2-1)/2, exact in REAL*4
    assert np.array_equal(stats["UBAR"]["data"][0], 0.5 * m2["ume"][rows] + 0.5 * m1["ume"][rows])
    assert np.array_equal(stats["THBAR01"]["data"][0], 0.5 * m2["thme01"][rows] + 0.5 * m1["thme01"][rows])


class _Profiles:
    def __init__(self, p, grid, value, t):
        self.p, self.grid, self.time, self.value = p, grid, t, value

    def mean_stats(self):
        ny2 = self.p.ny + 2
        m = {k: np.zeros(ny2) for k in MEAN_NAMES + ["epsilon"] + [f"{s}01" for s in SCAL_NAMES]}
        m["ume"] = np.full(ny2, self.value)
        return m


def test_running_mean_weights_single_precision(tmp_path):
    """UBAR(j) = (1./FLOAT(N)) U + ((FLOAT(N)-1.)/FLOAT(N)) UBAR with REAL*4
    weights (save_stats.f:110-117): 1/3 and 2/3 are not the FP64 values."""
    p = P.kelvin_helmholtz(12, 9, 10)
    g = G.channel_grid(G.create_grid(2, p.ny, 20.0, 1.5))
    w = statsfile.StatsWriter(str(tmp_path))
    vals = [1.0, 2.0, 7.0]
    for v in vals:
        w.save(_Profiles(p, g, v, 0.0))
    w.save(_Profiles(p, g, 0.0, 0.0), final=True)
    ubar = 0.0
    for n, v in enumerate(vals, 1):
        n32 = np.float32(n)
        ubar = float(np.float32(1.0) / n32) * v + float((n32 - np.float32(1.0)) / n32) * ubar
    got = statsfile.read(str(tmp_path / "stats.h5"))["UBAR"]["data"][0]
    assert np.all(got == ubar) and ubar != 10.0 / 3.0


class _TextRun(_OracleRun):
    def __init__(self, o, t, step, dt):
        super().__init__(o, t)
        self.time_step, self.delta_t = step, dt


def test_fortran_edit_descriptors():
    assert statsfile.fortran_f(1.5, 30, 20) == "        1.50000000000000000000"
    assert statsfile.fortran_f(-1e-30, 16, 9) == "    -0.000000000"
    assert statsfile.fortran_f(1e20, 16, 9) == "*" * 16             # too wide: asterisks
    assert statsfile.fortran_i(7, 3) == "  7" and statsfile.fortran_i(1000, 3) == "***"
    # gfortran list-directed: I12, then 1PG25.17E3 after a blank
    assert statsfile.list_directed(10, 0.01, 1e-3) == \
        "          10   1.0000000000000000E-002   1.0000000000000000E-003"
    assert statsfile.list_directed(0.5) == "  0.50000000000000000     "
    assert statsfile.list_directed(1.5) == "   1.5000000000000000     "


def test_text_files(tmp_path):
    """mean.txt / mean_th.txt / tke.txt (appended per call) and stats.txt:
    the reference's FORMAT statements and columns (save_stats.f:427-447,
    639-658, 1191-1205, 68-89)."""
    p, g, o, _, _ = modes_case()
    w = statsfile.StatsWriter(str(tmp_path), formats=("txt",))
    m1 = w.save(_TextRun(o, 0.0, 0, 0.01))
    o.step(1)
    m2 = w.save(_TextRun(o, 0.01, 1, 0.01))
    w.save(_TextRun(o, 0.01, 1, 0.01), final=True)
    assert not (tmp_path / "mean.h5").exists()
    lines = (tmp_path / "mean.txt").read_text().splitlines()
    ny = p.ny
    assert len(lines) == 2 * (2 + ny)
    step, t, dt = lines[2 + ny].split()
    assert (int(step), float(t), float(dt)) == (1, 0.01, 0.01)
    ub = statsfile.ubulk(p, g, m2["ume"])
    assert float(lines[3 + ny]) == pytest.approx(ub, rel=1e-15, abs=1e-300)
    row = lines[4 + ny + 4]                                   # J = 5 of the second sample
    assert len(row) == 3 + 1 + 17 * 31 and row[:3] == "  5"
    v = [float(x) for x in row.split()[1:]]
    assert v[0] == pytest.approx(g.gyf[5], abs=1e-20)
    assert v[1] == pytest.approx(m2["ume"][5], abs=1e-20)
    assert v[2] == pytest.approx(0.5 * (m2["vme"][6] + m2["vme"][5]), abs=1e-20)
    assert v[16] == pytest.approx(m2["omega_z"][5], abs=1e-20)   # the true omega_z here
    th = (tmp_path / "mean_th.txt").read_text().splitlines()
    assert len(th) == 2 * (2 + ny) and float(th[2 + 6].split()[5]) == pytest.approx(m1["thv01"][7], abs=1e-20)
    tke = (tmp_path / "tke.txt").read_text().splitlines()
    assert len(tke) == 2 * (1 + ny - 2)
    j, y, eps = tke[1].split()
    assert (int(j), float(eps)) == (2, pytest.approx(m1["epsilon"][2], abs=1e-9))
    st = (tmp_path / "stats.txt").read_text().splitlines()
    assert len(st) == 2 * ny and st[0].count(",") == 4
    assert float(st[0].split(",")[2]) == pytest.approx(0.5 * (m1["ume"][1] + m2["ume"][1]), abs=1e-9)
    # a new writer (a new run) starts the files afresh
    statsfile.StatsWriter(str(tmp_path), formats=("txt",)).save(_TextRun(o, 0.02, 2, 0.01))
    assert len((tmp_path / "mean.txt").read_text().splitlines()) == 2 + ny


class _LesRun(_TextRun):
    """An LES oracle seen through the Channel calls the writer makes."""

    def download(self):
        return {"cu": self.o.cu, "cth": self.o.cth}

    def fft_xz_to_physical(self, vv, v, jmin, jmax):
        self.o.fft_xz_to_physical(vv, v, jmin, jmax)

    def download_nu_t(self):
        return self.o.nu_t


def test_epsilon_sgs_matches_oracle(tmp_path):
    """tkebudget_chan_les (save_stats.f:859-935): the writer's numpy form on
    the state's physical fields and NU_T against the oracle's restatement,
    and its tke.h5 group and tke_les.txt rows."""
    from test_gpu_les import les_channel
    p, g, u, th = les_channel(24, 33, 16)
    o = Oracle(p, g, 1e-3)
    o.init_from_physical(u, th)
    o.step(2)
    assert np.abs(o.nu_t).max() > 0
    centres = (0.5 * p.lx, float(g.gyf[p.ny // 2]), 0.25 * p.lz)
    w = statsfile.StatsWriter(str(tmp_path), formats=("h5", "txt"), movie=centres)
    m = w.save(_LesRun(o, 0.002, 2, 1e-3))
    nx_m, ny_m, nz_m = statsfile.movie_indices(p, g, *centres)
    mv = statsfile.read(str(tmp_path / "movie.h5"))
    assert np.array_equal(mv["nu_t_xy"]["data"][0], o.nu_t[1 : p.ny + 1, nz_m, :])
    assert np.array_equal(mv["nu_t_xz"]["data"][0], o.nu_t[ny_m])
    ref = o.epsilon_sgs()
    rows = slice(1, p.ny + 1)
    assert np.abs(ref[rows]).max() > 0
    assert np.allclose(m["epsilon_sgs"][rows], ref[rows], rtol=1e-12, atol=1e-14 * np.abs(ref).max())
    tke = statsfile.read(str(tmp_path / "tke.h5"))
    assert np.array_equal(tke["epsilon_sgs"]["data"][0], m["epsilon_sgs"][rows])
    lines = (tmp_path / "tke_les.txt").read_text().splitlines()
    assert len(lines) == 1 + p.ny and len(lines[1]) == 3 + 1 + 2 * 31
    assert float(lines[3].split()[2]) == pytest.approx(m["epsilon_sgs"][3], abs=1e-20)


def test_movie_planes(tmp_path):
    """movie.h5 slices (save_stats.f:538-580, 677-839; INIT_CHAN_MOVIE,
    channel.f:1516-1560) against the oracle's physical fields."""
    from test_checkpoint import oracle_physical
    p, g, o, _, _ = modes_case()
    xc, yc, zc = 0.3 * p.lx, float(g.gyf[10]) + 1e-9, 0.55 * p.lz
    nx_m, ny_m, nz_m = statsfile.movie_indices(p, g, xc, yc, zc)
    assert (nx_m, ny_m, nz_m) == (int(0.3 * p.nx), 10, int(0.55 * p.nz))
    w = statsfile.StatsWriter(str(tmp_path), movie=(xc, yc, zc))
    w.save(_LesRun(o, 0.0, 0, 0.01))
    o.step(1)
    w.save(_LesRun(o, 0.01, 1, 0.01))
    mv = statsfile.read(str(tmp_path / "movie.h5"))
    names = [f"{q}_{s}" for q in ("u", "v", "w", "th01", "epsilon") for s in ("xy", "xz", "zy")]
    assert sorted(mv) == sorted(names) and all(mv[k]["SAMPLES"] == 2 for k in names)
    u1, u2 = oracle_physical(o, o.cu[0]), oracle_physical(o, o.cu[1])
    th = oracle_physical(o, o.cth[0])
    rows = slice(1, p.ny + 1)
    assert mv["u_xy"]["data"][1].shape == (p.ny, p.nx) and np.array_equal(mv["u_xy"]["data"][1], u1[rows, nz_m, :])
    assert mv["th01_xz"]["data"][1].shape == (p.nz, p.nx) and np.array_equal(mv["th01_xz"]["data"][1], th[ny_m])
    assert mv["u_zy"]["data"][1].shape == (p.ny, p.nz) and np.array_equal(mv["u_zy"]["data"][1], u1[rows, :, nx_m])
    assert np.array_equal(mv["v_xz"]["data"][1], 0.5 * (u2[ny_m] + u2[ny_m + 1]))
    assert list(mv["v_xy"]["Time"]) == [0.0, 0.01]
    # outside the walls' GYF range no process holds the x-z slice; beyond LZ, the x-y one
    assert statsfile.movie_indices(p, g, xc, float(g.gyf[p.ny]) + 1.0, zc)[1] is None
    assert statsfile.movie_indices(p, g, xc, yc, 1.5 * p.lz)[2] is None
    with pytest.raises(ValueError):
        statsfile.movie_indices(p, g, 2.0 * p.lx, yc, zc)


def test_epsilon_field_matches_oracle(tmp_path):
    """tkebudget_chan's F1 (save_stats.f:957-1131): the writer's host form
    against the oracle's, and its plane means against the epsilon profile."""
    from test_checkpoint import kh
    p, g, u, th = kh(24, 33, 20)
    o = Oracle(p, g, 0.01)
    o.init_from_physical(u, th)
    o.step(2)
    o.stats()                                             # the statistics' APPLY_BC_VEL
    ref = o.epsilon_field()
    host = statsfile.epsilon_field(_LesRun(o, 0.02, 2, 0.01))
    scale = np.abs(ref).max()
    assert scale > 0 and np.abs(host - ref).max() <= 1e-12 * scale
    assert not ref[[0, 1, p.ny, p.ny + 1]].any()
    means = ref.sum(axis=(1, 2)) / (p.nx * p.nz)
    eps = o.mean_stats()["epsilon"]
    assert np.allclose(means, eps, rtol=1e-12, atol=1e-14 * np.abs(eps).max())
    centres = (0.25 * p.lx, float(g.gyf[p.ny // 2]), 0.5 * p.lz)
    statsfile.StatsWriter(str(tmp_path), movie=centres).save(_LesRun(o, 0.02, 2, 0.01))
    nx_m, ny_m, nz_m = statsfile.movie_indices(p, g, *centres)
    mv = statsfile.read(str(tmp_path / "movie.h5"))
    assert np.abs(mv["epsilon_xz"]["data"][0] - ref[ny_m]).max() <= 1e-12 * scale
    assert mv["epsilon_zy"]["data"][0].shape == (p.ny, p.nz)
