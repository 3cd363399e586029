"""Flow files (SAVE_FLOW / READ_FLOW, for/diablo_io.f:201-418; WriteHDF5 /
ReadHDF5, for/hdf5.f:5-546): the format layer on the CPU, and the
reference's restart semantics run on the CPU oracle."""
import numpy as np
import pytest

from diablo_b200 import checkpoint as ck, grid as G, h5, ics, layout, params as P
from oracle.oracle import ORC_CTH, ORC_P, ORC_U1, ORC_U2, ORC_U3, Oracle


def kh(nx=32, ny=33, nz=32, seed=3):
    p = P.kelvin_helmholtz(nx, ny, nz)
    g = G.channel_grid(G.create_grid(2, ny, 20.0, 1.5))
    u, th = ics.shear_layer(p, g, seed=seed, amp=0.2)
    return p, g, u, th


def channel(nx=32, ny=33, nz=24, seed=3):
    p = P.turbulent_channel(nx, ny, nz, re_tau=180.0)
    g = G.channel_grid(G.create_grid(1, p.ny, 2.0, 1.75))
    u, th = ics.poiseuille(p, g, u_center=10.0, seed=seed, noise=0.3)
    return p, g, u, th


# --- the reference's SAVE_FLOW / READ_FLOW on the oracle ------------------------
_TARGETS = {"U": (ORC_U1, 0), "V": (ORC_U2, 0), "W": (ORC_U3, 0), "P": (ORC_P, 0)}


def oracle_physical(o, cu):
    p = o.p
    v = layout.new_physical(p)
    o.fft_xz_to_physical(np.ascontiguousarray(cu).copy(), v, 0, p.ny + 1)
    return v[:, : p.nz, : p.nx].copy()


def oracle_save(o, path, save_pressure=False):
    t, _, ts, _ = o.time()
    f = {k: oracle_physical(o, cu) for k, cu in zip(("U", "V", "W"), o.cu)}
    for n, th in enumerate(ck.scalar_names(o.p)):
        f[th] = oracle_physical(o, o.cth[n])
    if save_pressure:
        f["P"] = oracle_physical(o, o.cp)
    ck.write(path, o.p, f, t, ts)


def oracle_load(o, path, reset_time=False):
    """READ_FLOW -> ReadHDF5 (hdf5.f:297-546) then APPLY_BC_VEL (diablo_io.f:294-301)."""
    p = o.p
    r = ck.read(path, p)
    targets = dict(_TARGETS, **{th: (ORC_CTH, n) for n, th in enumerate(ck.scalar_names(p))})
    for key, a in r["fields"].items():                      # the fields in physical space
        v = o.physical(*targets[key])
        v[...] = 0.0
        v[:, : p.nz, : p.nx] = a
    _, dt, _, _ = o.time()
    o.set_time(r["time"], dt, r["time_step"])
    if p.variable_dt:
        o.courant()                                         # on physical U1..U3 (hdf5.f:513-515)
    for key in r["fields"]:
        which, n = targets[key]
        o.fft_xz_to_fourier(o.physical(which, n), o.fourier(which, n), 0, p.ny + 1)
    if not r["pressure"]:
        o.poisson_p_chan()
    o.apply_bc_vel()
    if reset_time:
        o.set_time(0.0, o.time()[1], 0)
    return r


def oracle_load_legacy(o, path, scalar_paths=None):
    p = o.p
    r = ck.read_legacy(path, p)
    for cu, which in zip(r["cu"], (ORC_U1, ORC_U2, ORC_U3)):
        o.fourier(which, 0)[...] = cu
    for n, sp in (scalar_paths or {}).items():
        o.fourier(ORC_CTH, n)[...] = ck.read_legacy_scalar(sp, p)["cth"]
    o.set_time(r["time"], o.time()[1], r["time_step"])
    o.apply_bc_vel()


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def state(o):
    p = o.p
    return [layout.dealiased(p, x).copy() for x in o.cu + [o.cth[0], o.cp]]


# --- format -------------------------------------------------------------------------
def test_g2gf_gf2g_inverse_on_interior_rows():
    rng = np.random.default_rng(0)
    v = rng.standard_normal((19, 5, 6))
    w = ck.gf2g(ck.g2gf(v))
    assert np.allclose(w[2:18], v[2:18], rtol=0, atol=1e-14)
    assert np.array_equal(w[1], -w[2]) and np.array_equal(w[18], -w[17])
    g = ck.g2gf(v)                                  # V at GYF: the half sums, the end rows copied
    assert np.allclose(g[5], 0.5 * (v[5] + v[6]))
    assert np.array_equal(g[1], v[2]) and np.array_equal(g[17], v[17])


def test_write_read_layout_and_round_trip(tmp_path):
    p, _, _, _ = kh(12, 9, 10)
    rng = np.random.default_rng(1)
    f = {k: rng.standard_normal((p.ny + 2, p.nz, p.nx)) for k in ("U", "V", "W", "TH01", "P")}
    path = str(tmp_path / "out.h5")
    ck.write(path, p, f, 1.25, 17)
    raw = ck.datasets(path)
    tree = h5.read(path)                               # WriteHDF5's layout
    assert list(tree.attrs["Resolution"]) == [p.nx, p.ny, p.nz] and tree.attrs["Resolution"].dtype == np.int32
    assert tree.attrs["Date"].shape == (20,) and tree.attrs["Info"].shape == (80,)
    assert float(tree.children["Timestep"].attrs["Time"]) == 1.25
    assert sorted(tree.children["Timestep"].children) == ["P", "TH01", "U", "V", "W"]
    # SWAPZY: dataset (NZ, NY, NX) in C order = Fortran out(1:NX,1:NY,1:NZ)
    assert raw["U"].shape == (p.nz, p.ny, p.nx)
    assert raw["U"][3, 4, 5] == f["U"][5, 3, 5]
    assert raw["V"][2, 0, 1] == f["V"][2, 2, 1]               # G2GF row 1 = V(2)
    assert float(raw["Time"]) == 1.25 and int(raw["Timestep"]) == 17
    r = ck.read(path, p)
    assert r["time"] == 1.25 and r["time_step"] == 17 and r["pressure"]
    for k in ("U", "W", "TH01", "P"):
        assert np.array_equal(r["fields"][k][1:-1], f[k][1:-1])
        assert not r["fields"][k][0].any() and not r["fields"][k][-1].any()
    assert np.allclose(r["fields"]["V"][2:-1], f["V"][2:-1], rtol=0, atol=1e-14)


def test_read_names_and_errors(tmp_path):
    p, _, _, _ = kh(12, 9, 10)
    f = {k: np.ones((p.ny + 2, p.nz, p.nx)) for k in ("U", "V", "W", "TH01")}
    path = str(tmp_path / "a.h5")
    ck.write(path, p, f, 0.0, 0)
    tree = h5.read(path)
    ts = tree.children["Timestep"]
    th = ts.children.pop("TH01")
    ts.children["TH1"] = h5.Dataset(2 * th.data)               # the reader's name (hdf5.f:426-427)
    h5.write(str(tmp_path / "b.h5"), tree)
    r = ck.read(str(tmp_path / "b.h5"), p)
    assert np.all(r["fields"]["TH01"][1:-1] == 2) and not r["pressure"]
    ts.children.pop("TH1")
    h5.write(str(tmp_path / "c.h5"), tree)
    with pytest.raises(KeyError):
        ck.read(str(tmp_path / "c.h5"), p)
    assert "TH01" not in ck.read(str(tmp_path / "c.h5"), p, new_scalars=(0,))["fields"]
    q = p.copy()
    q.nx = 16
    with pytest.raises(ValueError):
        ck.read(path, q)
    ck.write(str(tmp_path / "d.h5"), p, f, 0.0, 0, th_reader_names=True)
    names = ck.datasets(str(tmp_path / "d.h5"))
    assert "TH1" in names and "TH01" not in names


def test_legacy_bytes_and_round_trip(tmp_path):
    p, _, _, _ = kh(12, 9, 10)
    rng = np.random.default_rng(2)
    cu = [layout.new_fourier(p) for _ in range(3)]
    for c in cu:
        c[...] = rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)
    path = str(tmp_path / "diablo.saved")
    ck.write_legacy(path, p, cu, 0.5, 7)
    raw = open(path, "rb").read()
    plane = (p.tnkz + 1) * (p.nkx + 1)
    body = 16 * plane * (3 * p.ny - 1)                         # CU1 1..NY, CU2 2..NY, CU3 1..NY
    assert len(raw) == (4 + 28 + 4) + (4 + body + 4)
    assert np.frombuffer(raw, "<i4", 1, 0)[0] == 28 and np.frombuffer(raw, "<i4", 1, 32)[0] == 28
    assert list(np.frombuffer(raw, "<i4", 4, 4)) == [p.nx, p.ny, p.nz, 2]
    assert np.frombuffer(raw, "<f8", 1, 20)[0] == 0.5 and np.frombuffer(raw, "<i4", 1, 28)[0] == 7
    assert np.frombuffer(raw, "<i4", 1, 36)[0] == body
    first = np.frombuffer(raw, "<c16", 2, 40)                  # CU1(0,0,1), CU1(1,0,1): I fastest
    assert first[0] == cu[0][1, 0, 0] and first[1] == cu[0][1, 0, 1]
    r = ck.read_legacy(path, p)
    assert r["time"] == 0.5 and r["time_step"] == 7
    for j0, a, b in zip((1, 2, 1), r["cu"], cu):
        assert np.array_equal(a[j0 : p.ny + 1, : p.tnkz + 1, : p.nkx + 1], b[j0 : p.ny + 1, : p.tnkz + 1, : p.nkx + 1])
        assert not a[: j0].any() and not a[p.ny + 1].any()
    q = p.copy()
    q.ny = 11
    with pytest.raises(ValueError, match="wrong dimensions"):
        ck.read_legacy(path, q)
    open(str(tmp_path / "bad"), "wb").write(raw[:-3])
    with pytest.raises(ValueError):
        ck.read_legacy(str(tmp_path / "bad"), p)


def test_legacy_scalar_rows(tmp_path):
    p, _, _, _ = kh(12, 9, 10)
    th = layout.new_fourier(p)
    th[...] = np.arange(th.size).reshape(th.shape)
    sp = str(tmp_path / "diablo_th01.saved")
    ck.write_legacy_scalar(sp, p, th, 0.0, 0)                  # J = 0..NY as SAVE_FLOW writes
    r = ck.read_legacy_scalar(sp, p)["cth"]
    blk = np.s_[: p.ny + 1, : p.tnkz + 1, : p.nkx + 1]
    assert np.array_equal(r[blk], th[blk])
    # a record of NY planes (the reference reader's J = 1..NY)
    plane = (p.tnkz + 1) * (p.nkx + 1)
    rec = np.ascontiguousarray(th[1 : p.ny + 1, : p.tnkz + 1, : p.nkx + 1]).tobytes()
    hdr = open(sp, "rb").read()[:36]
    m = np.int32(16 * plane * p.ny).tobytes()
    open(sp, "wb").write(hdr + m + rec + m)
    r = ck.read_legacy_scalar(sp, p)["cth"]
    assert np.array_equal(r[1 : p.ny + 1, : p.tnkz + 1, : p.nkx + 1], th[1 : p.ny + 1, : p.tnkz + 1, : p.nkx + 1])
    assert not r[0].any()


# --- restart semantics on the oracle ---------------------------------------------
@pytest.mark.parametrize("save_pressure", [False, True])
def test_oracle_restart_is_reference_restart(tmp_path, save_pressure):
    """Restarting from the file equals restarting from the in-memory state
    with READ_FLOW's steps (APPLY_BC_VEL, POISSON_P_CHAN without P); both
    then step to the same state."""
    p, g, u, th = kh()
    o = Oracle(p, g, 0.01)
    o.init_from_physical(u, th)
    o.step(4)
    path = str(tmp_path / "out.h5")
    oracle_save(o, path, save_pressure)
    if not save_pressure:
        o.poisson_p_chan()
    o.apply_bc_vel()
    o2 = Oracle(p, g, 0.01)
    oracle_load(o2, path)
    assert o2.time()[:3] == o.time()[:3]
    for a, b in zip(state(o2), state(o)):
        assert rel(a, b) < 1e-12
    o.step(4)
    o2.step(4)
    for a, b in zip(state(o2), state(o)):
        assert rel(a, b) < 1e-11


def test_oracle_restart_variable_dt_runs_courant(tmp_path):
    p, g, u, th = channel()
    o = Oracle(p, g, 1e-3)
    o.init_from_physical(u, th)
    o.step(3)
    path = str(tmp_path / "out.h5")
    oracle_save(o, path)
    o2 = Oracle(p, g, 5e-2)                                   # a DELTA_T that COURANT replaces
    oracle_load(o2, path, reset_time=True)
    t, dt, ts, _ = o2.time()
    # COURANT of the fields as read (V row 1 from GF2G): the CFL limit of
    # courant.f on the file's physical velocity
    f = ck.read(path, p)["fields"]
    dx, dz = p.lx / p.nx, p.lz / p.nz
    j = slice(1, p.ny + 1)
    np.seterr(divide="ignore")                              # V = 0 on the walls: no limit there
    lim = 0.5 * min(dx, g.dy[1]) ** 2 / p.nu
    for n in range(p.n_th):
        lim = min(lim, lim * p.pr[n])
    ref = min(lim, float(np.min(p.cfl * dx / np.abs(f["U"][j]))),
              float(np.min(p.cfl * g.dy[j, None, None] / np.abs(f["V"][j]))),
              float(np.min(p.cfl * dz / np.abs(f["W"][j]))))
    np.seterr(divide="warn")
    assert (t, ts) == (0.0, 0) and dt == pytest.approx(ref, rel=1e-13)


def test_oracle_restart_from_legacy_files(tmp_path):
    p, g, u, th = kh()
    o = Oracle(p, g, 0.01)
    o.init_from_physical(u, th)
    o.step(3)
    t, _, ts, _ = o.time()
    flow, sp = str(tmp_path / "diablo.saved"), str(tmp_path / "diablo_th01.saved")
    ck.write_legacy(flow, p, o.cu, t, ts)
    ck.write_legacy_scalar(sp, p, o.cth[0], t, ts)
    o2 = Oracle(p, g, 0.01)
    o2.raw(ORC_P)[:] = o.raw(ORC_P)                            # READ_FLOW keeps CP
    oracle_load_legacy(o2, flow, {0: sp})
    o.apply_bc_vel()
    for a, b in zip(state(o2), state(o)):
        assert np.array_equal(a[1:-1], b[1:-1])
    o.step(3)
    o2.step(3)
    for a, b in zip(state(o2), state(o)):
        assert rel(a, b) < 1e-13


@pytest.mark.parametrize("n_th", [0, 2])
def test_scalar_counts_round_trip(tmp_path, n_th):
    """No scalar and two scalars through both formats."""
    p, _, _, _ = kh(12, 9, 10)
    p.n_th = n_th
    if n_th > 1:
        p.pr[1], p.ri[1] = 2.0, 0.0
    rng = np.random.default_rng(5)
    f = {k: rng.standard_normal((p.ny + 2, p.nz, p.nx)) for k in ["U", "V", "W"] + ck.scalar_names(p)}
    path = str(tmp_path / "out.h5")
    ck.write(path, p, f, 0.5, 3)
    r = ck.read(path, p)
    assert sorted(r["fields"]) == sorted(["U", "V", "W"] + ck.scalar_names(p))
    for k in ck.scalar_names(p):
        assert np.array_equal(r["fields"][k][1:-1], f[k][1:-1])
    for n in range(n_th):
        th = layout.new_fourier(p)
        th[...] = rng.standard_normal(th.shape)
        sp = str(tmp_path / f"diablo_th{n + 1:02d}.saved")
        ck.write_legacy_scalar(sp, p, th, 0.5, 3)
        got = ck.read_legacy_scalar(sp, p)["cth"]
        blk = np.s_[: p.ny + 1, : p.tnkz + 1, : p.nkx + 1]
        assert np.array_equal(got[blk], th[blk])
