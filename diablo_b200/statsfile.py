"""SAVE_STATS_CHAN's HDF5 outputs (for/save_stats.f:38-66, 349-425,
597-637, 1136-1149) -- mean.h5, tke.h5 and, on the final call, stats.h5 --
with WriteStatH5 / WriteHDF5_real's layout (for/hdf5.f:1345-1622): one group
per quantity, an int32 ``SAMPLES`` attribute counting its datasets, and
datasets ``0001``, ``0002``, .. of NY float64 values (rows 1..NY), each with
a ``Time`` attribute (the ``time`` group holds one value per dataset and no
attribute).

The files are HDF5 (diablo_b200.h5, written without an HDF5 library): group
``<name>`` with its scalar int32 ``SAMPLES`` attribute, datasets ``<NNNN>``
of float64 with a scalar float64 ``Time`` attribute, as WriteStatH5 creates
them.  An append reads the file's tree, adds the call's datasets and writes
it again, so a caller groups the datasets of one SAVE_STATS call into one
write_many.

The reference writes omega_y into mean.h5's ``omega_z`` group
(save_stats.f:421-423); ``StatsWriter(omega_z_quirk=True)``, the default,
does the same, and ``False`` writes the true omega_z.

``formats`` may add ``"txt"``: the files the reference writes when it is
built without HDF5 (save_stats.f:68-89, 427-447, 639-658, 1191-1205) --
mean.txt, mean_th.txt, tke.txt and, with LES, tke_les.txt, which a run
appends to (the reference never closes their units), and stats.txt on the
final call.  With LES, tke.h5 also gets tkebudget_chan_les's epsilon_sgs.  Their rows use
the reference's FORMAT statements and are reproduced byte for byte (F
editing rounds like Python's fixed-point formatting; a value too wide for
its field prints as asterisks); the list-directed header lines (TIME_STEP,
TIME, DELTA_T and UBULK) follow gfortran's list-directed style: integers in
12 columns, REAL*8 as G25.17E3 after one blank.
"""
from __future__ import annotations

import os

import numpy as np

from . import h5
from .channel import MEAN_NAMES, SCAL_NAMES


class StatFile:
    """One mean.h5-style HDF5 file, opened for appending.  Every append
    rewrites the file, so a caller groups the datasets of one SAVE_STATS call
    into one write_many."""

    def __init__(self, path: str):
        self.path = path
        self.root = h5.read(path) if os.path.exists(path) else h5.Group()

    def samples(self, gname: str) -> int:
        g = self.root.children.get(gname)
        return int(g.attrs["SAMPLES"]) if g is not None and "SAMPLES" in g.attrs else 0

    def write_many(self, entries) -> list[int]:
        """Append datasets (gname, value, time or None): each gets the group's
        next number; returns them."""
        numbers = []
        for gname, value, time in entries:
            g = self.root.group(gname)
            n = self.samples(gname) + 1                   # NSAMP = NSAMP + 1; dname = '(I0.4)'
            g.attrs["SAMPLES"] = np.int32(n)
            attrs = {} if time is None else {"Time": np.float64(time)}
            g.children[f"{n:04d}"] = h5.Dataset(np.asarray(value, dtype="<f8"), attrs)
            numbers.append(n)
        h5.write(self.path, self.root)
        return numbers

    def write_real(self, gname: str, value: float) -> int:
        """WriteHDF5_real (hdf5.f:1345-1464): one value, no attribute."""
        return self.write_many([(gname, np.array([value]), None)])[0]

    def write_stat(self, gname: str, diag: np.ndarray, time: float) -> int:
        """WriteStatH5 (hdf5.f:1466-1622): Diag(1:NY) with its Time."""
        return self.write_many([(gname, np.asarray(diag, dtype=np.float64), time)])[0]


def read(path: str) -> dict:
    """{group: {"SAMPLES": n, "data": [n][...] float64, "Time": [n] or None}}."""
    out: dict = {}
    for gname, g in h5.read(path).children.items():
        names = sorted(k for k in g.children if k.isdigit())
        if not names:
            continue
        data = np.stack([g.children[k].data for k in names])
        has_t = "Time" in g.children[names[0]].attrs
        t = np.array([float(g.children[k].attrs["Time"]) for k in names]) if has_t else None
        out[gname] = {"SAMPLES": int(g.attrs.get("SAMPLES", len(names))), "data": data, "Time": t}
    return out


def fortran_f(x: float, w: int, d: int) -> str:
    """Fortran Fw.d of one value."""
    t = f"{x:{w}.{d}f}"
    return "*" * w if len(t) > w else t


def fortran_i(i: int, w: int) -> str:
    t = f"{i:{w}d}"
    return "*" * w if len(t) > w else t


def list_directed(*items) -> str:
    """One gfortran list-directed record: INTEGER in 12 columns, REAL*8 as
    1PG25.17E3 preceded by a blank."""
    out = []
    for v in items:
        if isinstance(v, (int, np.integer)):
            out.append(f"{int(v):12d}")
            continue
        x = float(v)
        a = abs(x)
        r = float(f"{a:.16e}") if a != 0.0 else 0.0          # 17 significant digits
        if r == 0.0 or 0.1 <= r < 1e17:
            # G editing: 10**(k-1) <= |x| < 10**k prints d - k = 17 - k decimals (zero: 16)
            k = 1 if r == 0.0 else (0 if r < 1.0 else len(str(int(r))))
            body = f"{x:.{17 - k}f}".rjust(20) + " " * 5
        else:
            m, e = f"{x:.16E}".split("E")
            body = f"{m}E{int(e):+04d}".rjust(25)
        out.append(" " + body)
    return "".join(out)


def ubulk(p, grid, ume: np.ndarray) -> float:
    """INTEGRATE_Y_VAR of the mean velocity (mpi.f:1610-1632): the GY-point
    trapezoid sum over J = 2..NY divided by LY."""
    dy = np.asarray(grid.dy, dtype=np.float64)
    res = 0.0
    for j in range(2, p.ny + 1):
        res = res + 0.5 * (ume[j] + ume[j - 1]) * dy[j]
    return res / p.ly


def epsilon_sgs(p, grid, u1: np.ndarray, u2: np.ndarray, u3: np.ndarray, nu_t: np.ndarray) -> np.ndarray:
    """tkebudget_chan_les (save_stats.f:859-900) on physical [J][K][I] fields
    (planes 0..NY+1): per plane J = 1..NY, the sum over the plane of U_i
    times the implicit vertical eddy-viscosity term of U_i (U1, U3 at GYF,
    U2 at GY, NU_T at GY).  Plane sums, not means, as the reference writes."""
    dy = np.asarray(grid.dy, dtype=np.float64)[:, None, None]
    dyf = np.asarray(grid.dyf, dtype=np.float64)[:, None, None]
    c, n, m = slice(1, p.ny + 1), slice(2, p.ny + 2), slice(0, p.ny)
    nt = nu_t

    def gyf_term(u):
        return u[c] * ((nt[n] * (u[n] - u[c]) / dy[n] - nt[c] * (u[c] - u[m]) / dy[c]) / dyf[c])

    def flux(coef, du, h):
        # a zero eddy viscosity carries no flux: at J = 1 the reference
        # divides 0 by DYF(0), which it never sets (0), and gets NaN
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.where(coef == 0.0, 0.0, coef * du / h)

    t = gyf_term(u1) + gyf_term(u3) + u2[c] * (
        (flux(0.5 * (nt[c] + nt[n]), u2[n] - u2[c], dyf[c]) - flux(0.5 * (nt[c] + nt[m]), u2[c] - u2[m], dyf[m]))
        / dy[c])
    out = np.zeros(p.ny + 2)
    out[1 : p.ny + 1] = t.sum(axis=(1, 2))
    return out


def _physical(c, cu: np.ndarray) -> np.ndarray:
    from .layout import new_physical
    p = c.p
    v = new_physical(p)
    c.fft_xz_to_physical(np.ascontiguousarray(cu).copy(), v, 0, p.ny + 1)
    return v[:, : p.nz, : p.nx]


def epsilon_field(c) -> np.ndarray:
    """tkebudget_chan's 3-D dissipation field F1 (save_stats.f:957-1131) of an
    instance's current state (after the statistics' APPLY_BC_VEL): NU times
    du/dx, dv/dx, du/dy, dw/dx, du/dz, dv/dy, dw/dy, dv/dz, dw/dz squared, the
    x and z derivatives of U1 and U3 interpolated from GYF to GY, the y
    derivatives with the mean removed; rows 2..NY-1 of [J][K][I] (rows 1 and
    NY read rows of S1 that earlier code left behind in the reference: 0
    here).  The x and z derivatives go to physical space through the
    instance's own transforms."""
    from .layout import new_fourier
    p = c.p
    s = c.download()
    cu = s["cu"]
    nkx, nkz, tnkz = p.nx // 3, p.nz // 3, 2 * (p.nz // 3)
    kx = np.zeros(p.nx // 2 + 1)
    kx[: nkx + 1] = np.arange(nkx + 1) * 2.0 * np.pi / p.lx
    kk = np.arange(tnkz + 1)
    kz = np.zeros(p.nz + 2)
    kz[: tnkz + 1] = np.where(kk <= nkz, kk, kk - tnkz - 1) * 2.0 * np.pi / p.lz

    def deriv(f, along):                     # ikx or ikz of CU on rows 1..NY, to physical space
        a = new_fourier(p)
        k = kx[None, None, :] if along == "x" else kz[None, :, None]
        a[1 : p.ny + 1] = 1j * k * f[1 : p.ny + 1]
        return _physical(c, a)

    u1, u2, u3 = (_physical(c, f) for f in cu)
    ume, vme, wme = (f[:, 0, 0].real for f in cu)
    dy = np.asarray(c.grid.dy, dtype=np.float64)[:, None, None]
    dyf = np.asarray(c.grid.dyf, dtype=np.float64)[:, None, None]
    gy = np.asarray(c.grid.gy, dtype=np.float64)
    j, jm = slice(2, p.ny), slice(1, p.ny - 1)

    def interp(sq):                          # (DYF(j-1) S(j)^2 + DYF(j) S(j-1)^2) / (2 DY(j))
        return (dyf[jm] * sq[j] ** 2 + dyf[j] * sq[jm] ** 2) / (2.0 * dy[j])

    e = interp(deriv(cu[0], "x")) + deriv(cu[1], "x")[j] ** 2
    e = e + (((u1[j] - ume[j, None, None]) - (u1[jm] - ume[jm, None, None])) / dy[j]) ** 2
    e = e + interp(deriv(cu[2], "x")) + interp(deriv(cu[0], "z"))
    e = e + (((u2[3 : p.ny + 1] - vme[j, None, None]) - (u2[jm] - vme[jm, None, None]))
             / (gy[3 : p.ny + 1] - gy[1 : p.ny - 1])[:, None, None]) ** 2
    e = e + (((u3[j] - wme[j, None, None]) - (u3[jm] - wme[jm, None, None])) / dy[j]) ** 2
    e = e + deriv(cu[1], "z")[j] ** 2 + interp(deriv(cu[2], "z"))
    out = np.zeros((p.ny + 2, p.nz, p.nx))
    out[j] = p.nu * e
    return out


def les_epsilon_sgs(c) -> np.ndarray:
    """epsilon_sgs of an LES instance's current state (after the APPLY_BC_VEL
    of the statistics) and its NU_T."""
    s = c.download()
    u = [_physical(c, s["cu"][k]) for k in range(3)]
    return epsilon_sgs(c.p, c.grid, *u, c.download_nu_t())


def movie_indices(p, grid, xc: float, yc: float, zc: float) -> tuple:
    """INIT_CHAN_MOVIE (channel.f:1516-1560) for one process: NxMovie,
    NyMovie, NzMovie from the slice centres of MOVIE.dat.  NyMovie is the
    GYF interval holding yc when GYF(JSTART) <= yc < GYF(JEND+1) (JSTART = 2,
    JEND = NY-1); otherwise no process holds the x-z slice (RankYMovie = -1)
    and it is None, as is NzMovie when it falls outside 0..NZ-1 (no process
    holds the x-y slice).  An NxMovie outside 0..NX-1 is an error here; the
    reference would index outside its arrays."""
    gyf = np.asarray(grid.gyf, dtype=np.float64)
    nx_m = int(xc * p.nx / p.lx)
    nz_m = int(zc * p.nz / p.lz)
    if not 0 <= nx_m < p.nx:
        raise ValueError(f"XcMovie {xc} gives NxMovie {nx_m} outside 0..{p.nx - 1}")
    ny_m = None
    if gyf[2] <= yc < gyf[p.ny]:
        i = 1
        while not (gyf[i] <= yc < gyf[i + 1]):
            i += 1
        ny_m = i
    return nx_m, ny_m, (nz_m if 0 <= nz_m < p.nz else None)


def movie_planes(p, u1, u2, u3, th, nu_t, idx, eps=None) -> list:
    """The movie.h5 slices of SAVE_STATS_CHAN (save_stats.f:538-580, 677-839)
    from physical [J][K][I] fields: (group, 2-D array) in the byte order of
    WriteHDF5_XYPLANE / _XZPLANE / _ZYPLANE (Fortran (NX,NY), (NX,NZ), (NZ,NY)
    arrays, i.e. C-order (NY,NX), (NZ,NX), (NY,NZ)).  V is averaged to GYF;
    NU_T planes only with LES; eps, tkebudget_chan's F1, adds the epsilon
    slices (save_stats.f:1151-1189)."""
    nxm, nym, nzm = idx
    rows = slice(1, p.ny + 1)
    vg = 0.5 * (u2[1 : p.ny + 1] + u2[2 : p.ny + 2])             # V at GYF, J = 1..NY
    out = []
    for n in range(p.n_th):
        f = th[n]
        if nzm is not None:
            out.append((f"th{n + 1:02d}_xy", f[rows, nzm, :]))
        if nym is not None:
            out.append((f"th{n + 1:02d}_xz", f[nym, :, :]))
        out.append((f"th{n + 1:02d}_zy", f[rows, :, nxm]))
    fields = [("u", u1[rows], u1), ("v", vg, None), ("w", u3[rows], u3)]
    if p.les:
        fields.append(("nu_t", nu_t[rows], nu_t))
    if nzm is not None:
        out += [(f"{name}_xy", vol[:, nzm, :]) for name, vol, _ in fields]
    if nym is not None:
        out += [(f"{name}_xz", 0.5 * (u2[nym] + u2[nym + 1]) if full is None else full[nym])
                for name, _, full in fields]
    out += [(f"{name}_zy", vol[:, :, nxm]) for name, vol, _ in fields]
    if eps is not None:
        if nzm is not None:
            out.append(("epsilon_xy", eps[rows, nzm, :]))
        if nym is not None:
            out.append(("epsilon_xz", eps[nym]))
        out.append(("epsilon_zy", eps[rows, :, nxm]))
    return [(g, np.ascontiguousarray(a, dtype=np.float64)) for g, a in out]


class StatsWriter:
    """The output side of SAVE_STATS_CHAN for one channel run: mean.h5 and
    tke.h5 on every call, the running means UBAR, VBAR, WBAR, THBARnn
    (save_stats.f:104-123) and stats.h5 on the final call."""

    def __init__(self, directory: str, omega_z_quirk: bool = True, formats=("h5",), movie=None):
        self.dir = directory
        self.omega_z_quirk = omega_z_quirk
        self.formats = tuple(formats)
        self.movie = movie            # MOVIE.dat's (XcMovie, YcMovie, ZcMovie), or None
        self.nsamples = 0
        self.bar: dict[str, np.ndarray] = {}
        self._opened: set[str] = set()

    def _text(self, name: str, lines: list[str]) -> None:
        """Write records to a text file the run keeps open: the first write
        of the run starts it afresh, later ones append."""
        path = os.path.join(self.dir, name)
        mode = "a" if name in self._opened else "w"
        self._opened.add(name)
        with open(path, mode) as f:
            f.write("".join(line + "\n" for line in lines))

    def _f(self, name: str) -> StatFile:
        return StatFile(os.path.join(self.dir, name))

    def save(self, c, final: bool = False) -> dict | None:
        """SAVE_STATS_CHAN(FINAL) on a Channel's current state; returns the
        profiles written (None on the final call)."""
        p, gyf, t = c.p, np.asarray(c.grid.gyf, dtype=np.float64), float(c.time)
        rows = slice(1, p.ny + 1)
        if final:
            zero = np.zeros(p.ny + 2)
            if "h5" in self.formats:
                names = ["UBAR", "VBAR", "WBAR"] + [f"THBAR{n + 1:02d}" for n in range(p.n_th)]
                self._f("stats.h5").write_many([("GYF", gyf[rows], t)] +
                                               [(k, self.bar.get(k, zero)[rows], t) for k in names])
            if "txt" in self.formats:
                # 201 FORMAT(I3,',',F16.9,',',F16.9,',',F16.9,',',F16.9), 202 for each scalar
                ub, vb, wb = (self.bar.get(k, zero) for k in ("UBAR", "VBAR", "WBAR"))
                lines = [",".join([fortran_i(j, 3)] + [fortran_f(v, 16, 9) for v in (gyf[j], ub[j], vb[j], wb[j])])
                         for j in range(1, p.ny + 1)]
                for n in range(p.n_th):
                    tb = self.bar.get(f"THBAR{n + 1:02d}", zero)
                    lines += [",".join([fortran_i(j, 3), fortran_f(gyf[j], 16, 9), fortran_f(tb[j], 16, 9)])
                              for j in range(1, p.ny + 1)]
                with open(os.path.join(self.dir, "stats.txt"), "w") as f:
                    f.write("".join(line + "\n" for line in lines))
            return None
        m = c.mean_stats()
        if p.les:                     # tkebudget_chan_les (save_stats.f:170, 859-935)
            m["epsilon_sgs"] = les_epsilon_sgs(c)
        if self.movie is not None and "h5" in self.formats:
            st = c.download()        # the state after the statistics' APPLY_BC_VEL
            u = [_physical(c, st["cu"][k]) for k in range(3)]
            th = [_physical(c, st["cth"][n]) for n in range(p.n_th)]
            nt = c.download_nu_t() if p.les else None
            idx = movie_indices(p, c.grid, *self.movie)
            eps = epsilon_field(c)
            self._f("movie.h5").write_many([(g, a, t) for g, a in movie_planes(p, *u, th, nt, idx, eps)])
        # running means with REAL*4 weights: (1./FLOAT(N)) and ((FLOAT(N)-1.)/FLOAT(N))
        self.nsamples += 1
        n32 = np.float32(self.nsamples)
        w1 = float(np.float32(1.0) / n32)
        w2 = float((n32 - np.float32(1.0)) / n32)
        src = {"UBAR": m["ume"], "VBAR": m["vme"], "WBAR": m["wme"]}
        for n in range(p.n_th):
            src[f"THBAR{n + 1:02d}"] = m[f"thme{n + 1:02d}"]
        for name, v in src.items():
            old = self.bar.get(name, np.zeros(p.ny + 2))
            new = old.copy()
            new[rows] = w1 * v[rows] + w2 * old[rows]
            self.bar[name] = new
        if "h5" in self.formats:
            entries = [("time", np.array([t]), None), ("gyf", gyf[rows], t)]
            for name in MEAN_NAMES:
                v = m["omega_y"] if (name == "omega_z" and self.omega_z_quirk) else m[name]
                entries.append((name, v[rows], t))
            for n in range(p.n_th):
                for name in SCAL_NAMES:
                    entries.append((f"{name}{n + 1:02d}", m[f"{name}{n + 1:02d}"][rows], t))
            self._f("mean.h5").write_many(entries)
            tke = [("time", np.array([t]), None), ("gyf", gyf[rows], t), ("epsilon", m["epsilon"][rows], t)]
            if p.les:
                tke.append(("epsilon_sgs", m["epsilon_sgs"][rows], t))
            self._f("tke.h5").write_many(tke)
        if "txt" in self.formats:
            step, dt = int(c.time_step), float(c.delta_t)
            ub = ubulk(p, c.grid, m["ume"])
            head = [list_directed(step, t, dt), list_directed(ub)]
            # 401 FORMAT(I3,' ',17(F30.20,' ')): V averaged to GYF, the true omega_z
            cols = ["ume", None, "wme", "urms", "vrms", "wrms", "uv", "uw", "wv", "dudy", "dwdy", "cp", "shear",
                    "omega_x", "omega_y", "omega_z"]
            lines = []
            for j in range(1, p.ny + 1):
                vals = [gyf[j]] + [0.5 * (m["vme"][j + 1] + m["vme"][j]) if k is None else m[k][j] for k in cols]
                lines.append(fortran_i(j, 3) + " " + "".join(fortran_f(v, 30, 20) + " " for v in vals))
            self._text("mean.txt", head + lines)
            # 402 FORMAT(I3,' ',6(F30.20,' '))
            lines = []
            for n in range(p.n_th):
                for j in range(1, p.ny + 1):
                    vals = [gyf[j]] + [m[f"{k}{n + 1:02d}"][j] for k in SCAL_NAMES]
                    lines.append(fortran_i(j, 3) + " " + "".join(fortran_f(v, 30, 20) + " " for v in vals))
            self._text("mean_th.txt", head + lines)
            # tkebudget_chan's 401 FORMAT(I3,' ',2(F20.9,' ')), J = 2..NY-1
            lines = [fortran_i(j, 3) + " " + fortran_f(gyf[j], 20, 9) + " " + fortran_f(m["epsilon"][j], 20, 9) + " "
                     for j in range(2, p.ny)]
            self._text("tke.txt", [list_directed(step, t, dt)] + lines)
            if p.les:                 # 460 FORMAT(I3,' ',2(F30.20,' ')), J = 1..NY
                lines = [fortran_i(j, 3) + " " + fortran_f(gyf[j], 30, 20) + " " +
                         fortran_f(m["epsilon_sgs"][j], 30, 20) + " " for j in range(1, p.ny + 1)]
                self._text("tke_les.txt", [list_directed(step, t, dt)] + lines)
        return m
