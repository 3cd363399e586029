"""Flow checkpoints with the reference's SAVE_FLOW / READ_FLOW semantics
(for/diablo_io.f:201-418) in its two file formats.

HDF5 files (WriteHDF5 / ReadHDF5, for/hdf5.f:5-295, 297-546), written and
read by diablo_b200.h5 (no HDF5 library in the image) in WriteHDF5's layout:

* file attributes ``Resolution`` (int32 [NX, NY, NZ]), ``Date`` and ``Info``
  (20 and 80 one-character strings);
* group ``/Timestep`` with attribute ``Time`` (scalar float64) and this
  library's ``TimeStep`` (scalar int32, TIME_STEP, which the reference's
  reader does not look for);
* its datasets ``U``, ``W``, ``TH01``.., ``P``: physical fields on rows
  J = 1..NY as SWAPZY writes them (hdf5.f:1243-1262), i.e. the Fortran array
  out(1:NX,1:NY,1:NZ) -- float64 with shape (NZ, NY, NX) in C order, the
  reference's dataset byte for byte;
* ``V``: U2 moved to GYF points by G2GF before it is written and moved back
  by GF2G when read (hdf5.f:1177-1241), which also imposes V(1) = -V(2),
  V(NY+1) = -V(NY).

`read` also takes the .npz container earlier versions of this library
wrote.

The reference's writer names the scalars ``TH01``.. (hdf5.f:211-213) and its
reader asks for ``TH1``.. (hdf5.f:426-427), so it cannot read back its own
scalars.  `read` takes either name; `write` gives the writer's name, or the
reader's with ``th_reader_names=True``.

Unformatted binary (the SAVE_FLOW / READ_FLOW path for other file names,
diablo_io.f:230-297, 376-412): gfortran sequential records -- a 4-byte
length before and after each record -- byte for byte:

* diablo.start / diablo.saved / diablo.res: a header record NX, NY, NZ,
  NUM_PER_DIR (int32), TIME (float64), TIME_STEP (int32), then one record
  of CU1 (J = 1..NY), CU2 (J = 2..NY), CU3 (J = 1..NY), each ((I = 0..NKX),
  K = 0..TNKZ) complex128;
* diablo_thNN.*: the same header, then CTH(n) for J = 0..NY.  The
  reference's reader takes J = 1..NY from that record (diablo_io.f:257-258),
  i.e. the first NY planes shifted up one row; `read_legacy_scalar` instead
  places each plane on the row it was written from, and reads a record of
  NY planes as J = 1..NY.

On a load, READ_FLOW's order: the state replaced, COURANT with VARIABLE_DT
and POISSON_P_CHAN when the file held no pressure (hdf5.f:513-541, HDF5
only), then APPLY_BC_VEL (diablo_io.f:294-301), then TIME and TIME_STEP
zeroed with RESET_TIME (diablo_io.f:166-171).  Neither format holds rows 0
and NY+1, which APPLY_BC_VEL rewrites; a restarted run is therefore the
reference's restarted run, not a bit-for-bit continuation of the run that
wrote the file.
"""
from __future__ import annotations

import os
import time as _time

import numpy as np

from . import h5
from .layout import new_fourier, new_physical
from .params import DiabloParams

NUM_PER_DIR = 2
_HEADER = np.dtype([("nx", "<i4"), ("ny", "<i4"), ("nz", "<i4"), ("num_per_dir", "<i4"),
                    ("time", "<f8"), ("time_step", "<i4")])


def g2gf(v: np.ndarray) -> np.ndarray:
    """G2GF (hdf5.f:1177-1196) on a [J][K][I] array, one y process."""
    v = v.copy()
    ny = v.shape[0] - 2
    v[1] = v[2]
    v[ny + 1] = v[ny]
    for y in range(1, ny + 1):
        v[y] = 0.5 * (v[y] + v[y + 1])
    return v


def gf2g(v: np.ndarray) -> np.ndarray:
    """GF2G (hdf5.f:1198-1241) on a [J][K][I] array, one y process."""
    v = v.copy()
    ny = v.shape[0] - 2
    v[ny + 1] = v[ny]
    for y in range(ny, 0, -1):
        v[y] = 2 * v[y] - v[y + 1]
    v[1] = -v[2]
    v[ny + 1] = -v[ny]
    return v


def scalar_names(p: DiabloParams) -> list[str]:
    return [f"TH{n + 1:02d}" for n in range(p.n_th)]


# --- HDF5 datasets ------------------------------------------------------------
def write(path: str, p: DiabloParams, fields: dict, time: float, time_step: int,
          th_reader_names: bool = False) -> None:
    """WriteHDF5's datasets from physical [J][K][I] fields (NY+2, NZ, NX)
    keyed U, V, W, TH01.. and, with SAVE_PRESSURE, P."""
    root = h5.Group()
    root.attrs["Resolution"] = np.array([p.nx, p.ny, p.nz], dtype=np.int32)
    root.attrs["Date"] = np.frombuffer(_time.strftime("%Y-%m-%d %H:%M:%S").ljust(20)[:20].encode(), dtype="S1")
    root.attrs["Info"] = np.frombuffer(" (Put here what you want) ".ljust(80).encode(), dtype="S1")
    ts = root.group("Timestep")
    ts.attrs["Time"] = np.float64(time)
    ts.attrs["TimeStep"] = np.int32(time_step)
    for name in ["U", "V", "W"] + scalar_names(p) + (["P"] if "P" in fields else []):
        a = np.asarray(fields[name], dtype=np.float64)
        if a.shape != (p.ny + 2, p.nz, p.nx):
            raise ValueError(f"{name}: shape {a.shape}, expected {(p.ny + 2, p.nz, p.nx)}")
        d = g2gf(a) if name == "V" else a
        key = f"TH{int(name[2:])}" if th_reader_names and name.startswith("TH") else name
        ts.children[key] = h5.Dataset(np.ascontiguousarray(d[1 : p.ny + 1].transpose(1, 0, 2)))   # SWAPZY
    h5.write(path, root)


def datasets(path: str) -> dict:
    """The file's datasets by name, with ``Time``, ``Timestep`` (0 when the
    file has none) and ``Resolution``."""
    if h5.is_hdf5(path):
        root = h5.read(path)
        ts = root.children["Timestep"]
        out = {k: v.data for k, v in ts.children.items()}
        out["Time"] = np.float64(ts.attrs["Time"])
        out["Timestep"] = np.int64(ts.attrs["TimeStep"]) if "TimeStep" in ts.attrs else np.int64(0)
        if "Resolution" in root.attrs:
            out["Resolution"] = np.asarray(root.attrs["Resolution"], dtype=np.int64)
        return out
    with np.load(path if os.path.exists(path) else path + ".npz") as f:
        return {k: f[k] for k in f.files}


def read(path: str, p: DiabloParams, new_scalars=()) -> dict:
    """ReadHDF5's datasets as physical [J][K][I] fields (rows 0 and NY+1
    zero).  Scalars listed in `new_scalars` (0-based; CREATE_NEW_TH) are not
    read.  Returns {"fields", "time", "time_step", "pressure"}."""
    data = datasets(path)
    if "Resolution" in data:
        res = tuple(int(v) for v in data["Resolution"])
        if res != (p.nx, p.ny, p.nz):
            raise ValueError(f"flow file resolution {res} differs from ({p.nx}, {p.ny}, {p.nz})")
    names = {"U": "U", "V": "V", "W": "W"}
    for n, th in enumerate(scalar_names(p)):
        if n in new_scalars:
            continue
        src = next((c for c in (f"TH{n + 1}", th) if c in data), None)
        if src is None:
            raise KeyError(f"scalar {th} missing from the flow file")
        names[th] = src
    if "P" in data:
        names["P"] = "P"
    fields = {}
    for name, src in names.items():
        d = data[src]
        if d.shape != (p.nz, p.ny, p.nx):
            raise ValueError(f"{src}: shape {d.shape}, expected {(p.nz, p.ny, p.nx)}")
        a = np.zeros((p.ny + 2, p.nz, p.nx))
        a[1 : p.ny + 1] = d.transpose(1, 0, 2)                                # SWAPYZ
        fields[name] = gf2g(a) if name == "V" else a
    return {"fields": fields, "time": float(data["Time"]), "time_step": int(data.get("Timestep", 0)),
            "pressure": "P" in fields}


# --- unformatted binary ---------------------------------------------------------
def _records(path: str) -> list[bytes]:
    raw = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(raw):
        n = int(np.frombuffer(raw, "<i4", 1, pos)[0])
        if n < 0:
            raise ValueError(f"{path}: record split into sub-records (over 2 GiB) is not supported")
        if pos + 8 + n > len(raw) or int(np.frombuffer(raw, "<i4", 1, pos + 4 + n)[0]) != n:
            raise ValueError(f"{path}: corrupt record at byte {pos}")
        out.append(raw[pos + 4 : pos + 4 + n])
        pos += 8 + n
    return out


def _write_records(path: str, records: list[bytes]) -> None:
    with open(path, "wb") as f:
        for r in records:
            if len(r) > 0x7FFFFFFF:
                raise ValueError("record over 2 GiB: sub-records are not written")
            m = np.int32(len(r)).tobytes()
            f.write(m + r + m)


def _header(p: DiabloParams, time: float, time_step: int) -> bytes:
    h = np.zeros(1, _HEADER)
    h[0] = (p.nx, p.ny, p.nz, NUM_PER_DIR, time, time_step)
    return h.tobytes()


def _check_header(path: str, rec: bytes, p: DiabloParams) -> tuple[float, int]:
    if len(rec) != _HEADER.itemsize:
        raise ValueError(f"{path}: header record of {len(rec)} bytes")
    h = np.frombuffer(rec, _HEADER)[0]
    if (int(h["nx"]), int(h["ny"]), int(h["nz"])) != (p.nx, p.ny, p.nz):
        raise ValueError("Error: old flowfield wrong dimensions.")
    if int(h["num_per_dir"]) != NUM_PER_DIR:
        raise ValueError("Error: old flowfield wrong NUM_PER_DIR.")
    return float(h["time"]), int(h["time_step"])


def _planes(cu: np.ndarray, p: DiabloParams, j0: int, j1: int) -> np.ndarray:
    return np.ascontiguousarray(cu[j0 : j1 + 1, : p.tnkz + 1, : p.nkx + 1], dtype="<c16")


def write_legacy(path: str, p: DiabloParams, cu: list, time: float, time_step: int) -> None:
    """SAVE_FLOW's flow file from Fourier [J][K][I] arrays CU1..3."""
    body = b"".join(_planes(c, p, j0, p.ny).tobytes() for c, j0 in zip(cu, (1, 2, 1)))
    _write_records(path, [_header(p, time, time_step), body])


def write_legacy_scalar(path: str, p: DiabloParams, cth: np.ndarray, time: float, time_step: int) -> None:
    """SAVE_FLOW's diablo_thNN file from one Fourier scalar (J = 0..NY)."""
    _write_records(path, [_header(p, time, time_step), _planes(cth, p, 0, p.ny).tobytes()])


def read_legacy(path: str, p: DiabloParams) -> dict:
    """READ_FLOW's flow file: {"cu": [CU1, CU2, CU3] with zeros outside the
    record's planes, "time", "time_step"}."""
    recs = _records(path)
    if len(recs) < 2:
        raise ValueError(f"{path}: expected a header and a flow record")
    time, step = _check_header(path, recs[0], p)
    plane = (p.tnkz + 1) * (p.nkx + 1)
    counts = (p.ny, p.ny - 1, p.ny)
    flat = np.frombuffer(recs[1], "<c16")
    if flat.size != plane * sum(counts):
        raise ValueError(f"{path}: flow record of {flat.size} values, expected {plane * sum(counts)}")
    cu, pos = [], 0
    for j0, n in zip((1, 2, 1), counts):
        a = new_fourier(p)
        a[j0 : j0 + n, : p.tnkz + 1, : p.nkx + 1] = flat[pos : pos + n * plane].reshape(n, p.tnkz + 1, p.nkx + 1)
        cu.append(a)
        pos += n * plane
    return {"cu": cu, "time": time, "time_step": step}


def read_legacy_scalar(path: str, p: DiabloParams) -> dict:
    """A diablo_thNN file: {"cth", "time", "time_step"}."""
    recs = _records(path)
    if len(recs) < 2:
        raise ValueError(f"{path}: expected a header and a scalar record")
    time, step = _check_header(path, recs[0], p)
    plane = (p.tnkz + 1) * (p.nkx + 1)
    flat = np.frombuffer(recs[1], "<c16")
    if flat.size == plane * (p.ny + 1):
        j0, n = 0, p.ny + 1
    elif flat.size == plane * p.ny:
        j0, n = 1, p.ny
    else:
        raise ValueError(f"{path}: scalar record of {flat.size} values")
    a = new_fourier(p)
    a[j0 : j0 + n, : p.tnkz + 1, : p.nkx + 1] = flat.reshape(n, p.tnkz + 1, p.nkx + 1)
    return {"cth": a, "time": time, "time_step": step}


# --- a Channel's state ----------------------------------------------------------
def _to_physical(c, cu: np.ndarray) -> np.ndarray:
    p = c.p
    v = new_physical(p)
    c.fft_xz_to_physical(np.ascontiguousarray(cu).copy(), v, 0, p.ny + 1)
    return v[:, : p.nz, : p.nx].copy()


def _to_fourier(c, a: np.ndarray) -> np.ndarray:
    p = c.p
    v = new_physical(p)
    v[:, : p.nz, : p.nx] = a
    out = new_fourier(p)
    c.fft_xz_to_fourier(v, out, 0, p.ny + 1)
    return out


def save(c, path: str, save_pressure: bool = False, th_reader_names: bool = False) -> None:
    """WriteHDF5 of a Channel's state (SAVE_FLOW saves the pressure only in
    its final file, diablo_io.f:315-318)."""
    s = c.download()
    fields = {k: _to_physical(c, s["cu"][i]) for i, k in enumerate(("U", "V", "W"))}
    for n, th in enumerate(scalar_names(c.p)):
        fields[th] = _to_physical(c, s["cth"][n])
    if save_pressure:
        fields["P"] = _to_physical(c, s["cp"])
    write(path, c.p, fields, c.time, c.time_step, th_reader_names)


def _finish_load(c, hdf5: bool, pressure: bool, time: float, step: int, reset_time: bool) -> None:
    if hdf5:
        if c.p.variable_dt:
            c.courant()
        if not pressure:
            c.poisson_p_chan()
    c.apply_bc_vel()
    c.time, c.time_step = (0.0, 0) if reset_time else (time, step)


def load(c, path: str, new_scalars=(), reset_time: bool = False) -> dict:
    """READ_FLOW from an HDF5-dataset file into a Channel.  Scalars in
    `new_scalars` (CREATE_NEW_TH) keep the instance's current values, as
    does CF.  Returns {"pressure": bool}."""
    p = c.p
    r = read(path, p, new_scalars)
    f = r["fields"]
    s = c.download()
    cu = [_to_fourier(c, f[k]) for k in ("U", "V", "W")]
    cth = new_fourier(p, max(p.n_th, 1))
    for n, th in enumerate(scalar_names(p)):
        cth[n] = _to_fourier(c, f[th]) if th in f else s["cth"][n]
    cp = _to_fourier(c, f["P"]) if r["pressure"] else s["cp"]
    c.upload(cu, cp, cth, s["cf"], s["cfth"])
    _finish_load(c, True, r["pressure"], r["time"], r["time_step"], reset_time)
    return {"pressure": r["pressure"]}


def save_legacy(c, path: str, scalar_paths: list | None = None) -> None:
    """SAVE_FLOW's unformatted files: the flow file and one file per scalar."""
    s = c.download()
    write_legacy(path, c.p, s["cu"], c.time, c.time_step)
    for n, sp in enumerate(scalar_paths or []):
        write_legacy_scalar(sp, c.p, s["cth"][n], c.time, c.time_step)


def load_legacy(c, path: str, scalar_paths: dict | None = None, reset_time: bool = False) -> None:
    """READ_FLOW from unformatted files: CU1..3 from `path`, CTH(n) from
    scalar_paths[n] (READ_TH_INDEX, 0-based); the pressure and the scalars
    not read keep the instance's values, then APPLY_BC_VEL."""
    p = c.p
    r = read_legacy(path, p)
    s = c.download()
    cth = new_fourier(p, max(p.n_th, 1))
    cth[: p.n_th] = s["cth"]
    for n, sp in (scalar_paths or {}).items():
        cth[n] = read_legacy_scalar(sp, p)["cth"]
    c.upload(r["cu"], s["cp"], cth, s["cf"], s["cfth"])
    _finish_load(c, False, True, r["time"], r["time_step"], reset_time)

