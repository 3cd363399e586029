"""SAVE_STATS_CHAN's HDF5 outputs (for/save_stats.f:38-66, 349-425,
597-637, 1136-1149) -- mean.h5, tke.h5 and, on the final call, stats.h5 --
with WriteStatH5 / WriteHDF5_real's layout (for/hdf5.f:1345-1622): one group
per quantity, an int32 ``SAMPLES`` attribute counting its datasets, and
datasets ``0001``, ``0002``, .. of NY float64 values (rows 1..NY), each with
a ``Time`` attribute (the ``time`` group holds one value per dataset and no
attribute).

The image has no HDF5 library, so a file is a zip archive of .npy members
that numpy reads with ``np.load``: dataset ``<group>/<NNNN>`` and its
attribute ``<group>/<NNNN>@Time``.  A dataset is appended as a new member,
so a call costs the size of what it adds, as with HDF5.  ``SAMPLES`` is not
stored: it is the number of datasets in the group, the value the reference
keeps (it increments it once per dataset written).

The reference writes omega_y into mean.h5's ``omega_z`` group
(save_stats.f:421-423); ``StatsWriter(omega_z_quirk=True)``, the default,
does the same, and ``False`` writes the true omega_z.
"""
from __future__ import annotations

import io
import os
import re
import zipfile

import numpy as np

from .channel import MEAN_NAMES, SCAL_NAMES

_MEMBER = re.compile(r"^(?P<g>[^/]+)/(?P<n>\d{4,})(?P<a>@Time)?\.npy$")


class StatFile:
    """One mean.h5-style file, opened for appending."""

    def __init__(self, path: str):
        self.path = path
        self._samples: dict[str, int] = {}
        if os.path.exists(path):
            with zipfile.ZipFile(path) as z:
                for name in z.namelist():
                    m = _MEMBER.match(name)
                    if m and not m["a"]:
                        self._samples[m["g"]] = max(self._samples.get(m["g"], 0), int(m["n"]))

    def samples(self, gname: str) -> int:
        return self._samples.get(gname, 0)

    def _append(self, gname: str, value: np.ndarray, time: float | None) -> int:
        n = self.samples(gname) + 1                       # NSAMP = NSAMP + 1; dname = '(I0.4)'
        members = [(f"{gname}/{n:04d}.npy", np.ascontiguousarray(value, dtype="<f8"))]
        if time is not None:
            members.append((f"{gname}/{n:04d}@Time.npy", np.array(time, dtype="<f8")))
        with zipfile.ZipFile(self.path, "a") as z:
            for name, a in members:
                buf = io.BytesIO()
                np.lib.format.write_array(buf, a, allow_pickle=False)
                z.writestr(name, buf.getvalue())
        self._samples[gname] = n
        return n

    def write_real(self, gname: str, value: float) -> int:
        """WriteHDF5_real (hdf5.f:1345-1464): one value, no attribute."""
        return self._append(gname, np.array([value]), None)

    def write_stat(self, gname: str, diag: np.ndarray, time: float) -> int:
        """WriteStatH5 (hdf5.f:1466-1622): Diag(1:NY) with its Time."""
        return self._append(gname, np.asarray(diag, dtype=np.float64), time)


def read(path: str) -> dict:
    """{group: {"SAMPLES": n, "data": [n][...] float64, "Time": [n] or None}}."""
    out: dict = {}
    with np.load(path) as f:
        keys = f.files
        groups: dict[str, list[int]] = {}
        for k in keys:
            m = _MEMBER.match(k + ".npy")
            if m and not m["a"]:
                groups.setdefault(m["g"], []).append(int(m["n"]))
        for g, ns in groups.items():
            ns.sort()
            data = np.stack([f[f"{g}/{n:04d}"] for n in ns])
            has_t = f"{g}/{ns[0]:04d}@Time" in keys
            t = np.array([float(f[f"{g}/{n:04d}@Time"]) for n in ns]) if has_t else None
            out[g] = {"SAMPLES": len(ns), "data": data, "Time": t}
    return out


class StatsWriter:
    """The output side of SAVE_STATS_CHAN for one channel run: mean.h5 and
    tke.h5 on every call, the running means UBAR, VBAR, WBAR, THBARnn
    (save_stats.f:104-123) and stats.h5 on the final call."""

    def __init__(self, directory: str, omega_z_quirk: bool = True):
        self.dir = directory
        self.omega_z_quirk = omega_z_quirk
        self.nsamples = 0
        self.bar: dict[str, np.ndarray] = {}

    def _f(self, name: str) -> StatFile:
        return StatFile(os.path.join(self.dir, name))

    def save(self, c, final: bool = False) -> dict | None:
        """SAVE_STATS_CHAN(FINAL) on a Channel's current state; returns the
        profiles written (None on the final call)."""
        p, gyf, t = c.p, np.asarray(c.grid.gyf, dtype=np.float64), float(c.time)
        rows = slice(1, p.ny + 1)
        if final:
            f = self._f("stats.h5")
            f.write_stat("GYF", gyf[rows], t)
            for name in ["UBAR", "VBAR", "WBAR"] + [f"THBAR{n + 1:02d}" for n in range(p.n_th)]:
                f.write_stat(name, self.bar.get(name, np.zeros(p.ny + 2))[rows], t)
            return None
        m = c.mean_stats()
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
        mean = self._f("mean.h5")
        mean.write_real("time", t)
        mean.write_stat("gyf", gyf[rows], t)
        for name in MEAN_NAMES:
            v = m["omega_y"] if (name == "omega_z" and self.omega_z_quirk) else m[name]
            mean.write_stat(name, v[rows], t)
        for n in range(p.n_th):
            for name in SCAL_NAMES:
                mean.write_stat(f"{name}{n + 1:02d}", m[f"{name}{n + 1:02d}"][rows], t)
        tke = self._f("tke.h5")
        tke.write_real("time", t)
        tke.write_stat("gyf", gyf[rows], t)
        tke.write_stat("epsilon", m["epsilon"][rows], t)
        return m
