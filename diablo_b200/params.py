"""Run parameters of the channel solver: grid_def + input.dat + input_chan.dat.

`DiabloParams` mirrors ``struct diablo_params`` of ``include/diablo_gpu.h``
field by field.  The two readers below parse the reference's own input files
with the reference's fixed comment-line layout:

* ``input.dat``      -- ``INITIALIZE`` (for/diablo_io.f:11-46)
* ``input_chan.dat`` -- ``INPUT_CHAN`` (for/channel.f:1456-1512)

Like the Fortran ``READ(11,*)`` list reads, values are whitespace separated,
``.TRUE.``/``.FALSE.`` are logicals and quoted strings are single tokens.
"""
from __future__ import annotations

import ctypes
import math
import shlex
from dataclasses import dataclass

MAX_TH = 4
PREC_FP64 = 0
PREC_FP32SPLIT = 1


class DiabloParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("n_th", ctypes.c_int),
        ("nu", ctypes.c_double), ("beta", ctypes.c_double), ("lx", ctypes.c_double),
        ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("nu_v_scale", ctypes.c_double),
        ("variable_dt", ctypes.c_int), ("update_dt", ctypes.c_int),
        ("cfl", ctypes.c_double),
        ("les", ctypes.c_int), ("create_new_flow", ctypes.c_int),
        ("i_ro", ctypes.c_double),
        ("grav_x", ctypes.c_double), ("grav_y", ctypes.c_double), ("grav_z", ctypes.c_double),
        ("f_type", ctypes.c_int),
        ("ubulk0", ctypes.c_double), ("px0", ctypes.c_double), ("omega0", ctypes.c_double),
        ("amp_omega0", ctypes.c_double),
        ("u_bc_ymin", ctypes.c_int), ("v_bc_ymin", ctypes.c_int), ("w_bc_ymin", ctypes.c_int),
        ("u_bc_ymax", ctypes.c_int), ("v_bc_ymax", ctypes.c_int), ("w_bc_ymax", ctypes.c_int),
        ("u_bc_ymin_c1", ctypes.c_double), ("v_bc_ymin_c1", ctypes.c_double),
        ("w_bc_ymin_c1", ctypes.c_double),
        ("u_bc_ymax_c1", ctypes.c_double), ("v_bc_ymax_c1", ctypes.c_double),
        ("w_bc_ymax_c1", ctypes.c_double),
        ("th_bc_ymin", ctypes.c_int * MAX_TH), ("th_bc_ymax", ctypes.c_int * MAX_TH),
        ("th_bc_ymin_c1", ctypes.c_double * MAX_TH), ("th_bc_ymax_c1", ctypes.c_double * MAX_TH),
        ("ri", ctypes.c_double * MAX_TH), ("pr", ctypes.c_double * MAX_TH),
        ("drhodx", ctypes.c_double * MAX_TH), ("drhodz", ctypes.c_double * MAX_TH),
        ("precision", ctypes.c_int),
        ("les_model_type", ctypes.c_int),
    ]

    def copy(self) -> "DiabloParams":
        out = DiabloParams()
        ctypes.pointer(out)[0] = self
        return out

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d

    # Derived sizes of for/header:20-28 and header_mpi:13-14 (NPROCZ = 1).
    @property
    def nkx(self) -> int:
        return self.nx // 3

    @property
    def nkz(self) -> int:
        return self.nz // 3

    @property
    def tnkz(self) -> int:
        return 2 * (self.nz // 3)

    @property
    def nxp(self) -> int:
        return self.nx // 2


@dataclass
class RunControl:
    """Time-march settings of input.dat that stay on the host."""

    n_time_steps: int = 1
    time_limit: float = 1e30
    delta_t: float = 0.01
    reset_time: bool = False
    verbosity: int = 0
    save_flow_int: int = 10**9
    save_stats_int: int = 10**9
    movie: bool = False
    ic_type: int = 0
    kick: float = 0.0
    flavor: str = "Basic"


def _tokens(line: str) -> list[str]:
    lex = shlex.shlex(line, posix=True)
    lex.whitespace += ","
    lex.whitespace_split = True
    return list(lex)


def _logical(tok: str) -> bool:
    t = tok.strip().upper().strip(".")
    if t in ("TRUE", "T"):
        return True
    if t in ("FALSE", "F"):
        return False
    raise ValueError(f"not a Fortran logical: {tok!r}")


def _num(tok: str) -> float:
    return float(tok.lower().replace("d", "e"))


class _Reader:
    """Sequential Fortran list-directed READ over the lines of a file."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0

    def skip(self, n: int = 1) -> None:
        self.pos += n

    def read(self) -> list[str]:
        while self.pos < len(self.lines):
            toks = _tokens(self.lines[self.pos])
            self.pos += 1
            if toks:
                return toks
        raise ValueError("unexpected end of input file")


def read_input_dat(text: str, p: DiabloParams, ctl: RunControl) -> None:
    """Parse input.dat exactly as INITIALIZE does (for/diablo_io.f:17-46)."""
    r = _Reader(text)
    r.skip(4)
    t = r.read()
    ctl.flavor = t[0]
    if abs(_num(t[1]) - 2.0) > 1e-6:
        raise ValueError("Wrong input data format.")
    r.skip()
    t = r.read()
    _use_mpi, p.les = _logical(t[0]), int(_logical(t[1]))
    r.skip()
    t = r.read()
    p.nu, p.beta, p.lx, p.ly, p.lz = (_num(x) for x in t[:5])
    r.skip()
    p.nu_v_scale = _num(r.read()[0])
    r.skip()
    t = r.read()
    num_per_dir, p.create_new_flow = int(_num(t[0])), int(_logical(t[1]))
    if num_per_dir != 2:
        raise ValueError("only the channel geometry (NUM_PER_DIR=2) is provided")
    r.skip()
    t = r.read()
    ctl.n_time_steps = int(_num(t[0]))
    ctl.time_limit = _num(t[1])
    ctl.delta_t = _num(t[2])
    ctl.reset_time = _logical(t[3])
    p.variable_dt = int(_logical(t[4]))
    p.cfl = _num(t[5])
    p.update_dt = int(_num(t[6]))
    r.skip()
    t = r.read()
    ctl.verbosity, ctl.save_flow_int, ctl.save_stats_int = int(_num(t[0])), int(_num(t[1])), int(_num(t[2]))
    ctl.movie = _logical(t[3])
    r.skip()
    r.read()  # binning parameters (diagnostic only)
    r.skip()
    for n in range(p.n_th):
        r.skip()
        r.read()  # CREATE_NEW_TH(N)
        r.skip()
        t = r.read()
        p.ri[n], p.pr[n] = _num(t[0]), _num(t[1])


def read_input_chan_dat(text: str, p: DiabloParams, ctl: RunControl) -> None:
    """Parse input_chan.dat exactly as INPUT_CHAN does (for/channel.f:1466-1509)."""
    r = _Reader(text)
    r.skip(4)
    if abs(_num(r.read()[0]) - 2.0) > 1e-6:
        raise ValueError("Wrong input data format input_chan")
    r.skip()
    time_ad_meth = int(_num(r.read()[0]))
    if time_ad_meth != 1:
        raise ValueError("RK_CHAN_2 is not supported (for/channel.f:1076-1100)")
    r.skip()
    p.les_model_type = int(_num(r.read()[0]))
    r.skip()
    t = r.read()
    ctl.ic_type, ctl.kick = int(_num(t[0])), _num(t[1])
    r.skip()
    p.i_ro = _num(r.read()[0])
    r.skip()
    t = r.read()
    p.grav_x, p.grav_y, p.grav_z = (_num(x) for x in t[:3])
    r.skip()
    t = r.read()
    p.f_type = int(_num(t[0]))
    p.ubulk0, p.px0, p.omega0, p.amp_omega0 = (_num(x) for x in t[1:5])
    for name in ("u_bc_ymin", "v_bc_ymin", "w_bc_ymin", "u_bc_ymax", "v_bc_ymax", "w_bc_ymax"):
        r.skip()
        t = r.read()
        setattr(p, name, int(_num(t[0])))
        setattr(p, name + "_c1", _num(t[1]))
    r.skip()
    for n in range(p.n_th):
        r.skip()
        t = r.read()
        p.th_bc_ymin[n], p.th_bc_ymin_c1[n] = int(_num(t[0])), _num(t[1])
        r.skip()
        t = r.read()
        p.th_bc_ymax[n], p.th_bc_ymax_c1[n] = int(_num(t[0])), _num(t[1])
        r.skip()
        t = r.read()
        p.drhodx[n], p.drhodz[n] = _num(t[0]), _num(t[1])


def validate(p: DiabloParams) -> None:
    """Host-side checks the library repeats (a negative status there)."""
    for name, v in (("NX", p.nx), ("NZ", p.nz)):
        m = v
        for r in (2, 3, 5):
            while m % r == 0 and m > 1:
                m //= r
        if v < 8 or m != 1:
            raise ValueError(f"{name}={v} must be a product of 2, 3 and 5")
    if p.nx % 2:
        raise ValueError("NX must be even")
    if p.ny < 4:
        raise ValueError("NY must be at least 4")
    if not (0 <= p.n_th <= MAX_TH):
        raise ValueError(f"N_TH must be in 0..{MAX_TH}")
    if p.les:
        if p.les_model_type not in (1, 2, 4):
            # 1: constant Smagorinsky (les.f); 2: the dynamic model of this
            # library (the reference stops for 2 and 3, les.f:269-272); 4: the
            # learned closure of this library
            raise ValueError("LES_MODEL_TYPE must be 1 (constant), 2 (dynamic) or 4 (learned closure)")
        if p.v_bc_ymin == 2 or p.v_bc_ymax == 2:
            # APPLY_BC_VEL_PHYS stops for V_BC = 2 (channel.f:2554, 2656)
            raise ValueError("LES needs V_BC_YMIN, V_BC_YMAX in 0, 1")


def kelvin_helmholtz(nx: int = 64, ny: int = 65, nz: int = 64, precision: int = PREC_FP64) -> DiabloParams:
    """Stratified shear layer: Lx=4pi, Lz=2pi, y in [-10,10], Re=1000, Pr=1,
    Ri=0.1, fixed dt; BCs of KH_test/input_chan.dat (U, W, TH Neumann 0,
    V Dirichlet 0, no forcing)."""
    p = DiabloParams()
    p.nx, p.ny, p.nz, p.n_th = nx, ny, nz, 1
    p.nu, p.beta = 1.0e-3, 1.0
    p.lx, p.ly, p.lz = 4.0 * math.pi, 20.0, 2.0 * math.pi
    p.nu_v_scale = 1.0
    p.variable_dt, p.update_dt, p.cfl = 0, 1, 0.5
    p.grav_y = 1.0
    p.f_type = 3
    p.u_bc_ymin = p.w_bc_ymin = 1
    p.u_bc_ymax = p.w_bc_ymax = 1
    p.v_bc_ymin = p.v_bc_ymax = 0
    p.th_bc_ymin[0] = p.th_bc_ymax[0] = 1
    p.ri[0], p.pr[0] = 0.1, 1.0
    p.create_new_flow = 1
    p.precision = precision
    return p


def turbulent_channel(nx: int = 192, ny: int = 129, nz: int = 160, re_tau: float = 180.0,
                      precision: int = PREC_FP64, variable_dt: bool = True) -> DiabloParams:
    """Closed channel on [-1,1]: no-slip walls, constant mean pressure
    gradient (F_TYPE=1, PX0=-1), NU=1/Re_tau, Lx=4pi, Lz=4pi/3, passive scalar
    with Pr=0.71, CFL-adaptive dt."""
    p = DiabloParams()
    p.nx, p.ny, p.nz, p.n_th = nx, ny, nz, 1
    p.nu, p.beta = 1.0 / re_tau, 1.0
    p.lx, p.ly, p.lz = 4.0 * math.pi, 2.0, 4.0 * math.pi / 3.0
    p.nu_v_scale = 1.0
    p.variable_dt, p.update_dt, p.cfl = int(variable_dt), 1, 0.5
    p.f_type, p.px0 = 1, -1.0
    p.u_bc_ymin = p.v_bc_ymin = p.w_bc_ymin = 0
    p.u_bc_ymax = p.v_bc_ymax = p.w_bc_ymax = 0
    p.th_bc_ymin[0] = p.th_bc_ymax[0] = 0
    p.th_bc_ymin_c1[0], p.th_bc_ymax_c1[0] = 0.0, 1.0
    p.ri[0], p.pr[0] = 0.0, 0.71
    p.create_new_flow = 1
    p.precision = precision
    return p
