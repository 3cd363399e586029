"""CPU checks of the C ABI library: it loads, exports every entry point of
include/diablo_gpu.h, and rejects bad arguments before touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from diablo_b200 import build, channel, grid as G, params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "diablo_gpu.h")).read()
    return sorted(set(re.findall(r"\b(diablo_gpu_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return channel.load_library()


def test_header_declarations_are_all_exported(lib):
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(channel.EXPORTS)


def _create(lib, p, ny=None):
    g = G.channel_grid(G.uniform_gy(p.ny, -1.0, 1.0))
    h = ctypes.c_void_p()
    arrs = [np.ascontiguousarray(a) for a in (g.gy, g.gyf, g.dy, g.dyf)]
    ptrs = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in arrs]
    rc = lib.diablo_gpu_create(ctypes.byref(p), *ptrs, ctypes.byref(h))
    return rc, h


@pytest.mark.parametrize("mut,code", [
    (lambda p: setattr(p, "nx", 28), channel.DIABLO_ERADIX),
    (lambda p: setattr(p, "nz", 14), channel.DIABLO_ERADIX),
    (lambda p: setattr(p, "ny", 3), channel.DIABLO_EINVAL),
    (lambda p: setattr(p, "n_th", 5), channel.DIABLO_EINVAL),
    (lambda p: setattr(p, "les", 1), channel.DIABLO_ENOTSUP),
    (lambda p: setattr(p, "v_bc_ymin", 2), channel.DIABLO_EINVAL),
    (lambda p: setattr(p, "precision", 7), channel.DIABLO_EINVAL),
])
def test_create_rejects_bad_parameters(lib, mut, code):
    p = P.kelvin_helmholtz(32, 17, 24)
    mut(p)
    rc, h = _create(lib, p)
    assert rc == code and not h.value
    assert lib.diablo_gpu_last_error()


def test_null_pointers_and_unsupported_routines(lib):
    p = P.kelvin_helmholtz(32, 17, 24)
    h = ctypes.c_void_p()
    assert lib.diablo_gpu_create(ctypes.byref(p), None, None, None, None, ctypes.byref(h)) == channel.DIABLO_EINVAL
    assert lib.diablo_gpu_rk_chan_2(None) == channel.DIABLO_ENOTSUP
    assert lib.diablo_gpu_destroy(None) == channel.DIABLO_EINVAL
    assert lib.diablo_gpu_kernel_launches(None) == -1


def test_params_struct_matches_header_field_order():
    text = open(os.path.join(ROOT, "include", "diablo_gpu.h")).read()
    body = text[text.index("typedef struct diablo_params"):text.index("} diablo_params;")]
    names = []
    for line in body.splitlines():
        line = line.split("/*")[0].strip().rstrip(";")
        m = re.match(r"(int|double)\s+(.*)", line)
        if m:
            names += [n.strip().split("[")[0] for n in m.group(2).split(",")]
    assert names == [f for f, _ in P.DiabloParams._fields_]


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """sizeof and field offsets of diablo_params and diablo_user_rhs_args as
    gcc lays them out, against the ctypes mirrors."""
    import subprocess
    from diablo_b200.channel import UserRhsArgs
    structs = {"diablo_params": P.DiabloParams, "diablo_user_rhs_args": UserRhsArgs}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "diablo_gpu.h"', "int main(void) {"]
    for cname, ct in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in ct._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, ct in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(ct), cname
        for f, _ in ct._fields_:
            assert got[(cname, f)] == getattr(ct, f).offset, (cname, f)
