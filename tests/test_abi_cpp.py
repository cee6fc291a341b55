"""The C ABI from compiled C++: tests/abi_driver.cpp is built with g++
against include/dgmx.h and linked to dgm_b200/libdgmx.so, so a drift between
the header and the library fails to compile or link here.  On a GPU the
driver runs create -> time_derivative -> set_state -> advance -> get_state
-> destroy on a small Taylor-Green box and its output is checked against the
oracle."""
import math
import os
import subprocess

import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _build(tmp):
    import dgm_b200
    lib = dgm_b200.lib()._name
    exe = os.path.join(tmp, "abi_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "abi_driver.cpp"), "-o", exe, lib, "-Wl,-rpath," + os.path.dirname(lib)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_driver_compiles_and_links_against_the_header(tmp_path):
    exe = _build(str(tmp_path))
    assert os.path.exists(exe)
    out = subprocess.run(["nm", "-u", exe], check=True, capture_output=True, text=True).stdout
    for sym in ("dgmx_create", "dgmx_time_derivative", "dgmx_set_state", "dgmx_advance", "dgmx_get_state",
                "dgmx_destroy", "dgmx_sizes", "dgmx_last_error"):
        assert sym in out, sym


@pytest.mark.gpu
@pytest.mark.parametrize("flux,inttype", [(0, 14), (1, 3)])
def test_driver_matches_oracle(tmp_path, flux, inttype):
    import dgm_b200
    exe = _build(str(tmp_path))
    m = dgm_b200.meshgen.box(3, (3, 2, 3), 0.0, 2 * math.pi, 3)
    P = oracle.Problem(dgm_io.Mesh(3, m.verts, m.con, m.porder, m.qorder), oracle.EULER3D,
                       flux="roe" if flux else "laxfriedrichs")
    x, y, z = P.coords()
    f = ics.taylor_green(x, y, z, Ma=0.1)
    U0 = P.project(f)
    dt, steps = 2e-3, 3
    case = os.path.join(str(tmp_path), "case.bin")
    con = np.ascontiguousarray(m.con, dtype=np.int32).reshape(-1)
    with open(case, "wb") as fh:
        np.array([3, m.ne, con.size // 4, oracle.EULER3D, flux, inttype, steps], dtype=np.int32).tofile(fh)
        np.array([dt], dtype=np.float64).tofile(fh)
        np.ascontiguousarray(m.verts, dtype=np.float64).tofile(fh)
        con.tofile(fh)
        np.ascontiguousarray(m.porder, dtype=np.int32).tofile(fh)
        np.ascontiguousarray(m.qorder, dtype=np.int32).tofile(fh)
        np.ascontiguousarray(U0, dtype=np.float64).tofile(fh)
    out = os.path.join(str(tmp_path), "out.bin")
    subprocess.run([exe, case, out], check=True, capture_output=True, text=True)
    r = np.fromfile(out, dtype=np.float64).reshape(2, *U0.shape)
    F_o = P.rhs(U0)
    scale = np.linalg.norm(F_o) + np.linalg.norm(U0)
    assert np.linalg.norm(r[0] - F_o) / scale < 1e-12
    P.set_state(U0)
    assert P.advance(inttype, dt, steps) == 0
    O = P.state()
    assert np.linalg.norm(r[1] - O) / np.linalg.norm(O) < 1e-12
