"""Restart files in DGM's format and the Domain::diff comparison (host code).

The reader is pinned to the reference's own golden restart (runs/vhex.ref,
read directly when the reference checkout is present, else skipped) and to
the fixtures decoded from it; the writer round-trips through both the
library's reader and the test-side decoder; the diff tool's Linf/L2 norms
are checked against a numpy restatement of Field::norm
(src/Field.cpp:4675-4697) and its H1 norm against an independent GLL
derivative.  The GPU test writes a domain's state and reads it back.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics
from tests.cases import diff_norms

# The reference checkout (read-only), when one is mounted: DGM_REFERENCE_ROOT
# names its root; the tests that read its files skip without it.
REF_ROOT = os.environ.get("DGM_REFERENCE_ROOT", "")
REF = os.path.join(REF_ROOT, "runs", "vhex.ref") if REF_ROOT else ""
CHAN_REF = os.path.join(REF_ROOT, "runs", "chan", "chan.ref") if REF_ROOT else ""


def test_reads_the_references_golden_restart():
    import dgm_b200
    if not os.path.exists(REF):
        pytest.skip("reference checkout not mounted")
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "vhex.npz"))
    nm, fields, info = dgm_b200.restart_read(REF, 5)
    assert info["ne"] == 8 and info["nsd"] == 3 and info["lmax"] == 1331 and info["step"] == 1000
    assert info["t"] == 1.0 and info["dt"] == 0.001
    assert np.array_equal(nm, g["nmodes"])
    assert np.array_equal(np.stack(fields), g["modal"])


def _json_restart(path, modes, step, t, dt, scalar="float64"):
    """A restart file with the JSON header the reference writes
    (src/Domain.cpp:1500-1560): the object, a newline, the binary body."""
    nf, ne, nm = modes.shape
    hdr = ('{\n   "Basis type" : "Normalized",\n   "Field names" : [ "r", "ru", "rv", "rw", "rE" ],\n'
           '   "Lmax" : %d,\n   "Nel" : %d,\n   "Nsd" : 3,\n   "Step" : %d,\n   "Time" : %r,\n'
           '   "Time step" : %r,\n   "Types" : {\n      "ByteOrder" : "LittleEndian",\n'
           '      "GlobalSize" : "int32",\n      "LocalSize" : "int32",\n      "Scalar" : "%s"\n   }\n}\n'
           % (nm, ne, step, t, dt, scalar))
    with open(path, "wb") as f:
        f.write(hdr.encode())
        for n in range(nf):
            f.write(np.int32(ne * nm).tobytes())
            f.write(np.full(ne, nm, np.int32).tobytes())
            f.write((np.arange(ne, dtype=np.int32) * nm).tobytes())
            f.write(modes[n].astype(np.float64).tobytes())


def test_reads_json_headers():
    import dgm_b200
    rng = np.random.default_rng(7)
    modes = rng.standard_normal((5, 6, 27))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "j.rst")
        _json_restart(path, modes, 40, 0.5, 0.0125)
        nm, fields, info = dgm_b200.restart_read(path, 5)
        assert np.array_equal(np.stack(fields).reshape(5, 6, 27), modes)
        assert info["ne"] == 6 and info["lmax"] == 27 and info["step"] == 40 and info["t"] == 0.5
        assert info["dt"] == 0.0125
        header, ofields, _ = dgm_io.read_restart(path, 5, 6)
        assert header["Step"] == 40 and np.array_equal(np.stack(ofields).reshape(5, 6, 27), modes)
        bad = os.path.join(d, "f32.rst")
        _json_restart(bad, modes, 1, 0.0, 0.1, scalar="float32")
        with pytest.raises(Exception):
            dgm_b200.restart_read(bad, 5)
    if os.path.exists(CHAN_REF):
        g = np.load(os.path.join(os.path.dirname(__file__), "golden", "chan.npz"))
        nm, fields, info = dgm_b200.restart_read(CHAN_REF, 5)
        assert info["step"] == 100 and np.array_equal(np.stack(fields), g["modal"])


def test_write_then_read_round_trip():
    import dgm_b200
    rng = np.random.default_rng(4)
    modes = rng.standard_normal((5, 7, 64))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "case.rst")
        dgm_b200.restart_write(path, dgm_b200.EULER3D, modes, step=12, t=0.25, dt=0.01, vis=0.002)
        nm, fields, info = dgm_b200.restart_read(path, 5)
        assert np.array_equal(np.stack(fields).reshape(5, 7, 64), modes)
        assert (nm == 64).all() and info["step"] == 12 and info["t"] == 0.25 and info["vis"] == 0.002
        header, ofields, onm = dgm_io.read_restart(path, 5, 7)
        assert np.array_equal(np.stack(ofields).reshape(5, 7, 64), modes)
        assert header[3].split()[:3] == ["7", "3", "64"] and header[3].rstrip().endswith("Nel, Nsd, Lmax")
        assert header[8].split()[:5] == ["R", "U", "V", "W", "E"]
        assert header[9].startswith("Normalized")


def _gll_D(q):
    from numpy.polynomial import legendre as lg
    n = q - 1
    c = np.zeros(n + 1)
    c[-1] = 1
    x = np.concatenate(([-1.0], np.sort(np.real(lg.legroots(lg.legder(c)))), [1.0]))
    pn = lg.legval(x, c)
    D = np.zeros((q, q))
    for i in range(q):
        for j in range(q):
            if i != j:
                D[i, j] = pn[i] / pn[j] / (x[i] - x[j])
    D[0, 0], D[-1, -1] = -n * (n + 1) / 4.0, n * (n + 1) / 4.0
    return D


def test_diff_norms_match_field_norm():
    import dgm_b200
    nx, ny, p = 6, 5, 3
    mesh = dgm_io.box_mesh(2, (nx, ny), -5.0, 5.0, p, 0)
    P = oracle.Problem(mesh, oracle.EULER2D)
    x, y, _ = P.coords()
    U1 = P.project(ics.isentropic_vortex(x, y, beta=5.0, period=(10.0, 10.0)))
    U2 = P.project(ics.isentropic_vortex(x, y, beta=4.9, x0=0.05, period=(10.0, 10.0)))
    M1, M2 = P.forward(U1), P.forward(U2)
    ne, q = mesh.verts.shape[0], p + 2
    with tempfile.TemporaryDirectory() as d:
        r1, r2 = os.path.join(d, "a.rst"), os.path.join(d, "b.rst")
        dgm_b200.restart_write(r1, dgm_b200.EULER2D, M1.reshape(4, ne, -1))
        dgm_b200.restart_write(r2, dgm_b200.EULER2D, M2.reshape(4, ne, -1))
        status, norms = dgm_b200.restart_diff(mesh, dgm_b200.EULER2D, r1, r2, aeps=1e-3, reps=1e-2)
        same, zero = dgm_b200.restart_diff(mesh, dgm_b200.EULER2D, r1, r1, aeps=0.0, reps=0.0)
    assert same == 0 and np.all(zero[:, :3] == 0.0)
    V1, V2 = P.backward(M1), P.backward(M2)
    ref = diff_norms(V1, V2, P.wj())
    D = _gll_D(q)
    hx, hy = 10.0 / nx, 10.0 / ny
    wj = P.wj()
    for n in range(4):
        assert norms[n, 0] == pytest.approx(ref[n]["linf"], rel=1e-12)
        assert norms[n, 1] == pytest.approx(ref[n]["l2"], rel=1e-10)
        assert norms[n, 3] == pytest.approx(np.abs(V1[n]).max(), rel=1e-12)
        # H1 of the difference: u^2 + |grad u|^2 with the collocation derivative
        u = (V1[n] - V2[n]).reshape(ne, q, q)
        gx = np.einsum("im,emj->eij", D, u) * (2.0 / hx)
        gy = np.einsum("jm,eim->eij", D, u) * (2.0 / hy)
        h1 = np.sqrt(((u ** 2 + gx ** 2 + gy ** 2).reshape(-1) * wj).sum() / wj.sum())
        assert norms[n, 2] == pytest.approx(h1, rel=1e-10)
    # status bits as the reference sets them
    expect = 0
    for n in range(4):
        for k in range(3):
            if norms[n, k] > 1e-3:
                expect |= 1 << k
            if norms[n, 3 + k] > np.sqrt(np.finfo(float).eps) and norms[n, k] / norms[n, 3 + k] > 1e-2:
                expect |= 8 << k
    assert status == expect and status != 0


@pytest.mark.gpu
def test_domain_restart_round_trip_and_diff_against_oracle():
    """A GPU state written and read back is the same state; a GPU run written
    as a restart passes DGM's diff against the oracle's run of the same case
    (1e-12 absolute, 1e-8 relative)."""
    import dgm_b200
    m = dgm_b200.meshgen.box(3, (3, 3, 3), 0.0, 2 * np.pi, 3)
    mesh = dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder)
    P = oracle.Problem(mesh, oracle.EULER3D)
    x, y, z = P.coords()
    f = ics.taylor_green(x, y, z, Ma=0.1)
    P.set_state(P.project(f))
    P.advance(3, 0.002, 3)
    D = dgm_b200.Domain(m, dgm_b200.EULER3D, inttype=dgm_b200.TVD3)
    D.set_state(f)
    D.advance(0.002, 3)
    ne = m.verts.shape[0]
    with tempfile.TemporaryDirectory() as d:
        gpu, ora = os.path.join(d, "gpu.rst"), os.path.join(d, "oracle.rst")
        D.write_restart(gpu, step=3, t=0.006, dt=0.002)
        dgm_b200.restart_write(ora, dgm_b200.EULER3D, P.forward(P.state()).reshape(5, ne, -1), step=3, t=0.006)
        # the w-momentum of the Taylor-Green case is ~1e-6 after three steps, so
        # its relative error at round-off is ~1e-9: the relative test uses 1e-8
        status, norms = dgm_b200.restart_diff(m, dgm_b200.EULER3D, ora, gpu, aeps=1e-12, reps=1e-8)
        assert status == 0, norms
        assert norms[:, :3].max() < 1e-12
        D2 = dgm_b200.Domain(m, dgm_b200.EULER3D, inttype=dgm_b200.TVD3)
        step, t = D2.read_restart(gpu)
        assert step == 3 and t == 0.006
        assert np.array_equal(D2.modes(), D.modes())
        # continuing from the restart equals continuing the original
        D.advance(0.002, 2)
        D2.advance(0.002, 2)
        assert np.array_equal(D2.state(), D.state())
