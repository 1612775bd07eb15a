"""The reference's I/O and init-strategy tests (tests/test_io.c) restated on
the CPU: results are attached to the handle the way those tests inject them
(host arrays in bdg_t), then written through the C API and read back.

Covered here: load_wf_fmt (:113-139), write_eigenvalues (:145-185),
write_mode_1d_real (:190-226), write_mode_2d_real (:228-283),
write_mode_out_of_range (:285-302), set_init_mode (:307-319),
reuse_modes_packs_buffer (:332-368), init_survives_reset (:370-381).
load_wf_real / complex / file_not_found and reuse_modes_no_results are in
test_library_cpu.py; sweep_reuse_1d needs solves (GPU).
"""
import ctypes as C
import ctypes.util

import numpy as np
import pytest

LIBC = C.CDLL(ctypes.util.find_library("c"))
LIBC.malloc.restype = C.c_void_p
LIBC.malloc.argtypes = [C.c_size_t]


def _host(values):
    """A malloc'd copy (bdg_free releases results with free())."""
    values = np.ascontiguousarray(values, dtype=np.float64)
    p = LIBC.malloc(values.nbytes)
    C.memmove(p, values.ctypes.data, values.nbytes)
    return p


def _problem(bdg, N, nev, m):
    p = bdg.Problem(len(N), N, [1.0] * len(N))
    p.set_system()
    p.set_solver_params(nev, m, 100, 1e-6)
    return p


def test_load_wf_fmt(bdg, tmp_path):
    (tmp_path / "test_wf_007.dat").write_text("1.5 0.0\n2.5 0.0\n")
    p = bdg.Problem(1, [2], [1.0])
    p.set_system()
    lib = C.CDLL(bdg.lib()._name)  # own handle: the variadic call without fixed argtypes
    f = lib.bdg_load_wavefunction_fmt
    f.restype = C.c_int
    rc = f(C.c_void_p(p._h.value), b"%s/test_wf_%03d.dat", str(tmp_path).encode(), C.c_int(7))
    assert rc == 0
    assert np.allclose(p.wavefunction(), [1.5, 2.5], atol=1e-12)


def test_write_eigenvalues_appends(bdg, tmp_path):
    p = _problem(bdg, [4], 3, 6)
    p.raw.eigvals = C.cast(_host([1.0, 2.0, 3.0]), C.POINTER(C.c_double))
    f = tmp_path / "ev.dat"
    assert p.write_eigenvalues(str(f)) == 0
    assert p.write_eigenvalues(str(f)) == 0  # append mode
    lines = f.read_text().splitlines()
    assert len(lines) == 2
    for ln in lines:
        assert np.allclose([float(v) for v in ln.split()], [1.0, 2.0, 3.0], rtol=1e-6)
    p.close()


def test_write_mode_1d_real(bdg, tmp_path):
    p = _problem(bdg, [4], 1, 2)
    p.raw.modes_u = _host([1.0, 2.0, 3.0, 4.0])
    base = str(tmp_path / "m")
    assert p.write_mode_u(0, base) == 0
    rows = [ln.split() for ln in (tmp_path / "m_u_0.dat").read_text().splitlines()]
    assert len(rows) == 4
    for i, r in enumerate(rows):
        assert np.allclose([float(r[0]), float(r[1])], [i + 1.0, 0.0], atol=1e-6)
    p.close()


def test_write_mode_2d_real(bdg, tmp_path):
    p = _problem(bdg, [3, 2], 1, 2)
    p.raw.modes_u = _host(np.arange(1.0, 7.0))
    base = str(tmp_path / "m2")
    assert p.write_mode_u(0, base) == 0
    with open(tmp_path / "m2_u_0.dat") as fh:
        l1, blank, l3 = fh.readline(), fh.readline(), fh.readline()
    v1 = [float(v) for v in l1.split()]
    v3 = [float(v) for v in l3.split()]
    assert len(v1) == 6 and np.allclose(v1[0::2], [1.0, 2.0, 3.0], atol=1e-6)
    assert blank == "\n"  # a blank line between y rows
    assert len(v3) == 6 and np.allclose(v3[0::2], [4.0, 5.0, 6.0], atol=1e-6)
    p.close()


def test_write_mode_out_of_range(bdg, tmp_path):
    p = _problem(bdg, [4], 2, 4)
    p.raw.modes_u = _host(np.zeros(8))
    assert p.write_mode_u(5, str(tmp_path / "oor")) == -2
    p.close()


def test_set_init_mode_and_survives_reset(bdg):
    p = bdg.Problem(1, [4], [1.0])
    p.set_init_mode(bdg.INIT_WF_WEIGHTED)
    assert p.raw.init_mode == bdg.INIT_WF_WEIGHTED
    p.set_init_mode(bdg.INIT_PLANEWAVE)
    assert p.raw.init_mode == bdg.INIT_PLANEWAVE
    p.set_system()
    p.set_init_mode(bdg.INIT_WF_WEIGHTED)
    bdg.lib().bdg_reset(p._h)
    assert p.raw.init_mode == bdg.INIT_WF_WEIGHTED
    p.close()


def test_reuse_modes_packs_buffer(bdg):
    p = _problem(bdg, [4], 2, 4)
    p.raw.modes_u = _host(np.ones(8))
    p.raw.modes_v = _host(np.ones(8))
    p.raw.converged = 2
    p.set_wavefunction(np.ones(4))
    assert p.reuse_modes(0.01) == 0
    r = p.raw
    assert r.init_mode == bdg.INIT_REUSE and r.reuse_buf and r.reuse_n == 8 and r.reuse_cols == 4
    buf = np.ctypeslib.as_array(C.cast(r.reuse_buf, C.POINTER(C.c_double)), shape=(8 * 4,))
    assert np.sum(np.abs(buf)) > 0.0
    p.close()
