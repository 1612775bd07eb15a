"""Binary files of the library (bdg/bdg_b200.h), on the CPU.

* psi0 round trip, real and complex, bit for bit, through the C writer and
  loader and through the numpy reader/writer (bdg_lobpcg_b200.binio);
* loader errors: missing file -1; wrong magic, wrong grid, wrong path (real
  file into a complex problem) and a short payload -2;
* modes and eigenvalues of a solve (host results attached to the handle, as
  bdg_solve leaves them) written exactly, with the header describing them;
  nothing to write -3, a bad part -2.
"""
import ctypes as C
import ctypes.util

import numpy as np
import pytest

from bdg_lobpcg_b200 import binio


def _problem(bdg, N, cplx=False):
    p = bdg.Problem(len(N), N, [4.0] * len(N), cplx)
    p.set_system()
    return p


@pytest.mark.parametrize("cplx", [False, True])
def test_wavefunction_roundtrip(bdg, tmp_path, cplx):
    N = [6, 5, 4]
    rng = np.random.default_rng(1)
    psi = rng.standard_normal(120) + (1j * rng.standard_normal(120) if cplx else 0)
    p = _problem(bdg, N, cplx)
    p.set_wavefunction(psi)
    f = str(tmp_path / "psi.bin")
    assert p.write_wavefunction_bin(f) == 0
    h, a = binio.read(f)
    assert h == {"kind": binio.WAVEFUNCTION, "dtype": binio.C128 if cplx else binio.F64, "dim": 3, "N": N,
                 "count": 1}
    assert a.shape == (1, 4, 5, 6) and np.array_equal(a.reshape(-1), psi)
    q = _problem(bdg, N, cplx)
    assert q.load_wavefunction_bin(f) == 0
    assert np.array_equal(q.wavefunction(), psi)
    # a file written by the numpy writer loads the same
    g = str(tmp_path / "psi_np.bin")
    binio.write_wavefunction(g, psi, N)
    r = _problem(bdg, N, cplx)
    assert r.load_wavefunction_bin(g) == 0
    assert np.array_equal(r.wavefunction(), psi)


def test_load_errors(bdg, tmp_path):
    N = [8, 4]
    psi = np.arange(32.0)
    good = str(tmp_path / "good.bin")
    binio.write_wavefunction(good, psi, N)
    p = _problem(bdg, N)
    assert p.load_wavefunction_bin(str(tmp_path / "missing.bin")) == -1
    raw = open(good, "rb").read()
    bad = tmp_path / "magic.bin"
    bad.write_bytes(b"NOTABDG!" + raw[8:])
    assert p.load_wavefunction_bin(str(bad)) == -2
    short = tmp_path / "short.bin"
    short.write_bytes(raw[:-8])
    assert p.load_wavefunction_bin(str(short)) == -2
    assert _problem(bdg, [4, 8]).load_wavefunction_bin(good) == -2  # other grid
    assert _problem(bdg, N, True).load_wavefunction_bin(good) == -2  # real file, complex problem
    assert p.load_wavefunction_bin(good) == 0
    assert np.array_equal(p.wavefunction(), psi)


def _attach(p, name, values):
    """Host results owned by the handle (freed by bdg_free with free())."""
    libc = C.CDLL(ctypes.util.find_library("c"))
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    ptr = libc.malloc(values.nbytes)
    C.memmove(ptr, values.ctypes.data, values.nbytes)
    setattr(p.raw, name, C.cast(ptr, type(getattr(p.raw, name))) if name == "eigvals" else ptr)


@pytest.mark.parametrize("cplx", [False, True])
def test_modes_and_eigenvalues(bdg, tmp_path, cplx):
    N = [4, 3, 2]
    size, nev = 24, 3
    p = _problem(bdg, N, cplx)
    assert p.write_modes_bin(0, str(tmp_path / "u.bin")) == -3
    assert p.write_eigenvalues_bin(str(tmp_path / "e.bin")) == -3
    rng = np.random.default_rng(2)
    u = rng.standard_normal((nev, size)) + (1j * rng.standard_normal((nev, size)) if cplx else 0)
    v = rng.standard_normal((nev, size)) + (1j * rng.standard_normal((nev, size)) if cplx else 0)
    ev = np.array([0.5, 1.0, 1.5])
    p.raw.nev = nev
    _attach(p, "modes_u", np.ascontiguousarray(u))
    _attach(p, "modes_v", np.ascontiguousarray(v))
    _attach(p, "eigvals", ev)
    assert p.write_modes_bin(2, str(tmp_path / "x.bin")) == -2
    for part, ref in ((0, u), (1, v)):
        f = str(tmp_path / f"m{part}.bin")
        assert p.write_modes_bin(part, f) == 0
        h, a = binio.read(f)
        assert h["kind"] == (binio.MODES_V if part else binio.MODES_U) and h["count"] == nev
        assert a.shape == (nev, 2, 3, 4) and np.array_equal(a.reshape(nev, size), ref)
    f = str(tmp_path / "ev.bin")
    assert p.write_eigenvalues_bin(f) == 0
    h, a = binio.read(f)
    assert h["kind"] == binio.EIGENVALUES and np.array_equal(a, ev)
    p.close()
