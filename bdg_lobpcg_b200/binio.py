"""Binary files of the library (bdg_write_*_bin / bdg_load_wavefunction_bin).

Layout: a 64-byte header (magic "BDGBIN01", version, kind, dtype, dim,
N[3], count, reserved; bdg_bin_header_t in bdg/bdg_b200.h), then `count`
fields of N[0]*N[1]*N[2] values (float64, or complex128 as interleaved
re, im), x fastest, in the host's (little-endian) byte order.
"""
import numpy as np

MAGIC = b"BDGBIN01"
VERSION = 1
WAVEFUNCTION, MODES_U, MODES_V, EIGENVALUES = 0, 1, 2, 3
F64, C128 = 0, 1
HEADER = np.dtype([("magic", "S8"), ("version", "<u4"), ("kind", "<u4"), ("dtype", "<u4"), ("dim", "<u4"),
                   ("N", "<u8", (3,)), ("count", "<u8"), ("reserved", "<u8")])
assert HEADER.itemsize == 64


def read(path):
    """(header dict, array): fields shaped (count, N[2], N[1], N[0]) for the
    first `dim` axes, eigenvalues shaped (count,)."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < HEADER.itemsize:
        raise ValueError(f"{path}: shorter than the header")
    h = np.frombuffer(raw[:HEADER.itemsize], dtype=HEADER)[0]
    if h["magic"] != MAGIC or int(h["version"]) != VERSION:
        raise ValueError(f"{path}: not a version-{VERSION} BDGBIN file")
    dt = np.complex128 if int(h["dtype"]) == C128 else np.float64
    N = [int(v) for v in h["N"]]
    count, kind, dim = int(h["count"]), int(h["kind"]), int(h["dim"])
    per = 1 if kind == EIGENVALUES else int(np.prod(N))
    data = np.frombuffer(raw[HEADER.itemsize:], dtype=dt)
    if data.size != count * per:
        raise ValueError(f"{path}: {data.size} values, header says {count * per}")
    shape = (count,) if kind == EIGENVALUES else (count,) + tuple(reversed(N[:dim]))
    header = {"kind": kind, "dtype": int(h["dtype"]), "dim": dim, "N": N, "count": count}
    return header, data.reshape(shape).copy()


def write_wavefunction(path, psi, N):
    """A psi0 file for bdg_load_wavefunction_bin: psi on the grid N (x
    fastest), float64 for the real path, complex128 for the complex one."""
    psi = np.ascontiguousarray(psi).reshape(-1)
    cplx = np.iscomplexobj(psi)
    psi = psi.astype(np.complex128 if cplx else np.float64)
    if psi.size != int(np.prod(N)):
        raise ValueError("psi does not match the grid")
    h = np.zeros(1, dtype=HEADER)
    h["magic"] = MAGIC
    h["version"] = VERSION
    h["kind"] = WAVEFUNCTION
    h["dtype"] = C128 if cplx else F64
    h["dim"] = len(N)
    h["N"][0] = list(N) + [1] * (3 - len(N))
    h["count"] = 1
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(psi.tobytes())
