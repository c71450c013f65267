"""PQR atoms in, OpenDX potential out (pmg_read_pqr / pmg_write_dx).

The reference reads atoms with read_pqr_file (fileio.cc:10-53), shifts them
by the user's box origin (PBE_example.cc:124-129) and writes the potential
with Domain::print_dx_to_stream (Domain.h:136-185); these are the same
steps over the native library.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_lib._sig("pmg_read_pqr", ctypes.c_int, ctypes.c_char_p, _lib.PD,
          ctypes.c_int, ctypes.POINTER(ctypes.c_int))
_lib._sig("pmg_write_dx", ctypes.c_int, ctypes.c_char_p, _lib.PD,
          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
          ctypes.c_double, ctypes.c_double, ctypes.c_double)


def read_pqr(path: str, origin=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Atoms of a PQR file as rows (x, y, z, radius, charge), shifted into
    the grid frame by subtracting `origin` (the box's lower corner)."""
    n = ctypes.c_int()
    bpath = str(path).encode()
    _lib.check("pmg_read_pqr", _lib.lib.pmg_read_pqr(bpath, None, 0,
                                                     ctypes.byref(n)))
    out = np.zeros((n.value, 5))
    if n.value:
        _lib.check("pmg_read_pqr", _lib.lib.pmg_read_pqr(
            bpath, out.ctypes.data_as(_lib.PD), n.value, ctypes.byref(n)))
    out[:, :3] -= np.asarray(origin, dtype=np.float64)
    return out


def write_dx(path: str, values: np.ndarray, origin=(0.0, 0.0, 0.0),
             box_length: float | None = None) -> None:
    """Writes an (nz, ny, nx) array (x fastest in memory) as an OpenDX grid
    with the given origin and spacing box_length / (nz - 1) (box_length is
    the extent of the slowest axis, as in the reference's writer)."""
    v = np.ascontiguousarray(values, dtype=np.float64)
    if v.ndim != 3:
        raise ValueError("values must be a 3-D array")
    nz, ny, nx = v.shape
    if box_length is None:
        box_length = float(nz - 1)
    _lib.check("pmg_write_dx", _lib.lib.pmg_write_dx(
        str(path).encode(), v.ctypes.data_as(_lib.PD), nx, ny, nz,
        float(origin[0]), float(origin[1]), float(origin[2]),
        float(box_length)))
