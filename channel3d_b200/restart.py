"""Restart files in the reference's layout (write_restart / read_restart,
src/CFD_2nd/m_IOAndVisu.f90:352-480): RestartFor<RunName><itime %10.10d>,
raw FP64 global arrays in Fortran order, ux, uy, uz, pressure, optionally
followed by HistXOld, HistYOld, HistZOld; the reader accepts 4 or 7 arrays
and rejects any other size ("file byte wrong")."""
import os

import numpy as np


def restart_name(restart_dir, run_name, itime):
    return os.path.join(restart_dir, "RestartFor%s%010d" % (run_name.strip(), itime))


def write_restart(path, ux, uy, uz, p, hist=None):
    with open(path, "wb") as f:
        for a in (ux, uy, uz, p):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        if hist is not None:
            for a in hist:
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)


def read_restart(path, cfg):
    n = cfg.npoints
    size = os.path.getsize(path)
    if size not in (4 * 8 * n, 7 * 8 * n):
        raise ValueError("Read_Restart: file byte wrong (%d bytes, expected %d or %d)" % (size, 32 * n, 56 * n))
    data = np.fromfile(path, dtype=np.float64)
    arrs = [data[q * n:(q + 1) * n].reshape(cfg.shape) for q in range(size // (8 * n))]
    hist = arrs[4:7] if len(arrs) == 7 else None
    return arrs[0], arrs[1], arrs[2], arrs[3], hist
