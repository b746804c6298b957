"""Channel statistics of clcStat_CH (src/CFD_2nd/m_FlowType_Channel.f90:175-362):
35 plane-averaged moments per y row (rows 1..nyp), accumulated on the device,
the stats<itime> file writer, and derived profiles (mean U(y), rms, Re_tau)."""
import numpy as np

NSTAT = 35


def write_stats(path, sumstat, nfstime, prgradsum, itime, ivstats, is_ux_const=True):
    """stats%10.10d in the reference's text layout (:333-360)."""
    inf = 1.0 / nfstime
    with open(path, "w") as f:
        f.write("  The time step range for this fluid statistics is %7d:%7d:%7d\n"
                % (itime - (nfstime - 1) * ivstats, ivstats, itime))
        f.write("  \n")
        if is_ux_const:
            f.write("  Constant velocity in x-dir by adding a pressure gradient.\n")
            f.write("    time averaged pressure gradient is: %24.15E\n" % (prgradsum * inf))
        else:
            f.write("  Variable velocity in x-dir while adding a constant body force.\n")
        f.write("  \n")
        for row in np.asarray(sumstat).reshape(-1, NSTAT):
            f.write("".join("%24.15E" % (v * inf) for v in row) + "\n")


def profiles(sumstat, nfstime, prgradsum, xnu, h=1.0):
    """Mean profiles and rms from the moment sums (Tool/readStat_CH.m formulas):
    U = <u>, u' = sqrt(<u^2> - <u>^2) (likewise v, w), Re_tau = u_tau h / nu with
    u_tau = sqrt(h <dp/dx>)."""
    s = np.asarray(sumstat).reshape(-1, NSTAT)[:-1] / nfstime  # rows 1..nyc
    U, V, W = s[:, 0], s[:, 1], s[:, 2]
    urms = np.sqrt(np.maximum(s[:, 4] - U * U, 0.0))
    vrms = np.sqrt(np.maximum(s[:, 5] - V * V, 0.0))
    wrms = np.sqrt(np.maximum(s[:, 6] - W * W, 0.0))
    dpdx = prgradsum / nfstime
    utau = np.sqrt(max(h * dpdx, 0.0))
    return {"U": U, "urms": urms, "vrms": vrms, "wrms": wrms, "dpdx": dpdx, "Re_tau": utau * h / xnu}
