"""Channel statistics: the moments of clcStat_CH (2nd order,
src/CFD_2nd/m_FlowType_Channel.f90:175-362) and of clcStat (4th order,
src/CFD_4th/m_FlowCase.f90:330-998), 35 plane-averaged moments per y row (rows
1..nyp) plus, for the 4th order, 98 gradient moments; accumulated on the
device.  The stats<itime> and vGrad<itime> file writers, and derived profiles
(mean U(y), rms, Re_tau)."""
import numpy as np

NSTAT = 35
NGRAD = 98


def write_stats(path, sumstat, nfstime, prgradsum, itime, ivstats, is_ux_const=True, order=2):
    """stats%10.10d in the reference's text layout (2nd order :333-360; the 4th
    order writes the magnitude of the mean pressure gradient,
    src/CFD_4th/m_FlowCase.f90:958-980)."""
    inf = 1.0 / nfstime
    with open(path, "w") as f:
        f.write("  The time step range for this fluid statistics is %7d:%7d:%7d\n"
                % (itime - (nfstime - 1) * ivstats, ivstats, itime))
        f.write("  \n")
        if is_ux_const:
            pg = abs(prgradsum) if order == 4 else prgradsum
            f.write("  Constant velocity in x-dir by adding a pressure gradient.\n")
            f.write("    time averaged pressure gradient is: %24.15E\n" % (pg * inf))
        else:
            f.write("  Variable velocity in x-dir while adding a constant body force.\n")
        f.write("  \n")
        for row in np.asarray(sumstat).reshape(-1, NSTAT):
            f.write("".join("%24.15E" % (v * inf) for v in row) + "\n")


def write_vgrad(path, sumgrad, nfstime):
    """vGrad%10.10d of the 4th order (src/CFD_4th/m_FlowCase.f90:983-997): per
    row jc = 1..nyp the 98 gradient moments / nfstime."""
    inf = 1.0 / nfstime
    with open(path, "w") as f:
        for row in np.asarray(sumgrad).reshape(-1, NGRAD):
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


def write_spectra(path_x, path_z, specx, specz, nspectime):
    """SpecX%10.10d and SpecZ%10.10d of the 4th order (src/CFD_4th/m_FlowCase.f90:1000-1045):
    EnergySpecX(nxc/2+1, nyc, 18) and EnergySpecZ(nzc/2+1, nyc, 18) / nSpectime as raw
    native-endian FP64 in Fortran order (the C order of the (18, nyc, n) arrays)."""
    inf = 1.0 / nspectime
    for path, a in ((path_x, specx), (path_z, specz)):
        (np.ascontiguousarray(a, dtype=np.float64) * inf).tofile(path)


def write_spectra2d(path, spec2d, nspectime):
    """Spec2D%10.10d of the 4th order (src/CFD_4th/m_FlowCase.f90:1047-1140): the
    EnergySpec2D(nxc/2+1, nyc/2, nzc/2+1, 9) sums / nSpectime weighted by Ratio2D
    (4 inside, 2 on the kx = 0, nxc/2 and kz = 0, nzc/2 edges, 1 at the corners: the
    wavenumbers the half spectra stand for), as native-endian FP32 (SAVE_SINGLE_Spec2D)
    in Fortran order (the C order of the (9, nzc/2+1, nyc/2, nxc/2+1) array)."""
    a = np.asarray(spec2d, dtype=np.float64)
    nzh1, nxh = a.shape[1], a.shape[3]
    r = np.full((nzh1, nxh), 4.0)
    r[:, 0] = r[:, -1] = 2.0
    r[0, :] = r[-1, :] = 2.0
    r[0, 0] = r[0, -1] = r[-1, 0] = r[-1, -1] = 1.0
    (a * (r[None, :, None, :] / nspectime)).astype(np.float32).tofile(path)


def write_tg_dissipation(path, rows):
    """The TG_dissp file of clcStat_TG (src/CFD_2nd/m_FlowType_TGVortex.f90:
    69-80, 105-109): one line per sample, SimTime and xnu <2 S_ij S_ij> in the
    format (2ES24.15)."""
    with open(path, "w") as f:
        for t, eps in rows:
            f.write("%24.15E%24.15E\n" % (t, eps))

