"""Host-side checks that need no GPU: the C ABI library, the mesh, the
namelist reader, restart files and the CPU multi-rank path."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from helpers import small_channel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_library_exports_every_declared_symbol(built):
    from channel3d_b200 import _lib
    lib = _lib.load_library()
    hdr = open(os.path.join(ROOT, "include", "ch3d.h")).read()
    names = re.findall(r"CH3D_API\s+(?:const\s+char\*|int)\s+(ch3d_\w+)\(", hdr)
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, n
    assert lib.ch3d_version().startswith(b"ch3d-b200")


def test_mesh_matches_oracle(built):
    from channel3d_b200 import mesh_y
    from oracle import oracle as O
    for st, opt in (([1, 1], [0, 1]), ([0, 0], [0, 0]), ([2, 2], [0, 1]), ([3, 3], [0, 1])):
        cfg = small_channel(16, 40, 8, StretType=st, StretOption=opt, SectioncStret=[1.2, 1.2])
        a = mesh_y(cfg)
        b = O.Oracle(cfg).mesh()[0]
        assert np.array_equal(a, b), st


def test_invalid_configs_fail_cleanly(built):
    import ctypes
    from channel3d_b200 import _lib
    lib = _lib.load_library()
    yp = np.linspace(0, 2, 13)
    for change, code in ((dict(nxc=15), _lib.CH3D_ERR_INVALID), (dict(IsImplicit=3), _lib.CH3D_ERR_UNSUPPORTED),
                         (dict(IsImplicit=0, precision="mixed", BcOption=[0, 0, 0, 0, 0, 0]),
                          _lib.CH3D_ERR_UNSUPPORTED),  # periodic y is FP64 only
                         (dict(IsImplicit=0, order=4), _lib.CH3D_ERR_UNSUPPORTED),
                         (dict(IsImplicit=2, LES_type=2), _lib.CH3D_ERR_UNSUPPORTED),  # no FIMP+LES
                         (dict(ischeme=4), _lib.CH3D_ERR_INVALID),  # "Time scheme WRONG" 
                         (dict(BcOption=[-1, -1, -1, -1, 0, 0]), _lib.CH3D_ERR_UNSUPPORTED),
                         # periodic y: both sides ("Periodic Bc Wrong"), and only the FP64 2nd-order step without LES
                         (dict(BcOption=[0, 0, 0, -1, 0, 0], IsImplicit=2), _lib.CH3D_ERR_INVALID),
                         (dict(BcOption=[0, 0, 0, 0, 0, 0], LES_type=2), _lib.CH3D_ERR_UNSUPPORTED),
                         (dict(BcOption=[0, 0, 0, 0, 0, 0], IsImplicit=2, precision="mixed"), _lib.CH3D_ERR_UNSUPPORTED),
                         (dict(dtMax=-1.0), _lib.CH3D_ERR_INVALID)):
        cfg = small_channel(16, 12, 8).copy(**change)
        c = cfg.to_c()
        h = ctypes.c_void_p()
        rc = lib.ch3d_create(ctypes.byref(c), _lib.dptr(yp), ctypes.byref(h))
        assert rc == code, (change, rc, lib.ch3d_last_error())
        assert not h.value
    bad = np.array([0, 1, 0.5] + [2.0] * 10)
    c = small_channel(16, 12, 8).to_c()
    h = ctypes.c_void_p()
    assert lib.ch3d_create(ctypes.byref(c), _lib.dptr(bad), ctypes.byref(h)) == _lib.CH3D_ERR_INVALID
    c = small_channel(16, 12, 8, device=64).to_c()  # beyond the per-device set-up tables
    assert lib.ch3d_create(ctypes.byref(c), _lib.dptr(yp), ctypes.byref(h)) == _lib.CH3D_ERR_INVALID
    assert b"device 64" in lib.ch3d_last_error()


def test_noalloc_argument_checks(built):
    """ch3d_poisson_noalloc rejects, before touching the GPU, grids whose
    spectrum exceeds its static scratch array and narrow tall grids whose
    y-solve block would need more shared memory than its kernels may use."""
    import ctypes
    from channel3d_b200 import _lib
    lib = _lib.load_library()
    fake = ctypes.c_void_p(256)  # never dereferenced: the checks fail first
    yp = np.linspace(0.0, 2.0, 257)
    assert lib.ch3d_poisson_noalloc(512, 256, 512, 6.28, 3.14, _lib.dptr(yp), -1, -1, fake, fake,
                                    None) == _lib.CH3D_ERR_INVALID
    assert b"CH3D_NOALLOC_SCRATCH_BYTES" in lib.ch3d_last_error()
    yp = np.linspace(0.0, 2.0, 801)
    assert lib.ch3d_poisson_noalloc(4, 800, 2, 6.28, 3.14, _lib.dptr(yp), -1, -1, fake, fake,
                                    None) == _lib.CH3D_ERR_UNSUPPORTED
    assert b"shared memory" in lib.ch3d_last_error()
    assert lib.ch3d_poisson_noalloc(4, 800, 2, 6.28, 3.14, _lib.dptr(yp), -1, 0, fake, fake,
                                    None) == _lib.CH3D_ERR_UNSUPPORTED


PRM = """
&BasicParam
  RestartFlag = T          ! Restart or not
  FlowType = 1
  xlx = 6.283185307, yly = 2.0
  zlz = 3.141592654
  nxc = 64, nyc = 48, nzc = 32
  xnu = 3.5714E-4
  gravity = 0.0 0.0 0.0
  dtMax= 0.002, iCFL = 2, CFLc = 1.0
  ifirst= 1, ilast = 200
  ischeme = 3, IsImplicit= 1, FFTW_plan_type = 2
  BcOption  =   0,    0,   -1,   -1,    0,    0
  uxBcValue = 6*0.0
  RunName   = "Cha_test"
  vel_limit = 2.0
  div_limit = 0.2
/End
&ubulk_Param
  IsUxConst= T
  IsUbulkGlobal =T
  ubulk = 1.0
/End
&MeshSection
  nSection = 2
/End
&MeshOptions
  SectionLength =   1     1
  nycSection    =  24    24
  StretType     =   1     1
  StretOption   =   0     1
  SectioncStret =  2.0  2.0
/End
&LesOptions
  LES_type = 0
  FilterType = 1
/End
"""


def test_prm_reader(tmp_path):
    from channel3d_b200 import ChannelConfig
    f = tmp_path / "c.prm"
    f.write_text(PRM)
    cfg = ChannelConfig.from_prm(str(f))
    assert (cfg.nxc, cfg.nyc, cfg.nzc) == (64, 48, 32)
    assert cfg.BcOption == [0, 0, -1, -1, 0, 0]
    assert cfg.uxBcValue == [0.0] * 6
    assert cfg.RunName == "Cha_test" and cfg.IsUxConst is True
    assert cfg.nycSection == [24, 24] and cfg.SectioncStret == [2.0, 2.0]
    assert abs(cfg.xnu - 3.5714e-4) < 1e-12


REF_DECKS = os.environ.get("CH3D_REFERENCE_INPUT", "")


@pytest.mark.skipif(not REF_DECKS or not os.path.isdir(REF_DECKS),
                    reason="set CH3D_REFERENCE_INPUT to the reference's Input/ folder to read its decks")
def test_prm_reader_reads_reference_decks():
    from channel3d_b200 import ChannelConfig
    cfg = ChannelConfig.from_prm(os.path.join(REF_DECKS, "TurbulentChannel_2nd.prm"))
    assert (cfg.nxc, cfg.nyc, cfg.nzc) == (256, 150, 256)
    assert cfg.IsImplicit == 1 and cfg.BcOption == [0, 0, -1, -1, 0, 0]
    assert cfg.nycSection == [75, 75] and cfg.StretType == [1, 1]
    # the Taylor-Green deck (explicit, triply periodic) passes the library's
    # argument checks: ch3d_create gets as far as the device
    import ctypes
    from channel3d_b200 import _lib, mesh_y
    tg = ChannelConfig.from_prm(os.path.join(REF_DECKS, "TaylorGreenVortex.prm"))
    assert tg.IsImplicit == 0 and tg.BcOption == [0, 0, 0, 0, 0, 0] and tg.FlowType == 3
    lib = _lib.load_library()
    c, h = tg.to_c(), ctypes.c_void_p()
    rc = lib.ch3d_create(ctypes.byref(c), _lib.dptr(mesh_y(tg)), ctypes.byref(h))
    assert rc in (_lib.CH3D_OK, _lib.CH3D_ERR_CUDA), (rc, lib.ch3d_last_error())
    if h.value:
        lib.ch3d_destroy(h)
    # the lid-driven cavity deck (walls on all faces, FlowType 5): read as written,
    # rejected by the library (walls in x and z are in the oracle only)
    cav = ChannelConfig.from_prm(os.path.join(REF_DECKS, "LidDrivenCavity.prm"))
    assert cav.FlowType == 5 and cav.BcOption == [-1] * 6 and cav.uxBcValue[3] == 1.0 and cav.IsImplicit == 2
    c, h = cav.to_c(), ctypes.c_void_p()
    assert lib.ch3d_create(ctypes.byref(c), _lib.dptr(mesh_y(cav)), ctypes.byref(h)) == _lib.CH3D_ERR_UNSUPPORTED
    assert not h.value


def test_restart_roundtrip_and_size_check(tmp_path):
    from channel3d_b200 import restart
    cfg = small_channel(8, 6, 4)
    rng = np.random.default_rng(0)
    arrs = [rng.standard_normal(cfg.shape) for _ in range(4)]
    path = restart.restart_name(str(tmp_path), cfg.RunName, 0)
    assert path.endswith("RestartFor" + cfg.RunName + "0000000000")
    restart.write_restart(path, *arrs)
    back = restart.read_restart(path, cfg)
    for a, b in zip(arrs, back[:4]):
        assert np.array_equal(a, b)
    assert back[4] is None
    with open(path, "ab") as f:
        f.write(b"\0" * 8)
    with pytest.raises(ValueError):
        restart.read_restart(path, cfg)


def test_stats_writers(tmp_path):
    """The stats file of both trees and the 4th order's vGrad file: one line per
    row jc = 1..nyp, 35 / 98 values of 24 characters, averaged over nfstime;
    the 4th-order header writes the magnitude of the mean pressure gradient
    (src/CFD_4th/m_FlowCase.f90:958-997)."""
    from channel3d_b200 import stats
    nyp = 7
    s = np.arange(35 * nyp, dtype=float).reshape(nyp, 35)
    g = -np.arange(98 * nyp, dtype=float).reshape(nyp, 98)
    for order in (2, 4):
        p = tmp_path / ("stats%d" % order)
        stats.write_stats(str(p), s * 4, 4, -0.8, itime=400, ivstats=100, order=order)
        lines = p.read_text().splitlines()
        assert lines[0] == "  The time step range for this fluid statistics is     100:    100:    400"
        pg = float(lines[3].split()[-1])
        assert pg == (0.2 if order == 4 else -0.2)
        rows = lines[5:]
        assert len(rows) == nyp and all(len(r) == 35 * 24 for r in rows)
        assert np.allclose(np.array([[float(r[24 * q:24 * q + 24]) for q in range(35)] for r in rows]), s)
    p = tmp_path / "vGrad"
    stats.write_vgrad(str(p), g * 2, 2)
    rows = p.read_text().splitlines()
    assert len(rows) == nyp and all(len(r) == 98 * 24 for r in rows)
    assert np.allclose(np.array([[float(r[24 * q:24 * q + 24]) for q in range(98)] for r in rows]), g)


def test_two_rank_reference_arm_on_cpu():
    """bench.py --impl reference under torchrun with 2 gloo ranks: rank 0 prints
    the JSON line, rank 1 exits without work."""
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--workload", "channel48_les"]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    import json
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"


def test_max_over_ranks_gloo(tmp_path):
    """The replica timing of bench.py (one process per GPU): dist_init, the
    barriers around the timed region and the max over ranks of the device
    time, here with 2 gloo ranks on the CPU; every rank must see the slowest
    rank's time."""
    script = tmp_path / "ranks.py"
    script.write_text(
        "import sys\n"
        "sys.path.insert(0, %r)\n"
        "import bench\n"
        "ws, rank, local = bench.dist_init()\n"
        "bench.barrier(ws)\n"
        "v = bench.allmax(ws, 10.0 + 5.0 * rank)\n"
        "bench.barrier(ws)\n"
        "print('RANK%%d %%d %%.1f' %% (rank, ws, v))\n" % ROOT)
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(script)]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    # the two ranks share the pipe, so their lines may interleave
    got = sorted(re.findall(r"RANK\d \d+ [\d.]+", out.stdout))
    assert got == ["RANK0 2 15.0", "RANK1 2 15.0"], (got, out.stderr[-1000:])


def test_spectra_writer(tmp_path):
    """SpecX / SpecZ: the sums / nSpectime as raw FP64 in Fortran order of
    (nxc/2+1, nyc, 18), i.e. 18 blocks of nyc rows (src/CFD_4th/m_FlowCase.f90:1000-1045)."""
    from channel3d_b200 import stats
    sx = np.arange(18 * 5 * 9, dtype=float).reshape(18, 5, 9)
    sz = -np.arange(18 * 5 * 4, dtype=float).reshape(18, 5, 4)
    stats.write_spectra(str(tmp_path / "SpecX"), str(tmp_path / "SpecZ"), sx * 3, sz * 3, 3)
    bx = np.fromfile(str(tmp_path / "SpecX"), dtype=np.float64)
    bz = np.fromfile(str(tmp_path / "SpecZ"), dtype=np.float64)
    assert bx.size == sx.size and np.allclose(bx.reshape(9, 5, 18, order="F"), np.moveaxis(sx, [0, 1, 2], [2, 1, 0]))
    assert np.allclose(bz, sz.ravel())
    s2 = np.ones((9, 3, 5, 4))
    stats.write_spectra2d(str(tmp_path / "Spec2D"), s2 * 2, 2)
    b2 = np.fromfile(str(tmp_path / "Spec2D"), dtype=np.float32).reshape(9, 3, 5, 4)
    assert b2[0, 1, 2, 1] == 4 and b2[0, 0, 2, 1] == 2 and b2[0, 1, 2, 3] == 2 and b2[0, 2, 0, 0] == 1


def test_taylor_green_field_and_writer(tmp_path):
    """InitVelocity_TG on the staggered mesh: the analytic values, uy zero on
    the y = 0 plane, discretely divergence-free when dy = dx; and the
    TG_dissp lines in the reference's (2ES24.15) format."""
    from channel3d_b200 import initfield, stats, workloads
    cfg = workloads.taylor_green(16)
    yp = np.linspace(0.0, np.pi, cfg.nyc + 1)
    ux, uy, uz, p = initfield.taylor_green(cfg, yp=yp)
    h = cfg.xlx / cfg.nxc
    i, j, k = 3, 5, 7
    yc = 0.5 * (yp[j] + yp[j + 1])
    assert abs(ux[k, j, i] - np.sin(i * h) * np.cos(yc) * np.cos((k + 0.5) * h)) < 1e-15
    assert abs(uy[k, j, i] + np.cos((i + 0.5) * h) * np.sin(yp[j]) * np.cos((k + 0.5) * h)) < 1e-15
    assert not uy[:, 0, :].any() and not uz.any() and not p.any()
    uyp = np.concatenate([uy[:, 1:, :], np.zeros_like(uy[:, :1, :])], axis=1)
    div = (np.roll(ux, -1, axis=2) - ux) / h + (uyp - uy) / np.diff(yp)[None, :, None]
    assert np.abs(div).max() < 1e-13
    path = tmp_path / "TG_dissp0000001000"
    stats.write_tg_dissipation(path, [(0.0, 4.6426766105924085e-4), (0.01, 4.64e-4)])
    lines = path.read_text().splitlines()
    assert lines[0] == "   0.000000000000000E+00   4.642676610592409E-04"
    assert len(lines[1]) == 48

