"""ctypes binding of libch3d.so (include/ch3d.h).

The library is built in-tree by channel3d_b200/build.py.  Loading fails loudly
when it is missing: there is no CPU fallback for the time step.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libch3d.so")

CH3D_OK = 0
CH3D_ERR_INVALID = 1
CH3D_ERR_UNSUPPORTED = 2
CH3D_ERR_CUDA = 3
CH3D_ERR_DIVERGED = 4
CH3D_ERR_NOMEM = 5

LAYOUT_INTERIOR = 0
LAYOUT_GHOST2 = 1
LAYOUT_GHOST4 = 2

PREC_FP64 = 0
PREC_MIXED = 1

_D6 = ctypes.c_double * 6
_I6 = ctypes.c_int * 6
_D3 = ctypes.c_double * 3


class Ch3dConfig(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int),
        ("nxc", ctypes.c_int), ("nyc", ctypes.c_int), ("nzc", ctypes.c_int),
        ("xlx", ctypes.c_double), ("yly", ctypes.c_double), ("zlz", ctypes.c_double),
        ("xnu", ctypes.c_double),
        ("dtMax", ctypes.c_double),
        ("iCFL", ctypes.c_int),
        ("CFLc", ctypes.c_double),
        ("ischeme", ctypes.c_int),
        ("IsImplicit", ctypes.c_int),
        ("FlowType", ctypes.c_int),
        ("BcOption", _I6),
        ("uxBcValue", _D6), ("uyBcValue", _D6), ("uzBcValue", _D6),
        ("gravity", _D3),
        ("IsUxConst", ctypes.c_int),
        ("ubulk", ctypes.c_double), ("ybulk1", ctypes.c_double), ("ybulk2", ctypes.c_double),
        ("LES_type", ctypes.c_int),
        ("FilterType", ctypes.c_int),
        ("Cs", ctypes.c_double),
        ("vel_limit", ctypes.c_double), ("div_limit", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class Ch3dStepInfo(ctypes.Structure):
    _fields_ = [
        ("SimTime", ctypes.c_double), ("dt", ctypes.c_double), ("cflmp", ctypes.c_double),
        ("divmax1", ctypes.c_double), ("divmax2", ctypes.c_double), ("vmax", _D3),
        ("uxm", ctypes.c_double), ("PrGradAver", ctypes.c_double),
        ("itime", ctypes.c_int), ("status", ctypes.c_int),
    ]

    def as_dict(self):
        return {"SimTime": self.SimTime, "dt": self.dt, "cflmp": self.cflmp, "divmax1": self.divmax1,
                "divmax2": self.divmax2, "vmax": list(self.vmax), "uxm": self.uxm,
                "PrGradAver": self.PrGradAver, "itime": self.itime, "status": self.status}


_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p

# name -> (restype, argtypes); mirrors include/ch3d.h
SIGNATURES = {
    "ch3d_version": (ctypes.c_char_p, []),
    "ch3d_last_error": (ctypes.c_char_p, []),
    "ch3d_mesh_section": (ctypes.c_int, [_DP, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "ch3d_mesh_y": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int, _DP, _IP, _IP, _IP, _DP, _DP]),
    "ch3d_create": (ctypes.c_int, [ctypes.POINTER(Ch3dConfig), _DP, ctypes.POINTER(_VP)]),
    "ch3d_destroy": (ctypes.c_int, [_VP]),
    "ch3d_upload_state": (ctypes.c_int, [_VP, ctypes.c_int, _DP, _DP, _DP, _DP, _DP]),
    "ch3d_download_state": (ctypes.c_int, [_VP, ctypes.c_int, _DP, _DP, _DP, _DP, _DP]),
    "ch3d_step": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(Ch3dStepInfo)]),
    "ch3d_stage": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    "ch3d_get_array": (ctypes.c_int, [_VP, ctypes.c_int, _DP]),
    "ch3d_set_array": (ctypes.c_int, [_VP, ctypes.c_int, _DP]),
    "ch3d_poisson": (ctypes.c_int, [_VP, _DP, _DP]),
    "ch3d_project": (ctypes.c_int, [_VP, _DP, _DP]),
    "ch3d_set_dt": (ctypes.c_int, [_VP, ctypes.c_double]),
    "ch3d_stats_accumulate": (ctypes.c_int, [_VP]),
    "ch3d_sgs_viscosity": (ctypes.c_int, [_VP]),
    "ch3d_sgs_mlp_set": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "ch3d_sgs_training_samples": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "ch3d_stats_fetch": (ctypes.c_int, [_VP, _DP, _IP, _DP, ctypes.c_int]),
    "ch3d_stats_fetch_grad": (ctypes.c_int, [_VP, _DP]),
    "ch3d_dissipation": (ctypes.c_int, [_VP, _DP]),
    "ch3d_interp_state": (ctypes.c_int, [_VP, _VP]),
    "ch3d_spectra_accumulate": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    "ch3d_spectra_fetch": (ctypes.c_int, [_VP, _DP, _DP, _DP, _IP, ctypes.c_int]),
    "ch3d_memory_bytes": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_longlong)]),
    "ch3d_last_step_ms": (ctypes.c_int, [_VP, _DP]),
    "ch3d_path_flags": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)]),
    "ch3d_kernel_times": (ctypes.c_int, [_VP, ctypes.c_int, _DP, ctypes.c_int]),
    "ch3d_mlp_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    "ch3d_mlp_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int]),
    "ch3d_mlp_wait_check": (ctypes.c_int, [ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p]),
    "ch3d_mlp_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "ch3d_mlp_adam": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                     ctypes.c_void_p]),
    "ch3d_poisson_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, _DP, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p]),
}

_lib = None


class Ch3dError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ch3d error {code}: {msg}")
        self.code = code


def load_library(path=None):
    """Loads libch3d.so (once).  Raises if the library or a symbol is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libch3d.so not built at {p}; run channel3d_b200/build.py (no CPU fallback exists)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if not exported
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(rc, lib=None):
    if rc != CH3D_OK:
        lib = lib or load_library()
        raise Ch3dError(rc, lib.ch3d_last_error().decode())
    return rc


def dptr(a):
    """ctypes double pointer of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], "need contiguous float64"
    return a.ctypes.data_as(_DP)
