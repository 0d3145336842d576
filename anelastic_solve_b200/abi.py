"""ctypes mirrors of the C-ABI structs declared in include/anel.h."""
from __future__ import annotations

import ctypes as C

import numpy as np

MAX_LEVELS = 16

OK = 0
ERR_SIZE = -1
ERR_BC = -2
ERR_NOCONV = -3
ERR_CUDA = -4
ERR_TIMEOUT = -5
ERR_ARG = -6
ERR_NOMEM = -7
ERR_UNSUPPORTED = -8
ERR_NONFINITE = -9

SMOOTHER_RBPGS = 0
SMOOTHER_LJ = 1
SMOOTHER_ZLINE = 2
MODE_LITERAL = 0
MODE_METRIC = 1
PREC_FP64 = 0
PREC_MIXED = 1
STOP_RELMAX = 0
STOP_RESID = 1
MEM_HOST = 0
MEM_DEVICE = 1
BC_PERIODIC = 0
BC_NEUMANN = 1
BC_DIRICHLET = 2

_DP = C.POINTER(C.c_double)


class GridDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("xL", C.c_double), ("yL", C.c_double), ("zL", C.c_double),
        ("xe", _DP), ("xc", _DP), ("dxe", _DP), ("dxc", _DP), ("rdxe", _DP), ("rdxc", _DP),
        ("ye", _DP), ("yc", _DP), ("dye", _DP), ("dyc", _DP), ("rdye", _DP), ("rdyc", _DP),
        ("ze", _DP), ("zc", _DP), ("dze", _DP), ("dzc", _DP), ("rdze", _DP), ("rdzc", _DP)]


class MGParams(C.Structure):
    _fields_ = [("levels", C.c_int32 * 3), ("maxcy", C.c_int32), ("tolmax", C.c_double),
                ("smoother", C.c_int32), ("pre_relax", C.c_int32 * MAX_LEVELS),
                ("post_relax", C.c_int32 * MAX_LEVELS), ("tbc", C.c_int32 * 6),
                ("vbc", C.c_double * 6), ("mode", C.c_int32), ("precision", C.c_int32),
                ("stop", C.c_int32), ("verbose", C.c_int32)]


class MGReport(C.Structure):
    _fields_ = [("iter", C.c_int32), ("status", C.c_int32), ("relmax", C.c_double),
                ("resid", C.c_double), ("ms", C.c_double), ("launches", C.c_int64),
                ("fine_sweeps", C.c_int32), ("reserved", C.c_int32),
                ("fine_sweep_ms", C.c_double)]


def dptr(a: np.ndarray):
    """Pointer to the data of a C- or Fortran-contiguous float64 array."""
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(_DP)


def make_grid_desc(grid):
    """Build a GridDesc from an anelastic_solve_b200.grid.Grid; returns
    (desc, keepalive) -- keep the second item alive while desc is used."""
    keep = []
    d = GridDesc()
    d.nx, d.ny, d.nz = grid.x.n, grid.y.n, grid.z.n
    d.xL, d.yL, d.zL = grid.x.L, grid.y.L, grid.z.L
    for ax, pfx in ((grid.x, "x"), (grid.y, "y"), (grid.z, "z")):
        for name, arr in zip(("e", "c", "de", "dc", "rde", "rdc"), ax.arrays()):
            a = np.ascontiguousarray(arr, dtype=np.float64)
            keep.append(a)
            fld = {"e": f"{pfx}e", "c": f"{pfx}c", "de": f"d{pfx}e", "dc": f"d{pfx}c",
                   "rde": f"rd{pfx}e", "rdc": f"rd{pfx}c"}[name]
            setattr(d, fld, dptr(a))
    return d, keep


def make_mg_params(levels, maxcy=99, tolmax=1e-10, pre=None, post=None, tbc=(0, 1, 0, 1, 0, 0),
                   vbc=(0.0,) * 6, smoother=SMOOTHER_RBPGS, mode=MODE_LITERAL,
                   precision=PREC_FP64, stop=STOP_RELMAX, verbose=0) -> MGParams:
    """``pre``/``post`` are per-level sweep counts listed coarsest -> finest,
    as in the ini file; a scalar applies to every level."""
    p = MGParams()
    ngrid = max(levels)
    for d in range(3):
        p.levels[d] = int(levels[d])
    p.maxcy = int(maxcy)
    p.tolmax = float(tolmax)
    p.smoother = int(smoother)
    pre = [2] * ngrid if pre is None else ([pre] * ngrid if np.isscalar(pre) else list(pre))
    post = [2] * ngrid if post is None else ([post] * ngrid if np.isscalar(post) else list(post))
    if len(pre) != ngrid or len(post) != ngrid:
        raise ValueError("pre/post must list one sweep count per level")
    for l in range(ngrid):
        p.pre_relax[l] = int(pre[l])
        p.post_relax[l] = int(post[l])
    for f in range(6):
        p.tbc[f] = int(tbc[f])
        p.vbc[f] = float(vbc[f])
    p.mode, p.precision, p.stop, p.verbose = int(mode), int(precision), int(stop), int(verbose)
    return p


# ------------------------------------------------------------------ stepper
MODEL_DNS = 0
MODEL_SSM = 1
MODEL_DSM = 2
DELTA_3ROOT = 0
DELTA_2ROOT = 1
DAMP_LITERAL = 0
DAMP_NONE = 1

# boundC variable index (1-based in the reference) -> name
BC_VARS = ("U1", "U2", "U3", "P", "RHO", "FLUC", "TEMP", "SCAL1")


class NSParams(C.Structure):
    _fields_ = [("Re", C.c_double), ("Pr", C.c_double), ("Sc", C.c_double),
                ("cfl", C.c_double), ("dtmax", C.c_double),
                ("g_init", C.c_double), ("g_final", C.c_double), ("gt1", C.c_double),
                ("gt2", C.c_double), ("vmodel", C.c_int32), ("rmodel", C.c_int32),
                ("smodel", C.c_int32), ("les_delta", C.c_int32), ("les_damp", C.c_int32),
                ("ssm_const", C.c_double), ("pr_sgs", C.c_double), ("les_start", C.c_int32),
                ("les_freq", C.c_int32), ("tb", ((C.c_int32 * 8) * 2) * 3),
                ("vb", ((C.c_double * 8) * 2) * 3), ("ew", C.c_int32), ("scal1_on", C.c_int32),
                ("test_ratio", C.c_double), ("filt", C.c_int32 * 3), ("stretched", C.c_int32 * 3),
                ("interp", C.c_int32), ("clip", C.c_int32), ("pguess", C.c_int32),
                ("rho_min", C.c_double), ("rho_max", C.c_double),
                ("scal1_min", C.c_double), ("scal1_max", C.c_double)]


class Fields(C.Structure):
    _fields_ = [(n, _DP) for n in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG",
                                   "q_u", "q_v", "q_w", "q_rho", "q_s", "psrc",
                                   "nuT", "kappaT", "nappaT")]


FIELD_NAMES = [n for n, _ in Fields._fields_]


INIT_SHEAR = 0
INIT_FIELDS = 1
INIT_POISSON = 2


class Request(C.Structure):
    """anel_request: one serving member."""
    _fields_ = [("grid", GridDesc), ("mg", MGParams), ("ns", NSParams), ("nsteps", C.c_int32),
                ("init", C.c_int32), ("seed", C.c_uint32), ("reserved", C.c_int32),
                ("amp", C.c_double), ("fields_in", C.POINTER(Fields)),
                ("fields_out", C.POINTER(Fields))]


class Result(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int32), ("nsteps", C.c_int32),
                ("cells", C.c_int64), ("queue_ms", C.c_double), ("run_ms", C.c_double),
                ("latency_ms", C.c_double), ("dt_last", C.c_double), ("max_div", C.c_double),
                ("mg_iter", C.c_int32), ("reserved", C.c_int32), ("resid", C.c_double)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("bytes_in_use", C.c_int64), ("peak_bytes", C.c_int64), ("active", C.c_int32),
                ("peak_active", C.c_int32), ("contexts", C.c_int32), ("queued", C.c_int32),
                ("peak_cohort", C.c_int32), ("reserved", C.c_int32)]


class StepReport(C.Structure):
    _fields_ = [("nstep", C.c_int32), ("mg_iter", C.c_int32 * 3), ("dt", C.c_double),
                ("time", C.c_double), ("mg_relmax", C.c_double * 3), ("max_div", C.c_double),
                ("avg_div", C.c_double), ("ms", C.c_double), ("mg_ms", C.c_double),
                ("launches", C.c_int64), ("fine_sweeps", C.c_int32), ("reserved", C.c_int32),
                ("fine_sweep_ms", C.c_double), ("diag_ms", C.c_double)]


class RestartHeader(C.Structure):
    """Header record of a restart file (Restart.F90 write_flow_*)."""
    _fields_ = [("nstep", C.c_int32), ("time", C.c_double), ("delt", C.c_double), ("g", C.c_double),
                ("rho_0", C.c_double), ("scal1_0", C.c_double), ("Re", C.c_double), ("Pr", C.c_double),
                ("Sc", C.c_double)]


RESTART_SMALL = 0  # serial dump (write_flow_small / Greadfile)
RESTART_BIG = 1    # one rank's file (write_flow_big / start_big)
RESTART_FIELDS = ("u", "v", "w", "p", "rho", "scal1")


# plane statistics of the driver's dk/dt block (NSsolver.F90:288-395)
DIAG_LITERAL = 0    # center_velocity's stretched-axis interpolation as written
DIAG_CORRECTED = 1  # the same 5-point interpolation of the values over the coordinates
DIAG_NAMES = ["U1", "U2", "T", "S", "MKE", "TKE", "t2", "s2",
              "dU1dt", "dU2dt", "dTdt", "dSdt", "dMKEdt", "dkdt", "dt2dt", "ds2dt"]


def free_slip_bcs(p: NSParams, rho_value=(0.0, 0.0)):
    """x, y periodic; z walls free-slip: U1, U2 Neumann 0, U3 Dirichlet 0,
    P Neumann 0, RHO Neumann (values), FLUC Neumann 0, SCAL1 Neumann 0,
    temporaries Dirichlet 0 (BC.F90:741-742)."""
    for d in range(2):
        for f in range(2):
            for v in range(8):
                p.tb[d][f][v] = 3
                p.vb[d][f][v] = -1.0
    ztypes = {0: 2, 1: 2, 2: 1, 3: 2, 4: 2, 5: 2, 6: 1, 7: 2}
    for f in range(2):
        for v in range(8):
            p.tb[2][f][v] = ztypes[v]
            p.vb[2][f][v] = 0.0
        p.vb[2][f][4] = float(rho_value[f])
    return p


def make_ns_params(Re=1000.0, Pr=1.0, Sc=1.0, cfl=1e6, dtmax=0.01, g=-0.12, les=False,
                   ssm_const=0.0289, pr_sgs=0.7, les_start=0, les_freq=1,
                   les_damp=DAMP_NONE, les_delta=DELTA_3ROOT, ew=1, scal1_on=1, models=None,
                   test_ratio=2.449489742783178, filt=(1, 1, 1), stretched=(0, 0, 0),
                   interp=None, clip=None, pguess=0) -> NSParams:
    """Shear-layer parameters: gravity constant g from t = 0 (Ginit = Gfinal
    = g, GT1 = GT2 = 0), free-slip z walls, periodic x and y."""
    p = NSParams()
    p.Re, p.Pr, p.Sc = float(Re), float(Pr), float(Sc)
    p.cfl, p.dtmax = float(cfl), float(dtmax)
    p.g_init = p.g_final = float(g)
    p.gt1 = p.gt2 = 0.0
    m = MODEL_SSM if les else MODEL_DNS
    p.vmodel, p.rmodel, p.smodel = models if models is not None else (m, m, m)
    # TestGrid_ratio / xfilter.. of the reference's runfile (run_dir/Sturb.ini:15-18)
    p.test_ratio = float(test_ratio)
    for d in range(3):
        p.filt[d] = int(filt[d])
        p.stretched[d] = int(stretched[d])
    p.interp = int(DIAG_LITERAL if interp is None else interp)
    p.les_delta, p.les_damp = int(les_delta), int(les_damp)
    p.ssm_const, p.pr_sgs = float(ssm_const), float(pr_sgs)
    p.les_start, p.les_freq = int(les_start), int(les_freq)
    p.ew = int(ew)
    p.scal1_on = int(scal1_on)
    p.pguess = int(pguess)
    # clip: None (off) or (rho_min, rho_max, scal1_min, scal1_max)
    if clip is not None:
        p.clip = 1
        p.rho_min, p.rho_max, p.scal1_min, p.scal1_max = (float(v) for v in clip)
    return free_slip_bcs(p)
