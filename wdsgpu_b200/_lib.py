"""ctypes binding of libwds_b200.so (the C ABI declared in include/wds_b200.h).

The library is loaded from the package directory only; if it is missing the
import of the solver fails loudly -- there is no CPU or library fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwds_b200.so")

c_int8_p = ctypes.POINTER(ctypes.c_int8)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_double_p = ctypes.POINTER(ctypes.c_double)

KIND_PIPE, KIND_CVPIPE, KIND_TCV, KIND_PUMP, KIND_PRV_FIXED, KIND_PRV, KIND_FCV, KIND_PSV = range(8)
F_ZERO_SPEED, F_PUMP_LIVE, F_CHP, F_IS_PIPE = 1, 2, 4, 8
TL_OVERFLOW, TL_IS_PUMP, TL_PUMP_IN, TL_PUMP_OUT = 1, 2, 4, 8
INFO_NOT_PD, INFO_UNCONVERGED, INFO_EMITTER_CAP, INFO_BAD_HEAD = 1, 2, 4, 8
LAYOUT_AUTO, LAYOUT_SHARED, LAYOUT_GLOBAL = 0, 1, 2
E_NAMES = {-1: "bad argument", -2: "CUDA error", -3: "out of memory",
           -4: "unsupported network", -5: "no forward state"}

EXPORTS = ("wds_plan", "wds_forward", "wds_adjoint", "wds_plan_stats",
           "wds_plan_symbolic", "wds_state_generation", "wds_free", "wds_last_error", "wds_forward_noalloc",
           "wds_forward_multi", "wds_adjoint_multi", "wds_adjoint_rhs", "wds_adjoint_pumps",
           "wds_unrolled_adjoint")
MULTI_MAX = 8


class WdsNetwork(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int32), ("n_links", ctypes.c_int32),
        ("node_type", c_int8_p), ("elev", c_double_p),
        ("link_n1", c_int32_p), ("link_n2", c_int32_p),
        ("link_kind", c_int8_p), ("link_flags", c_uint8_p),
        ("km", c_double_p), ("km_tcv", c_double_p), ("q_init", c_double_p),
        ("status0", c_int8_p), ("pump_type", c_int8_p),
        ("pump_h0", c_double_p), ("pump_r", c_double_p), ("pump_n", c_double_p),
        ("pump_speed", c_double_p), ("pump_hmax", c_double_p),
        ("curve_ptr", c_int32_p), ("curve_x", c_double_p), ("curve_y", c_double_p),
        ("prv_hset", c_double_p),
        ("n_tank_links", ctypes.c_int32),
        ("tl_link", c_int32_p), ("tl_tank", c_int32_p), ("tl_other", c_int32_p),
        ("tl_qsign", c_double_p), ("tl_hmax", c_double_p), ("tl_hmin", c_double_p),
        ("tl_flags", c_uint8_p),
        ("hexp", ctypes.c_double), ("qexp", ctypes.c_double), ("rqtol", ctypes.c_double),
        ("htol", ctypes.c_double), ("qtol", ctypes.c_double),
        ("ucf_flow", ctypes.c_double), ("ucf_head", ctypes.c_double),
        ("checkfreq", ctypes.c_int32), ("maxcheck", ctypes.c_int32),
        ("extra_iter", ctypes.c_int32),
        ("perm", c_int32_p),
        ("emitter_capacity", ctypes.c_int32),
        ("layout", ctypes.c_int32), ("factor_fp32", ctypes.c_int32),
        ("pump_hunit", c_double_p),
        ("groups_per_cta", ctypes.c_int32), ("top_max", ctypes.c_int32),
        ("level_barrier_cost", ctypes.c_double),
    ]


class WdsForwardOpts(ctypes.Structure):
    _fields_ = [
        ("accuracy", ctypes.c_double), ("max_iter", ctypes.c_int32),
        ("status_machine", ctypes.c_int32), ("refine", ctypes.c_int32),
        ("polish_steps", ctypes.c_int32), ("ke_stride", ctypes.c_int64),
        ("r_stride", ctypes.c_int64), ("q0", ctypes.c_void_p), ("e0", ctypes.c_void_p),
        ("pump_speed", ctypes.c_void_p), ("pump_h0", ctypes.c_void_p),
        ("pump_r", ctypes.c_void_p), ("pump_stride", ctypes.c_int64),
        ("refine_band", ctypes.c_double), ("unroll_record", ctypes.c_void_p),
        ("diag_ratio", ctypes.c_void_p), ("sched_flags", ctypes.c_void_p),
        ("sched_chg", ctypes.c_void_p), ("status0", ctypes.c_void_p),
    ]


class WdsForwardIO(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "demand", "fixed_head", "ke", "r", "head", "flow", "emitter", "status", "iters",
        "relerr", "info")]


class WdsAdjointIO(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("gH", "gQ", "gE", "gd", "grh", "gke", "gr")]


_lib = None


def load():
    """Load the library (once).  Raises ImportError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libwds_b200.so is not built; run `python -m wdsgpu_b200.build` "
            "(nvcc, sm_100a).  There is no CPU fallback.")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    lib.wds_plan.argtypes = [ctypes.POINTER(WdsNetwork), ctypes.c_int32, ctypes.POINTER(vp)]
    lib.wds_plan.restype = ctypes.c_int
    lib.wds_forward.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(WdsForwardOpts)] + [vp] * 11 + [vp]
    lib.wds_forward.restype = ctypes.c_int
    lib.wds_forward_noalloc.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(WdsForwardOpts)] + [vp] * 11 + [vp]
    lib.wds_forward_noalloc.restype = ctypes.c_int
    lib.wds_adjoint.argtypes = [vp, ctypes.c_int32] + [vp] * 7 + [vp]
    lib.wds_adjoint.restype = ctypes.c_int
    lib.wds_forward_multi.argtypes = [ctypes.c_int32, ctypes.POINTER(vp), c_int32_p,
                                      ctypes.POINTER(WdsForwardOpts),
                                      ctypes.POINTER(WdsForwardIO), vp]
    lib.wds_forward_multi.restype = ctypes.c_int
    lib.wds_adjoint_multi.argtypes = [ctypes.c_int32, ctypes.POINTER(vp), c_int32_p,
                                      ctypes.POINTER(WdsAdjointIO), vp]
    lib.wds_adjoint_multi.restype = ctypes.c_int
    lib.wds_adjoint_rhs.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32] + \
        [vp] * 7 + [vp]
    lib.wds_adjoint_rhs.restype = ctypes.c_int
    lib.wds_adjoint_pumps.argtypes = [vp, ctypes.c_int32] + [vp] * 10 + [vp]
    lib.wds_adjoint_pumps.restype = ctypes.c_int
    lib.wds_unrolled_adjoint.argtypes = [vp, ctypes.c_int32, ctypes.c_int32] + [vp] * 4 + \
        [ctypes.c_int64, vp, ctypes.c_int64] + [vp] * 9 + [vp]
    lib.wds_unrolled_adjoint.restype = ctypes.c_int
    lib.wds_plan_stats.argtypes = [vp, c_int64_p]
    lib.wds_plan_stats.restype = ctypes.c_int
    lib.wds_plan_symbolic.argtypes = [vp] + [c_int32_p] * 5
    lib.wds_plan_symbolic.restype = ctypes.c_int
    lib.wds_state_generation.argtypes = [vp, c_int64_p]
    lib.wds_state_generation.restype = ctypes.c_int
    lib.wds_free.argtypes = [vp]
    lib.wds_free.restype = ctypes.c_int
    lib.wds_last_error.argtypes = []
    lib.wds_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def check(rc, what):
    if rc != 0:
        msg = load().wds_last_error().decode(errors="replace")
        kind = E_NAMES.get(rc, "error %d" % rc)
        if rc == -4:
            raise NotImplementedError("%s: %s (%s)" % (what, msg, kind))
        if rc == -1:
            raise ValueError("%s: %s (%s)" % (what, msg, kind))
        raise RuntimeError("%s: %s (%s)" % (what, msg, kind))
