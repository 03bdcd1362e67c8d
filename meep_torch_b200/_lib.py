"""ctypes binding of the C ABI in include/meep_b200.h (libmeep_b200.so).

The library is built in-tree (``meep_torch_b200/lib/libmeep_b200.so``, see
``meep_torch_b200.build``). There is no fallback: if the library cannot be
loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# MEEP_B200_LIB selects another build of the same library (tuning variants)
LIB_PATH = os.environ.get("MEEP_B200_LIB") or os.path.join(HERE, "lib", "libmeep_b200.so")

MTB_OK, MTB_INVALID_ARG, MTB_UNSUPPORTED, MTB_DEVICE_TIMEOUT, MTB_CUDA_ERROR = 0, 1, 2, 3, 4
MTB_MAX_POLES = 8
MTB_TM, MTB_TE = 0, 1
C2_MAIN, C2_X, C2_Y = 0, 1, 2
EX, EY, EZ, HX, HY, HZ = range(6)

f32p = C.POINTER(C.c_float)
vp = C.c_void_p


class Cells(C.Structure):
    _fields_ = [("row_ptr", vp), ("col", vp), ("w", vp), ("n", C.c_int32), ("amp_col", C.c_int32),
                ("row_lo", C.c_int32), ("row_hi", C.c_int32)]


class LineSample(C.Structure):
    _fields_ = [("comp", C.c_int32), ("kind", C.c_int32), ("index", C.c_int32),
                ("lo", C.c_int32), ("hi", C.c_int32), ("pad_", C.c_int32),
                ("ring_off", C.c_int64)]


class Yee2DStruct(C.Structure):
    _fields_ = [("pol", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("pitch", C.c_int32),
                ("y_pmc", C.c_int32), ("explicit_e", C.c_int32),
                ("dt", C.c_float), ("dx", C.c_float),
                ("f_main", vp * 2), ("f_x", vp * 2), ("f_y", vp * 2),
                ("inv_eps_a", vp), ("inv_eps_b", vp), ("e_explicit", vp),
                ("psi", (vp * 2) * 4),
                ("hx_b", vp), ("hx_a", vp), ("hy_b", vp), ("hy_a", vp),
                ("ex_b", vp), ("ex_a", vp), ("ey_b", vp), ("ey_a", vp),
                ("src_e", Cells), ("src_h1", Cells), ("src_h2", Cells),
                ("lines", vp), ("n_lines", C.c_int32), ("xband", C.c_int32 * 4),
                ("yband", C.c_int32 * 4), ("pad_", C.c_int32), ("ring_full", C.c_int64 * 3),
                ("cond_d1", vp * 2), ("cond_d2", vp * 2),
                ("n_poles", C.c_int32), ("n_poles_y", C.c_int32), ("pol_p", vp * 3),
                ("pol_c", vp * 3), ("pol_py", vp * 3), ("pol_cy", vp * 3),
                ("mag_h1", vp * 2), ("mag_h2", vp * 2),
                ("cut_y", C.c_int32), ("cut_x", C.c_int32), ("cut_map_y", C.c_int32),
                ("cut_map_x", C.c_int32), ("cut_ph_y", C.c_float), ("cut_ph_x", C.c_float),
                ("pad2_", C.c_int32 * 2),
                ("f_x0", vp * 2), ("f_y0", vp * 2),
                ("chi2", vp), ("chi3", vp), ("eps_nl", vp), ("pad3_", vp),
                ("n_mpoles", C.c_int32), ("pad4_", C.c_int32 * 3), ("f_b", (vp * 2) * 2),
                ("mpol", (vp * 3) * 2), ("mpc", (vp * 3) * 2),
                ("te3", C.c_int32), ("pad5_", C.c_int32 * 3), ("tinv", vp * 4),
                ("e_x", vp), ("e_y", vp), ("c3xy", vp), ("c3yx", vp),
                ("nlx", vp * 3), ("nly", vp * 3), ("e_t", vp * 2)]


class PhaseGroup(C.Structure):
    _fields_ = [("freqs", C.POINTER(C.c_double)), ("nf", C.c_int32), ("mode", C.c_int32),
                ("dt", C.c_double)]


class DftRegion(C.Structure):
    _fields_ = [("acc", vp), ("re_off", C.c_int64), ("im_off", C.c_int64),
                ("f_stride", C.c_int64), ("ring_a", C.c_int64), ("ring_b", C.c_int64),
                ("rows", C.c_int32), ("cols", C.c_int32), ("ring_pitch", C.c_int32),
                ("acc_pitch", C.c_int32), ("group", C.c_int32), ("toff", C.c_int32)]


class Tuning(C.Structure):
    _fields_ = [("rows_per_warp", C.c_int32), ("ring_slots", C.c_int32),
                ("graph", C.c_int32), ("variant", C.c_int32), ("geometry", C.c_int32)]


class Yee3DStruct(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("zpitch", C.c_int32),
                ("dt", C.c_float), ("dx", C.c_float),
                ("point_sign", C.c_int32), ("pad_", C.c_int32),
                ("f", (vp * 2) * 6), ("eps", vp), ("psi", (vp * 2) * 12),
                ("prof_b", (vp * 2) * 3), ("prof_a", (vp * 2) * 3),
                ("src_comp", C.c_int32), ("src_is_point", C.c_int32), ("src", Cells),
                ("planes", vp), ("plane_ring_off", vp), ("n_planes", C.c_int32),
                ("pad2_", C.c_int32), ("damp", (vp * 2) * 6),
                ("n_poles", C.c_int32), ("pmc_axes", C.c_int32), ("pol_p", (vp * 2) * 3),
                ("pol_c3", vp * 3), ("pol_c1", C.c_float * 8), ("pol_c2", C.c_float * 8)]


class Adj2DBuffers(C.Structure):
    _fields_ = [("g", vp * 5), ("g_psi", vp * 4), ("tmp", vp * 4), ("g_eps", vp * 2),
                ("g_pol", vp * 2), ("g_pol_y", vp * 2), ("g_cut", (vp * 2) * 2),
                ("g_b", vp * 2), ("g_mpol", (vp * 2) * 2)]


class Adj3DBuffers(C.Structure):
    _fields_ = [("g", vp * 6), ("g_psi", vp * 12), ("tmp", vp * 15), ("g_eps", vp),
                ("g_pol", (vp * 2) * 3)]


STRUCTS = [Cells, LineSample, Yee2DStruct, PhaseGroup, DftRegion, Tuning, Yee3DStruct,
           Adj2DBuffers, Adj3DBuffers]

# name -> (restype, argtypes); the exported C ABI (include/meep_b200.h)
SIGNATURES = {
    "mtb_yee2d_plan_create": (C.c_int, [C.POINTER(Yee2DStruct), C.c_int32, C.POINTER(DftRegion),
                                        C.c_int32, C.POINTER(PhaseGroup), C.c_int32, C.c_int64,
                                        C.c_int32, C.POINTER(Tuning), C.POINTER(vp)]),
    "mtb_yee2d_run": (C.c_int, [vp, C.c_int64, C.c_int32, C.POINTER(C.c_double),
                                C.POINTER(C.c_double), vp]),
    "mtb_yee2d_current": (C.c_int32, [vp]),
    "mtb_yee2d_pole_slot": (C.c_int32, [vp]),
    "mtb_yee2d_check": (C.c_int, [vp, vp]),
    "mtb_yee2d_run_noalloc": (C.c_int, [C.POINTER(Yee2DStruct), C.POINTER(DftRegion), C.c_int32,
                                        C.POINTER(PhaseGroup), C.c_int32, C.c_int64, C.c_int32,
                                        C.c_int32, C.c_int64, C.c_int32, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), vp]),
    "mtb_yee2d_last_launches": (C.c_int64, [vp]),
    "mtb_yee2d_plan_destroy": (None, [vp]),
    "mtb_yee2d_ring": (C.c_int, [vp, C.POINTER(vp), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int32)]),
    "mtb_yee2d_ring_gather": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp, vp]),
    "mtb_yee2d_adjoint_create": (C.c_int, [C.POINTER(Yee2DStruct), C.POINTER(Adj2DBuffers),
                                           C.POINTER(DftRegion), C.c_int32,
                                           C.POINTER(PhaseGroup), C.c_int32, C.c_int64,
                                           C.c_int32, C.POINTER(vp)]),
    "mtb_yee2d_adjoint_run": (C.c_int, [vp, C.c_int64, C.c_int32, vp, C.c_int64,
                                        C.POINTER(C.c_int64), vp]),
    "mtb_yee2d_adjoint_last_launches": (C.c_int64, [vp]),
    "mtb_yee2d_adjoint_destroy": (None, [vp]),
    "mtb_yee2d_set_timing": (C.c_int, [vp, C.c_int32]),
    "mtb_yee2d_timing": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "mtb_yee3d_plan_create": (C.c_int, [C.POINTER(Yee3DStruct), C.POINTER(DftRegion), C.c_int32,
                                        C.POINTER(PhaseGroup), C.c_int32, C.c_int64,
                                        C.POINTER(Tuning), C.POINTER(vp)]),
    "mtb_yee3d_run": (C.c_int, [vp, C.c_int64, C.c_int32, C.POINTER(C.c_double), vp]),
    "mtb_yee3d_check": (C.c_int, [vp, vp]),
    "mtb_yee3d_set_slab": (C.c_int, [vp, C.c_int32, C.c_int32]),
    "mtb_yee3d_begin": (C.c_int, [vp, C.c_int64, C.c_int32, C.POINTER(C.c_double), vp]),
    "mtb_yee3d_half": (C.c_int, [vp, C.c_int32, vp]),
    "mtb_yee3d_current": (C.c_int32, [vp]),
    "mtb_yee3d_last_launches": (C.c_int64, [vp]),
    "mtb_yee3d_plan_destroy": (None, [vp]),
    "mtb_yee3d_adjoint_create": (C.c_int, [C.POINTER(Yee3DStruct), C.POINTER(Adj3DBuffers),
                                           C.POINTER(DftRegion), C.c_int32,
                                           C.POINTER(PhaseGroup), C.c_int32, C.c_int64,
                                           C.c_int32, C.POINTER(vp)]),
    "mtb_yee3d_adjoint_run": (C.c_int, [vp, C.c_int64, C.c_int32, vp, C.c_int64, C.c_int64, vp]),
    "mtb_yee3d_adjoint_last_launches": (C.c_int64, [vp]),
    "mtb_yee3d_adjoint_destroy": (None, [vp]),
    "mtb_yee3d_set_timing": (C.c_int, [vp, C.c_int32]),
    "mtb_yee3d_timing": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "mtb_pack": (C.c_int, [vp, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, vp,
                           C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                           C.c_int64, C.c_int64, vp]),
    "mtb_unpack": (C.c_int, [vp, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                             C.c_int64, C.c_int64, C.c_int64, vp, C.c_int64, C.c_int64, vp]),
    "mtb_unpack_ratio": (C.c_int, [vp, vp, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                   C.c_int64, C.c_int64, C.c_int64, C.c_int64, vp, C.c_int64,
                                   C.c_int64, vp]),
    "mtb_count_outside": (C.c_int, [vp, C.c_int64, C.c_int64, C.c_int64, vp, vp, vp, vp]),
    "mtb_last_error": (C.c_char_p, []),
    "mtb_abi_version": (C.c_int32, []),
    "mtb_struct_size": (C.c_int64, [C.c_int32]),
    "mtb_launch_count": (C.c_int64, []),
    "mtb_fno_mix": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_int32,
                              C.c_int64, C.c_int32, vp]),
    "mtb_fno_mix_dx": (C.c_int, [vp, vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_int32,
                                 C.c_int64, C.c_int32, vp]),
    "mtb_fno_mix_dw": (C.c_int, [vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int64, vp]),
    "mtb_fno_status": (C.c_int, [vp]),
}

_lib = None


def load():
    """Load the in-tree library (raises OSError with the build hint if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not built; run meep_torch_b200.build.build() "
                      "(or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for i, cls in enumerate(STRUCTS):
        n = lib.mtb_struct_size(i)
        if n != C.sizeof(cls):
            raise OSError(f"ABI mismatch for {cls.__name__}: C sizeof {n}, ctypes {C.sizeof(cls)}")
    _lib = lib
    return lib


class MtbError(RuntimeError):
    pass


class MtbUnsupported(NotImplementedError):
    pass


def check(rc: int, what: str = ""):
    """Map a status code to the reference's exception style."""
    if rc == MTB_OK:
        return
    msg = load().mtb_last_error().decode(errors="replace")
    if what:
        msg = f"{what}: {msg}"
    if rc == MTB_INVALID_ARG:
        raise ValueError(msg)
    if rc == MTB_UNSUPPORTED:
        raise MtbUnsupported(msg)
    raise MtbError(f"[status {rc}] {msg}")


def ptr(t) -> int:
    """Raw device pointer of a torch tensor (0 for None)."""
    return 0 if t is None else int(t.data_ptr())
