"""ctypes binding of libpmb200.so (the C ABI of include/pmb200.h).

The library is built in-tree by ``python -m protomol3_b200.build``.  There is no CPU fallback:
if the shared library is missing, loading raises immediately.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmb200.so")

PMB_OK, PMB_ERR_ARG, PMB_ERR_CUDA, PMB_ERR_CAPACITY = 0, 1, 2, 3
PMB_ERR_UNSUPPORTED, PMB_ERR_STATE, PMB_ERR_NUMERIC = 4, 5, 6
FP64, MIXED = 0, 1
SWITCH = {"Cutoff": 0, "cutoff": 0, "C1": 1, "C2": 2}
FORCE_CUTOFF, FORCE_PME, FORCE_BONDED = 1, 2, 3
LEAPFROG, LANGEVIN = 0, 1
E_COULOMB, E_LJ, E_BOND, E_ANGLE, E_VIRIAL, E_STRIDE = 0, 1, 2, 3, 4, 16


class BoxDesc(C.Structure):
    _fields_ = [("n_atoms", C.c_int), ("n_types", C.c_int), ("charge", C.c_void_p),
                ("mass", C.c_void_p), ("type", C.c_void_p), ("molecule", C.c_void_p),
                ("lj", C.c_void_p), ("n_excl", C.c_int), ("excl_pairs", C.c_void_p),
                ("excl_kind", C.c_void_p), ("n_bonds", C.c_int), ("bonds", C.c_void_p),
                ("bond_k", C.c_void_p), ("bond_r0", C.c_void_p), ("n_angles", C.c_int),
                ("angles", C.c_void_p), ("angle_k", C.c_void_p), ("angle_theta0", C.c_void_p),
                ("ub_k", C.c_void_p), ("ub_r0", C.c_void_p), ("box", C.c_double * 3),
                ("coulomb_scaling", C.c_double)]


class ForceDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("lj", C.c_int), ("lj_switch", C.c_int),
                ("lj_switchon", C.c_double), ("lj_cutoff", C.c_double), ("coulomb", C.c_int),
                ("coulomb_switch", C.c_int), ("coulomb_switchon", C.c_double),
                ("coulomb_cutoff", C.c_double), ("grid", C.c_int * 3), ("box_grids", C.c_void_p),
                ("order", C.c_int), ("cutoff", C.c_double), ("accuracy", C.c_double),
                ("alpha", C.c_double), ("real_switch", C.c_int), ("real", C.c_int),
                ("reciprocal", C.c_int), ("correction", C.c_int)]


class IntegratorDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("timestep_fs", C.c_double), ("temperature", C.c_double),
                ("gamma_ps", C.c_double), ("seed", C.c_ulonglong)]


class Tuning(C.Structure):
    _fields_ = [("skin", C.c_double), ("sort_cell", C.c_double), ("pair_ctas_per_sm", C.c_int)]


class ConstraintDesc(C.Structure):
    _fields_ = [("n_constraints", C.c_int), ("atom1", C.c_void_p), ("atom2", C.c_void_p),
                ("rest_length", C.c_void_p), ("shake", C.c_int), ("shake_epsilon", C.c_double),
                ("shake_max_iter", C.c_int), ("rattle", C.c_int), ("rattle_epsilon", C.c_double),
                ("rattle_max_iter", C.c_int)]


# (name, restype, argtypes)
_PROTOS = [
    ("pmb_last_error", C.c_char_p, []),
    ("pmb_device_count", C.c_int, []),
    ("pmb_system_create", C.c_void_p, [C.c_void_p, C.c_int, C.c_int]),
    ("pmb_system_destroy", C.c_int, [C.c_void_p]),
    ("pmb_system_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_system_n_atoms", C.c_int, [C.c_void_p]),
    ("pmb_system_n_boxes", C.c_int, [C.c_void_p]),
    ("pmb_system_set_skin", C.c_int, [C.c_void_p, C.c_double]),
    ("pmb_system_set_tuning", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_system_get_tuning", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_vacuum_box", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    ("pmb_system_set_vacuum", C.c_int, [C.c_void_p, C.c_int]),
    ("pmb_ewald_reciprocal", C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p,
                                       C.c_void_p, C.c_int]),
    ("pmb_system_check", C.c_int, [C.c_void_p]),
    ("pmb_system_list_builds", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_system_list_tiles", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_system_evaluate_times", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_force_create", C.c_void_p, [C.c_void_p, C.c_void_p]),
    ("pmb_force_destroy", C.c_int, [C.c_void_p]),
    ("pmb_force_alpha", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_force_evaluate", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    ("pmb_evaluate", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_int]),
    ("pmb_evaluate_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int]),
    ("pmb_md_create", C.c_void_p, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    ("pmb_md_destroy", C.c_int, [C.c_void_p]),
    ("pmb_md_set_state", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pmb_md_get_checkpoint", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pmb_md_set_checkpoint", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong]),
    ("pmb_md_write_checkpoint", C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_longlong, C.c_char_p,
                                          C.c_char_p, C.c_void_p]),
    ("pmb_md_get_state", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pmb_md_get_forces", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_md_run", C.c_int, [C.c_void_p, C.c_int]),
    ("pmb_md_energies", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pmb_md_use_graph", C.c_int, [C.c_void_p, C.c_int]),
    ("pmb_md_time", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("pmb_md_set_box_noise", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pmb_md_get_box_noise", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pmb_md_set_virial", C.c_int, [C.c_void_p, C.c_int]),
    ("pmb_md_set_constraints", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_md_constraint_sweeps", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pmb_traj_open_dcd", C.c_void_p, [C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_char_p]),
    ("pmb_traj_open_xyz", C.c_void_p, [C.c_char_p, C.c_int, C.c_void_p]),
    ("pmb_traj_open_xyz_trajectory", C.c_void_p, [C.c_char_p, C.c_int, C.c_void_p]),
    ("pmb_traj_set_minimal_image", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_void_p, C.c_void_p]),
    ("pmb_traj_write_host", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_md_write_frame", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_md_write_force_frame", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_traj_flush", C.c_int, [C.c_void_p]),
    ("pmb_traj_frames", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_traj_close", C.c_int, [C.c_void_p]),
    ("pmb_md_kernels_per_step", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_md_device_bytes", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pmb_profile", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                              C.c_void_p, C.c_int, C.c_void_p, C.c_char_p, C.c_int]),
    ("pmb_fp32_peak", C.c_int, [C.c_void_p]),
    ("pmb_cutoff_evaluate_static", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_int]),
]
STATIC_MAX_BOXES = 1024

_lib = None


class PMBError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("libpmb200 error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Loads libpmb200.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libpmb200.so not built: run `python -m protomol3_b200.build` "
                              "(expected at %s)" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, res, args in _PROTOS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    m = lib().pmb_last_error()
    return m.decode() if m else ""


def check(code):
    if code != PMB_OK:
        raise PMBError(code, last_error())
    return code


def checked_ptr(p):
    if not p:
        raise PMBError(-1, last_error())
    return p
