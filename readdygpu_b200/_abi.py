"""ctypes mirror of include/readdy_b200.h (structures and constants).

The structures are plain C layouts; this module only declares them so the
host-side Python API and the tests can fill a system description.
"""
import ctypes as C

ABI_VERSION = 1
MAX_TYPES = 16
MAX_PAIR_POTS = 32
MAX_EXT_POTS = 16

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_OVERFLOW = -3
ERR_NONFINITE = -4
ERR_STATE = -5
ERR_NOMEM = -6
ERR_JUMP = -7

PREC_F64 = 0
PREC_F32C = 1

P2_HARMONIC = 1
P2_WEAK_PIECEWISE = 2

P1_DISK = 1
P1_CYLINDER = 2
P1_SPHERE = 3
P1_CUBE = 4

SUB_ATTRACTIVE = 1
SUB_REPULSIVE = 2
SUB_SPRING = 3
SUB_MEMBRANE = 4

SUBTYPES = {"attractive": SUB_ATTRACTIVE, "repulsive": SUB_REPULSIVE,
            "spring": SUB_SPRING, "membrane": SUB_MEMBRANE}


class PairPot(C.Structure):
    _fields_ = [("kind", C.c_int32), ("subtype", C.c_int32), ("k", C.c_double),
                ("r0", C.c_double), ("length", C.c_double), ("depth", C.c_double),
                ("pairs", C.c_uint8 * (MAX_TYPES * MAX_TYPES))]


class ExtPot(C.Structure):
    _fields_ = [("kind", C.c_int32), ("subtype", C.c_int32), ("k", C.c_double),
                ("center", C.c_double * 3), ("normal", C.c_double * 3),
                ("radius", C.c_double), ("height", C.c_double),
                ("origin", C.c_double * 3), ("extension", C.c_double * 3),
                ("consider_radius", C.c_int32), ("types", C.c_uint8 * MAX_TYPES)]


class SystemDesc(C.Structure):
    _fields_ = [("n_types", C.c_int32), ("D", C.c_double * MAX_TYPES),
                ("coll_radius", C.c_double * (MAX_TYPES * MAX_TYPES)),
                ("p_radius", C.c_double * MAX_TYPES),
                ("n_pair", C.c_int32), ("pair", PairPot * MAX_PAIR_POTS),
                ("n_ext", C.c_int32), ("ext", ExtPot * MAX_EXT_POTS),
                ("kB", C.c_double), ("T", C.c_double), ("dt", C.c_double),
                ("lo", C.c_double * 3), ("hi", C.c_double * 3),
                ("periodic", C.c_int32 * 3), ("max_cutoff", C.c_double),
                ("cell_size", C.c_double)]


class Box(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3),
                ("periodic", C.c_int32 * 3), ("seed", C.c_uint64)]


NB_AUTO, NB_CELLS, NB_LIST = 0, 1, 2


class Options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("neighbour_mode", C.c_int32),
                ("graph_steps", C.c_int32), ("skin", C.c_double), ("seed", C.c_uint64)]


class Metrics(C.Structure):
    _fields_ = [("energy", C.c_double), ("msd", C.c_double * MAX_TYPES),
                ("count", C.c_int64 * MAX_TYPES), ("step", C.c_int64),
                ("neighbour_mode", C.c_int32), ("list_builds", C.c_int32), ("skin", C.c_double),
                ("list_capacity", C.c_int32), ("list_entry_bytes", C.c_int32)]


# C-ABI functions and their signatures: (name, restype, argtypes)
P = C.c_void_p
DP = C.POINTER(C.c_double)
FP = C.POINTER(C.c_float)
I32P = C.POINTER(C.c_int32)
I64P = C.POINTER(C.c_int64)
U64P = C.POINTER(C.c_uint64)

FUNCTIONS = [
    ("rdgpu_create", C.c_int, [C.POINTER(SystemDesc), C.POINTER(Options), C.POINTER(P)]),
    ("rdgpu_create_batch", C.c_int, [C.POINTER(SystemDesc), C.c_int32, C.POINTER(Box),
                                     C.POINTER(Options), C.POINTER(P)]),
    ("rdgpu_destroy", C.c_int, [P]),
    ("rdgpu_last_error", C.c_char_p, [P]),
    ("rdgpu_set_particles", C.c_int, [P, I64P, C.c_int64, DP, I32P]),
    ("rdgpu_get_particles", C.c_int, [P, DP, I32P]),
    ("rdgpu_set_particles_f32", C.c_int, [P, I64P, C.c_int64, FP, I32P]),
    ("rdgpu_get_particles_f32", C.c_int, [P, FP, I32P]),
    ("rdgpu_num_particles", C.c_int, [P, I64P]),
    ("rdgpu_step", C.c_int, [P, C.c_int64]),
    ("rdgpu_step_with_noise", C.c_int, [P, DP]),
    ("rdgpu_set_seed", C.c_int, [P, C.c_int32, C.c_uint64]),
    ("rdgpu_forces", C.c_int, [P, DP, DP]),
    ("rdgpu_neighbor_digest", C.c_int, [P, I32P, U64P]),
    ("rdgpu_debug_noise", C.c_int, [P, C.c_int64, DP]),
    ("rdgpu_rdf", C.c_int, [P, C.c_int32, C.c_double, C.c_int32, U64P, I64P]),
    ("rdgpu_rdf_normalized", C.c_int, [P, DP]),
    ("rdgpu_metrics_get", C.c_int, [P, C.POINTER(Metrics)]),
    ("rdgpu_stream", C.c_void_p, [P]),
    ("rdgpu_launch_count", C.c_int64, [P]),
    ("rdgpu_step_profile", C.c_int, [P, C.c_int64, DP, DP]),
    ("rdgpu_autotune", C.c_int, [P]),
    ("rdgpu_apply_edits", C.c_int, [P, C.POINTER(C.c_float), C.c_int64]),
    ("rdgpu_set_bonds", C.c_int, [P, C.c_int64, I32P, I32P, C.c_int32, C.c_void_p]),
    ("rdgpu_rdf_counts_noalloc", C.c_int, [P, P, C.c_int64, C.c_int32, DP, DP, I32P, C.c_int32, C.c_double,
                                           P, P]),
]


def bind(lib):
    """Attach restype/argtypes to every C-ABI function of a loaded library."""
    for name, res, args in FUNCTIONS:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib
