"""ctypes binding of libfluamsl.so (the C ABI declared in include/fluamsl.h).

The library is built in-tree by ``fluam_b200/build.py``.  There is no CPU
fallback: if the shared library is missing or cannot be loaded, every entry
point raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfluamsl.so")

FSL_OK = 0
ERRORS = {-1: "FSL_E_ARG", -2: "FSL_E_CUDA", -3: "FSL_E_NOMEM", -4: "FSL_E_KERNEL",
          -5: "FSL_E_IO", -6: "FSL_E_INPUT"}
PAIR_NONE, PAIR_TABLE_LJ, PAIR_SOFT = 0, 1, 2
RFD_REFERENCE, RFD_PAPER = 0, 1
SCHEME_MIDPOINT, SCHEME_FIRST_ORDER, SCHEME_QUASI2D, SCHEME_STOKES2D, SCHEME_INCOMPRESSIBLE = 0, 1, 2, 3, 4
PRECISION_FIXED64, PRECISION_FLOAT_ATOMIC, PRECISION_FP64 = 0, 1, 2

# Every symbol include/fluamsl.h declares.
EXPORTS = [
    "fsl_config_defaults", "fsl_create", "fsl_load_bonds", "fsl_load_bonds_directed", "fsl_step", "fsl_sync",
    "fsl_get_positions", "fsl_set_positions", "fsl_get_forces", "fsl_get_velocity",
    "fsl_get_velocity_f64", "fsl_set_velocity_f64",
    "fsl_get_status", "fsl_get_observables", "fsl_reset_observables", "fsl_set_step", "fsl_clear_errors", "fsl_set_graph", "fsl_stream",
    "fsl_profile", "fsl_profile_read",
    "fsl_destroy", "fsl_last_error", "fsl_run_data_main", "fsl_parse_data_main",
    "fsl_write_fluid_final", "fsl_write_fluid_vtk",
    "fsl_neighbor_grid", "fsl_cell_list", "fsl_compute_forces", "fsl_spread", "fsl_solve",
    "fsl_interpolate", "fsl_noise", "fsl_cell_list_noalloc",
    "fsl_batch_create", "fsl_batch_load_bonds", "fsl_batch_step", "fsl_batch_sync",
    "fsl_batch_get_positions", "fsl_batch_get_forces", "fsl_batch_get_status",
    "fsl_batch_get_observables", "fsl_batch_reset_observables",
    "fsl_batch_get_positions_packed", "fsl_batch_set_positions_packed",
    "fsl_batch_get_positions_packed_async", "fsl_batch_set_positions_packed_async",
    "fsl_batch_set_graph", "fsl_batch_get_info", "fsl_batch_stream", "fsl_batch_destroy",
    "fsl_batch_get_class_tuning", "fsl_get_tuning", "fsl_step_io", "fsl_batch_step_io",
    "fsl_server_config_defaults", "fsl_server_create", "fsl_server_submit", "fsl_server_poll",
    "fsl_server_wait", "fsl_server_result", "fsl_server_get_stats", "fsl_server_destroy",
]
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class Config(ctypes.Structure):
    _fields_ = [
        ("mx", ctypes.c_int32), ("my", ctypes.c_int32), ("mz", ctypes.c_int32),
        ("kernel", ctypes.c_int32),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("shearviscosity", ctypes.c_double), ("temperature", ctypes.c_double),
        ("dt", ctypes.c_double), ("cutoff", ctypes.c_double),
        ("extra_mobility", ctypes.c_double), ("soft_epsilon", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("pair", ctypes.c_int32), ("rfd", ctypes.c_int32),
        ("nonbonded", ctypes.c_int32), ("device", ctypes.c_int32),
        ("scheme", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("ndrift", ctypes.c_int32), ("use_rfd", ctypes.c_int32),
        ("predictor_corrector", ctypes.c_int32), ("observables", ctypes.c_int32),
        ("radius", ctypes.c_double), ("saffman_kc", ctypes.c_double),
        ("saffman_width", ctypes.c_double), ("shear_amp", ctypes.c_double),
        ("density", ctypes.c_double),
    ]


class Status(ctypes.Structure):
    _fields_ = [
        ("step", ctypes.c_uint64), ("error_bits", ctypes.c_int32), ("np", ctypes.c_int32),
        ("nc", ctypes.c_int64), ("graph", ctypes.c_int32), ("launches_per_step", ctypes.c_int32),
    ]


class Observables(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64), ("msd", ctypes.c_double), ("msd_sum", ctypes.c_double),
        ("displacement", ctypes.c_double * 3), ("force", ctypes.c_double * 3),
        ("momentum", ctypes.c_double * 3), ("momentum_sum", ctypes.c_double * 3),
    ]

    def as_dict(self):
        return dict(steps=self.steps, msd=self.msd, msd_sum=self.msd_sum,
                    displacement=list(self.displacement), force=list(self.force),
                    momentum=list(self.momentum), momentum_sum=list(self.momentum_sum))


class StageTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_int64),
                ("total_ms", ctypes.c_double)]


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32), ("classes", ctypes.c_int32), ("graph", ctypes.c_int32),
        ("launches_per_step", ctypes.c_int32), ("np_total", ctypes.c_int64),
        ("nc_total", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
    ]


class ClassTuning(ctypes.Structure):
    _fields_ = [
        ("mx", ctypes.c_int32), ("my", ctypes.c_int32), ("mz", ctypes.c_int32),
        ("kernel", ctypes.c_int32), ("precision", ctypes.c_int32), ("scheme", ctypes.c_int32),
        ("n", ctypes.c_int32), ("tuned", ctypes.c_int32), ("fft_schedule", ctypes.c_int32),
        ("z_tile_kx", ctypes.c_int32), ("z_tile_ky", ctypes.c_int32), ("z_threads", ctypes.c_int32),
        ("z_candidates", ctypes.c_int32), ("z_us", ctypes.c_float * 8),
        ("schedule_us", ctypes.c_float * 2), ("list_build", ctypes.c_int32),
        ("list_us", ctypes.c_float * 2), ("plane_pb", ctypes.c_int32),
        ("plane_candidates", ctypes.c_int32), ("plane_us", ctypes.c_float * 4),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["z_us"] = list(self.z_us)[:self.z_candidates]
        d["schedule_us"] = list(self.schedule_us)
        d["list_us"] = list(self.list_us)
        d["plane_us"] = list(self.plane_us)[:self.plane_candidates]
        d["fft_schedule"] = {0: "plane", 1: "lines"}.get(self.fft_schedule, "other")
        d["list_build"] = {0: "separate", 1: "block_per_instance", 2: "cooperative"}.get(
            self.list_build, "none")
        return d


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_int64), ("device", ctypes.c_int32),
                ("max_round_steps", ctypes.c_int32)]


class RequestInfo(ctypes.Structure):
    _fields_ = [
        ("state", ctypes.c_int32), ("error_bits", ctypes.c_int32), ("np", ctypes.c_int64),
        ("steps", ctypes.c_int64), ("steps_done", ctypes.c_int64), ("submit_s", ctypes.c_double),
        ("start_s", ctypes.c_double), ("done_s", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int64) for f in (
        "submitted", "completed", "failed", "queued", "running", "rounds", "steps",
        "particle_steps", "bytes_held", "slots", "groups", "captures")] + [
        ("busy_s", ctypes.c_double), ("now_s", ctypes.c_double)]


class FslError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int32)
_VP = ctypes.c_void_p


def load(path=None):
    """Load libfluamsl.so (raises OSError if it is not built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"{p} is not built; run fluam_b200/build.py (nvcc, sm_100a)")
    L = ctypes.CDLL(p)
    L.fsl_config_defaults.argtypes = [ctypes.POINTER(Config)]
    L.fsl_create.argtypes = [ctypes.POINTER(Config), ctypes.c_int64, _D, ctypes.POINTER(_VP)]
    L.fsl_load_bonds.argtypes = [_VP, ctypes.c_int64, _I, _I, _D, _D, ctypes.c_int64, _I, _D, _D, _D]
    L.fsl_load_bonds_directed.argtypes = L.fsl_load_bonds.argtypes
    L.fsl_step.argtypes = [_VP, ctypes.c_int64]
    L.fsl_sync.argtypes = [_VP]
    L.fsl_get_positions.argtypes = [_VP, _D]
    L.fsl_set_positions.argtypes = [_VP, _D]
    L.fsl_get_forces.argtypes = [_VP, _D]
    L.fsl_get_velocity.argtypes = [_VP, _F]
    L.fsl_get_velocity_f64.argtypes = [_VP, _D]
    L.fsl_set_velocity_f64.argtypes = [_VP, _D]
    L.fsl_get_status.argtypes = [_VP, ctypes.POINTER(Status)]
    L.fsl_set_step.argtypes = [_VP, ctypes.c_uint64]
    L.fsl_get_observables.argtypes = [_VP, ctypes.POINTER(Observables)]
    L.fsl_reset_observables.argtypes = [_VP]
    L.fsl_clear_errors.argtypes = [_VP]
    L.fsl_set_graph.argtypes = [_VP, ctypes.c_int]
    L.fsl_stream.argtypes = [_VP]
    L.fsl_stream.restype = _VP
    L.fsl_profile.argtypes = [_VP, ctypes.c_int]
    L.fsl_profile_read.argtypes = [_VP, ctypes.POINTER(StageTime), ctypes.c_int32,
                                   ctypes.POINTER(ctypes.c_int32)]
    L.fsl_destroy.argtypes = [_VP]
    L.fsl_destroy.restype = None
    L.fsl_last_error.restype = ctypes.c_char_p
    L.fsl_run_data_main.argtypes = [ctypes.c_char_p]
    L.fsl_write_fluid_final.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config), ctypes.c_double, _D,
                                        ctypes.c_int32, _D]
    L.fsl_write_fluid_vtk.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _D]
    L.fsl_parse_data_main.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config),
                                      ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    L.fsl_neighbor_grid.argtypes = [_VP, _I]
    L.fsl_cell_list.argtypes = [_VP, _I, _I, _I]
    L.fsl_compute_forces.argtypes = [_VP, _D]
    L.fsl_spread.argtypes = [_VP, _D, _D]
    L.fsl_solve.argtypes = [_VP, _D, _D]
    L.fsl_interpolate.argtypes = [_VP, _D, _D]
    L.fsl_noise.argtypes = [_VP, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int64, _F]
    L.fsl_cell_list_noalloc.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int64, _VP, _VP, _VP, _VP, _VP]
    L.fsl_batch_create.argtypes = [ctypes.c_int32, ctypes.POINTER(Config),
                                   ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(_D),
                                   ctypes.POINTER(_VP)]
    L.fsl_batch_load_bonds.argtypes = [_VP, ctypes.c_int32, ctypes.c_int64, _I, _I, _D, _D,
                                       ctypes.c_int64, _I, _D, _D, _D]
    L.fsl_batch_step.argtypes = [_VP, ctypes.c_int64]
    L.fsl_batch_sync.argtypes = [_VP]
    L.fsl_batch_get_positions.argtypes = [_VP, ctypes.c_int32, _D]
    L.fsl_batch_get_forces.argtypes = [_VP, ctypes.c_int32, _D]
    L.fsl_batch_get_status.argtypes = [_VP, ctypes.c_int32, ctypes.POINTER(Status)]
    L.fsl_batch_get_observables.argtypes = [_VP, ctypes.c_int32, ctypes.POINTER(Observables)]
    L.fsl_batch_reset_observables.argtypes = [_VP, ctypes.c_int32]
    L.fsl_batch_get_positions_packed.argtypes = [_VP, _D]
    L.fsl_batch_set_positions_packed.argtypes = [_VP, _D]
    L.fsl_batch_get_positions_packed_async.argtypes = [_VP, _VP]
    L.fsl_batch_set_positions_packed_async.argtypes = [_VP, _VP]
    L.fsl_batch_set_graph.argtypes = [_VP, ctypes.c_int]
    L.fsl_batch_get_info.argtypes = [_VP, ctypes.POINTER(BatchInfo)]
    L.fsl_batch_get_class_tuning.argtypes = [_VP, ctypes.c_int32, ctypes.POINTER(ClassTuning)]
    L.fsl_get_tuning.argtypes = [_VP, ctypes.POINTER(ClassTuning)]
    L.fsl_step_io.argtypes = [_VP, _VP, _VP]
    L.fsl_batch_step_io.argtypes = [_VP, _VP, _VP]
    L.fsl_batch_stream.argtypes = [_VP]
    L.fsl_batch_stream.restype = _VP
    L.fsl_batch_destroy.argtypes = [_VP]
    L.fsl_batch_destroy.restype = None
    L.fsl_server_config_defaults.argtypes = [ctypes.POINTER(ServerConfig)]
    L.fsl_server_config_defaults.restype = None
    L.fsl_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(_VP)]
    L.fsl_server_submit.argtypes = [_VP, ctypes.POINTER(Config), ctypes.c_int64, _D, ctypes.c_int64,
                                    ctypes.POINTER(ctypes.c_int64)]
    L.fsl_server_poll.argtypes = [_VP, ctypes.c_int64, ctypes.POINTER(RequestInfo)]
    L.fsl_server_wait.argtypes = [_VP, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(RequestInfo)]
    L.fsl_server_result.argtypes = [_VP, ctypes.c_int64, _D, _D]
    L.fsl_server_get_stats.argtypes = [_VP, ctypes.POINTER(ServerStats)]
    L.fsl_server_destroy.argtypes = [_VP]
    L.fsl_server_destroy.restype = None
    if path is None:
        _lib = L
    return L


def check(rc):
    if rc != FSL_OK:
        msg = load().fsl_last_error()
        raise FslError(rc, msg.decode() if msg else "")
    return rc


def last_error():
    m = load().fsl_last_error()
    return m.decode() if m else ""
