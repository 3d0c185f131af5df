"""ctypes binding of include/ssim2b200.h (libssim2b200.so)."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(HERE, "libssim2b200.so")

if not os.path.exists(library_path):
    raise ImportError(
        "libssim2b200.so is not built (run `python turbo-metrics_b200/build.py`); "
        "the SSIMULACRA2 engine has no CPU fallback")

lib = ctypes.CDLL(library_path)

NUM_STATS = 108

S2_OK = 0
S2_ERR_OOM = 1
S2_ERR_INVALID_SIZE = 2
S2_ERR_DIM_MISMATCH = 3
S2_ERR_NO_REFERENCE = 4
S2_ERR_CUDA = 5
S2_ERR_TIMEOUT = 6
S2_ERR_BUSY = 7
S2_ERR_INVALID_ARG = 8
S2_ERR_NOT_READY = 9
S2_ERR_CANCELLED = 10

BLUR = {"fir": 0, "iir_ref": 1}
STORAGE = {"f32": 0, "f16": 1, "bf16": 2}
SCALE_RULE = {"cpu": 0, "min8": 1, "all6": 2}
FMT = {"linear_f32": 0, "srgb8": 1, "nv12": 2, "rgb16": 3, "p016": 4}
MATRIX = {"bt709": 0, "bt601_525": 1, "bt601_625": 2}
RANGE = {"limited": 0, "full": 1}


class S2Error(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = lib.s2_status_string(status).decode()
        detail = lib.s2_last_error().decode()
        super().__init__(f"{what}: {msg}" + (f" ({detail})" if detail else ""))


class OutOfMemory(S2Error):
    pass


class InvalidImageSize(S2Error):
    pass


class DimensionMismatch(S2Error):
    pass


class NoCachedReference(S2Error):
    pass


class InvalidArgument(S2Error):
    """A NULL pointer, an unknown enum value or a bad pitch (S2_ERR_INVALID_ARG)."""
    pass


class Busy(S2Error):
    """The server holds its maximum of unfinished jobs (S2_ERR_BUSY)."""
    pass


class Timeout(S2Error):
    """A bounded device-side wait ran out (S2_ERR_TIMEOUT)."""
    pass


_ERRS = {S2_ERR_OOM: OutOfMemory, S2_ERR_INVALID_SIZE: InvalidImageSize,
         S2_ERR_DIM_MISMATCH: DimensionMismatch, S2_ERR_NO_REFERENCE: NoCachedReference, S2_ERR_BUSY: Busy,
         S2_ERR_INVALID_ARG: InvalidArgument, S2_ERR_TIMEOUT: Timeout}


def check(status, what=""):
    if status != S2_OK:
        raise _ERRS.get(status, S2Error)(status, what)


class Config(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("device", ctypes.c_int32), ("blur", ctypes.c_int32),
                ("storage", ctypes.c_int32), ("scale_rule", ctypes.c_int32), ("strip_rows", ctypes.c_int32),
                ("hbm_budget", ctypes.c_uint64)]


class Result(ctypes.Structure):
    _fields_ = [("score", ctypes.c_double), ("stats", ctypes.c_double * NUM_STATS),
                ("sums", ctypes.c_double * NUM_STATS), ("n_scales", ctypes.c_int32), ("status", ctypes.c_int32),
                ("dssim", ctypes.c_double), ("dssim_scale", ctypes.c_double * 5)]


METRIC = {"ssimulacra2": 1, "dssim": 2}


def metrics_mask(metrics):
    """'ssimulacra2', 'dssim' or an iterable of them -> S2_METRIC_* bits."""
    if isinstance(metrics, str):
        metrics = (metrics,)
    m = 0
    for name in metrics:
        m |= METRIC[name]
    return m


class PairDescC(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("format", ctypes.c_int32),
                ("bits", ctypes.c_int32), ("ref", ctypes.c_void_p), ("dis", ctypes.c_void_p),
                ("ref_uv", ctypes.c_void_p), ("dis_uv", ctypes.c_void_p), ("ref_pitch", ctypes.c_size_t),
                ("dis_pitch", ctypes.c_size_t), ("matrix", ctypes.c_int32), ("range", ctypes.c_int32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("device", ctypes.c_int32), ("max_batch_pairs", ctypes.c_uint32),
                ("max_batch_pixels", ctypes.c_uint64), ("hbm_budget", ctypes.c_uint64),
                ("max_queued_jobs", ctypes.c_uint32)]


class JobDesc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("format", ctypes.c_int32),
                ("ref", ctypes.c_void_p), ("ref_pitch", ctypes.c_size_t), ("n_candidates", ctypes.c_uint32),
                ("candidates", ctypes.POINTER(ctypes.c_void_p)), ("cand_pitch", ctypes.c_size_t)]


class ServerReport(ctypes.Structure):
    _fields_ = [("jobs_done", ctypes.c_uint64), ("pairs_done", ctypes.c_uint64), ("rounds", ctypes.c_uint64),
                ("queued_jobs", ctypes.c_uint64), ("hbm_in_use", ctypes.c_uint64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("uptime_s", ctypes.c_double),
                ("gpu_busy_s", ctypes.c_double), ("worker_wait_s", ctypes.c_double),
                ("worker_upload_s", ctypes.c_double), ("worker_submit_s", ctypes.c_double),
                ("copy_busy_s", ctypes.c_double), ("bytes_uploaded", ctypes.c_uint64)]


P = ctypes.c_void_p
D = ctypes.POINTER(ctypes.c_double)
_sig = {
    "s2_version": (ctypes.c_char_p, []),
    "s2_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "s2_last_error": (ctypes.c_char_p, []),
    "s2_config_default": (None, [ctypes.POINTER(Config)]),
    "s2_num_scales": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32]),
    "s2_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(P)]),
    "s2_destroy": (None, [P]),
    "s2_mem_usage": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_size_t)]),
    "s2_dimensions": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "s2_compute_linear_f32": (ctypes.c_int, [P, P, ctypes.c_size_t, P, ctypes.c_size_t, P]),
    "s2_compute_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_int32, P]),
    "s2_compute_nv12": (ctypes.c_int, [P, P, P, ctypes.c_size_t, P, P, ctypes.c_size_t, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_int32, P]),
    "s2_compute_p016": (ctypes.c_int, [P, P, P, ctypes.c_size_t, P, P, ctypes.c_size_t, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_int32, P]),
    "s2_compute_rgb16": (ctypes.c_int, [P, P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_int32,
                                        ctypes.c_int32, P]),
    "s2_get_result": (ctypes.c_int, [P, D, D, D]),
    "s2_compute_sync_linear_f32": (ctypes.c_int, [P, P, ctypes.c_size_t, P, ctypes.c_size_t, P, D]),
    "s2_set_reference_linear_f32": (ctypes.c_int, [P, P, ctypes.c_size_t, P]),
    "s2_set_reference_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, ctypes.c_int32, P]),
    "s2_compute_with_reference_linear_f32": (ctypes.c_int, [P, P, ctypes.c_size_t, P]),
    "s2_compute_with_reference_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, ctypes.c_int32, P]),
    "s2_clear_reference": (ctypes.c_int, [P]),
    "s2_has_reference": (ctypes.c_int32, [P]),
    "s2_batch_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(P)]),
    "s2_batch_destroy": (None, [P]),
    "s2_batch_submit": (ctypes.c_int, [P, ctypes.POINTER(PairDescC), ctypes.c_uint32, P]),
    "s2_batch_submit_host": (ctypes.c_int, [P, ctypes.POINTER(PairDescC), ctypes.c_uint32, P]),
    "s2_set_graphs": (ctypes.c_int, [P, ctypes.c_int32]),
    "s2_error_maps": (ctypes.c_int, [P, ctypes.c_int32, P, ctypes.c_size_t, P]),
    "s2_batch_results": (ctypes.c_int, [P, ctypes.POINTER(Result), ctypes.c_uint32]),
    "s2_batch_mem_usage": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_size_t)]),
    "s2_batch_set_graphs": (ctypes.c_int, [P, ctypes.c_int32]),
    "s2_profile_enable": (ctypes.c_int, [P, ctypes.c_int32]),
    "s2_profile_last": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_float)]),
    "s2_batch_set_profiling": (ctypes.c_int, [P, ctypes.c_int32]),
    "s2_batch_last_timings": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_float)]),
    "s2_fused_blocks_per_sm": (ctypes.c_int32, [ctypes.c_int32]),
    "s2_debug_tile_timeout": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int64]),
    "s2_server_config_default": (None, [ctypes.POINTER(ServerConfig)]),
    "s2_server_create": (ctypes.c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(P)]),
    "s2_server_destroy": (None, [P]),
    "s2_server_submit": (ctypes.c_int, [P, ctypes.POINTER(JobDesc), ctypes.POINTER(ctypes.c_uint64)]),
    "s2_server_wait": (ctypes.c_int, [P, ctypes.c_uint64, ctypes.c_uint32, D, ctypes.POINTER(ctypes.c_int32), D]),
    "s2_server_cancel": (ctypes.c_int, [P, ctypes.c_uint64]),
    "s2_server_stats": (ctypes.c_int, [P, ctypes.POINTER(ServerReport)]),
    "s2_server_reset_stats": (ctypes.c_int, [P]),
    "s2_compute_srgb8_noalloc": (ctypes.c_int, [P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_uint32,
                                                ctypes.c_uint32, P, P]),
    "s2_set_metrics": (ctypes.c_int, [P, ctypes.c_int32]),
    "s2_batch_set_metrics": (ctypes.c_int, [P, ctypes.c_int32]),
    "s2_get_dssim": (ctypes.c_int, [P, D, D]),
    "s2_batch_last_dssim_ms": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_float)]),
    "s2_dssim_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(P)]),
    "s2_dssim_destroy": (None, [P]),
    "s2_dssim_compute_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_int32, P, D]),
    "s2_dssim_compute_dis_only_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, ctypes.c_int32, P, D]),
    "s2_dssim_mem_usage": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_size_t)]),
    "s2_zensim_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(P)]),
    "s2_zensim_destroy": (None, [P]),
    "s2_zensim_set_reference_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, ctypes.c_int32, P]),
    "s2_zensim_compute_with_reference_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, ctypes.c_int32, P, D,
                                                              ctypes.POINTER(ctypes.c_int32)]),
    "s2_zensim_compute_features_srgb8": (ctypes.c_int, [P, P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_int32,
                                                        P, D, ctypes.POINTER(ctypes.c_int32)]),
    "s2_zensim_has_reference": (ctypes.c_int32, [P]),
    "s2_zensim_clear_reference": (ctypes.c_int, [P]),
    "s2_zensim_raw": (ctypes.c_int, [P, D, ctypes.POINTER(ctypes.c_uint32)]),
    "s2_zensim_mem_usage": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_size_t)]),
}
for _name, (_res, _args) in _sig.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def version():
    return lib.s2_version().decode()


def num_scales(width, height, rule="cpu"):
    return lib.s2_num_scales(width, height, SCALE_RULE[rule])


def make_config(device=0, blur="fir", storage="f32", scale_rule="cpu", strip_rows=0, hbm_budget=0):
    cfg = Config()
    lib.s2_config_default(ctypes.byref(cfg))
    cfg.device = device
    cfg.blur = BLUR[blur]
    cfg.storage = STORAGE[storage]
    cfg.scale_rule = SCALE_RULE[scale_rule]
    cfg.strip_rows = strip_rows
    cfg.hbm_budget = hbm_budget
    return cfg
