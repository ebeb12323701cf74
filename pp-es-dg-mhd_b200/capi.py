"""ctypes binding of the C ABI in include/mhd_gpu.h (libmhd_gpu.so, built in-tree).

There is no fallback: if the shared library is missing or cannot be loaded this module raises,
and every solver call goes through the CUDA kernels.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmhd_gpu.so")

MHD_OK = 0
MHD_FLAG_NEG_AVG = 1
MHD_FLAG_PP_RELIMIT = 2
MHD_FLAG_DT_COLLAPSE = 4
MHD_FLAG_INIT_NEG_AVG = 8
MHD_FLAG_DEVICE_WAIT = 16

IC_OT2PI, IC_OT_UNIT, IC_VORTEX, IC_BLAST, IC_ROTOR, IC_ALFVEN, IC_CLOUD_SHOCK, IC_JET = range(8)
MHD_ERR_INVALID = -1
MHD_ERR_UNSUPPORTED = -2
MHD_ERR_CUDA = -3
MHD_ERR_NO_DEVICE = -4
MHD_ERR_STATE = -5

BC_PERIODIC, BC_EXTRAPOLATE, BC_FIXED, BC_XEXTRAP_YPER, BC_CLOUD_SHOCK, BC_JET = 0, 1, 2, 3, 4, 5


class Status(C.Structure):
    """mhd_gpu_status"""
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("dt_lim", C.c_double),
                ("tot_ent", C.c_double), ("steps", C.c_longlong), ("retries", C.c_longlong),
                ("num_negcell_total", C.c_longlong), ("num_negcell_last", C.c_int),
                ("done", C.c_int), ("flags", C.c_int), ("pad_", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


class LogEntry(C.Structure):
    """mhd_log_entry"""
    _fields_ = [("seq", C.c_longlong), ("step", C.c_longlong), ("kind", C.c_int), ("stage", C.c_int),
                ("try_num", C.c_int), ("num_negcell", C.c_int), ("neg_avg", C.c_int), ("flags", C.c_int),
                ("t", C.c_double), ("dt", C.c_double), ("dt_lim", C.c_double), ("tot_ent", C.c_double),
                ("rho_min", C.c_double), ("p_min", C.c_double), ("total", C.c_double * 8)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "total"}
        d["total"] = list(self.total)
        return d


LOG_STAGE, LOG_STEP = 1, 2


class Request(C.Structure):
    """mhd_request"""
    _fields_ = [("id", C.c_longlong), ("nx", C.c_int), ("ny", C.c_int), ("p", C.c_int),
                ("rknstg", C.c_int), ("left", C.c_double), ("right", C.c_double),
                ("bottom", C.c_double), ("top", C.c_double), ("gamma", C.c_double),
                ("bc_kind", C.c_int), ("pad_", C.c_int), ("bc_state8", C.c_double * 8),
                ("final_T", C.c_double), ("cfl", C.c_double), ("use_oedg", C.c_int),
                ("use_ldf", C.c_int), ("ent_offset", C.c_int), ("pad2_", C.c_int),
                ("arrival", C.c_double), ("u0", C.c_void_p), ("u_avg_out", C.c_void_p)]


class RequestResult(C.Structure):
    """mhd_request_result"""
    _fields_ = [("id", C.c_longlong), ("arrival", C.c_double), ("admitted", C.c_double),
                ("finished", C.c_double), ("t", C.c_double), ("steps", C.c_longlong),
                ("retries", C.c_longlong), ("done", C.c_int), ("flags", C.c_int),
                ("error", C.c_int), ("pad_", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


class ServerStats(C.Structure):
    """mhd_server_stats"""
    _fields_ = [("rounds", C.c_longlong), ("admitted", C.c_longlong), ("retired", C.c_longlong),
                ("graph_captures", C.c_longlong), ("admit_s", C.c_double), ("launch_s", C.c_double),
                ("wait_s", C.c_double), ("retire_s", C.c_double), ("idle_s", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p

# name -> (restype, argtypes); exactly the functions declared in include/mhd_gpu.h
SIGNATURES = {
    "mhd_gpu_create": (C.c_int, [C.c_int] * 5 + [C.c_double] * 5 + [C.c_int, _dp, C.POINTER(_vp)]),
    "mhd_gpu_destroy": (C.c_int, [_vp]),
    "mhd_gpu_set_stream": (C.c_int, [_vp, _vp]),
    "mhd_gpu_device_bytes": (C.c_int, [_vp, C.POINTER(C.c_size_t)]),
    "mhd_gpu_synchronize": (C.c_int, [_vp]),
    "mhd_gpu_status_string": (C.c_char_p, [C.c_int]),
    "mhd_gpu_nodes": (C.c_int, [_vp, _dp, _dp]),
    "mhd_gpu_gll_tables": (C.c_int, [C.c_int] + [_dp] * 7),
    "mhd_gpu_ldf_operator": (C.c_int, [C.c_int, C.c_double, C.c_double, _dp]),
    "mhd_gpu_upload_state": (C.c_int, [_vp, C.c_int, _dp]),
    "mhd_gpu_download_state": (C.c_int, [_vp, C.c_int, _dp]),
    "mhd_gpu_upload_ut": (C.c_int, [_vp, C.c_int, _dp]),
    "mhd_gpu_download_ut": (C.c_int, [_vp, C.c_int, _dp]),
    "mhd_gpu_download_avg": (C.c_int, [_vp, _dp]),
    "mhd_gpu_apply_bc": (C.c_int, [_vp, C.c_int]),
    "mhd_gpu_post_process": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                       _ip, _ip, _dp]),
    "mhd_gpu_semidiscretize": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
    "mhd_gpu_rk_combine": (C.c_int, [_vp, C.c_int, C.c_double]),
    "mhd_gpu_rk_accept": (C.c_int, [_vp]),
    "mhd_gpu_solve_begin": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _dp]),
    "mhd_gpu_step": (C.c_int, [_vp, C.POINTER(Status)]),
    "mhd_gpu_advance": (C.c_int, [_vp, C.c_longlong, C.c_int, C.POINTER(Status)]),
    "mhd_gpu_get_status": (C.c_int, [_vp, C.POINTER(Status)]),
    "mhd_gpu_state_device_ptr": (C.c_int, [_vp, C.c_int, C.POINTER(_dp)]),
    "mhd_gpu_step_graph_kernels": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "mhd_batch_create": (C.c_int, [C.POINTER(_vp)]),
    "mhd_batch_destroy": (C.c_int, [_vp]),
    "mhd_batch_add": (C.c_int, [_vp, _vp]),
    "mhd_batch_remove": (C.c_int, [_vp, _vp]),
    "mhd_batch_size": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "mhd_batch_advance": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    "mhd_batch_launch": (C.c_int, [_vp, C.c_int]),
    "mhd_batch_wait": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "mhd_batch_member_status": (C.c_int, [_vp, _vp, C.POINTER(Status)]),
    "mhd_gpu_footprint": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
    "mhd_server_create": (C.c_int, [C.c_size_t, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "mhd_server_submit": (C.c_int, [_vp, C.POINTER(Request)]),
    "mhd_server_run": (C.c_int, [_vp, C.c_double]),
    "mhd_server_pending": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
    "mhd_server_results": (C.c_int, [_vp, C.POINTER(RequestResult), C.c_int, C.POINTER(C.c_int)]),
    "mhd_server_get_stats": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "mhd_server_destroy": (C.c_int, [_vp]),
    "mhd_gpu_download_avg_primitive": (C.c_int, [_vp, C.POINTER(C.c_float), _dp, _dp]),
    "mhd_gpu_init_problem": (C.c_int, [_vp, C.c_int, _dp, C.c_int]),
    "mhd_gpu_set_log": (C.c_int, [_vp, C.c_int, C.c_int]),
    "mhd_gpu_read_log": (C.c_int, [_vp, C.POINTER(LogEntry), C.c_int, C.POINTER(C.c_int),
                                   C.POINTER(C.c_longlong)]),
    "mhd_gpu_semidiscretize_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                                 C.c_double, _vp, _vp, _dp, _vp]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libmhd_gpu.so (raises if it is missing: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libmhd_gpu.so not built ({path}); run pp-es-dg-mhd_b200/build.py")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if a declared symbol is not exported
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(code: int) -> str:
    return load().mhd_gpu_status_string(int(code)).decode()


class MHDError(RuntimeError):
    """A C-ABI call returned an API error (< 0) or a fatal solver flag."""

    def __init__(self, fn, code):
        self.code = code
        super().__init__(f"{fn} failed: {code} ({status_string(code)})")
