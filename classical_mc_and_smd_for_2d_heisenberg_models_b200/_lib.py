"""ctypes binding of libsmd_b200.so (the C ABI declared in include/smd_b200.h).

The library is built in-tree (``csrc/Makefile``) and loaded from this
package folder.  There is no fallback: if the library is missing the import
fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsmd_b200.so")

SMD_OK, SMD_EINVAL, SMD_ENOMEM_ADMIT, SMD_ECUDA = 0, 1, 2, 3
SMD_ETIMEOUT, SMD_ECANCELLED, SMD_ENOTFOUND, SMD_EBUSY = 4, 5, 6, 7
SMD_FP64, SMD_FP32 = 0, 1
GEOMS = {"square": 0, "triang": 1, "hexagn": 2, "kagome": 3, "lieb": 4}

STATUS_NAMES = {0: "SMD_OK", 1: "SMD_EINVAL", 2: "SMD_ENOMEM_ADMIT", 3: "SMD_ECUDA",
                4: "SMD_ETIMEOUT", 5: "SMD_ECANCELLED", 6: "SMD_ENOTFOUND", 7: "SMD_EBUSY"}

# Every entry point of include/smd_b200.h, in declaration order.
EXPORTS = [
    "smd_ctx_create", "smd_ctx_destroy", "smd_last_error", "smd_version",
    "smd_geometry_info", "smd_build_lattice", "smd_build_bonds", "smd_window",
    "smd_lattice_upload", "smd_lattice_free", "smd_qset_upload", "smd_qset_size",
    "smd_lattice_sites", "smd_run", "smd_run_device", "smd_dyn_spectrum_ref",
    "smd_static_prepass", "smd_evolve", "smd_batch_create", "smd_batch_info", "smd_batch_run",
    "smd_batch_run_device", "smd_batch_free", "smd_submit", "smd_poll", "smd_wait", "smd_cancel",
    "smd_job_info",
    "smd_serve_shutdown", "smd_mc_run", "smd_mc_colouring", "smd_evolve_fp64_noalloc",
    "smd_measure_fma_peak",
]


class SMDError(RuntimeError):
    def __init__(self, code: int, msg: str = ""):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class DeviceOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget", C.c_size_t)]


class LatticeDesc(C.Structure):
    _fields_ = [("N", C.c_int), ("zn", C.c_int * 3), ("nbr", C.c_void_p * 3),
                ("shell_on", C.c_int * 3), ("J", C.c_double * 12),
                ("lambda_", C.c_double * 9), ("lieb_delta_on", C.c_int),
                ("j2_delta", C.c_double), ("h", C.c_double), ("nbonds", C.c_int * 3),
                ("bonds", C.c_void_p), ("G", C.c_int), ("grid_map", C.c_void_p),
                ("pos", C.c_void_p)]


class JobDesc(C.Structure):
    _fields_ = [("lattice", C.c_int), ("qset", C.c_int), ("n_samples", C.c_int),
                ("dt", C.c_double), ("n_rec", C.c_int), ("stride", C.c_int),
                ("precision", C.c_int), ("fix_every", C.c_int), ("imp", C.c_void_p)]


class BatchMember(C.Structure):
    _fields_ = [("lattice", C.c_int), ("qset", C.c_int), ("n_samples", C.c_int),
                ("imp", C.c_void_p)]


class BatchDesc(C.Structure):
    _fields_ = [("n_members", C.c_int), ("members", C.POINTER(BatchMember)), ("dt", C.c_double),
                ("n_rec", C.c_int), ("stride", C.c_int), ("precision", C.c_int),
                ("fix_every", C.c_int)]


class BatchTuning(C.Structure):
    _fields_ = [("cluster_ctas", C.c_int), ("sites_per_thread", C.c_int), ("threads", C.c_int),
                ("edge_slots", C.c_int), ("records_per_launch", C.c_int), ("clusters", C.c_int),
                ("items", C.c_int), ("candidates", C.c_int), ("probe_ms", C.c_double),
                ("member_ctas", C.c_int * 24)]


class NoAllocModel(C.Structure):
    _fields_ = [("N", C.c_int), ("zn", C.c_int * 3), ("d_nbr", C.c_void_p),
                ("J", C.c_double * 3), ("lambda_", C.c_double * 9), ("h", C.c_double)]


NOALLOC_SCRATCH_BYTES = 16 << 20


class MCDesc(C.Structure):
    _fields_ = [("lattice", C.c_int), ("n_temps", C.c_int), ("temps", C.POINTER(C.c_double)),
                ("chains", C.c_int), ("n_therm", C.c_int), ("n_meas", C.c_int),
                ("cr_skip", C.c_int), ("pt", C.c_int), ("n_micro", C.c_int),
                ("n_canon", C.c_int), ("n_micro2", C.c_int), ("n_canon2", C.c_int),
                ("seed", C.c_ulonglong), ("imp", C.POINTER(C.c_int))]


class Report(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_h2d", C.c_double), ("ms_d2h", C.c_double),
                ("site_steps", C.c_double), ("drift_max", C.c_double),
                ("drift_final", C.c_double), ("waves", C.c_int),
                ("kernel_launches", C.c_int), ("ms_device", C.c_double), ("ms_rk", C.c_double),
                ("ms_proj", C.c_double), ("ms_tfft", C.c_double), ("rk_launches", C.c_int),
                ("rk_kind", C.c_int), ("rk_ctas", C.c_int)]


_lib = None


def load():
    """Load libsmd_b200.so; raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          f"`make -C {os.path.join(HERE, 'csrc')}` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.smd_ctx_create.argtypes = [C.POINTER(DeviceOpts), C.POINTER(vp)]
    L.smd_ctx_destroy.argtypes = [vp]
    L.smd_last_error.argtypes = [vp]
    L.smd_last_error.restype = C.c_char_p
    L.smd_version.restype = C.c_char_p
    L.smd_geometry_info.argtypes = [C.c_int, C.c_int, ip, ip, ip, ip]
    L.smd_build_lattice.argtypes = [C.c_int, C.c_int, dp, ip, ip, ip, ip]
    L.smd_build_bonds.argtypes = [C.c_int, ip, ip, ip, ip, C.c_int, C.c_int, ip, C.c_int, ip]
    L.smd_window.argtypes = [C.c_char_p, C.c_int, dp]
    L.smd_lattice_upload.argtypes = [vp, C.POINTER(LatticeDesc), ip]
    L.smd_lattice_free.argtypes = [vp, C.c_int]
    L.smd_qset_upload.argtypes = [vp, C.c_int, C.c_int, C.c_int, dp, C.c_double, ip]
    L.smd_qset_size.argtypes = [vp, C.c_int, ip]
    L.smd_lattice_sites.argtypes = [vp, C.c_int, ip]
    L.smd_run.argtypes = [vp, C.POINTER(JobDesc), dp, dp, dp, dp, dp, C.POINTER(Report)]
    L.smd_run_device.argtypes = [vp, C.POINTER(JobDesc), vp, vp, vp, vp, vp, C.POINTER(Report)]
    L.smd_dyn_spectrum_ref.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_int, dp, dp, ip,
                                       dp, dp, dp, dp]
    L.smd_static_prepass.argtypes = [vp, C.c_int, C.c_int, C.c_int, dp, ip, dp,
                                     C.POINTER(C.c_longlong), dp]
    L.smd_evolve.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, ip,
                             dp, C.POINTER(Report)]
    L.smd_batch_create.argtypes = [vp, C.POINTER(BatchDesc), ip]
    L.smd_batch_info.argtypes = [vp, C.c_int, C.POINTER(BatchTuning)]
    L.smd_batch_run.argtypes = [vp, C.c_int, C.POINTER(dp), dp, C.POINTER(dp), C.POINTER(dp),
                                C.POINTER(Report)]
    L.smd_batch_run_device.argtypes = [vp, C.c_int, C.POINTER(vp), vp, C.POINTER(vp),
                                       C.POINTER(vp), C.POINTER(Report)]
    L.smd_batch_free.argtypes = [vp, C.c_int]
    L.smd_submit.argtypes = [vp, C.POINTER(JobDesc), dp, dp, dp, dp, C.POINTER(C.c_longlong)]
    L.smd_poll.argtypes = [vp, C.c_longlong, dp]
    L.smd_wait.argtypes = [vp, C.c_longlong, C.c_double, dp]
    L.smd_cancel.argtypes = [vp, C.c_longlong]
    L.smd_job_info.argtypes = [vp, C.c_longlong, C.POINTER(Report)]
    L.smd_serve_shutdown.argtypes = [vp]
    L.smd_serve_shutdown.restype = None
    L.smd_evolve_fp64_noalloc.argtypes = [C.POINTER(NoAllocModel), C.c_int, C.c_double, C.c_int,
                                          vp, vp, vp, vp]
    L.smd_measure_fma_peak.argtypes = [C.c_int, C.c_int, dp]
    L.smd_mc_run.argtypes = [vp, C.POINTER(MCDesc), dp, dp, dp, ip, C.POINTER(Report)]
    L.smd_mc_colouring.argtypes = [vp, C.c_int, ip, ip, ip]
    _lib = L
    return L
