"""ctypes binding of libcqfock.so (declarations in include/cqfock.h).

The library is the only compute path: if it is missing or fails to load this
module raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcqfock.so")

CQF_OK, CQF_EINVAL, CQF_ENOMEM, CQF_ECUDA, CQF_ENOTSUP, CQF_ETIMEDOUT, \
    CQF_ENODEV = range(7)
CQF_COULOMB, CQF_EXCHANGE = 0, 1
CQF_FP64, CQF_MIXED = 0, 1

# every entry point declared in include/cqfock.h
EXPORTS = ("cqf_opts_default", "cqf_basis_create", "cqf_basis_destroy",
           "cqf_basis_info", "cqf_basis_schwarz", "cqf_basis_one_electron",
           "cqf_basis_nuclear", "cqf_basis_nuclear_pvp",
           "cqf_four_comp_core_hamiltonian",
           "cqf_two_body_contract", "cqf_two_body_contract_noalloc", "cqf_autotune",
           "cqf_graph_create", "cqf_graph_launch", "cqf_graph_destroy",
           "cqf_rel_two_body_contract", "cqf_dc_opts_default",
           "cqf_four_comp_gd", "cqf_grad_two_body_contract",
           "cqf_server_opts_default", "cqf_fock_footprint",
           "cqf_server_create", "cqf_server_submit", "cqf_server_wait",
           "cqf_server_get_stats", "cqf_server_destroy", "cqf_last_error")
# cqf_rel_comp / cqf_rel_type (DIRAC_PAULI_SPINOR_COMP order)
(CQF_CLLMS, CQF_XLLMS, CQF_XLLMX, CQF_XLLMY, CQF_XLLMZ, CQF_CSSMS, CQF_CSSMX,
 CQF_CSSMY, CQF_CSSMZ, CQF_XSSMS, CQF_XSSMX, CQF_XSSMY, CQF_XSSMZ, CQF_XLSMS,
 CQF_XLSMX, CQF_XLSMY, CQF_XLSMZ, CQF_REL_NMAT) = range(18)
# the GAUNT list continues with LS Coulomb, SL Coulomb and SL exchange
(CQF_CLSMS, CQF_CLSMX, CQF_CLSMY, CQF_CLSMZ, CQF_CSLMS, CQF_CSLMX, CQF_CSLMY,
 CQF_CSLMZ, CQF_XSLMS, CQF_XSLMX, CQF_XSLMY, CQF_XSLMZ,
 CQF_REL_NMAT_GAUNT) = range(17, 30)
CQF_REL_BARE_COULOMB, CQF_REL_LLSS, CQF_REL_SSSS, CQF_REL_GAUNT, CQF_REL_GAUGE = range(5)
NOALLOC_SCRATCH_BYTES = 32 * 1024 * 1024


class CqfShell(C.Structure):
    _fields_ = [("l", C.c_int), ("pure", C.c_int), ("nprim", C.c_int),
                ("alpha", C.POINTER(C.c_double)),
                ("coeff", C.POINTER(C.c_double)),
                ("origin", C.c_double * 3)]


class CqfContraction(C.Structure):
    _fields_ = [("X", C.c_void_p), ("AX", C.c_void_p),
                ("hermitian", C.c_int), ("type", C.c_int)]


class CqfOpts(C.Structure):
    _fields_ = [("is_complex", C.c_int), ("screen", C.c_int),
                ("device_pointers", C.c_int), ("precision", C.c_int),
                ("fp32_cutoff", C.c_double), ("stream", C.c_void_p),
                ("shard_index", C.c_int), ("shard_count", C.c_int)]


class CqfStats(C.Structure):
    _fields_ = [("quartets_total", C.c_longlong),
                ("quartets_screened", C.c_longlong),
                ("quartets_fp32", C.c_longlong),
                ("quartets_fp64", C.c_longlong),
                ("device_ms", C.c_double)]


class CqfDcOpts(C.Structure):
    _fields_ = [("bare_coulomb", C.c_int), ("dirac_coulomb", C.c_int),
                ("dirac_coulomb_ssss", C.c_int), ("libcint", C.c_int),
                ("xHFX", C.c_double), ("gaunt", C.c_int), ("gauge", C.c_int)]


class CqfServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int),
                ("mem_budget", C.c_ulonglong), ("cache_entries", C.c_int)]


class CqfFockRequest(C.Structure):
    _fields_ = [("shells", C.POINTER(CqfShell)), ("nshell", C.c_int),
                ("thresh_schwarz", C.c_double), ("D", C.POINTER(C.c_double)),
                ("G", C.POINTER(C.c_double)), ("xHFX", C.c_double),
                ("precision", C.c_int), ("fp32_cutoff", C.c_double)]


class CqfRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("queue_ms", C.c_double),
                ("setup_ms", C.c_double), ("build_ms", C.c_double),
                ("latency_ms", C.c_double)]


class CqfServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("failed", C.c_longlong), ("peak_inflight", C.c_int),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double)]


class CqfError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("cqfock error %d: %s" % (status, msg))
        self.status = status


_lib = None


def lib():
    """Load libcqfock.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libcqfock.so not built (%s); run python -m "
            "chronusq_public_b200.build" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    L.cqf_opts_default.argtypes = [C.POINTER(CqfOpts)]
    L.cqf_opts_default.restype = None
    L.cqf_basis_create.argtypes = [C.POINTER(CqfShell), C.c_int, C.c_double,
                                   C.c_int, C.POINTER(C.c_void_p)]
    L.cqf_basis_create.restype = C.c_int
    L.cqf_basis_destroy.argtypes = [C.c_void_p]
    L.cqf_basis_destroy.restype = C.c_int
    L.cqf_basis_info.argtypes = [C.c_void_p, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.cqf_basis_info.restype = C.c_int
    L.cqf_basis_schwarz.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.cqf_basis_schwarz.restype = C.c_int
    L.cqf_basis_one_electron.argtypes = [C.c_void_p, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
    L.cqf_basis_one_electron.restype = C.c_int
    L.cqf_basis_nuclear.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]
    L.cqf_basis_nuclear.restype = C.c_int
    L.cqf_basis_nuclear_pvp.argtypes = L.cqf_basis_nuclear.argtypes
    L.cqf_basis_nuclear_pvp.restype = C.c_int
    L.cqf_four_comp_core_hamiltonian.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                                 C.POINTER(C.c_void_p)]
    L.cqf_four_comp_core_hamiltonian.restype = C.c_int
    L.cqf_two_body_contract.argtypes = [C.c_void_p, C.POINTER(CqfContraction),
                                        C.c_int, C.POINTER(CqfOpts),
                                        C.POINTER(CqfStats)]
    L.cqf_two_body_contract.restype = C.c_int
    L.cqf_autotune.argtypes = [C.c_void_p, C.POINTER(CqfContraction), C.c_int,
                               C.POINTER(CqfOpts), C.c_char_p, C.POINTER(C.c_int)]
    L.cqf_autotune.restype = C.c_int
    L.cqf_two_body_contract_noalloc.argtypes = L.cqf_two_body_contract.argtypes
    L.cqf_two_body_contract_noalloc.restype = C.c_int
    L.cqf_graph_create.argtypes = [C.c_void_p, C.POINTER(CqfContraction), C.c_int,
                                   C.POINTER(CqfOpts), C.POINTER(C.c_void_p)]
    L.cqf_graph_create.restype = C.c_int
    L.cqf_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
    L.cqf_graph_launch.restype = C.c_int
    L.cqf_graph_destroy.argtypes = [C.c_void_p]
    L.cqf_graph_destroy.restype = C.c_int
    L.cqf_rel_two_body_contract.argtypes = [
        C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int,
        C.c_int, C.POINTER(CqfOpts), C.POINTER(CqfStats)]
    L.cqf_rel_two_body_contract.restype = C.c_int
    L.cqf_dc_opts_default.argtypes = [C.POINTER(CqfDcOpts)]
    L.cqf_dc_opts_default.restype = None
    L.cqf_four_comp_gd.argtypes = [
        C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
        C.POINTER(CqfDcOpts), C.POINTER(CqfOpts), C.POINTER(CqfStats)]
    L.cqf_four_comp_gd.restype = C.c_int
    L.cqf_grad_two_body_contract.argtypes = [
        C.c_void_p, C.POINTER(C.c_int), C.c_int, C.POINTER(CqfContraction), C.c_int,
        C.POINTER(C.c_void_p), C.POINTER(CqfOpts), C.POINTER(CqfStats)]
    L.cqf_grad_two_body_contract.restype = C.c_int
    L.cqf_server_opts_default.argtypes = [C.POINTER(CqfServerOpts)]
    L.cqf_server_opts_default.restype = None
    L.cqf_fock_footprint.argtypes = [C.POINTER(CqfShell), C.c_int]
    L.cqf_fock_footprint.restype = C.c_ulonglong
    L.cqf_server_create.argtypes = [C.POINTER(CqfServerOpts), C.POINTER(C.c_void_p)]
    L.cqf_server_create.restype = C.c_int
    L.cqf_server_submit.argtypes = [C.c_void_p, C.POINTER(CqfFockRequest),
                                    C.POINTER(C.c_longlong)]
    L.cqf_server_submit.restype = C.c_int
    L.cqf_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double,
                                  C.POINTER(CqfRequestInfo)]
    L.cqf_server_wait.restype = C.c_int
    L.cqf_server_get_stats.argtypes = [C.c_void_p, C.POINTER(CqfServerStats)]
    L.cqf_server_get_stats.restype = C.c_int
    L.cqf_server_destroy.argtypes = [C.c_void_p]
    L.cqf_server_destroy.restype = C.c_int
    L.cqf_last_error.argtypes = []
    L.cqf_last_error.restype = C.c_char_p
    _lib = L
    return L


def check(status):
    if status != CQF_OK:
        raise CqfError(status, lib().cqf_last_error().decode())
    return status
