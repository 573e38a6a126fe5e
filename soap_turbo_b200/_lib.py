"""Loads libsoapb200.so and declares its C ABI (include/soap_b200.h).

There is no fallback: if the library is missing or cannot be loaded, importing
the package's compute entry points raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsoapb200.so")

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p

SOAPB_OK = 0
ERRORS = {
    1: "SOAPB_ERR_ARGUMENT", 2: "SOAPB_ERR_ALPHA_TOO_LARGE", 3: "SOAPB_ERR_CONTRACT_STATE",
    4: "SOAPB_ERR_COMPRESS_MODE", 5: "SOAPB_ERR_BASIS", 6: "SOAPB_ERR_CUDA",
    7: "SOAPB_ERR_NO_DEVICE", 8: "SOAPB_ERR_INPUT", 9: "SOAPB_ERR_BASIS_MATRIX",
    10: "SOAPB_ERR_HESSIAN_STATE",
}
BASIS = {"poly3": 0, "poly3gauss": 1, "poly3operator": 2}
PREC_MIXED, PREC_FP64 = 0, 1
G_SITE_FASTEST, G_SOAP_FASTEST = 0, 1


class SoapError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class Hyper(C.Structure):
    _fields_ = [
        ("n_species", C.c_int32), ("l_max", C.c_int32), ("basis", C.c_int32),
        ("scaling_mode", C.c_int32), ("radial_enhancement", C.c_int32),
        ("legacy_filter_seed", C.c_int32), ("alpha_max", i32p),
        ("rcut_hard", f64p), ("rcut_soft", f64p), ("nf", f64p), ("global_scaling", f64p),
        ("atom_sigma_r", f64p), ("atom_sigma_r_scaling", f64p),
        ("atom_sigma_t", f64p), ("atom_sigma_t_scaling", f64p),
        ("amplitude_scaling", f64p), ("central_weight", f64p),
        ("compress", C.c_int32), ("P_nonzero", C.c_int32), ("P_i", i32p), ("P_j", i32p),
        ("P_el", f64p),
    ]


class Batch(C.Structure):
    _fields_ = [
        ("n_sites", C.c_int32), ("n_atom_pairs", C.c_int32),
        ("max_species_multiplicity", C.c_int32),
        ("n_neigh", C.c_void_p), ("species", C.c_void_p), ("species_multiplicity", C.c_void_p),
        ("mask", C.c_void_p), ("rjs", C.c_void_p), ("thetas", C.c_void_p), ("phis", C.c_void_p),
    ]


# every exported symbol of include/soap_b200.h with (restype, argtypes)
SIGNATURES = {
    "soapb_last_error": (C.c_char_p, []),
    "soapb_version": (C.c_char_p, []),
    # the drop-in calls take their host arrays as addresses (ndarray.ctypes.data):
    # per-call conversions dominate their Python overhead otherwise
    "soapb_get_soap": (C.c_int, [
        C.c_int32, vp, C.c_int32, vp, C.c_int32, vp, C.c_int32, vp, vp, vp, vp,
        vp, C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int32, vp,
        C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp,
        vp, C.c_int32, vp, C.c_int32]),
    "soapb_soap_contract": (C.c_int, [vp, vp, C.c_double, vp, C.c_int32, C.c_int32,
                                      C.c_int32]),
    "soapb_set_legacy_filter_seed": (C.c_int, [C.c_int32]),
    "soapb_get_legacy_filter_seed": (C.c_int, [i32p]),
    "soapb_set_soap_hessian_enabled": (C.c_int, [C.c_int32]),
    "soapb_get_soap_hessian_enabled": (C.c_int, [i32p]),
    "soapb_get_soap_central_hessian": (C.c_int, [
        C.c_int32, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, C.c_int32, vp, vp, vp, C.c_int32,
        C.c_int32, vp, vp, vp, vp, C.c_int32, C.c_int32, vp, vp]),
    "soapb_set_precision": (C.c_int, [C.c_int32]),
    "soapb_set_basis_matrices": (C.c_int, [C.c_int32, f64p, f64p]),
    "soapb_get_compress_indices": (C.c_int, [C.c_char_p, C.c_int32, i32p, C.c_int32, i32p, i32p,
                                             i32p, i32p, f64p, C.c_char_p]),
    "soapb_orthonormalization_matrix": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double,
                                                  f64p, f64p]),
    "soapb_create": (C.c_int, [C.POINTER(Hyper), C.c_int32, C.POINTER(C.c_void_p)]),
    "soapb_destroy": (C.c_int, [C.c_void_p]),
    "soapb_set_basis": (C.c_int, [C.c_void_p, f64p, f64p]),
    "soapb_get_basis": (C.c_int, [C.c_void_p, f64p, f64p]),
    "soapb_n_soap": (C.c_int, [C.c_void_p, i32p]),
    "soapb_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "soapb_set_threads_per_site": (C.c_int, [C.c_void_p, C.c_int32]),
    "soapb_descriptor": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_int32]),
    "soapb_contract": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_void_p, C.c_int32,
                                 C.c_double, C.c_void_p]),
    "soapb_descriptor_noalloc": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p]),
    "soapb_descriptor_and_vjp": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_int32,
                                           C.c_double, C.c_void_p, C.c_void_p]),
    "soapb_descriptor_fp64": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_void_p]),
    "soapb_contract_cart_der": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_void_p,
                                          C.c_int32, C.c_double, C.c_void_p]),
    "soapb_central_hessian": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_int32,
                                        C.c_void_p, C.c_void_p]),
    "soapb_autotune": (C.c_int, [C.c_void_p, C.POINTER(Batch), i32p]),
    "soapb_check_inputs": (C.c_int, [C.c_void_p, i64p]),
    "soapb_launch_count": (C.c_int, [C.c_void_p, i64p]),
    "soapb_build_neighbors": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, f64p, C.c_void_p,
                                        C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_double,
                                        C.POINTER(Batch), C.POINTER(C.c_void_p)]),
    "soapb_kernel_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "soapb_kernel_times": (C.c_int, [C.c_void_p, i64p, f64p, i64p]),
    "soapb_selftest_scan_wait": (C.c_int, [C.c_int32, C.c_int32, i64p]),
    "soapb_set_radial_tables": (C.c_int, [C.c_void_p, C.c_int32]),
    "soapb_radial_tables": (C.c_int, [C.c_void_p, i32p, f64p]),
    "soapb_set_tensor_cores": (C.c_int, [C.c_void_p, C.c_int32]),
}
KERNEL_KINDS = ("prep", "pair", "descriptor", "contract")

_lib = None


def load():
    """The loaded library; raises if it is absent (build it with build())."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`make -C soap_turbo_b200/csrc` (or __graft_entry__.build())")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(rc):
    if rc != SOAPB_OK:
        raise SoapError(rc, load().soapb_last_error().decode())
