"""The reference's host interface for the descriptor path, on the GPU.

``get_soap``, ``soap_contract`` and ``get_soap_central_hessian`` take the
arguments of soap_turbo's Fortran routines (src/soap_turbo.f90:139-169,
:1723-1730 and :1151-1160) in the same order, with
numpy arrays in the same (Fortran) shapes, and write their outputs in place
like the Fortran ``intent(inout)`` / ``intent(out)`` arguments.  They call the
drop-in layer of libsoapb200.so, which keeps the reference's module state:
the basis cache, ``legacy_filter_seed``, ``soap_hessian_enabled`` and the
contract and Hessian state.
"""
from __future__ import annotations

import numpy as np

from . import _lib

_i32 = np.int32
_f64 = np.float64


def _f(a, dtype):
    a = np.asarray(a, dtype=dtype)
    return np.asfortranarray(a)


def _p(a, t):
    return a.ctypes.data_as(t)


def _a(a):
    """The array's address, for the drop-in calls' void-pointer arguments."""
    return a.ctypes.data


def _per_species(v, n):
    if isinstance(v, (float, int)):
        return np.full(n, float(v))
    v = np.atleast_1d(np.asarray(v, dtype=_f64))
    if v.shape[0] == 1 and n > 1:
        v = np.repeat(v, n)
    if v.shape[0] != n:
        raise ValueError("per-species array has the wrong length")
    return np.ascontiguousarray(v)


def get_soap(n_sites, n_neigh, n_species, species, species_multiplicity, n_atom_pairs, mask, rjs,
             thetas, phis, alpha_max, l_max, rcut_hard, rcut_soft, nf, global_scaling,
             atom_sigma_r, atom_sigma_r_scaling, atom_sigma_t, atom_sigma_t_scaling,
             amplitude_scaling, radial_enhancement, central_weight, basis, scaling_mode,
             do_timing, do_derivatives, compress_soap, compress_P_nonzero, compress_P_i,
             compress_P_j, compress_P_el, soap, soap_cart_der, contract=False):
    """get_soap (src/soap_turbo.f90:139-169).

    Shapes as in Fortran: species (max_mult, n_sites), mask (n_atom_pairs,
    n_species), soap (n_soap, n_sites) and soap_cart_der (3, n_soap,
    n_atom_pairs), all Fortran-ordered float64 / int32 / bool arrays.  soap
    receives the normalised descriptor; soap_cart_der is written when
    do_derivatives and not contract (pass None otherwise).  As in the
    reference, a compressed soap is added into (the caller's values count in
    the norm) and the self columns of soap_cart_der are accumulated into, so
    callers pass both zeroed (src/soap_turbo.f90:798-802, 888-892)."""
    lib = _lib.load()
    if not (isinstance(soap, np.ndarray) and soap.dtype == _f64 and soap.flags.f_contiguous):
        raise TypeError("soap must be a Fortran-ordered float64 array (written in place)")
    species = _f(species, _i32)
    if species.ndim == 1:
        species = species.reshape(1, -1, order="F")
    mask_u8 = _f(mask, np.uint8)  # no copy when already uint8 and Fortran-ordered
    n_neigh = np.ascontiguousarray(n_neigh, dtype=_i32)
    species_multiplicity = np.ascontiguousarray(species_multiplicity, dtype=_i32)
    rjs = np.ascontiguousarray(rjs, dtype=_f64)
    thetas = np.ascontiguousarray(thetas, dtype=_f64)
    phis = np.ascontiguousarray(phis, dtype=_f64)
    alpha_max = np.ascontiguousarray(alpha_max, dtype=_i32)
    ps = [_per_species(v, n_species) for v in (rcut_hard, rcut_soft, nf, global_scaling,
                                               atom_sigma_r, atom_sigma_r_scaling, atom_sigma_t,
                                               atom_sigma_t_scaling, amplitude_scaling)]
    cw = _per_species(central_weight, n_species)
    if compress_soap:
        P_i = np.ascontiguousarray(compress_P_i, dtype=_i32)
        P_j = np.ascontiguousarray(compress_P_j, dtype=_i32)
        P_el = np.ascontiguousarray(compress_P_el, dtype=_f64)
    else:
        P_i = np.zeros(1, _i32)
        P_j = np.zeros(1, _i32)
        P_el = np.zeros(1, _f64)
    cart_ptr = None
    if soap_cart_der is not None:
        if not (soap_cart_der.dtype == _f64 and soap_cart_der.flags.f_contiguous):
            raise TypeError("soap_cart_der must be a Fortran-ordered float64 array")
        cart_ptr = _a(soap_cart_der)
    _lib.check(lib.soapb_get_soap(
        int(n_sites), _a(n_neigh), int(n_species), _a(species), int(species.shape[0]),
        _a(species_multiplicity), int(n_atom_pairs), _a(mask_u8), _a(rjs), _a(thetas), _a(phis),
        _a(alpha_max), int(l_max), *[_a(v) for v in ps[:9]], int(radial_enhancement), _a(cw),
        basis.encode(), scaling_mode.encode(), int(bool(do_timing)), int(bool(do_derivatives)),
        int(bool(compress_soap)), int(compress_P_nonzero), _a(P_i), _a(P_j), _a(P_el), _a(soap),
        int(soap.shape[0]), cart_ptr, int(bool(contract))))


def soap_contract(soap, G, sgn, pair):
    """soap_contract (src/soap_turbo.f90:1723-1730): soap (n_soap, n_sites), G
    (n_sites, n_soap), pair (3, n_pairs) written in place."""
    lib = _lib.load()
    soap = _f(soap, _f64)
    G = _f(G, _f64)
    if not (isinstance(pair, np.ndarray) and pair.dtype == _f64 and pair.flags.f_contiguous):
        raise TypeError("pair must be a Fortran-ordered float64 array (written in place)")
    _lib.check(lib.soapb_soap_contract(_a(soap), _a(G), float(sgn), _a(pair), int(soap.shape[1]),
                                       int(soap.shape[0]), int(pair.shape[1])))


def get_soap_central_hessian(n_sites, n_neigh, n_atom_pairs, n_species, mask, rjs, thetas, phis,
                             l_max, rcut_hard, atom_sigma_t, atom_sigma_t_scaling, compress_soap,
                             compress_P_nonzero, compress_P_i, compress_P_j, compress_P_el, soap,
                             n_vec, vecs, hess):
    """get_soap_central_hessian (src/soap_turbo.f90:1151-1160): soap (n_soap,
    n_sites) as get_soap returned it, vecs (n_soap, n_vec, n_sites), hess (3, 3,
    n_vec, n_atom_pairs) written in place: hess[a, b, v, k] = sum_d vecs[d, v, i]
    d^2 soap[d, i] / dr_ia dr_jb.  Follows a get_soap on the same batch with
    do_derivatives and soap_hessian_enabled set."""
    lib = _lib.load()
    soap = _f(soap, _f64)
    vecs = _f(vecs, _f64)
    if not (isinstance(hess, np.ndarray) and hess.dtype == _f64 and hess.flags.f_contiguous):
        raise TypeError("hess must be a Fortran-ordered float64 array (written in place)")
    if hess.size != 9 * int(n_vec) * int(n_atom_pairs) or vecs.size != soap.size * int(n_vec):
        raise ValueError("hess must be (3, 3, n_vec, n_atom_pairs) and vecs (n_soap, n_vec, n_sites)")
    _lib.check(lib.soapb_get_soap_central_hessian(
        int(n_sites), None, int(n_atom_pairs), int(n_species), None, None, None, None, int(l_max),
        None, None, None, int(bool(compress_soap)), int(compress_P_nonzero), None, None, None,
        _a(soap), int(soap.shape[0]), int(n_vec), _a(vecs), _a(hess)))


def set_soap_hessian_enabled(enabled: bool):
    """The reference's module flag soap_hessian_enabled (src/soap_turbo.f90:76)."""
    _lib.check(_lib.load().soapb_set_soap_hessian_enabled(int(bool(enabled))))


def get_soap_hessian_enabled() -> bool:
    import ctypes as C
    v = C.c_int32(0)
    _lib.check(_lib.load().soapb_get_soap_hessian_enabled(C.byref(v)))
    return bool(v.value)


def get_compress_indices(compress_mode, alpha_max, l_max, what_to_do="set_indices"):
    """get_compress_indices (src/soap_turbo_compress.f90:44): returns
    (dim, P_nonzero, P_i, P_j, P_el), the index arrays 1-based."""
    lib = _lib.load()
    am = np.ascontiguousarray(alpha_max, dtype=_i32)
    import ctypes as C
    dim = C.c_int32(0)
    nz = C.c_int32(0)
    _lib.check(lib.soapb_get_compress_indices(compress_mode.encode(), len(am), _p(am, _lib.i32p),
                                              int(l_max), C.byref(dim), C.byref(nz), None, None,
                                              None, b"get_dim"))
    if what_to_do == "get_dim":
        return dim.value, nz.value, None, None, None
    P_i = np.zeros(nz.value, _i32)
    P_j = np.zeros(nz.value, _i32)
    P_el = np.zeros(nz.value, _f64)
    _lib.check(lib.soapb_get_compress_indices(compress_mode.encode(), len(am), _p(am, _lib.i32p),
                                              int(l_max), C.byref(dim), C.byref(nz),
                                              _p(P_i, _lib.i32p), _p(P_j, _lib.i32p),
                                              _p(P_el, _lib.f64p), what_to_do.encode()))
    return dim.value, nz.value, P_i, P_j, P_el


def set_legacy_filter_seed(legacy: bool):
    """The reference's module flag legacy_filter_seed (src/soap_turbo_radial.f90:67)."""
    _lib.check(_lib.load().soapb_set_legacy_filter_seed(int(bool(legacy))))


def get_legacy_filter_seed() -> bool:
    import ctypes as C
    v = C.c_int32(0)
    _lib.check(_lib.load().soapb_get_legacy_filter_seed(C.byref(v)))
    return bool(v.value)


def set_precision(precision: str):
    """"mixed" (default) or "fp64" for the drop-in calls."""
    _lib.check(_lib.load().soapb_set_precision(
        {"mixed": _lib.PREC_MIXED, "fp64": _lib.PREC_FP64}[precision]))


def set_basis_matrices(W=None, S=None):
    """Use these W and S (n_max x n_max, block diagonal) in the drop-in calls;
    None restores the library's own."""
    lib = _lib.load()
    if W is None:
        _lib.check(lib.soapb_set_basis_matrices(0, None, None))
        return
    W = _f(W, _f64)
    S = _f(S, _f64)
    _lib.check(lib.soapb_set_basis_matrices(int(W.shape[0]), _p(W, _lib.f64p), _p(S, _lib.f64p)))


def orthonormalization_matrix(basis, alpha_max, atom_sigma_r=0.5, rcut_hard=5.0):
    """(S, W) of one species, alpha x alpha, Fortran order."""
    S = np.zeros((alpha_max, alpha_max), order="F")
    W = np.zeros((alpha_max, alpha_max), order="F")
    _lib.check(_lib.load().soapb_orthonormalization_matrix(
        _lib.BASIS[basis], int(alpha_max), float(atom_sigma_r), float(rcut_hard),
        _p(S, _lib.f64p), _p(W, _lib.f64p)))
    return S, W
