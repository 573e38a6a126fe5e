"""ctypes wrapper of the FP64 CPU oracle (soap_oracle.c).

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py import this module, always as the checker or the timed CPU
baseline -- never as the thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsoap_oracle.so")
_lib = None

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


class _Args(C.Structure):
    _fields_ = [
        ("n_sites", C.c_int), ("n_species", C.c_int), ("n_pairs", C.c_int), ("max_mult", C.c_int),
        ("l_max", C.c_int), ("radial_enhancement", C.c_int), ("basis", C.c_int),
        ("scaling_poly", C.c_int), ("legacy_filter_seed", C.c_int),
        ("n_neigh", _i32p), ("species", _i32p), ("species_multiplicity", _i32p),
        ("mask", _u8p), ("rjs", _f64p), ("thetas", _f64p), ("phis", _f64p),
        ("alpha_max", _i32p),
        ("rcut_hard", _f64p), ("rcut_soft", _f64p), ("nf", _f64p), ("global_scaling", _f64p),
        ("atom_sigma_r", _f64p), ("atom_sigma_r_scaling", _f64p),
        ("atom_sigma_t", _f64p), ("atom_sigma_t_scaling", _f64p),
        ("amplitude_scaling", _f64p), ("central_weight", _f64p),
        ("compress", C.c_int), ("P_nonzero", C.c_int), ("P_i", _i32p), ("P_j", _i32p), ("P_el", _f64p),
        ("W", _f64p), ("S", _f64p),
    ]


def build() -> str:
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "soap_oracle.c")):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.or_get_soap.restype = C.c_int
        _lib.or_get_soap.argtypes = [C.POINTER(_Args), C.c_int, _f64p, _f64p, C.POINTER(C.c_void_p)]
        _lib.or_soap_contract.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double, _f64p]
        _lib.or_get_soap2.restype = C.c_int
        _lib.or_get_soap2.argtypes = [C.POINTER(_Args), C.c_int, C.c_int, _f64p, _f64p,
                                      C.POINTER(C.c_void_p)]
        _lib.or_central_hessian.restype = C.c_int
        _lib.or_central_hessian.argtypes = [C.POINTER(_Args), C.c_void_p, _f64p, C.c_int, _f64p,
                                            _f64p, _f64p]
        _lib.or_ctx_free.argtypes = [C.c_void_p]
        for name in ("or_ctx_cnk", "or_ctx_rad", "or_ctx_rad_der", "or_ctx_norm"):
            getattr(_lib, name).restype = _f64p
            getattr(_lib, name).argtypes = [C.c_void_p]
        _lib.or_ctx_ang.restype = _f64p
        _lib.or_ctx_ang.argtypes = [C.c_void_p, C.c_int]
        _lib.or_plm_double.restype = C.c_double
        _lib.or_plm_double.argtypes = [C.c_int, C.c_int, C.c_double]
        _lib.or_ilexp_double.restype = C.c_double
        _lib.or_ilexp_double.argtypes = [C.c_int, C.c_double]
        _lib.or_plm_array.argtypes = [C.c_int, C.c_double, _f64p]
        _lib.or_plm_array_der.argtypes = [C.c_int, _f64p, _f64p, _f64p]
        _lib.or_ilexp_array.argtypes = [C.c_int, C.c_double, _f64p]
        _lib.or_preflm.argtypes = [C.c_int, _f64p]
        _lib.or_inverse_sqrt.argtypes = [C.c_int, _f64p, _f64p]
        _lib.or_overlap_poly3.argtypes = [C.c_int, _f64p]
        _lib.or_overlap_poly3gauss.argtypes = [C.c_int, C.c_double, C.c_double, _f64p]
        _lib.or_compress_trivial.argtypes = [C.c_int, _i32p, C.c_int, _i32p, _i32p, _f64p]
        _lib.or_compress_darby.argtypes = [C.c_int, _i32p, C.c_int, C.c_int, C.c_int, _i32p,
                                           _i32p, _i32p, _f64p]
        _lib.or_radial_eval.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_double, _f64p, C.c_int, C.c_int,
                                        C.c_double, C.c_int, C.c_int, C.c_int, _f64p, _f64p, _f64p,
                                        _f64p]
        _lib.or_num_threads.restype = C.c_int
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def num_threads() -> int:
    return lib().or_num_threads()


# ---------------------------------------------------------------- basis
def overlap(basis: str, alpha: int, sigma: float = 0.5, rcut: float = 5.0) -> np.ndarray:
    S = np.zeros((alpha, alpha), order="F")
    if basis in ("poly3", "poly3operator"):  # poly3operator uses poly3's W (src/soap_turbo.f90:380-381)
        lib().or_overlap_poly3(alpha, _p(S, _f64p))
    else:
        lib().or_overlap_poly3gauss(alpha, sigma, rcut, _p(S, _f64p))
    return S


def inverse_sqrt(S: np.ndarray) -> np.ndarray:
    a = S.shape[0]
    S = np.asfortranarray(S, dtype=np.float64)
    W = np.zeros((a, a), order="F")
    rc = lib().or_inverse_sqrt(a, _p(S, _f64p), _p(W, _f64p))
    if rc:
        raise RuntimeError("overlap matrix not positive definite")
    return W


def inverse_sqrt_lapack_route(S: np.ndarray) -> np.ndarray:
    """W = (S^{1/2})^{-1} the way the reference forms it in FP64 LAPACK
    (src/soap_turbo_radial.f90:1052-1087 poly3, :1177-1212 poly3gauss): dgesvd
    of S, S^{1/2} = U diag(sqrt(svd)) VT, then dpotrf + dpotri of S^{1/2} and
    the upper triangle mirrored.  scipy's bundled LAPACK stands in for the
    (unpinned) LAPACK the reference links."""
    from scipy.linalg import lapack
    S = np.asfortranarray(S, dtype=np.float64)
    u, svd, vt, info = lapack.dgesvd(S, compute_uv=1, full_matrices=1)
    if info != 0:
        raise RuntimeError("dgesvd failed")
    half = np.asfortranarray((u * np.sqrt(svd)) @ vt)
    c, info = lapack.dpotrf(half, lower=0)
    if info != 0:
        raise RuntimeError("dpotrf failed")
    inv, info = lapack.dpotri(c, lower=0)
    if info != 0:
        raise RuntimeError("dpotri failed")
    up = np.triu(inv)
    return np.asfortranarray(up + np.triu(inv, 1).T)


def basis_matrices(hyper):
    """Block-diagonal (n_max, n_max) W and S, Fortran order."""
    n_max = hyper.n_max
    W = np.zeros((n_max, n_max), order="F")
    S = np.zeros((n_max, n_max), order="F")
    b = 0
    sig = hyper.arr("atom_sigma_r")
    rc = hyper.arr("rcut_hard")
    for s, a in enumerate(hyper.alpha_max):
        Ss = overlap(hyper.basis, a, sig[s], rc[s])
        S[b:b + a, b:b + a] = Ss
        W[b:b + a, b:b + a] = inverse_sqrt(Ss)
        b += a
    return W, S


# ---------------------------------------------------------------- scalars
def plm_double(l, m, x):
    return lib().or_plm_double(l, m, x)


def ilexp_double(l, x):
    return lib().or_ilexp_double(l, x)


def plm_array(lmax, x):
    out = np.zeros((lmax + 1) * (lmax + 2) // 2)
    lib().or_plm_array(lmax, x, _p(out, _f64p))
    return out


def ilexp_array(lmax, x):
    out = np.zeros(lmax + 1)
    lib().or_ilexp_array(lmax, x, _p(out, _f64p))
    return out


def preflm(lmax):
    out = np.zeros((lmax + 1) * (lmax + 2) // 2)
    lib().or_preflm(lmax, _p(out, _f64p))
    return out


BASIS_CODE = {"poly3": 0, "poly3gauss": 1, "poly3operator": 2}


def radial_eval(hyper, species: int, W_block, r, legacy_seed=True, is_central=False, der2=False):
    """The radial expansion of one species at distances r: (values, r-derivatives)
    and, with der2 (unified seed only), the second r-derivatives as well."""
    a = hyper.alpha_max[species]
    r = np.ascontiguousarray(r, dtype=np.float64)
    out = np.zeros((r.shape[0], a))
    der = np.zeros((r.shape[0], a))
    d2 = np.zeros((r.shape[0], a)) if der2 else None
    Wb = np.asfortranarray(W_block, dtype=np.float64)
    rc = lib().or_radial_eval(
        BASIS_CODE[hyper.basis], a, hyper.arr("rcut_soft")[species],
        hyper.arr("rcut_hard")[species], hyper.arr("atom_sigma_r")[species],
        hyper.arr("atom_sigma_r_scaling")[species], hyper.arr("amplitude_scaling")[species],
        hyper.arr("nf")[species], _p(Wb, _f64p), 1 if hyper.scaling_mode == "polynomial" else 0,
        hyper.radial_enhancement, hyper.arr("central_weight")[species], int(is_central),
        int(legacy_seed), r.shape[0], _p(r, _f64p), _p(out, _f64p), _p(der, _f64p),
        _p(d2, _f64p) if der2 else None)
    if rc:
        raise ValueError("second radial derivatives need the unified filter seed (and poly3 or "
                         "poly3gauss)")
    return (out, der, d2) if der2 else (out, der)


def compress_trivial(alpha_max, l_max):
    am = np.ascontiguousarray(alpha_max, dtype=np.int32)
    n = lib().or_compress_trivial(len(am), _p(am, _i32p), l_max, None, None, None)
    P_i = np.zeros(n, dtype=np.int32)
    P_j = np.zeros(n, dtype=np.int32)
    P_el = np.zeros(n)
    lib().or_compress_trivial(len(am), _p(am, _i32p), l_max, _p(P_i, _i32p), _p(P_j, _i32p),
                              _p(P_el, _f64p))
    return P_i, P_j, P_el


DARBY_MODES = ("0_0", "0_1", "0_2", "1_0", "1_1", "1_2", "2_0", "2_1", "2_2")


def compress_darby(mode, alpha_max, l_max):
    """get_compress_indices for the Darby modes "nu_R_nu_S"
    (src/soap_turbo_compress.f90:120-303): (dim, P_i, P_j, P_el), 1-based."""
    nu_R, nu_S = int(mode[0]), int(mode[2])
    am = np.ascontiguousarray(alpha_max, dtype=np.int32)
    dim = C.c_int(0)
    n = lib().or_compress_darby(len(am), _p(am, _i32p), l_max, nu_R, nu_S, C.byref(dim),
                                None, None, None)
    if n == -2:
        raise ValueError(f"compress_mode={mode} requires all species to have the same number "
                         "of radial basis functions")
    if n < 0:
        raise MemoryError("compression lookup does not fit")
    P_i = np.zeros(n, dtype=np.int32)
    P_j = np.zeros(n, dtype=np.int32)
    P_el = np.zeros(n)
    lib().or_compress_darby(len(am), _p(am, _i32p), l_max, nu_R, nu_S, C.byref(dim),
                            _p(P_i, _i32p), _p(P_j, _i32p), _p(P_el, _f64p))
    return dim.value, P_i, P_j, P_el


# ---------------------------------------------------------------- get_soap
class Result:
    """soap (n_sites, n_soap) == Fortran soap(n_soap, n_sites); the state
    soap_contract reads is kept in ``ctx``."""

    def __init__(self, soap, cart, ctx, keep):
        self.soap = soap
        self.soap_cart_der = cart
        self._ctx = ctx
        self._keep = keep

    def contract(self, G_fortran: np.ndarray, sgn: float = 1.0) -> np.ndarray:
        """soap_contract: G is Fortran G(n_sites, n_soap), given here as a
        (n_soap, n_sites) C-ordered array. Returns pair (n_pairs, 3)."""
        G = np.ascontiguousarray(G_fortran, dtype=np.float64)
        soap = np.ascontiguousarray(self.soap)
        n_pairs = self._keep["n_pairs"]
        pair = np.zeros((n_pairs, 3))
        rc = lib().or_soap_contract(self._ctx, _p(soap, _f64p), _p(G, _f64p), sgn, _p(pair, _f64p))
        if rc:
            raise RuntimeError("oracle soap_contract needs derivatives")
        return pair

    def central_hessian(self, vecs: np.ndarray):
        """get_soap_central_hessian (src/soap_turbo.f90:1151-1700) on this
        state (get_soap with hessian=True).  vecs: (n_sites, n_vec, n_soap),
        the reference's vecs(n_soap, n_vec, n_sites).  Returns (hess, err):
        hess (n_pairs, n_vec, 3, 3) with hess[k, v, b, a] the reference's
        hess(a, b, v, k) (a: central atom, b: neighbour), and the self-test's
        relative error of the rebuilt first derivative."""
        vecs = np.ascontiguousarray(vecs, dtype=np.float64)
        n_vec = vecs.shape[1]
        soap = np.ascontiguousarray(self.soap)
        hess = np.zeros((self._keep["n_pairs"], n_vec, 3, 3))
        err = C.c_double(0.0)
        rc = lib().or_central_hessian(C.byref(self._keep["args"]), self._ctx, _p(soap, _f64p), n_vec,
                                      _p(vecs, _f64p), _p(hess, _f64p), C.byref(err))
        if rc:
            raise RuntimeError("central_hessian needs get_soap(..., hessian=True)")
        return hess, err.value

    def cnk(self):
        c = self._keep
        ptr = lib().or_ctx_cnk(self._ctx)
        n = c["n_sites"] * c["n_max"] * c["k_max"] * 2
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy().reshape(c["n_sites"], c["n_max"], c["k_max"], 2)

    def radial(self):
        c = self._keep
        n = c["n_pairs"] * c["n_max"]
        r = np.ctypeslib.as_array(lib().or_ctx_rad(self._ctx), shape=(n,)).copy()
        d = np.ctypeslib.as_array(lib().or_ctx_rad_der(self._ctx), shape=(n,)).copy()
        return r.reshape(c["n_pairs"], c["n_max"]), d.reshape(c["n_pairs"], c["n_max"])

    def angular(self, which=0):
        c = self._keep
        n = c["n_pairs"] * c["k_max"] * 2
        a = np.ctypeslib.as_array(lib().or_ctx_ang(self._ctx, which), shape=(n,)).copy()
        return a.reshape(c["n_pairs"], c["k_max"], 2)

    def norm(self):
        c = self._keep
        return np.ctypeslib.as_array(lib().or_ctx_norm(self._ctx), shape=(c["n_sites"],)).copy()

    def __del__(self):
        if self._ctx:
            lib().or_ctx_free(self._ctx)
            self._ctx = None


def compress_arrays(hyper):
    if hyper.compress_mode in ("trivial", "Trivial"):
        return compress_trivial(hyper.alpha_max, hyper.l_max)
    if hyper.compress_mode in DARBY_MODES:
        return compress_darby(hyper.compress_mode, hyper.alpha_max, hyper.l_max)[1:]
    return None


def get_soap(hyper, nl, W, S, do_derivatives=True, cart_der=False, legacy_filter_seed=True,
             compress=None, hessian=False, soap_init=None, cart_init=None) -> Result:
    """Run the oracle get_soap.  ``cart_der`` materialises soap_cart_der
    (contract = .false.); the expansion is always kept for ``contract``;
    ``hessian`` also keeps the second radial derivatives central_hessian needs
    (the reference's soap_hessian_enabled; unified filter seed only).
    ``soap_init`` (n_sites, n_soap) and ``cart_init`` (n_pairs, n_soap, 3) are
    the caller's arrays on entry (zero when None): the reference adds the
    compressed descriptor into soap and the self columns into soap_cart_der
    (src/soap_turbo.f90:798-802, 888-892)."""
    n_species = hyper.n_species
    if compress is None:
        compress = compress_arrays(hyper)
    keep = {}
    arrays = {
        "n_neigh": np.ascontiguousarray(nl.n_neigh, dtype=np.int32),
        "species": np.ascontiguousarray(nl.species, dtype=np.int32),
        "species_multiplicity": np.ascontiguousarray(nl.species_multiplicity, dtype=np.int32),
        "mask": np.ascontiguousarray(nl.mask, dtype=np.uint8),
        "rjs": np.ascontiguousarray(nl.rjs, dtype=np.float64),
        "thetas": np.ascontiguousarray(nl.thetas, dtype=np.float64),
        "phis": np.ascontiguousarray(nl.phis, dtype=np.float64),
        "alpha_max": np.ascontiguousarray(hyper.alpha_max, dtype=np.int32),
        "W": np.asfortranarray(W, dtype=np.float64),
        "S": np.asfortranarray(S, dtype=np.float64),
    }
    for name in ("rcut_hard", "rcut_soft", "nf", "global_scaling", "atom_sigma_r",
                 "atom_sigma_r_scaling", "atom_sigma_t", "atom_sigma_t_scaling",
                 "amplitude_scaling", "central_weight"):
        arrays[name] = hyper.arr(name)
    a = _Args()
    a.n_sites = nl.n_sites
    a.n_species = n_species
    a.n_pairs = nl.n_pairs
    a.max_mult = arrays["species"].shape[1]
    a.l_max = hyper.l_max
    a.radial_enhancement = hyper.radial_enhancement
    a.basis = BASIS_CODE[hyper.basis]
    a.scaling_poly = 1 if hyper.scaling_mode == "polynomial" else 0
    a.legacy_filter_seed = int(legacy_filter_seed)
    for name in ("n_neigh", "species", "species_multiplicity", "alpha_max"):
        setattr(a, name, _p(arrays[name], _i32p))
    a.mask = _p(arrays["mask"], _u8p)
    for name in ("rjs", "thetas", "phis", "rcut_hard", "rcut_soft", "nf", "global_scaling",
                 "atom_sigma_r", "atom_sigma_r_scaling", "atom_sigma_t", "atom_sigma_t_scaling",
                 "amplitude_scaling", "central_weight", "W", "S"):
        setattr(a, name, _p(arrays[name], _f64p))
    n_max = hyper.n_max
    n_unc = n_max * (n_max + 1) // 2 * (hyper.l_max + 1)
    if compress is not None:
        P_i, P_j, P_el = (np.ascontiguousarray(compress[0], dtype=np.int32),
                          np.ascontiguousarray(compress[1], dtype=np.int32),
                          np.ascontiguousarray(compress[2], dtype=np.float64))
        arrays.update(P_i=P_i, P_j=P_j, P_el=P_el)
        a.compress = 1
        a.P_nonzero = P_i.shape[0]
        a.P_i = _p(P_i, _i32p)
        a.P_j = _p(P_j, _i32p)
        a.P_el = _p(P_el, _f64p)
        n_soap = int(P_i.max())
    else:
        a.compress = 0
        n_soap = n_unc
    soap = np.zeros((nl.n_sites, n_soap))
    if soap_init is not None:
        soap[...] = soap_init
    cart = np.zeros((nl.n_pairs, n_soap, 3)) if (do_derivatives and cart_der) else None
    if cart is not None and cart_init is not None:
        cart[...] = cart_init
    ctx = C.c_void_p()
    rc = lib().or_get_soap2(C.byref(a), int(do_derivatives), int(bool(hessian)), _p(soap, _f64p),
                            _p(cart, _f64p) if cart is not None else None, C.byref(ctx))
    if rc < 0:
        raise RuntimeError(f"oracle get_soap failed ({rc})")
    keep.update(n_sites=nl.n_sites, n_pairs=nl.n_pairs, n_max=n_max,
                k_max=(hyper.l_max + 1) * (hyper.l_max + 2) // 2, arrays=arrays, args=a)
    return Result(soap, cart, ctx.value, keep)


def _slice_sites(nl, lo, hi):
    """The CSR rows of sites [lo, hi) as a neighbour list of their own."""
    import copy
    off = np.concatenate([[0], np.cumsum(nl.n_neigh)])
    p0, p1 = int(off[lo]), int(off[hi])
    out = copy.copy(nl)
    out.n_sites = hi - lo
    out.n_neigh = nl.n_neigh[lo:hi]
    out.rjs, out.thetas, out.phis = nl.rjs[p0:p1], nl.thetas[p0:p1], nl.phis[p0:p1]
    out.mask = nl.mask[:, p0:p1]
    out.species = nl.species[lo:hi]
    out.species_multiplicity = nl.species_multiplicity[lo:hi]
    return out, p0, p1


def soap_and_vjp_chunked(hyper, nl, W, S, G, sgn=1.0, max_pairs=400_000, legacy_filter_seed=True,
                         sites=None):
    """get_soap + soap_contract over contiguous site ranges of at most
    ``max_pairs`` pairs each: every site's descriptor and every pair's force
    depend on its own site's CSR row alone (src/soap_turbo.f90:619-664,
    1723-1884), so this equals one call on the whole list while bounding the
    oracle's memory (~3.5 KB of expansions per pair) at full configuration
    sizes.  G: (n_soap, n_sites), the reference's G(n_sites, n_soap).
    ``sites`` (optional, sorted) restricts the work to those sites; rows of
    the others are left NaN.  Returns soap (n_sites, n_soap), pair (n_pairs, 3)."""
    off = np.concatenate([[0], np.cumsum(nl.n_neigh)]).astype(np.int64)
    n_soap = G.shape[0]
    soap = np.full((nl.n_sites, n_soap), np.nan)
    pair = np.full((nl.n_pairs, 3), np.nan)
    want = np.ones(nl.n_sites, bool) if sites is None else np.zeros(nl.n_sites, bool)
    if sites is not None:
        want[np.asarray(sites)] = True
    lo = 0
    while lo < nl.n_sites:
        if not want[lo]:
            lo += 1
            continue
        hi = lo + 1
        while hi < nl.n_sites and want[hi] and off[hi + 1] - off[lo] <= max_pairs:
            hi += 1
        sub, p0, p1 = _slice_sites(nl, lo, hi)
        r = get_soap(hyper, sub, W, S, do_derivatives=True, legacy_filter_seed=legacy_filter_seed)
        soap[lo:hi] = r.soap
        pair[p0:p1] = r.contract(np.ascontiguousarray(G[:, lo:hi]), sgn)
        del r
        lo = hi
    return soap, pair
