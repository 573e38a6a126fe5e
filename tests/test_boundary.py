"""The C ABI of libsoapb200.so without a GPU: it loads, exports every entry
point include/soap_b200.h declares, and its host-only entry points (basis
matrices, compression indices, argument checks) behave like the reference."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import oracle as O
from conftest import ROOT
from soap_turbo_b200 import _lib, descriptor as D
from soap_turbo_b200 import synthetic as syn

HEADER = os.path.join(ROOT, "include", "soap_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(soapb_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding declares exactly the header's functions
    assert sorted(_lib.SIGNATURES) == names
    assert lib.soapb_version().startswith(b"soap_b200")


def test_no_oracle_in_the_product_library():
    lib = _lib.load()
    for n in ("or_get_soap", "or_soap_contract", "or_radial_eval"):
        assert not hasattr(lib, n)


GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "poly3tab.json")))["tables"]


@pytest.mark.parametrize("a", range(1, 9))
def test_library_basis_matches_reference_table_and_oracle(a):
    S, W = D.orthonormalization_matrix("poly3", a)
    St = np.array(GOLDEN[str(a)]["S"]).reshape(a, a, order="F")
    Wt = np.array(GOLDEN[str(a)]["W"]).reshape(a, a, order="F")
    np.testing.assert_array_equal(S, St)
    assert np.abs(W - Wt).max() / np.abs(Wt).max() < 2e-5
    Wo = O.inverse_sqrt(St)
    assert np.abs(W - Wo).max() / np.abs(Wo).max() < 1e-12


@pytest.mark.parametrize("a", [2, 6, 8, 11])
def test_library_poly3gauss_basis_matches_oracle(a):
    S, W = D.orthonormalization_matrix("poly3gauss", a, 0.5, 5.0)
    So = O.overlap("poly3gauss", a, 0.5, 5.0)
    assert np.abs(S - So).max() < 1e-15
    Wo = O.inverse_sqrt(So)
    assert np.abs(W - Wo).max() / np.abs(Wo).max() < 1e-12


def test_alpha_limits_like_the_reference():
    # poly3 refuses alpha_max > 10, poly3gauss > 11 (src/soap_turbo_radial.f90:144-153, 210-219)
    with pytest.raises(_lib.SoapError) as e:
        D.orthonormalization_matrix("poly3", 11)
    assert e.value.code == 2
    D.orthonormalization_matrix("poly3", 10)
    with pytest.raises(_lib.SoapError) as e:
        D.orthonormalization_matrix("poly3gauss", 12)
    assert e.value.code == 2
    D.orthonormalization_matrix("poly3gauss", 11)


@pytest.mark.parametrize("am,L", [([8, 8, 8], 8), ([8], 8), ([4, 6], 3), ([3, 3, 3, 3], 5), ([1], 0)])
def test_compress_indices_bit_exact(am, L):
    dim, nz, P_i, P_j, P_el = D.get_compress_indices("trivial", am, L)
    Q_i, Q_j, Q_el = O.compress_trivial(am, L)
    assert dim == nz == Q_i.shape[0]
    np.testing.assert_array_equal(P_i, Q_i)
    np.testing.assert_array_equal(P_j, Q_j)
    np.testing.assert_array_equal(P_el, Q_el)
    dim2, nz2, *_ = D.get_compress_indices("Trivial", am, L, what_to_do="get_dim")
    assert (dim2, nz2) == (dim, nz)


DARBY = ("0_0", "0_1", "0_2", "1_0", "1_1", "1_2", "2_0", "2_1", "2_2")


@pytest.mark.parametrize("mode", DARBY)
@pytest.mark.parametrize("am,L", [([4], 3), ([3, 3], 2), ([8, 8, 8], 8), ([2, 2, 2, 2], 4)])
def test_darby_indices_bit_exact(mode, am, L):
    """The library's Darby maps against the oracle's literal restatement
    (dense lookup and all) of src/soap_turbo_compress.f90:120-303."""
    dim, nz, P_i, P_j, P_el = D.get_compress_indices(mode, am, L)
    qdim, Q_i, Q_j, Q_el = O.compress_darby(mode, am, L)
    assert dim == qdim and nz == Q_i.shape[0]
    np.testing.assert_array_equal(P_i, Q_i)
    np.testing.assert_array_equal(P_j, Q_j)
    np.testing.assert_array_equal(P_el, Q_el)
    assert P_i.min() >= 1 and P_i.max() == dim
    n_unc = sum(am) * (sum(am) + 1) // 2 * (L + 1)
    assert P_j.min() >= 1 and P_j.max() == n_unc
    assert (dim, nz) == D.get_compress_indices(mode, am, L, what_to_do="get_dim")[:2]


def test_darby_2_2_keeps_every_component_once():
    """nu_R = nu_S = 2 is the full power spectrum: the map is the identity."""
    dim, nz, P_i, P_j, P_el = D.get_compress_indices("2_2", [3, 3], 2)
    assert dim == nz == 6 * 7 // 2 * 3
    np.testing.assert_array_equal(P_i, P_j)
    np.testing.assert_array_equal(P_el, np.ones(nz))


def test_darby_0_0_sums_every_radial_pair_per_l():
    """nu_R = nu_S = 0 keeps one component per l: each uncompressed (n <= n')
    enters it once, with sqrt 2 off the diagonal."""
    am, L = [2, 2], 3
    dim, nz, P_i, P_j, P_el = D.get_compress_indices("0_0", am, L)
    N = sum(am)
    assert dim == L + 1 and nz == N * (N + 1) // 2 * (L + 1)
    ls = (P_j - 1) % (L + 1)
    np.testing.assert_array_equal(P_i - 1, ls)
    diag = []
    for n in range(N):
        for m in range(n, N):
            diag += [n == m] * (L + 1)
    np.testing.assert_array_equal(P_el, np.where(np.asarray(diag)[P_j - 1], 1.0, np.sqrt(2.0)))


def test_compress_errors():
    with pytest.raises(_lib.SoapError) as e:
        D.get_compress_indices("2_2", [8, 6], 8)  # Darby modes need equal alpha_max
    assert e.value.code == 4
    with pytest.raises(ValueError):
        O.compress_darby("2_2", [8, 6], 8)
    with pytest.raises(_lib.SoapError) as e:
        D.get_compress_indices("3_0", [8], 8)
    assert e.value.code == 4
    with pytest.raises(_lib.SoapError) as e:
        D.get_compress_indices("bogus", [8], 8)
    assert e.value.code == 4
    lib = _lib.load()
    am = np.array([8], dtype=np.int32)
    d, n = C.c_int32(0), C.c_int32(0)
    rc = lib.soapb_get_compress_indices(b"trivial", 1, am.ctypes.data_as(_lib.i32p), 8, C.byref(d),
                                        C.byref(n), None, None, None, b"neither")
    assert rc == 1


def test_legacy_filter_seed_flag_roundtrip():
    assert D.get_legacy_filter_seed() is True
    D.set_legacy_filter_seed(False)
    assert D.get_legacy_filter_seed() is False
    D.set_legacy_filter_seed(True)
    assert D.get_legacy_filter_seed() is True


def test_contract_without_get_soap_is_refused():
    # src/soap_turbo.f90:1744-1747
    pair = np.zeros((3, 1), order="F")
    with pytest.raises(_lib.SoapError) as e:
        D.soap_contract(np.zeros((324, 1)), np.zeros((1, 324)), 1.0, pair)
    assert e.value.code == 3


def _tiny_call(**over):
    w = syn.config(1, seed=1)
    hp, nl = w.hyper, w.nl
    n_soap = 324
    args = dict(n_sites=nl.n_sites, n_neigh=nl.n_neigh, n_species=1, species=nl.species.T,
                species_multiplicity=nl.species_multiplicity, n_atom_pairs=nl.n_pairs,
                mask=nl.mask.T, rjs=nl.rjs, thetas=nl.thetas, phis=nl.phis, alpha_max=[8],
                l_max=8, rcut_hard=5.0, rcut_soft=4.5, nf=4.0, global_scaling=1.0,
                atom_sigma_r=0.5, atom_sigma_r_scaling=0.0, atom_sigma_t=0.5,
                atom_sigma_t_scaling=0.0, amplitude_scaling=1.0, radial_enhancement=0,
                central_weight=1.0, basis="poly3", scaling_mode="polynomial", do_timing=False,
                do_derivatives=False, compress_soap=False, compress_P_nonzero=0, compress_P_i=None,
                compress_P_j=None, compress_P_el=None,
                soap=np.zeros((n_soap, nl.n_sites), order="F"), soap_cart_der=None)
    args.update(over)
    return args


def test_argument_checks_before_any_device_work():
    # a bad basis name or inconsistent CSR is refused on the host
    with pytest.raises(_lib.SoapError) as e:
        D.get_soap(**_tiny_call(basis="poly3tab"))  # no radial expansion of its own in the reference
    assert e.value.code == 5
    a = _tiny_call()
    a["n_atom_pairs"] = a["n_atom_pairs"] - 1
    a["rjs"] = a["rjs"][:-1]
    with pytest.raises(_lib.SoapError) as e:
        D.get_soap(**a)
    assert e.value.code == 8


def test_get_soap_without_a_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.SoapError) as e:
        D.get_soap(**_tiny_call())
    assert e.value.code == 7


def test_central_hessian_state_checks_on_the_host():
    """get_soap_central_hessian without a matching get_soap stops the reference
    (src/soap_turbo.f90:1206-1227); soap_hessian_enabled with the legacy filter
    seed is refused before any device work (src/soap_turbo_radial.f90:318-323)."""
    args = _tiny_call()
    n_soap, n_sites, n_pairs = 324, args["n_sites"], args["n_atom_pairs"]
    hess = np.zeros((3, 3, 1, n_pairs), order="F")
    with pytest.raises(_lib.SoapError) as e:
        D.get_soap_central_hessian(
            n_sites, args["n_neigh"], n_pairs, 1, args["mask"], args["rjs"], args["thetas"],
            args["phis"], 8, 5.0, 0.5, 0.0, False, 0, None, None, None,
            np.zeros((n_soap, n_sites), order="F"), 1, np.zeros((n_soap, 1, n_sites), order="F"), hess)
    assert e.value.code == 10
    assert not D.get_soap_hessian_enabled()
    D.set_soap_hessian_enabled(True)
    try:
        assert D.get_legacy_filter_seed()
        with pytest.raises(_lib.SoapError) as e:
            D.get_soap(**_tiny_call(do_derivatives=True))
        assert e.value.code == 1 and "legacy_filter_seed" in str(e.value)
    finally:
        D.set_soap_hessian_enabled(False)


def test_poly3operator_has_no_hessian():
    """soap_hessian_enabled with the poly3operator basis stops get_soap in the
    reference (src/soap_turbo.f90:485-489): refused before any device work."""
    D.set_legacy_filter_seed(False)
    D.set_soap_hessian_enabled(True)
    try:
        with pytest.raises(_lib.SoapError) as e:
            D.get_soap(**_tiny_call(basis="poly3operator", do_derivatives=True))
        assert e.value.code == 5 and "poly3operator" in str(e.value)
    finally:
        D.set_soap_hessian_enabled(False)
        D.set_legacy_filter_seed(True)
