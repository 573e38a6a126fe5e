"""The drop-in get_soap keeps the reference's intent(inout) meaning of soap and
soap_cart_der: a compressed soap is added into before the norm is taken
(src/soap_turbo.f90:798-802), an uncompressed one is overwritten, and each
site's self column of soap_cart_der is accumulated into (:888-892).  Checked
against the oracle given the same arrays on entry; the contract that follows
reads the norms of the accumulated rows, as the reference's does."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import FP64_TOL, SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import descriptor as D
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context
from test_gpu_parity import _dropin_args

pytestmark = pytest.mark.gpu


def _host(a, pinned, keep):
    if not pinned:
        return np.asfortranarray(a)
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    out = t.numpy().reshape(a.shape, order="F")
    out[...] = a
    keep.append(t)
    return out


@pytest.mark.parametrize("case", ["chunked_pinned", "chunked_pageable", "single_launch", "timed"])
def test_compressed_soap_is_added_into(case):
    # 1703 sites: from pageable arrays the drop-in runs three site chunks, each
    # copying its soap rows in beside its pair inputs; a page-locked soap is
    # added into in place by the site kernel (one chunk); a quarter-size batch
    # runs as one launch, and do_timing takes the unchunked path
    w = syn.config(2, seed=41, scale=0.25 if case == "single_launch" else 1.0)
    nl = w.nl
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    rng = np.random.default_rng(3)
    ref_zero = O.get_soap(w.hyper, nl, W, S, do_derivatives=True)
    # entry values of the unnormalised descriptor's size (its norm per site), so
    # that they change the result visibly; Fortran soap(n_soap, n_sites)
    soap0 = (0.3 * ref_zero.norm() / np.sqrt(ctx.n_soap) *
             rng.standard_normal((ctx.n_soap, nl.n_sites)))
    ref = O.get_soap(w.hyper, nl, W, S, do_derivatives=True, soap_init=soap0.T)
    assert site_rel_err(ref.soap, ref_zero.soap) > 1e-2  # the caller's values matter
    G = rng.standard_normal((ctx.n_soap, nl.n_sites))
    keep = []
    pinned = case == "chunked_pinned"
    D.set_basis_matrices(W, S)
    try:
        for _ in range(2):  # the second call must not see the first call's rows
            soap = _host(soap0, pinned, keep)
            args = _dropin_args(w, soap)
            args["do_timing"] = case == "timed"
            D.get_soap(**args, contract=True)
            assert site_rel_err(soap.T, ref.soap) <= SOAP_TOL
            pair = _host(np.zeros((3, nl.n_pairs)), pinned, keep)
            D.soap_contract(soap, _host(G.T, pinned, keep), 1.0, pair)
            assert max_rel_err(pair.T, ref.contract(G, 1.0)) <= VJP_TOL
    finally:
        D.set_basis_matrices(None)


def test_uncompressed_soap_is_overwritten():
    w = syn.config(1, seed=7)
    nl = w.nl
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    ref = O.get_soap(w.hyper, nl, W, S, do_derivatives=True)
    D.set_basis_matrices(W, S)
    try:
        soap = np.asfortranarray(np.random.default_rng(4).standard_normal((ctx.n_soap, nl.n_sites)))
        D.get_soap(**_dropin_args(w, soap), contract=True)
        assert site_rel_err(soap.T, ref.soap) <= SOAP_TOL
    finally:
        D.set_basis_matrices(None)


def test_soap_cart_der_self_columns_are_accumulated_into():
    # do_derivatives without contract: the FP64 path writes soap_cart_der; its
    # neighbour columns are overwritten, its self columns accumulate
    w = syn.config(2, seed=11, scale=0.25)
    nl = w.nl
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    rng = np.random.default_rng(5)
    nrm = O.get_soap(w.hyper, nl, W, S, do_derivatives=True).norm()
    soap0 = 0.3 * nrm / np.sqrt(ctx.n_soap) * rng.standard_normal((ctx.n_soap, nl.n_sites))
    cart0 = rng.standard_normal((3, ctx.n_soap, nl.n_pairs))
    ref = O.get_soap(w.hyper, nl, W, S, do_derivatives=True, cart_der=True, soap_init=soap0.T,
                     cart_init=np.transpose(cart0, (2, 1, 0)))
    D.set_basis_matrices(W, S)
    try:
        soap = np.asfortranarray(soap0)
        cart = np.asfortranarray(cart0)
        D.get_soap(**_dropin_args(w, soap, cart=cart), contract=False)
        assert site_rel_err(soap.T, ref.soap) <= SOAP_TOL
        got = np.transpose(cart, (2, 1, 0))
        assert max_rel_err(got, ref.soap_cart_der) <= FP64_TOL
        # the self columns really carry the caller's values
        first = np.concatenate([[0], np.cumsum(nl.n_neigh)[:-1]])
        ref_zero = O.get_soap(w.hyper, nl, W, S, do_derivatives=True, cart_der=True, soap_init=soap0.T)
        d = got[first] - ref_zero.soap_cart_der[first]
        np.testing.assert_allclose(d, np.transpose(cart0, (2, 1, 0))[first], rtol=1e-9, atol=1e-9)
    finally:
        D.set_basis_matrices(None)


def test_pinned_soap_written_in_place_matches_the_staged_path():
    """A page-locked soap is written by the site kernel in place, in chunks of
    at least 4096 sites: a chunk whose entry rows are all zero is not read, any
    other is added into in place (read over the host link).  Two chunks here,
    the first entered all zero and the second partly not; soap, and the pair
    forces the contract writes into a page-locked pair array, equal bit for bit
    those of the same calls on pageable copies (staged through the library's
    buffers in 512-site chunks whose rows are copied in and out)."""
    w = syn.config(5, seed=43, scale=0.08)
    nl = w.nl
    assert nl.n_sites >= 2 * 4096
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    rng = np.random.default_rng(6)
    nrm = O.get_soap(w.hyper, nl, W, S, do_derivatives=False).norm()
    soap0 = np.zeros((ctx.n_soap, nl.n_sites))
    lo = 3 * nl.n_sites // 4  # inside the second chunk
    soap0[:, lo:] = 0.3 * nrm[lo:] / np.sqrt(ctx.n_soap) * rng.standard_normal((ctx.n_soap, nl.n_sites - lo))
    G = rng.standard_normal((ctx.n_soap, nl.n_sites))
    out = {}
    keep = []
    D.set_basis_matrices(W, S)
    try:
        for pinned in (True, False):
            soap = _host(soap0, pinned, keep)
            D.get_soap(**_dropin_args(w, soap), contract=True)
            pair = _host(np.zeros((3, nl.n_pairs)), pinned, keep)
            D.soap_contract(soap, _host(G.T, pinned, keep), 1.0, pair)
            out[pinned] = (np.array(soap), np.array(pair))
    finally:
        D.set_basis_matrices(None)
    assert np.all(np.isfinite(out[True][0])) and np.abs(out[True][1]).max() > 0
    np.testing.assert_array_equal(out[True][0], out[False][0])
    np.testing.assert_array_equal(out[True][1], out[False][1])
    # the entry rows mattered where they were not zero
    ref = Context(w.hyper)
    b = ref.batch(nl)
    plain = ref.descriptor(b, keep=False).cpu().numpy().T
    assert np.abs(out[True][0][:, :lo] - plain[:, :lo]).max() < 1e-12
    assert site_rel_err(out[True][0][:, lo:].T, plain[:, lo:].T) > 1e-4
