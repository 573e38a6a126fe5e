"""Parity with the FP64 oracle at the configurations' stated sizes.

The GPU runs each configuration whole -- 4096 atoms (config 2), all 512
structures as one concatenated CSR batch (config 3), 32768 atoms (config 4),
262144 atoms (config 5) -- and every site and pair is compared with the oracle,
which runs over contiguous site ranges (a site's descriptor and its pairs'
forces depend on its own CSR row alone).  Gates: descriptor max over sites of
|soap - ref|_inf / |ref|_inf <= 1e-6, force VJP max |pair - ref| / max |ref|
<= 1e-5.  Config 5 is also run in the plain FP64 GPU form on a 16384-atom
slice, beside the mixed path on the same slice, both against the oracle."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import FP64_TOL, SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu

SIZES = {2: "4096 atoms", 3: "512 structures", 4: "32768 atoms", 5: "262144 atoms"}


def _mixed(ctx, b, G):
    soap = ctx.descriptor(b, keep=True)
    pair = ctx.contract(b, soap, G)
    ctx.check_inputs()
    return soap.cpu().numpy(), pair.cpu().numpy()


@pytest.mark.parametrize("cfg", [2, 3, 4, 5])
def test_full_size_parity(cfg):
    w = syn.config(cfg, seed=2024)
    nl = w.nl
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    b = ctx.batch(nl)
    G = np.random.default_rng(cfg).standard_normal((ctx.n_soap, nl.n_sites))
    soap, pair = _mixed(ctx, b, torch.as_tensor(G).cuda())
    del b
    ref_soap, ref_pair = O.soap_and_vjp_chunked(w.hyper, nl, W, S, G)
    e_soap, e_vjp = site_rel_err(soap, ref_soap), max_rel_err(pair, ref_pair)
    print(f"config {cfg} ({SIZES[cfg]}: {nl.n_sites} sites, {nl.n_pairs} pairs): "
          f"soap {e_soap:.2e}, vjp {e_vjp:.2e}")
    assert e_soap <= SOAP_TOL
    assert e_vjp <= VJP_TOL


def test_config5_slice_fp64_form_beside_the_mixed_path():
    """The 16384-atom slice of config 5: the plain FP64 GPU form (materialised
    soap_cart_der, then contracted) and the mixed adjoint path, both against
    the oracle on every site and pair."""
    w = syn.config(5, seed=2024, scale=16384 / 262144)
    nl = w.nl
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    b = ctx.batch(nl)
    G = np.random.default_rng(55).standard_normal((ctx.n_soap, nl.n_sites))
    Gt = torch.as_tensor(G).cuda()
    ref_soap, ref_pair = O.soap_and_vjp_chunked(w.hyper, nl, W, S, G)
    soap, pair = _mixed(ctx, b, Gt)
    assert site_rel_err(soap, ref_soap) <= SOAP_TOL
    assert max_rel_err(pair, ref_pair) <= VJP_TOL
    s64, cart = ctx.descriptor_fp64(b, cart=True)
    p64 = ctx.contract_cart_der(b, cart, Gt)
    del cart
    assert site_rel_err(s64.cpu().numpy(), ref_soap) <= FP64_TOL
    assert max_rel_err(p64.cpu().numpy(), ref_pair) <= FP64_TOL
