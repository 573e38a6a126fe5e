"""Darby compression modes ("nu_R_nu_S", src/soap_turbo_compress.f90:120-303)
through the CUDA descriptor and force VJP, against the oracle fed the same
index maps: the kernels take any compression map, so these check the maps'
use (many kept components, several outputs per component, weights 1/sqrt 2
and sqrt 2) rather than new kernel code."""
import numpy as np
import pytest

import oracle as O
from conftest import FP64_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context
from test_gpu_edge import check, make_nl, random_sites

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["0_0", "0_1", "0_2", "1_0", "1_1", "1_2", "2_0", "2_1", "2_2"])
def test_darby_modes_small_basis(mode):
    hp = syn.Hyper(alpha_max=[4, 4, 4], l_max=4, basis="poly3gauss", compress_mode=mode)
    nl = make_nl(random_sites(np.random.default_rng(17), 24, 3), 3)
    check(hp, nl)


@pytest.mark.parametrize("mode", ["1_1", "2_2"])
def test_darby_modes_benchmark_basis(mode):
    """The 3-species alpha = 8, l_max = 8 basis: 2_2 keeps all 2700
    components, 1_1 compresses them to 216."""
    hp = syn.Hyper(alpha_max=[8, 8, 8], l_max=8, basis="poly3gauss", compress_mode=mode)
    nl = make_nl(random_sites(np.random.default_rng(23), 16, 3, lo=30, hi=80), 3)
    check(hp, nl)


@pytest.mark.parametrize("basis", ["poly3", "poly3operator"])
def test_darby_mode_other_bases(basis):
    hp = syn.Hyper(alpha_max=[4, 4, 4], l_max=4, basis=basis, compress_mode="1_2")
    nl = make_nl(random_sites(np.random.default_rng(29), 20, 3), 3)
    check(hp, nl)


@pytest.mark.parametrize("mode,alpha,l_max", [("0_1", 4, 4), ("1_2", 4, 4), ("1_1", 8, 8), ("2_2", 8, 8)])
def test_darby_modes_soap_cart_der(mode, alpha, l_max):
    """The FP64 form's soap_cart_der (src/soap_turbo.f90:816-902) when the
    compression map is not one-to-one: each output column a weighted sum of
    kept components' derivatives; at 2_2 (2700 outputs) the form whose rows
    do not fit the CTA's shared memory."""
    hp = syn.Hyper(alpha_max=[alpha] * 3, l_max=l_max, basis="poly3gauss", compress_mode=mode)
    nl = make_nl(random_sites(np.random.default_rng(31), 10, 3, lo=20, hi=60), 3)
    ctx = Context(hp)
    W, S = ctx.basis()
    ref = O.get_soap(hp, nl, W, S, do_derivatives=True, cart_der=True)
    soap, cart = ctx.descriptor_fp64(ctx.batch(nl), cart=True)
    assert site_rel_err(soap.cpu().numpy(), ref.soap) <= FP64_TOL
    assert max_rel_err(cart.cpu().numpy(), ref.soap_cart_der) <= FP64_TOL
