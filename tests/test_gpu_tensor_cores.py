"""The site kernels' contractions on the tensor cores (tcgen05, 3xTF32) against
the CUDA-core forms and the FP64 oracle: both forms meet the parity gates,
agree with each other within FP32 rounding, and repeat bit for bit."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu

CASES = {
    "config1": lambda: syn.config(1, seed=7),
    "config2_quarter": lambda: syn.config(2, seed=11, scale=0.25),
    "config3_8structs": lambda: syn.config(3, seed=5, scale=1 / 64),
}


@pytest.mark.parametrize("name", list(CASES))
def test_tensor_core_contract_matches_cuda_cores_and_oracle(name):
    w = CASES[name]()
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    ref = O.get_soap(w.hyper, w.nl, W, S, do_derivatives=True)
    G = np.random.default_rng(8).standard_normal((ctx.n_soap, w.nl.n_sites))
    ref_pair = ref.contract(G, 1.0)
    b = ctx.batch(w.nl)
    Gt = torch.as_tensor(G).cuda()
    out = {}
    for tc in (True, False):
        ctx.set_tensor_cores(tc)
        soap = ctx.descriptor(b, keep=True)
        p1 = ctx.contract(b, soap, Gt)
        p2 = ctx.contract(b, soap, Gt)
        ctx.check_inputs()
        assert torch.equal(p1, p2)  # bitwise reproducible
        out[tc] = (soap.cpu().numpy(), p1.cpu().numpy())
        assert site_rel_err(out[tc][0], ref.soap) <= SOAP_TOL
        assert max_rel_err(out[tc][1], ref_pair) <= VJP_TOL
    ctx.set_tensor_cores(True)
    assert max_rel_err(out[True][1], out[False][1]) <= VJP_TOL


def test_tensor_core_contract_on_many_neighbours():
    # sites with more than 128 neighbours: several chunks, and rounds of 64
    # entries per chunk on the tensor cores
    st = syn.random_structure(400, density=0.30, d_min=0.7, fractions=(0.4, 0.4, 0.2), seed=31)
    hp = syn.Hyper(alpha_max=[8, 8, 8], basis="poly3gauss", compress_mode="trivial")
    nl = syn.neighbour_list(st, 5.0, 3, central_species=1)
    assert nl.n_neigh.max() > 128
    ctx = Context(hp)
    W, S = ctx.basis()
    ref = O.get_soap(hp, nl, W, S, do_derivatives=True)
    G = np.random.default_rng(9).standard_normal((ctx.n_soap, nl.n_sites))
    b = ctx.batch(nl)
    soap = ctx.descriptor(b, keep=True)
    pair = ctx.contract(b, soap, torch.as_tensor(G).cuda()).cpu().numpy()
    assert max_rel_err(pair, ref.contract(G, 1.0)) <= VJP_TOL
