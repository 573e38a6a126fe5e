"""The batched path: every CTA size of the site kernels, the autotuner, and
descriptor + force VJP captured in one CUDA graph over a concatenated CSR
neighbour list of uneven structures (the batched-workload configuration at
reduced size), each checked against the FP64 oracle."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu


class Batched:
    def __init__(self, w):
        self.w = w
        self.ctx = Context(w.hyper)
        W, S = self.ctx.basis()
        self.ref = O.get_soap(w.hyper, w.nl, W, S, do_derivatives=True, cart_der=False)
        self.b = self.ctx.batch(w.nl)
        rng = np.random.default_rng(23)
        self.G = rng.standard_normal((self.ctx.n_soap, w.nl.n_sites))
        self.Gt = torch.as_tensor(self.G).cuda()
        self.pair_ref = self.ref.contract(self.G, 1.0)


@pytest.fixture(scope="module")
def batched():
    # 16 structures of 16..2048 atoms (log-uniform), densities 0.06..0.14
    return Batched(syn.config(3, seed=29, scale=1 / 32))


@pytest.mark.parametrize("tensor_cores,threads", [(True, 128), (False, 64), (False, 128), (False, 256)])
def test_every_cta_size_matches_the_oracle(batched, tensor_cores, threads):
    # the tensor-core kernels have one CTA size; the CUDA-core ones three
    c = batched.ctx
    c.set_threads_per_site(threads)
    c.set_tensor_cores(tensor_cores)
    try:
        soap = c.descriptor(batched.b)
        pair = c.contract(batched.b, soap, batched.Gt)
        assert site_rel_err(soap.cpu().numpy(), batched.ref.soap) <= SOAP_TOL
        assert max_rel_err(pair.cpu().numpy(), batched.pair_ref) <= VJP_TOL
        # bit-reproducible for a fixed launch configuration
        soap2 = c.descriptor(batched.b)
        pair2 = c.contract(batched.b, soap2, batched.Gt)
        assert torch.equal(soap, soap2) and torch.equal(pair, pair2)
    finally:
        c.set_threads_per_site(0)
        c.set_tensor_cores(True)


def test_autotuner_choice_is_valid_and_used(batched):
    c = batched.ctx
    choice = c.autotune(batched.b)
    # 0: the tensor-core kernel
    assert choice["descriptor_threads"] in (0, 64, 128, 256)
    assert choice["contract_threads"] in (0, 64, 128, 256)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for k in ("descriptor_max_ctas", "contract_max_ctas"):
        assert choice[k] in (0, sms, 2 * sms)
    # the autotuner discarded the kept state: contract must refuse until a descriptor
    from soap_turbo_b200 import _lib
    with pytest.raises(_lib.SoapError):
        c.contract(batched.b, torch.zeros(batched.w.nl.n_sites, c.n_soap, dtype=torch.float64,
                                          device="cuda"), batched.Gt)
    soap = c.descriptor(batched.b)
    pair = c.contract(batched.b, soap, batched.Gt)
    assert site_rel_err(soap.cpu().numpy(), batched.ref.soap) <= SOAP_TOL
    assert max_rel_err(pair.cpu().numpy(), batched.pair_ref) <= VJP_TOL


def test_descriptor_and_vjp_in_one_cuda_graph(batched):
    c = batched.ctx
    b = batched.b
    n_sites, n_pairs = batched.w.nl.n_sites, batched.w.nl.n_pairs
    soap = torch.empty(n_sites, c.n_soap, dtype=torch.float64, device="cuda")
    pair = torch.empty(n_pairs, 3, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        c.set_stream(side)
        # eager warm-up on the capture stream: the context's buffers reach
        # their size here, so the captured calls allocate nothing
        c.descriptor(b, out=soap)
        c.contract(b, soap, batched.Gt, out=pair)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    eager_soap, eager_pair = soap.clone(), pair.clone()
    n0 = c.launch_count
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        c.set_stream(torch.cuda.current_stream())
        c.descriptor(b, out=soap)
        c.contract(b, soap, batched.Gt, out=pair)
    n_captured = c.launch_count - n0
    assert n_captured == 3  # pair (with the CSR scan), descriptor and contract kernels
    for _ in range(3):
        soap.zero_()
        pair.zero_()
        g.replay()
    torch.cuda.synchronize()
    c.set_stream(torch.cuda.current_stream())
    assert torch.equal(soap, eager_soap) and torch.equal(pair, eager_pair)
    assert site_rel_err(soap.cpu().numpy(), batched.ref.soap) <= SOAP_TOL
    assert max_rel_err(pair.cpu().numpy(), batched.pair_ref) <= VJP_TOL
    del g
