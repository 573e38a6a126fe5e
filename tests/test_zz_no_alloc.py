"""soapb_descriptor_noalloc, the descriptor entry point that allocates no
device memory, against soapb_descriptor on the same batches.

Collected last (file name) so that it also runs after every other test has
used the library; it must pass alone in a fresh process as well."""
import numpy as np
import pytest

from conftest import SOAP_TOL, site_rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    from soap_turbo_b200 import synthetic as syn
    from soap_turbo_b200.context import Context
    torch.cuda.set_device(0)
    big = syn.config(2, seed=11, scale=0.25)
    small = syn.config(2, seed=12, scale=0.1)
    ctx = Context(big.hyper)
    return ctx, ctx.batch(big.nl), ctx.batch(small.nl)


def test_noalloc_matches_descriptor_on_consecutive_calls(setup):
    import torch
    ctx, b_big, b_small = setup
    ref_big = ctx.descriptor(b_big, keep=False).cpu().numpy()
    ref_small = ctx.descriptor(b_small, keep=False).cpu().numpy()
    # a larger batch, then a smaller one: the second call finds the first
    # call's contents in the shared array
    n0 = ctx.launch_count
    out_big = ctx.descriptor_noalloc(b_big)
    torch.cuda.synchronize()
    out_small = ctx.descriptor_noalloc(b_small)
    torch.cuda.synchronize()
    assert ctx.launch_count - n0 == 4  # pair (with the CSR scan) and site kernels, twice
    for out, ref in ((out_big, ref_big), (out_small, ref_small)):
        out = out.cpu().numpy()
        assert out.shape == ref.shape and np.all(np.isfinite(out))
        assert np.abs(ref).max() > 0
        assert site_rel_err(out, ref) < SOAP_TOL
    # and the larger batch again, after the smaller one
    again = ctx.descriptor_noalloc(b_big).cpu().numpy()
    assert site_rel_err(again, ref_big) < SOAP_TOL


def test_noalloc_rejects_batches_beyond_its_array(setup):
    from soap_turbo_b200 import _lib
    from soap_turbo_b200 import synthetic as syn
    ctx = setup[0]
    w = syn.config(2, seed=13, scale=1.5)  # about 133 thousand pairs: > 64 MiB of rows
    b = ctx.batch(w.nl)
    with pytest.raises(_lib.SoapError) as e:
        ctx.descriptor_noalloc(b)
    assert e.value.code == 1 and "scratch" in str(e.value)
    # the entry point stays usable after the rejection
    ctx2_out = ctx.descriptor_noalloc(setup[2])
    ref = ctx.descriptor(setup[2], keep=False)
    assert site_rel_err(ctx2_out.cpu().numpy(), ref.cpu().numpy()) < SOAP_TOL


def test_noalloc_allocates_no_device_memory(setup):
    """After the first call on the device (which loads the static array), the
    free device memory does not move across further calls: neither the library
    nor the CUDA runtime allocates for them."""
    import torch
    ctx, b_big, b_small = setup
    out_big = torch.empty(b_big.n_sites, ctx.n_soap, dtype=torch.float64, device="cuda")
    out_small = torch.empty(b_small.n_sites, ctx.n_soap, dtype=torch.float64, device="cuda")
    ctx.descriptor_noalloc(b_big, out=out_big)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        ctx.descriptor_noalloc(b_small, out=out_small)
        ctx.descriptor_noalloc(b_big, out=out_big)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_reports_bad_inputs(setup):
    """A non-finite pair input of an allocation-free call is reported by
    soapb_check_inputs (from the static array's error word), with its index;
    the next clean call clears it."""
    from soap_turbo_b200 import _lib
    ctx, _, b_small = setup
    ctx.descriptor_noalloc(b_small)
    ctx.check_inputs()
    saved = b_small.rjs[7].item()
    b_small.rjs[7] = float("nan")
    try:
        ctx.descriptor_noalloc(b_small)
        with pytest.raises(_lib.SoapError) as e:
            ctx.check_inputs()
        assert e.value.code == 8 and "pair 7" in str(e.value)
    finally:
        b_small.rjs[7] = saved
    ctx.descriptor_noalloc(b_small)
    ctx.check_inputs()
