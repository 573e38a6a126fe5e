"""Parity of the CUDA paths with the FP64 oracle, through the C ABI.

Tolerances (conftest): mixed-precision descriptor max over sites of
|soap - ref|_inf / |ref|_inf <= 1e-6; force VJP max |pair - ref| / max |ref|
<= 1e-5; the plain FP64 path <= 1e-8.  Both paths get the same W and S
(the reference's W is not reproducible across LAPACK builds, so parity runs
feed one FP64 W to both sides)."""
import copy

import numpy as np
import pytest
import torch

import oracle as O
from conftest import FP64_TOL, SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import _lib, descriptor as D
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu

WORKLOADS = {
    "config1": lambda: syn.config(1, seed=7),
    "config2_quarter": lambda: syn.config(2, seed=11, scale=0.25),
    "config3_8structs": lambda: syn.config(3, seed=5, scale=1 / 64),
    "config4_512": lambda: syn.config(4, seed=9, scale=1 / 64),
    "config5_1024": lambda: syn.config(5, seed=13, scale=1 / 256),
}


class Run:
    def __init__(self, w, legacy=True, cart=True):
        self.w = w
        self.ctx = Context(w.hyper, legacy_filter_seed=legacy)
        W, S = self.ctx.basis()
        self.ref = O.get_soap(w.hyper, w.nl, W, S, do_derivatives=True, cart_der=cart,
                              legacy_filter_seed=legacy)
        self.b = self.ctx.batch(w.nl)
        rng = np.random.default_rng(17)
        self.G = rng.standard_normal((self.ctx.n_soap, w.nl.n_sites))  # Fortran G(n_sites, n_soap)
        self.Gt = torch.as_tensor(self.G).cuda()
        self.pair_ref = self.ref.contract(self.G, 1.0)


@pytest.fixture(scope="module", params=list(WORKLOADS))
def run(request):
    return Run(WORKLOADS[request.param]())


def test_mixed_descriptor_parity(run):
    soap = run.ctx.descriptor(run.b).cpu().numpy()
    run.ctx.check_inputs()
    assert site_rel_err(soap, run.ref.soap) <= SOAP_TOL


def test_mixed_vjp_parity(run):
    soap = run.ctx.descriptor(run.b)
    pair = run.ctx.contract(run.b, soap, run.Gt).cpu().numpy()
    assert max_rel_err(pair, run.pair_ref) <= VJP_TOL
    # translation invariance: each site's self pair is minus the sum of the others
    off = np.concatenate([[0], np.cumsum(run.w.nl.n_neigh)])
    for i in range(0, run.w.nl.n_sites, max(1, run.w.nl.n_sites // 20)):
        seg = pair[off[i]:off[i + 1]]
        assert np.abs(seg.sum(0)).max() <= 1e-12 * max(1.0, np.abs(seg).max())


def test_g_layouts_agree(run):
    soap = run.ctx.descriptor(run.b)
    p0 = run.ctx.contract(run.b, soap, run.Gt, g_layout=_lib.G_SITE_FASTEST)
    p1 = run.ctx.contract(run.b, soap, run.Gt.T.contiguous(), g_layout=_lib.G_SOAP_FASTEST)
    assert torch.equal(p0, p1)


def test_fp64_path_parity(run):
    cart = run.ref.soap_cart_der is not None
    soap, c = run.ctx.descriptor_fp64(run.b, cart=cart)
    assert site_rel_err(soap.cpu().numpy(), run.ref.soap) <= FP64_TOL
    if cart:
        assert max_rel_err(c.cpu().numpy(), run.ref.soap_cart_der) <= FP64_TOL
        pair = run.ctx.contract_cart_der(run.b, c, run.Gt).cpu().numpy()
        assert max_rel_err(pair, run.pair_ref) <= FP64_TOL


def test_fused_equals_two_calls(run):
    soap = run.ctx.descriptor(run.b)
    pair = run.ctx.contract(run.b, soap, run.Gt)
    s2, p2 = run.ctx.descriptor_and_vjp(run.b, run.Gt)
    assert torch.equal(soap, s2) and torch.equal(pair, p2)


def test_bitwise_deterministic(run):
    outs = []
    for _ in range(3):
        s = run.ctx.descriptor(run.b)
        p = run.ctx.contract(run.b, s, run.Gt)
        outs.append((s.clone(), p.clone()))
    for s, p in outs[1:]:
        assert torch.equal(s, outs[0][0]) and torch.equal(p, outs[0][1])


def test_unified_seed_parity():
    w = syn.config(1, seed=21)
    r = Run(w, legacy=False, cart=False)
    soap = r.ctx.descriptor(r.b)
    assert site_rel_err(soap.cpu().numpy(), r.ref.soap) <= SOAP_TOL
    pair = r.ctx.contract(r.b, soap, r.Gt).cpu().numpy()
    assert max_rel_err(pair, r.pair_ref) <= VJP_TOL


# ---------------------------------------------------------------- drop-in
def _dropin_args(w, soap, cart=None, do_der=True, compress=None):
    hp, nl = w.hyper, w.nl
    if compress is None and hp.compress_mode == "trivial":
        _, _, P_i, P_j, P_el = D.get_compress_indices("trivial", hp.alpha_max, hp.l_max)
        compress = (P_i, P_j, P_el)
    return dict(n_sites=nl.n_sites, n_neigh=nl.n_neigh, n_species=hp.n_species,
                species=nl.species.T, species_multiplicity=nl.species_multiplicity,
                n_atom_pairs=nl.n_pairs, mask=nl.mask.T.astype(bool), rjs=nl.rjs,
                thetas=nl.thetas, phis=nl.phis, alpha_max=hp.alpha_max, l_max=hp.l_max,
                rcut_hard=hp.rcut_hard, rcut_soft=hp.rcut_soft, nf=hp.nf,
                global_scaling=hp.global_scaling, atom_sigma_r=hp.atom_sigma_r,
                atom_sigma_r_scaling=hp.atom_sigma_r_scaling, atom_sigma_t=hp.atom_sigma_t,
                atom_sigma_t_scaling=hp.atom_sigma_t_scaling,
                amplitude_scaling=hp.amplitude_scaling,
                radial_enhancement=hp.radial_enhancement, central_weight=hp.central_weight,
                basis=hp.basis, scaling_mode=hp.scaling_mode, do_timing=False,
                do_derivatives=do_der, compress_soap=compress is not None,
                compress_P_nonzero=0 if compress is None else len(compress[0]),
                compress_P_i=None if compress is None else compress[0],
                compress_P_j=None if compress is None else compress[1],
                compress_P_el=None if compress is None else compress[2], soap=soap,
                soap_cart_der=cart)


@pytest.mark.parametrize("name", ["config1", "config2_quarter"])
def test_dropin_get_soap_and_contract(name):
    w = WORKLOADS[name]()
    r = Run(w, cart=False)
    W, S = r.ctx.basis()
    D.set_basis_matrices(W, S)
    try:
        soap = np.zeros((r.ctx.n_soap, w.nl.n_sites), order="F")
        D.get_soap(**_dropin_args(w, soap), contract=True)
        assert site_rel_err(soap.T, r.ref.soap) <= SOAP_TOL
        # identical to the context layer on device arrays
        s_ctx = r.ctx.descriptor(r.b).cpu().numpy()
        np.testing.assert_array_equal(soap.T, s_ctx)
        pair = np.zeros((3, w.nl.n_pairs), order="F")
        G = np.asfortranarray(r.G.T)  # G(n_sites, n_soap)
        D.soap_contract(soap, G, 1.0, pair)
        assert max_rel_err(pair.T, r.pair_ref) <= VJP_TOL
    finally:
        D.set_basis_matrices(None)


@pytest.mark.parametrize("pinned", [True, False])
def test_dropin_site_chunks_match_the_context_layer(pinned):
    """The drop-in layer runs batches of 1024 sites or more in site chunks whose
    copies overlap the kernels (1703 sites here: three chunks in get_soap from
    pageable arrays, one when the kernel writes a page-locked soap in place;
    four in soap_contract, the last of them half size); every site's result is
    computed the same way, so soap and pair equal the single-launch context
    calls bit for bit, from pinned or pageable host arrays."""
    import torch
    w = syn.config(2, seed=41)
    nl = w.nl
    assert nl.n_sites >= 4 * 384
    ctx = Context(w.hyper)
    W, S = ctx.basis()
    b = ctx.batch(nl)
    s_ctx = ctx.descriptor(b, keep=True)
    G = np.random.default_rng(5).standard_normal((ctx.n_soap, nl.n_sites))
    p_ctx = ctx.contract(b, s_ctx, torch.as_tensor(G).cuda()).cpu().numpy()
    s_ctx = s_ctx.cpu().numpy()

    def host(a):
        if not pinned:
            return np.asfortranarray(a)
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        out = t.numpy().reshape(a.shape, order="F")
        out[...] = a
        host.keep.append(t)
        return out
    host.keep = []
    D.set_basis_matrices(W, S)
    try:
        for _ in range(2):  # a second step reuses the streams, events and buffers
            soap = host(np.zeros((ctx.n_soap, nl.n_sites)))
            D.get_soap(**_dropin_args(w, soap), contract=True)
            np.testing.assert_array_equal(soap.T, s_ctx)
            pair = host(np.zeros((3, nl.n_pairs)))
            D.soap_contract(soap, host(G.T), 1.0, pair)
            np.testing.assert_array_equal(pair.T, p_ctx)
    finally:
        D.set_basis_matrices(None)


def _empty_sites(n, n_species, like):
    """n sites with no pairs (not even the self pair) in the layout of `like`."""
    mm = like.species.shape[1]
    sp = np.zeros((n, mm), np.int32)
    sp[:, 0] = like.species[0, 0]
    return syn.NeighbourList(
        n_sites=n, n_neigh=np.zeros(n, np.int32), rjs=np.zeros(0), thetas=np.zeros(0),
        phis=np.zeros(0), mask=np.zeros((n_species, 0), np.uint8), species=sp,
        species_multiplicity=np.ones(n, np.int32), site_atom=np.zeros(n, np.int64),
        neigh_atom=np.zeros(0, np.int64), disp=np.zeros((0, 3)))


def test_dropin_chunks_without_pairs():
    """Site chunks whose sites have no pairs at all: get_soap's chunk 1 of 3 and
    soap_contract's chunks 1 and 2 of 5 copy no pair rows and launch the pair
    kernel on an empty range; the result still equals the context layer's.
    (An empty site's descriptor is the central-atom term alone, the same for
    all of them, src/soap_turbo.f90:646-662.)"""
    import torch
    hp = syn.Hyper(alpha_max=[8, 8, 8], basis="poly3gauss", compress_mode="trivial")
    parts = []
    for seed in (61, 62):
        st = syn.random_structure(700, density=0.10, d_min=0.9, fractions=(0.4, 0.4, 0.2), seed=seed)
        parts.append(syn.neighbour_list(st, 5.0, 3, central_species=1))
    nl = syn.concatenate([parts[0], _empty_sites(1400, 3, parts[0]), parts[1]])
    n = nl.n_sites
    lo, hi = parts[0].n_sites, parts[0].n_sites + 1400
    assert lo <= n // 3 and hi >= 2 * n // 3          # get_soap's middle chunk is empty
    assert lo <= 2 * n // 9 and hi >= 6 * n // 9      # so are two of soap_contract's
    w = syn.Workload("gaps", hp, nl, [])
    ctx = Context(hp)
    W, S = ctx.basis()
    b = ctx.batch(nl)
    s_ctx = ctx.descriptor(b, keep=True)
    G = np.random.default_rng(9).standard_normal((ctx.n_soap, n))
    p_ctx = ctx.contract(b, s_ctx, torch.as_tensor(G).cuda()).cpu().numpy()
    s_ctx = s_ctx.cpu().numpy()
    np.testing.assert_array_equal(s_ctx[lo:hi], np.broadcast_to(s_ctx[lo], (hi - lo, ctx.n_soap)))
    D.set_basis_matrices(W, S)
    try:
        soap = np.zeros((ctx.n_soap, n), order="F")
        D.get_soap(**_dropin_args(w, soap), contract=True)
        np.testing.assert_array_equal(soap.T, s_ctx)
        pair = np.zeros((3, nl.n_pairs), order="F")
        D.soap_contract(soap, np.asfortranarray(G.T), 1.0, pair)
        np.testing.assert_array_equal(pair.T, p_ctx)
    finally:
        D.set_basis_matrices(None)


def test_dropin_batches_of_changing_size():
    """Consecutive drop-in steps on batches of 1 chunk, 3 chunks and 1 chunk
    again (chunk plans, events and staging areas re-used or grown between
    calls), with pageable and page-locked arrays mixed: every step equals the
    context layer bit for bit."""
    hp = syn.Hyper(alpha_max=[8, 8, 8], basis="poly3gauss", compress_mode="trivial")
    ctx = Context(hp)
    W, S = ctx.basis()
    D.set_basis_matrices(W, S)
    try:
        for n_atoms, seed, pin in ((600, 71, False), (4096, 72, True), (900, 73, False), (4096, 74, False)):
            st = syn.random_structure(n_atoms, density=0.10, d_min=0.9, fractions=(0.4, 0.4, 0.2), seed=seed)
            nl = syn.neighbour_list(st, 5.0, 3, central_species=1)
            w = syn.Workload("step", hp, nl, [st])
            b = ctx.batch(nl)
            s_ctx = ctx.descriptor(b, keep=True)
            G = np.random.default_rng(seed).standard_normal((ctx.n_soap, nl.n_sites))
            p_ctx = ctx.contract(b, s_ctx, torch.as_tensor(G).cuda()).cpu().numpy()
            s_ctx = s_ctx.cpu().numpy()
            keep = []

            def host(a):
                if not pin:
                    return np.asfortranarray(a)
                t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
                keep.append(t)
                out = t.numpy().reshape(a.shape, order="F")
                out[...] = a
                return out
            soap = host(np.zeros((ctx.n_soap, nl.n_sites)))
            D.get_soap(**_dropin_args(w, soap), contract=True)
            np.testing.assert_array_equal(soap.T, s_ctx)
            pair = np.zeros((3, nl.n_pairs), order="F")
            D.soap_contract(soap, host(G.T), 1.0, pair)
            np.testing.assert_array_equal(pair.T, p_ctx)
    finally:
        D.set_basis_matrices(None)


def test_dropin_soap_cart_der_is_fp64():
    w = WORKLOADS["config1"]()
    r = Run(w, cart=True)
    W, S = r.ctx.basis()
    D.set_basis_matrices(W, S)
    try:
        soap = np.zeros((r.ctx.n_soap, w.nl.n_sites), order="F")
        cart = np.zeros((3, r.ctx.n_soap, w.nl.n_pairs), order="F")
        D.get_soap(**_dropin_args(w, soap, cart=cart), contract=False)
        assert site_rel_err(soap.T, r.ref.soap) <= FP64_TOL
        ref = np.transpose(r.ref.soap_cart_der, (2, 1, 0))
        assert max_rel_err(cart, ref) <= FP64_TOL
        # contract after a non-contract call is refused (src/soap_turbo.f90:1744-1747)
        with pytest.raises(_lib.SoapError) as e:
            D.soap_contract(soap, np.asfortranarray(r.G.T), 1.0, np.zeros((3, w.nl.n_pairs), order="F"))
        assert e.value.code == 3
    finally:
        D.set_basis_matrices(None)


def test_dropin_fp64_precision_contract():
    w = WORKLOADS["config2_quarter"]()
    r = Run(w, cart=False)
    W, S = r.ctx.basis()
    D.set_basis_matrices(W, S)
    D.set_precision("fp64")
    try:
        soap = np.zeros((r.ctx.n_soap, w.nl.n_sites), order="F")
        D.get_soap(**_dropin_args(w, soap), contract=True)
        assert site_rel_err(soap.T, r.ref.soap) <= FP64_TOL
        pair = np.zeros((3, w.nl.n_pairs), order="F")
        D.soap_contract(soap, np.asfortranarray(r.G.T), 1.0, pair)
        assert max_rel_err(pair.T, r.pair_ref) <= FP64_TOL
    finally:
        D.set_precision("mixed")
        D.set_basis_matrices(None)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_dropin_do_timing(precision, capfd):
    """do_timing (src/soap_turbo.f90:139-169): the call prints its timing table
    (GPU times of the copies and kernels; the mixed path then runs its kernels
    unchunked) and returns the same soap as without it; soap_contract works
    after it."""
    w = syn.config(2, seed=43)
    hp, nl = w.hyper, w.nl
    ctx = Context(hp)
    W, S = ctx.basis()
    G = np.asfortranarray(np.random.default_rng(6).standard_normal((nl.n_sites, ctx.n_soap)))
    D.set_basis_matrices(W, S)
    D.set_precision(precision)
    try:
        out = {}
        for timing in (False, True):
            args = _dropin_args(w, np.zeros((ctx.n_soap, nl.n_sites), order="F"))
            args["do_timing"] = timing
            D.get_soap(**args, contract=True)
            pair = np.zeros((3, nl.n_pairs), order="F")
            D.soap_contract(args["soap"], G, 1.0, pair)
            out[timing] = (args["soap"], pair)
        printed = capfd.readouterr().out
        assert printed.count("SOAP timings") == 1
        for line in ("Host to device copies:", "Descriptor kernels:", "Device to host copies:"):
            assert line in printed
        np.testing.assert_array_equal(out[True][0], out[False][0])
        np.testing.assert_array_equal(out[True][1], out[False][1])
    finally:
        D.set_precision("mixed")
        D.set_basis_matrices(None)


# ---------------------------------------------------------------- gradients
class SoapFunction(torch.autograd.Function):
    """soap(disp) for a fixed topology; backward is the adjoint contract.
    Test-harness only: the library exposes the VJP through its C ABI."""

    @staticmethod
    def forward(fctx, disp, ctx, b):
        r = torch.sqrt((disp * disp).sum(1))
        nz = r > 0
        th = torch.zeros_like(r)
        ph = torch.zeros_like(r)
        th[nz] = torch.acos(torch.clamp(disp[nz, 2] / r[nz], -1.0, 1.0))
        ph[nz] = torch.atan2(disp[nz, 1], disp[nz, 0])
        b.rjs.copy_(r)
        b.thetas.copy_(th)
        b.phis.copy_(ph)
        soap = ctx.descriptor(b, keep=True)
        fctx.save_for_backward(soap, nz)
        fctx.ctx, fctx.b = ctx, b
        return soap

    @staticmethod
    def backward(fctx, grad_soap):
        soap, nz = fctx.saved_tensors
        pair = fctx.ctx.contract(fctx.b, soap, grad_soap.contiguous(), g_layout=_lib.G_SOAP_FASTEST)
        pair = pair * nz[:, None]  # self pairs: their displacement is identically zero
        return pair, None, None


def test_autograd_vjp_against_finite_differences():
    # config 4 shapes (poly3, single species), FD on a 64-atom subset with
    # h = 1e-4 A and the unified filter seed; FD values from the FP64 path
    w = syn.config(4, seed=31, scale=1 / 64)
    st, hp, nl = w.structures[0], w.hyper, w.nl
    ctx = Context(hp, legacy_filter_seed=False)
    b = ctx.batch(nl)
    n_atoms = st.positions.shape[0]
    rng = np.random.default_rng(3)
    G = torch.as_tensor(rng.standard_normal((nl.n_sites, ctx.n_soap))).cuda()
    pos = torch.as_tensor(st.positions).cuda().requires_grad_(True)
    shift = torch.as_tensor(nl.disp - (st.positions[nl.neigh_atom] - st.positions[
        np.repeat(nl.site_atom, nl.n_neigh)])).cuda()
    site_atom = torch.as_tensor(np.repeat(nl.site_atom, nl.n_neigh)).cuda()
    neigh = torch.as_tensor(nl.neigh_atom).cuda()
    disp = pos[neigh] - pos[site_atom] + shift
    soap = SoapFunction.apply(disp, ctx, b)
    (soap * G).sum().backward()
    grad = pos.grad.cpu().numpy()
    ctx64 = Context(hp, legacy_filter_seed=False)

    def L(p):
        nl2 = syn.neighbour_list(syn.Structure(p, st.box, st.species), 5.0, 1)
        s, _ = ctx64.descriptor_fp64(ctx64.batch(nl2))
        return float((s * G).sum())
    h = 1e-4
    fd = np.zeros((64, 3))
    for a in range(64):
        for c in range(3):
            p, m = st.positions.copy(), st.positions.copy()
            p[a, c] += h
            m[a, c] -= h
            fd[a, c] = (L(p) - L(m)) / (2 * h)
    assert max_rel_err(grad[:64], fd) <= VJP_TOL
    assert n_atoms >= 64


# ---------------------------------------------------------------- full sizes
def _rotated(nl, R):
    d = nl.disp @ R.T
    r = np.sqrt((d * d).sum(1))
    th = np.zeros_like(r)
    ph = np.zeros_like(r)
    nz = r > 0
    th[nz] = np.arccos(np.clip(d[nz, 2] / r[nz], -1, 1))
    ph[nz] = np.arctan2(d[nz, 1], d[nz, 0])
    out = copy.copy(nl)
    out.rjs, out.thetas, out.phis = r, th, ph
    return out


@pytest.mark.parametrize("idx", [2, 4, 5])
def test_full_size_properties(idx):
    w = syn.config(idx, seed=100 + idx)
    ctx = Context(w.hyper)
    b = ctx.batch(w.nl)
    s1 = ctx.descriptor(b)
    # unit norm (src/soap_turbo.f90:904-909)
    nrm = torch.linalg.norm(s1, dim=1).cpu().numpy()
    assert np.abs(nrm - 1.0).max() < 1e-6
    # rotation invariance
    R = np.linalg.qr(np.random.default_rng(idx).standard_normal((3, 3)))[0]
    s2 = ctx.descriptor(ctx.batch(_rotated(w.nl, R)))
    assert site_rel_err(s2.cpu().numpy(), s1.cpu().numpy()) <= 2 * SOAP_TOL
    # determinism and the self-pair sum of the VJP
    s1 = ctx.descriptor(b)
    G = torch.randn(ctx.n_soap, w.nl.n_sites, dtype=torch.float64, device="cuda")
    p1 = ctx.contract(b, s1, G)
    s3 = ctx.descriptor(b)
    p3 = ctx.contract(b, s3, G)
    assert torch.equal(s1, s3) and torch.equal(p1, p3)
    site = torch.as_tensor(np.repeat(np.arange(w.nl.n_sites), w.nl.n_neigh)).cuda()
    tot = torch.zeros(w.nl.n_sites, 3, dtype=torch.float64, device="cuda").index_add_(0, site, p1)
    assert float(tot.abs().max()) <= 1e-10 * float(p1.abs().max())
