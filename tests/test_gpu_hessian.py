"""Central-atom Hessian (get_soap_central_hessian, src/soap_turbo.f90:1151-1700)
on the GPU against the FP64 oracle's restatement, which is pinned by finite
differences of its own force VJP (test_oracle.py).

Tolerance: FP64_TOL on max |hess - ref| / max |ref|, as for the plain FP64
descriptor path, except for alpha_max = 10 with poly3gauss: there |W| is 6e6
and the radial second derivatives amplify rounding further -- moving every
distance by 2e-16 relative moves the oracle's own Hessian by 4e-8 -- so that
case is held to 5e-7."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import FP64_TOL, max_rel_err
from soap_turbo_b200 import _lib, descriptor as D
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu

CASES = {
    # two species, poly3gauss, sigma scaling: the oracle's finite-difference case
    "gauss_2sp": dict(alpha_max=[4, 4], l_max=4, basis="poly3gauss", atom_sigma_t_scaling=0.05,
                      atom_sigma_r_scaling=0.05),
    # three species, the benchmark's hyperparameters, compressed
    "poly3_3sp_trivial": dict(alpha_max=[8, 8, 8], l_max=8, compress_mode="trivial"),
    # radial enhancement, central weight, amplitude scaling other than 1
    "poly3_enh_cw": dict(alpha_max=[6, 5], l_max=6, radial_enhancement=2, central_weight=0.5,
                         amplitude_scaling=2.0, atom_sigma_r_scaling=0.1),
    # alpha above 8: the wide radial instantiation
    "gauss_alpha10": dict(alpha_max=[10], l_max=5, basis="poly3gauss", radial_enhancement=1),
    # a Darby compression mode: its map spreads each output over several (n, n', l)
    "gauss_3sp_darby": dict(alpha_max=[4, 4, 4], l_max=4, basis="poly3gauss", compress_mode="1_1"),
}
TOL = {"gauss_alpha10": 5e-7}


def _case(name, seed=3, n_atoms=28):
    hp = syn.Hyper(**CASES[name])
    fr = tuple([1.0 / hp.n_species] * hp.n_species)
    st = syn.random_structure(n_atoms, density=0.1, d_min=1.0, fractions=fr, seed=seed)
    nl = syn.neighbour_list(st, 5.0, hp.n_species)
    return hp, nl


def _oracle(hp, nl, W, S, n_vec, seed=1):
    ref = O.get_soap(hp, nl, W, S, do_derivatives=True, legacy_filter_seed=False, hessian=True)
    vecs = np.random.default_rng(seed).standard_normal((nl.n_sites, n_vec, ref.soap.shape[1]))
    hess, err = ref.central_hessian(vecs)
    assert err < 1e-10
    return ref, vecs, hess


@pytest.mark.parametrize("name", list(CASES))
def test_central_hessian_matches_the_oracle(name):
    hp, nl = _case(name)
    ctx = Context(hp, legacy_filter_seed=False)
    W, S = ctx.basis()
    n_vec = 2
    ref, vecs, href = _oracle(hp, nl, W, S, n_vec)
    b = ctx.batch(nl)
    soap_t = torch.as_tensor(np.ascontiguousarray(ref.soap)).cuda()
    vecs_t = torch.as_tensor(vecs).cuda()
    hess = ctx.central_hessian(b, vecs_t, soap=soap_t).cpu().numpy()
    ctx.check_inputs()
    tol = TOL.get(name, FP64_TOL)
    assert max_rel_err(hess, href) <= tol
    # the descriptor the call computes itself in place of the caller's
    hess2 = ctx.central_hessian(b, vecs_t).cpu().numpy()
    assert max_rel_err(hess2, href) <= tol
    # each site's row of blocks sums to zero (a rigid shift leaves q alone)
    off = np.concatenate([[0], np.cumsum(nl.n_neigh)])
    scale = np.abs(hess).max()
    for i in range(nl.n_sites):
        assert np.abs(hess[off[i]:off[i + 1]].sum(axis=0)).max() <= 1e-11 * scale


def test_many_weight_vectors_and_repeat_calls():
    """More weight vectors than the kernel contracts per pass (8), and a second
    call on the same context giving the same bits."""
    hp, nl = _case("gauss_2sp", seed=9, n_atoms=20)
    ctx = Context(hp, legacy_filter_seed=False)
    W, S = ctx.basis()
    ref, vecs, href = _oracle(hp, nl, W, S, n_vec=11, seed=4)
    b = ctx.batch(nl)
    vecs_t = torch.as_tensor(vecs).cuda()
    soap_t = torch.as_tensor(np.ascontiguousarray(ref.soap)).cuda()
    h1 = ctx.central_hessian(b, vecs_t, soap=soap_t)
    h2 = ctx.central_hessian(b, vecs_t, soap=soap_t)
    assert torch.equal(h1, h2)
    assert max_rel_err(h1.cpu().numpy(), href) <= FP64_TOL


@pytest.mark.parametrize("basis", ["poly3", "poly3gauss"])
def test_edge_sites(basis):
    """A site with only itself, a neighbour beyond the cutoff (its block stays
    zero), neighbours on the poles and at a very short distance, a site whose
    descriptor is zero (poly3gauss, central weight 0, nothing in range: the
    norm floor), and ordinary sites beside them."""
    import dataclasses
    from test_gpu_edge import make_nl, random_sites
    rng = np.random.default_rng(11)
    if basis == "poly3":
        hp = syn.Hyper(alpha_max=[6], l_max=5, basis="poly3")
        sites = [(0, []), (0, [(6.0, 1.0, 0.5, 1), (2.0, 0.0, 0.0, 1), (3.0, np.pi, 1.0, 1)]),
                 (0, [(0.05, 1.2, -2.0, 1), (4.99, 0.7, 0.3, 1)])] + random_sites(rng, 4, 1, 5, 20)
        nl = make_nl(sites, 1)
    else:
        hp = syn.Hyper(alpha_max=[5, 5, 5], l_max=5, basis="poly3gauss", central_weight=[1.0, 0.0, 1.0])
        sites = [(1, []), (1, [(7.0, 0.3, 0.2, 1)]), (0, [(1.5, 0.0, 1.0, 4), (2.5, np.pi, 0.0, 2)])] + \
            random_sites(rng, 4, 3, 5, 20)
        nl = make_nl(sites, 3)
    ctx = Context(hp, legacy_filter_seed=False)
    W, S = ctx.basis()
    ref, vecs, href = _oracle(hp, nl, W, S, 2, seed=3)
    b = ctx.batch(nl)
    hess = ctx.central_hessian(b, torch.as_tensor(vecs).cuda(),
                               soap=torch.as_tensor(np.ascontiguousarray(ref.soap)).cuda()).cpu().numpy()
    ctx.check_inputs()
    assert np.isfinite(hess).all()
    assert max_rel_err(hess, href) <= FP64_TOL
    off = np.concatenate([[0], np.cumsum(nl.n_neigh)])
    assert np.abs(hess[off[0]:off[1]]).max() == 0.0  # a site with only itself
    if basis == "poly3":
        assert np.abs(hess[off[1] + 1]).max() == 0.0  # the neighbour beyond the cutoff


def test_legacy_seed_context_is_refused():
    hp, nl = _case("gauss_2sp", n_atoms=12)
    ctx = Context(hp, legacy_filter_seed=True)
    b = ctx.batch(nl)
    vecs = torch.zeros((nl.n_sites, 1, ctx.n_soap), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.SoapError) as e:
        ctx.central_hessian(b, vecs)
    assert e.value.code == 1
    # poly3operator has no second radial derivatives (src/soap_turbo.f90:485-489)
    op = syn.Hyper(alpha_max=[4, 4], l_max=4, basis="poly3operator")
    ctx = Context(op, legacy_filter_seed=False)
    with pytest.raises(_lib.SoapError) as e:
        ctx.central_hessian(ctx.batch(nl), torch.zeros((nl.n_sites, 1, ctx.n_soap), dtype=torch.float64,
                                                       device="cuda"))
    assert e.value.code == 5


def test_more_weight_vectors_than_one_pass_holds():
    """Past the kernel's shared-memory limit (about 100 vectors at this
    definition) the call works in chunks of vectors; every vector's block
    depends on that vector alone, so the result equals, bit for bit, a call on
    any subset -- here one straddling a chunk boundary."""
    hp, nl = _case("gauss_2sp", n_atoms=12)
    ctx = Context(hp, legacy_filter_seed=False)
    b = ctx.batch(nl)
    g = torch.Generator(device="cuda").manual_seed(7)
    vecs = torch.randn((nl.n_sites, 230, ctx.n_soap), dtype=torch.float64, device="cuda", generator=g)
    h_all = ctx.central_hessian(b, vecs)
    for lo, hi in ((0, 5), (95, 110), (220, 230)):
        h_part = ctx.central_hessian(b, vecs[:, lo:hi].contiguous())
        assert torch.equal(h_all[:, lo:hi], h_part)


def _dropin_args(hp, nl, soap, P):
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
                do_derivatives=True, compress_soap=P is not None,
                compress_P_nonzero=0 if P is None else len(P[0]),
                compress_P_i=None if P is None else P[0], compress_P_j=None if P is None else P[1],
                compress_P_el=None if P is None else P[2], soap=soap, soap_cart_der=None)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_dropin_central_hessian(precision):
    """The reference's call sequence: soap_hessian_enabled, get_soap with
    do_derivatives, then get_soap_central_hessian on the soap it returned."""
    hp, nl = _case("poly3_3sp_trivial", seed=6, n_atoms=24)
    ctx = Context(hp, legacy_filter_seed=False)
    W, S = ctx.basis()
    _, _, P_i, P_j, P_el = D.get_compress_indices("trivial", hp.alpha_max, hp.l_max)
    D.set_basis_matrices(W, S)
    D.set_legacy_filter_seed(False)
    D.set_precision(precision)
    D.set_soap_hessian_enabled(True)
    try:
        soap = np.zeros((ctx.n_soap, nl.n_sites), order="F")
        D.get_soap(**_dropin_args(hp, nl, soap, (P_i, P_j, P_el)), contract=True)
        vecs = np.asfortranarray(
            np.random.default_rng(2).standard_normal((ctx.n_soap, 3, nl.n_sites)))
        hess = np.zeros((3, 3, 3, nl.n_pairs), order="F")
        hargs = dict(n_sites=nl.n_sites, n_neigh=nl.n_neigh, n_atom_pairs=nl.n_pairs,
                     n_species=hp.n_species, mask=nl.mask.T.astype(bool), rjs=nl.rjs,
                     thetas=nl.thetas, phis=nl.phis, l_max=hp.l_max, rcut_hard=hp.rcut_hard,
                     atom_sigma_t=hp.atom_sigma_t, atom_sigma_t_scaling=hp.atom_sigma_t_scaling,
                     compress_soap=True, compress_P_nonzero=len(P_i), compress_P_i=P_i,
                     compress_P_j=P_j, compress_P_el=P_el, soap=soap, n_vec=3, vecs=vecs,
                     hess=hess)
        D.get_soap_central_hessian(**hargs)
        # the oracle on the same soap the drop-in call returned
        ref = O.get_soap(hp, nl, W, S, do_derivatives=True, legacy_filter_seed=False, hessian=True)
        ref.soap = np.ascontiguousarray(soap.T)
        href, _ = ref.central_hessian(np.ascontiguousarray(np.transpose(vecs, (2, 1, 0))))
        got = np.transpose(hess, (3, 2, 1, 0))  # [k, v, b, a]
        assert max_rel_err(got, href) <= FP64_TOL
        # the contract state of the same get_soap is still there
        pair = np.zeros((3, nl.n_pairs), order="F")
        D.soap_contract(soap, np.zeros((nl.n_sites, ctx.n_soap), order="F"), 1.0, pair)
        # a batch with other extents is refused (src/soap_turbo.f90:1220-1227)
        bad = dict(hargs, l_max=hp.l_max - 1)
        with pytest.raises(_lib.SoapError) as e:
            D.get_soap_central_hessian(**bad)
        assert e.value.code == 10
        # get_soap without do_derivatives clears the state
        D.get_soap(**dict(_dropin_args(hp, nl, soap, (P_i, P_j, P_el)), do_derivatives=False))
        with pytest.raises(_lib.SoapError) as e:
            D.get_soap_central_hessian(**hargs)
        assert e.value.code == 10
    finally:
        D.set_soap_hessian_enabled(False)
        D.set_precision("mixed")
        D.set_legacy_filter_seed(True)
        D.set_basis_matrices(None)


def test_two_species_atoms():
    """Neighbours and central atoms that carry two species (mask rows with
    both bits, species_multiplicity 2), as in test_gpu_edge, through the
    Hessian."""
    import dataclasses
    hp, nl = _case("gauss_2sp", seed=5)
    rng = np.random.default_rng(4)
    mask = nl.mask.copy()
    mask[:, rng.random(nl.n_pairs) < 0.2] = 1
    first = np.concatenate([[0], np.cumsum(nl.n_neigh)[:-1]])
    dual = np.arange(nl.n_sites) % 3 == 0
    mask[:, first[dual]] = 1
    species = np.zeros((nl.n_sites, 2), np.int32)
    species[:, 0] = nl.species[:, 0]
    species[dual] = (1, 2)
    nl = dataclasses.replace(nl, mask=mask, species=species,
                             species_multiplicity=np.where(dual, 2, 1).astype(np.int32))
    ctx = Context(hp, legacy_filter_seed=False)
    W, S = ctx.basis()
    ref, vecs, href = _oracle(hp, nl, W, S, 2)
    hess = ctx.central_hessian(ctx.batch(nl), torch.as_tensor(vecs).cuda()).cpu().numpy()
    assert max_rel_err(hess, href) <= FP64_TOL


def test_neighbour_list_with_a_skin():
    """Pairs beyond rcut_max (a list built to 5.6 A for rcut_hard 5.0) add
    nothing: their Hessian blocks are zero and the others match the oracle."""
    hp = syn.Hyper(**CASES["gauss_2sp"])
    st = syn.random_structure(28, density=0.1, d_min=1.0, fractions=(0.5, 0.5), seed=6)
    nl = syn.neighbour_list(st, 5.6, hp.n_species)
    assert (nl.rjs >= 5.0).any()
    ctx = Context(hp, legacy_filter_seed=False)
    W, S = ctx.basis()
    ref, vecs, href = _oracle(hp, nl, W, S, 2)
    hess = ctx.central_hessian(ctx.batch(nl), torch.as_tensor(vecs).cuda()).cpu().numpy()
    assert max_rel_err(hess, href) <= FP64_TOL
    assert not hess[nl.rjs >= 5.0].any()
