"""The poly3operator basis (src/soap_turbo_radial.f90:1549-2141) on the GPU
against the FP64 oracle's restatement, which test_oracle.py pins by quadrature
of the integrand and by finite differences.

Tolerances as for the other bases (conftest): mixed descriptor SOAP_TOL, mixed
force VJP VJP_TOL, plain FP64 path FP64_TOL; both sides get the context's W."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import FP64_TOL, SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import descriptor as D
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu

CASES = {
    # one species at the defaults (rcut 5.0 / 4.5): soft and buffer zones
    "op_1sp": dict(alpha_max=[8], l_max=8, basis="poly3operator"),
    # two species, a wide buffer, sigma scaling, central weight, enhancement,
    # amplitude exponent other than 0 and 1
    "op_2sp": dict(alpha_max=[6, 7], l_max=6, basis="poly3operator", rcut_soft=4.0,
                   atom_sigma_r_scaling=0.05, central_weight=0.5, radial_enhancement=1,
                   amplitude_scaling=1.5),
    # alpha 11 (the tables' limit, the wide instantiation); no buffer zone;
    # amplitude 1/sigma
    "op_alpha11": dict(alpha_max=[11], l_max=5, basis="poly3operator", rcut_soft=5.0,
                       amplitude_scaling=0.0, radial_enhancement=2),
    # species with different rcut_hard: the basis has no rcut_hard cut of its own
    "op_2rcut": dict(alpha_max=[5, 5], l_max=4, basis="poly3operator", rcut_hard=[5.0, 4.0],
                     rcut_soft=[4.5, 3.5]),
    # three species, compressed
    "op_3sp_trivial": dict(alpha_max=[8, 8, 8], l_max=8, basis="poly3operator",
                           compress_mode="trivial"),
}


def _case(name, seed=5, n_atoms=40):
    hp = syn.Hyper(**CASES[name])
    fr = tuple([1.0 / hp.n_species] * hp.n_species)
    st = syn.random_structure(n_atoms, density=0.1, d_min=1.0, fractions=fr, seed=seed)
    nl = syn.neighbour_list(st, float(np.max(hp.arr("rcut_hard"))), hp.n_species)
    return hp, nl


@pytest.fixture(scope="module", params=list(CASES))
def case(request):
    hp, nl = _case(request.param)
    ctx = Context(hp)
    W, S = ctx.basis()
    ref = O.get_soap(hp, nl, W, S, do_derivatives=True, cart_der=True)
    G = np.random.default_rng(3).standard_normal((ctx.n_soap, nl.n_sites))
    return hp, nl, ctx, ref, G


def test_mixed_descriptor_and_vjp(case):
    hp, nl, ctx, ref, G = case
    b = ctx.batch(nl)
    soap = ctx.descriptor(b, keep=True)
    ctx.check_inputs()
    assert site_rel_err(soap.cpu().numpy(), ref.soap) <= SOAP_TOL
    pair = ctx.contract(b, soap, torch.as_tensor(G).cuda()).cpu().numpy()
    assert max_rel_err(pair, ref.contract(G, 1.0)) <= VJP_TOL


def test_fp64_path(case):
    hp, nl, ctx, ref, G = case
    b = ctx.batch(nl)
    soap, cart = ctx.descriptor_fp64(b, cart=True)
    assert site_rel_err(soap.cpu().numpy(), ref.soap) <= FP64_TOL
    assert max_rel_err(cart.cpu().numpy(), ref.soap_cart_der) <= FP64_TOL


def test_dropin_matches_the_context_layer():
    hp, nl = _case("op_2sp", seed=8)
    ctx = Context(hp)
    W, S = ctx.basis()
    b = ctx.batch(nl)
    s_ctx = ctx.descriptor(b, keep=False).cpu().numpy()
    D.set_basis_matrices(W, S)
    try:
        soap = np.zeros((ctx.n_soap, nl.n_sites), order="F")
        D.get_soap(n_sites=nl.n_sites, n_neigh=nl.n_neigh, n_species=hp.n_species, species=nl.species.T,
                   species_multiplicity=nl.species_multiplicity, n_atom_pairs=nl.n_pairs,
                   mask=nl.mask.T.astype(bool), rjs=nl.rjs, thetas=nl.thetas, phis=nl.phis,
                   alpha_max=hp.alpha_max, l_max=hp.l_max, rcut_hard=hp.rcut_hard, rcut_soft=hp.rcut_soft,
                   nf=hp.nf, global_scaling=hp.global_scaling, atom_sigma_r=hp.atom_sigma_r,
                   atom_sigma_r_scaling=hp.atom_sigma_r_scaling, atom_sigma_t=hp.atom_sigma_t,
                   atom_sigma_t_scaling=hp.atom_sigma_t_scaling, amplitude_scaling=hp.amplitude_scaling,
                   radial_enhancement=hp.radial_enhancement, central_weight=hp.central_weight,
                   basis="poly3operator", scaling_mode=hp.scaling_mode, do_timing=False, do_derivatives=False,
                   compress_soap=False, compress_P_nonzero=0, compress_P_i=None, compress_P_j=None,
                   compress_P_el=None, soap=soap, soap_cart_der=None)
        np.testing.assert_array_equal(soap.T, s_ctx)
    finally:
        D.set_basis_matrices(None)


@pytest.mark.parametrize("basis", ["poly3operator", "poly3gauss"])
def test_neighbour_list_with_a_skin(basis):
    """A neighbour list built beyond the cutoff (5.6 A for rcut_hard 5.0, as an
    MD code's list with a skin): pairs at or beyond rcut_max have no angular
    coefficients in the reference (src/soap_turbo_angular.f90:549-574), so they
    add nothing -- also for poly3operator, whose radial part has no rcut_hard
    cut of its own."""
    hp = syn.Hyper(alpha_max=[6, 6], l_max=6, basis=basis)
    st = syn.random_structure(40, density=0.1, d_min=1.0, fractions=(0.5, 0.5), seed=12)
    nl = syn.neighbour_list(st, 5.6, 2)
    assert (nl.rjs >= 5.0).any()
    ctx = Context(hp)
    W, S = ctx.basis()
    ref = O.get_soap(hp, nl, W, S, do_derivatives=True, cart_der=True)
    b = ctx.batch(nl)
    soap = ctx.descriptor(b, keep=True)
    assert site_rel_err(soap.cpu().numpy(), ref.soap) <= SOAP_TOL
    G = np.random.default_rng(4).standard_normal((ctx.n_soap, nl.n_sites))
    pair = ctx.contract(b, soap, torch.as_tensor(G).cuda()).cpu().numpy()
    assert max_rel_err(pair, ref.contract(G, 1.0)) <= VJP_TOL
    assert not pair[nl.rjs >= 5.0].any()
    s64, cart = ctx.descriptor_fp64(b, cart=True)
    assert site_rel_err(s64.cpu().numpy(), ref.soap) <= FP64_TOL
    assert max_rel_err(cart.cpu().numpy(), ref.soap_cart_der) <= FP64_TOL
