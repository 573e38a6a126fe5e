"""Edge cases of the CUDA paths against the oracle: the reference's branches
(empty spheres, cutoff edges, poles, small-x series, zero-width filter,
amplitude/enhancement/central-weight variants, multi-species masks) and the
kernels' own (chunking of large sites, several entry rounds, empty sites and
batches, input checks)."""
import dataclasses

import numpy as np
import pytest
import torch

import oracle as O
from conftest import FP64_TOL, SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import _lib, descriptor as D
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu


def make_nl(sites, n_species):
    """sites: list of (central_species, [(r, theta, phi, species_bits), ...])."""
    n_neigh, rjs, th, ph, masks, species = [], [], [], [], [], []
    for cs, neigh in sites:
        rows = [(0.0, 0.0, 0.0, 1 << cs)] + list(neigh)
        n_neigh.append(len(rows))
        species.append([cs + 1])
        for r, t, p, bits in rows:
            rjs.append(r)
            th.append(t)
            ph.append(p)
            masks.append([(bits >> s) & 1 for s in range(n_species)])
    n_pairs = len(rjs)
    mask = np.asarray(masks, dtype=np.uint8).T.copy() if n_pairs else np.zeros((n_species, 0), np.uint8)
    disp = np.zeros((n_pairs, 3))
    return syn.NeighbourList(
        n_sites=len(sites), n_neigh=np.asarray(n_neigh, np.int32), rjs=np.asarray(rjs, float),
        thetas=np.asarray(th, float), phis=np.asarray(ph, float), mask=mask,
        species=np.asarray(species, np.int32).reshape(len(sites), 1),
        species_multiplicity=np.ones(len(sites), np.int32), site_atom=np.arange(len(sites)),
        neigh_atom=np.zeros(n_pairs, np.int64), disp=disp)


def random_sites(rng, n_sites, n_species, lo=12, hi=60, rmax=5.3):
    sites = []
    for _ in range(n_sites):
        k = int(rng.integers(lo, hi))
        neigh = []
        for _ in range(k):
            r = float(rng.uniform(0.9, rmax))
            neigh.append((r, float(np.arccos(rng.uniform(-1, 1))), float(rng.uniform(-np.pi, np.pi)),
                          1 << int(rng.integers(0, n_species))))
        sites.append((int(rng.integers(0, n_species)), neigh))
    return sites


def check(hp, nl, legacy=True, soap_tol=SOAP_TOL, vjp_tol=VJP_TOL, fp64=True):
    ctx = Context(hp, legacy_filter_seed=legacy)
    W, S = ctx.basis()
    ref = O.get_soap(hp, nl, W, S, do_derivatives=True, cart_der=False, legacy_filter_seed=legacy)
    b = ctx.batch(nl)
    soap = ctx.descriptor(b)
    ctx.check_inputs()
    s = soap.cpu().numpy()
    rng = np.random.default_rng(7)
    G = rng.standard_normal((ctx.n_soap, nl.n_sites))
    pair = ctx.contract(b, soap, torch.as_tensor(G).cuda()).cpu().numpy()
    pref = ref.contract(G, 1.0)
    ok = np.abs(ref.soap).max(axis=1) > 0
    if ok.any():
        assert site_rel_err(s[ok], ref.soap[ok]) <= soap_tol
    assert np.abs(s[~ok]).max(initial=0.0) == 0.0
    if np.abs(pref).max() > 0:
        assert max_rel_err(pair, pref) <= vjp_tol
    else:
        assert np.abs(pair).max() == 0.0
    if fp64:
        s64, _ = ctx.descriptor_fp64(b)
        if ok.any():
            assert site_rel_err(s64.cpu().numpy()[ok], ref.soap[ok]) <= FP64_TOL
    return s, ref


H3 = syn.Hyper(alpha_max=[8], basis="poly3")
HG = syn.Hyper(alpha_max=[8, 8, 8], basis="poly3gauss", compress_mode="trivial")


def test_isolated_sites_and_empty_spheres():
    nl = make_nl([(0, []), (0, [(6.0, 1.0, 0.5, 1)]), (0, [(2.0, 1.0, 0.5, 1)])], 1)
    s, ref = check(H3, nl)
    # poly3 with a central weight: the self pair alone gives an l = 0 descriptor
    assert np.abs(ref.soap[0]).max() > 0
    # poly3gauss with central_weight 0 and nothing in range: soap is zero and
    # the norm floor (src/soap_turbo.f90:806-809) keeps it finite
    hp = dataclasses.replace(HG, central_weight=[1.0, 0.0, 1.0])
    nl = make_nl([(1, []), (1, [(7.0, 0.3, 0.2, 1)]), (0, [(1.5, 2.0, 1.0, 4)])], 3)
    s, ref = check(hp, nl)
    assert np.abs(s[0]).max() == 0.0 and np.abs(s[1]).max() == 0.0


def test_cutoff_edges_poles_and_small_distances():
    neigh = [(4.999999, 1.0, 0.1, 1), (5.0, 1.2, 0.3, 1), (5.2, 0.4, 0.3, 1), (4.5, 0.0, 0.7, 1),
             (3.0, np.pi, -0.4, 1), (2.0, 0.0, 0.0, 1), (1.0, np.pi / 2, np.pi, 1),
             (1.0, np.pi / 2, -np.pi, 1), (1e-3, 0.9, 0.2, 1), (2e-5, 0.9, 0.2, 1),
             (4.75, 2.5, 2.5, 1)]
    nl = make_nl([(0, neigh), (0, neigh[::-1])], 1)
    check(H3, nl)
    check(H3, nl, legacy=False)


@pytest.mark.parametrize("variant", [
    dict(amplitude_scaling=0.0), dict(amplitude_scaling=2.0), dict(radial_enhancement=1),
    dict(radial_enhancement=2), dict(central_weight=0.5), dict(atom_sigma_r_scaling=0.1),
    dict(atom_sigma_t_scaling=0.05), dict(global_scaling=2.0), dict(nf=3.0),
    dict(rcut_soft=5.0), dict(scaling_mode="none"), dict(central_weight=0.0),
])
@pytest.mark.parametrize("basis", ["poly3", "poly3gauss", "poly3operator"])
def test_hyperparameter_variants(variant, basis):
    hp = dataclasses.replace(syn.Hyper(alpha_max=[7, 6], basis=basis), **variant)
    nl = make_nl(random_sites(np.random.default_rng(11), 12, 2), 2)
    check(hp, nl)


def test_per_species_cutoffs_and_multi_species_masks():
    hp = syn.Hyper(alpha_max=[6, 8], basis="poly3gauss", rcut_hard=[5.0, 4.0],
                   rcut_soft=[4.5, 3.2], atom_sigma_r=[0.5, 0.4], atom_sigma_t=[0.45, 0.5],
                   central_weight=[1.0, 0.7])
    rng = np.random.default_rng(5)
    sites = random_sites(rng, 10, 2)
    # some neighbours count as both species (mask bits 1 and 2)
    sites = [(cs, [(r, t, p, 3 if i % 4 == 0 else b) for i, (r, t, p, b) in enumerate(ng)])
             for cs, ng in sites]
    check(hp, make_nl(sites, 2))


@pytest.mark.parametrize("basis", ["poly3", "poly3gauss", "poly3operator"])
def test_central_atoms_of_two_species(basis):
    """Sites whose atom carries two species (species(:, i) = (1, 2),
    species_multiplicity = 2): the self pair has both mask bits, and poly3gauss
    adds the central-atom term of each species (src/soap_turbo.f90:646-662),
    with different central weights."""
    hp = syn.Hyper(alpha_max=[6, 5], basis=basis, central_weight=[1.0, 0.6])
    rng = np.random.default_rng(9)
    sites = random_sites(rng, 12, 2)
    sites = [(cs, [(r, t, p, 3 if i % 5 == 0 else b) for i, (r, t, p, b) in enumerate(ng)])
             for cs, ng in sites]
    nl = make_nl(sites, 2)
    dual = np.arange(nl.n_sites) % 3 == 0
    species = np.zeros((nl.n_sites, 2), np.int32)
    species[:, 0] = nl.species[:, 0]
    species[dual] = (1, 2)
    mult = np.where(dual, 2, 1).astype(np.int32)
    mask = nl.mask.copy()
    first = np.concatenate([[0], np.cumsum(nl.n_neigh)[:-1]])
    mask[:, first[dual]] = 1                      # the self pair of a two-species atom
    nl = dataclasses.replace(nl, species=species, species_multiplicity=mult, mask=mask)
    check(hp, nl)


@pytest.mark.parametrize("l_max", [1, 3, 6])
def test_small_l_max(l_max):
    hp = syn.Hyper(alpha_max=[8, 8, 8], l_max=l_max, basis="poly3gauss", compress_mode="trivial")
    check(hp, make_nl(random_sites(np.random.default_rng(l_max), 10, 3), 3))


@pytest.mark.parametrize("hp", [
    syn.Hyper(alpha_max=[6, 6], l_max=10, basis="poly3"),
    syn.Hyper(alpha_max=[10], l_max=8, basis="poly3gauss"),
    syn.Hyper(alpha_max=[1], l_max=4, basis="poly3"),
    syn.Hyper(alpha_max=[1, 2], l_max=4, basis="poly3gauss"),
    syn.Hyper(alpha_max=[5, 4], l_max=10, basis="poly3operator"),
    syn.Hyper(alpha_max=[2], l_max=3, basis="poly3operator"),
])
def test_generic_kernel_shapes(hp):
    # l_max > 8 or alpha > 8 take the generic kernel instantiation.  alpha = 10
    # poly3gauss is past the reference's stability warning (W ~ 1e8): the
    # FP32 pair arithmetic then carries more of W's conditioning
    big_alpha = max(hp.alpha_max) > 8
    check(hp, make_nl(random_sites(np.random.default_rng(3), 8, hp.n_species), hp.n_species),
          soap_tol=1e-4 if big_alpha else SOAP_TOL, vjp_tol=1e-3 if big_alpha else VJP_TOL,
          fp64=not big_alpha)


@pytest.mark.parametrize("basis", ["poly3", "poly3gauss"])
def test_eight_species(basis):
    """The species limit of the kernels (8: one mask byte per pair) with
    neighbours of two species at once; a ninth species is refused."""
    hp = syn.Hyper(alpha_max=[2, 3, 2, 1, 3, 2, 2, 3], l_max=4, basis=basis,
                   central_weight=[1.0, 0.5, 1.0, 0.8, 1.0, 1.0, 0.3, 1.0])
    rng = np.random.default_rng(31)
    sites = random_sites(rng, 16, 8)
    sites = [(cs, [(r, t, p, b | (1 << ((cs + i) % 8)) if i % 3 == 0 else b)
                   for i, (r, t, p, b) in enumerate(ng)]) for cs, ng in sites]
    check(hp, make_nl(sites, 8))
    with pytest.raises(_lib.SoapError):
        Context(syn.Hyper(alpha_max=[2] * 9, l_max=4, basis=basis))


def test_large_sites_span_chunks_and_rounds():
    rng = np.random.default_rng(9)
    sites = random_sites(rng, 3, 3, lo=140, hi=300, rmax=5.0) + random_sites(rng, 3, 3, lo=65, hi=90)
    check(HG, make_nl(sites, 3))


def test_empty_sites_inside_a_batch_and_empty_batch():
    rng = np.random.default_rng(2)
    sites = random_sites(rng, 4, 1)
    nl = make_nl(sites, 1)
    # a site with n_neigh = 0 between others: no pair belongs to it
    nl2 = dataclasses.replace(nl, n_sites=5, n_neigh=np.insert(nl.n_neigh, 2, 0),
                              species=np.insert(nl.species, 2, [[1]], axis=0),
                              species_multiplicity=np.ones(5, np.int32))
    ctx = Context(H3)
    W, S = ctx.basis()
    ref = O.get_soap(H3, nl, W, S, do_derivatives=False)
    s = ctx.descriptor(ctx.batch(nl2)).cpu().numpy()
    assert site_rel_err(np.delete(s, 2, axis=0), ref.soap) <= SOAP_TOL
    empty = make_nl([], 1)
    out = ctx.descriptor(ctx.batch(empty))
    assert out.shape == (0, ctx.n_soap)


def test_bad_inputs_are_reported():
    nl = make_nl(random_sites(np.random.default_rng(4), 3, 1), 1)
    nl.rjs[5] = np.nan
    ctx = Context(H3)
    ctx.descriptor(ctx.batch(nl))
    with pytest.raises(_lib.SoapError) as e:
        ctx.check_inputs()
    assert e.value.code == 8


def test_scan_wait_gives_up_and_reports():
    """The CSR offset scan's look-back wait is bounded: a tile whose predecessor
    never publishes gives up after its spin limit and the scan reports it
    (SOAPB_ERR_CUDA, "gave up waiting"); with the predecessor published (tile
    states prepared on the host) the same launch ends normally with the right
    total.  Nothing hangs or faults either way."""
    import ctypes as C
    lib = _lib.load()
    last = C.c_int64(-1)
    assert lib.soapb_selftest_scan_wait(1000, 1, C.byref(last)) == 0
    assert last.value == 4096
    rc = lib.soapb_selftest_scan_wait(1000, 0, C.byref(last))
    assert rc == 6 and b"gave up waiting" in lib.soapb_last_error()
    assert last.value == 2048  # the tile's own sum, no predecessor's prefix
