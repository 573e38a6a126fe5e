"""The pair kernel's tabulated radial expansion (atom_sigma_r_scaling = 0).

The context fits per-species piecewise polynomials to the FP64 expansion
(src/soap_turbo_radial.f90:550-1002) and uses them only when their FP32 check
passes (largest error relative to each function's largest value <= 5e-7).
Both forms -- the tables and the FP64 expansion per pair -- must meet the
parity gates against the oracle, and they must agree with each other."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import SOAP_TOL, VJP_TOL, max_rel_err, site_rel_err
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu


def _run(ctx, b, G):
    soap = ctx.descriptor(b, keep=True)
    pair = ctx.contract(b, soap, G)
    return soap.cpu().numpy(), pair.cpu().numpy()


@pytest.mark.parametrize("cfg,scale,legacy", [(1, 1.0, True), (2, 0.25, True), (2, 0.25, False),
                                              (4, 1 / 64, True)])
def test_tables_and_fp64_expansion_both_meet_the_gates(cfg, scale, legacy):
    w = syn.config(cfg, seed=19, scale=scale)
    ctx = Context(w.hyper, legacy_filter_seed=legacy)
    use, err = ctx.radial_tables()
    assert use and 0.0 <= err <= 5e-7
    W, S = ctx.basis()
    ref = O.get_soap(w.hyper, w.nl, W, S, do_derivatives=True, legacy_filter_seed=legacy)
    G = np.random.default_rng(3).standard_normal((ctx.n_soap, w.nl.n_sites))
    ref_pair = ref.contract(G, 1.0)
    b = ctx.batch(w.nl)
    Gt = torch.as_tensor(G).cuda()
    s_tab, p_tab = _run(ctx, b, Gt)
    ctx.set_radial_tables(False)
    assert ctx.radial_tables()[0] is False
    s_64, p_64 = _run(ctx, b, Gt)
    ctx.set_radial_tables(True)
    for s, p in ((s_tab, p_tab), (s_64, p_64)):
        assert site_rel_err(s, ref.soap) <= SOAP_TOL
        assert max_rel_err(p, ref_pair) <= VJP_TOL
    assert site_rel_err(s_tab, s_64) <= SOAP_TOL


def test_tables_cover_the_hyperparameter_variants():
    # radial enhancement, amplitude scaling 0 and 2, no polynomial scaling,
    # another nf, and species with different cutoffs and widths
    variants = [
        dict(radial_enhancement=1), dict(radial_enhancement=2), dict(amplitude_scaling=0.0),
        dict(amplitude_scaling=2.0), dict(scaling_mode="none"), dict(nf=2.0),
        dict(rcut_hard=[5.0, 4.0], rcut_soft=[4.5, 3.0]), dict(atom_sigma_r=[0.5, 0.35]),
    ]
    st = syn.random_structure(48, density=0.10, d_min=0.9, fractions=(0.5, 0.5), seed=23)
    for v in variants:
        hp = syn.Hyper(alpha_max=[8, 8], basis="poly3gauss", compress_mode="trivial", **v)
        nl = syn.neighbour_list(st, max(hp.arr("rcut_hard")), 2, central_species=None)
        ctx = Context(hp)
        use, err = ctx.radial_tables()
        assert use and err <= 5e-7, (v, err)
        W, S = ctx.basis()
        ref = O.get_soap(hp, nl, W, S, do_derivatives=True)
        G = np.random.default_rng(4).standard_normal((ctx.n_soap, nl.n_sites))
        s, p = _run(ctx, ctx.batch(nl), torch.as_tensor(G).cuda())
        assert site_rel_err(s, ref.soap) <= SOAP_TOL, v
        assert max_rel_err(p, ref.contract(G, 1.0)) <= VJP_TOL, v


def test_no_tables_where_r_alone_does_not_fix_the_expansion():
    # a sigma that grows with r, and the poly3operator basis, keep the FP64 form
    for hp in (syn.Hyper(alpha_max=[8], basis="poly3", atom_sigma_r_scaling=0.1),
               syn.Hyper(alpha_max=[8], basis="poly3operator")):
        ctx = Context(hp)
        assert ctx.radial_tables() == (False, -1.0)
