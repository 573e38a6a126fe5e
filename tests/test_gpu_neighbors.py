"""The GPU neighbour-list builder (soapb_build_neighbors) against the numpy
builder the tests and bench use, a brute-force builder for triclinic cells,
and a restatement of assign_species_multiplicity's mask loop
(src/soap_turbo.f90:2188-2214)."""
import numpy as np
import pytest
import torch

from conftest import site_rel_err
from soap_turbo_b200 import _lib
from soap_turbo_b200 import synthetic as syn
from soap_turbo_b200.context import Context

pytestmark = pytest.mark.gpu


def built(ctx, pos, lattice, atom_species, sites, rcut=0.0, atom_mult=None):
    sp = np.asarray(atom_species, dtype=np.int32)
    if sp.ndim == 1:
        sp = sp.reshape(-1, 1)
    am = None if atom_mult is None else torch.as_tensor(np.asarray(atom_mult, np.int32)).cuda()
    b = ctx.build_neighbors(torch.as_tensor(np.asarray(pos, np.float64)).cuda(), lattice,
                            torch.as_tensor(sp).cuda(), torch.as_tensor(np.asarray(sites, np.int32)).cuda(),
                            atom_mult=am, rcut=rcut)
    return b, b.arrays()


def canonical(n_neigh, atom, r, th, ph):
    """Row-wise order by (atom, distance to 1e-9, theta, phi): images of one atom
    at equal distance (up to rounding) may come in either order."""
    off = np.concatenate([[0], np.cumsum(n_neigh)])
    order = np.arange(atom.shape[0])
    for i in range(len(n_neigh)):
        a, b = off[i], off[i + 1]
        order[a:b] = a + np.lexsort((np.round(ph[a:b], 9), np.round(th[a:b], 9), np.round(r[a:b], 9), atom[a:b]))
    return order


def compare(a, nl, atol=1e-12):
    np.testing.assert_array_equal(a["n_neigh"], nl.n_neigh)
    o1 = canonical(a["n_neigh"], a["neigh_atom"], a["rjs"], a["thetas"], a["phis"])
    o2 = canonical(nl.n_neigh, nl.neigh_atom, nl.rjs, nl.thetas, nl.phis)
    np.testing.assert_array_equal(a["neigh_atom"][o1], nl.neigh_atom[o2])
    np.testing.assert_allclose(a["rjs"][o1], nl.rjs[o2], rtol=0, atol=atol)
    np.testing.assert_allclose(a["thetas"][o1], nl.thetas[o2], rtol=0, atol=atol * 1e3)
    np.testing.assert_allclose(a["phis"][o1], nl.phis[o2], rtol=0, atol=atol * 1e3)
    np.testing.assert_array_equal(a["mask"][:, o1], nl.mask[:, o2])
    np.testing.assert_array_equal(a["species"], nl.species)
    np.testing.assert_array_equal(a["species_multiplicity"], nl.species_multiplicity)


CASES = {
    "config1_images": lambda: syn.config(1, seed=3),              # 8 A box < 2 rcut: many images
    "config2_quarter": lambda: syn.config(2, seed=5, scale=0.25),  # central species only
    "config4_small": lambda: syn.config(4, seed=9, scale=1 / 64),
}


@pytest.mark.parametrize("name", list(CASES))
def test_matches_the_numpy_builder(name):
    w = CASES[name]()
    st = w.structures[0]
    ctx = Context(w.hyper)
    _, a = built(ctx, st.positions, np.eye(3) * st.box, st.species + 1, w.nl.site_atom)
    compare(a, w.nl)


def test_positions_outside_the_cell_give_the_same_list():
    w = syn.config(1, seed=4)
    st = w.structures[0]
    ctx = Context(w.hyper)
    shifted = st.positions + np.array([3.0, -2.0, 1.0]) * st.box
    _, a = built(ctx, shifted, np.eye(3) * st.box, st.species + 1, w.nl.site_atom)
    compare(a, w.nl, atol=1e-11)


def brute_force(pos, lat, sites, rcut):
    """Every image within rcut, for any cell, by enumeration."""
    inv = np.linalg.inv(lat)
    widths = 1.0 / np.linalg.norm(inv, axis=0)
    k = np.ceil(rcut / widths).astype(int) + 1
    g = [np.arange(-k[d], k[d] + 1) for d in range(3)]
    shifts = np.stack(np.meshgrid(*g, indexing="ij"), -1).reshape(-1, 3)
    trans = shifts @ lat
    rows = []
    for a in sites:
        d = (pos[None, :, :] + trans[:, None, :]) - pos[a][None, None, :]
        r = np.sqrt((d * d).sum(-1))
        s_i, j_i = np.nonzero(r < rcut)
        keep = ~((j_i == a) & np.all(shifts[s_i] == 0, axis=1))
        s_i, j_i = s_i[keep], j_i[keep]
        rr = r[s_i, j_i]
        order = np.lexsort((rr, j_i))
        rows.append((j_i[order], d[s_i[order], j_i[order]]))
    return rows


@pytest.mark.parametrize("cell", ["triclinic", "thin"])
def test_triclinic_and_thin_cells(cell):
    rng = np.random.default_rng(11)
    if cell == "triclinic":
        lat = np.array([[9.0, 0.0, 0.0], [3.1, 8.2, 0.0], [-2.3, 1.7, 7.5]])
        n = 70
    else:  # one axis far shorter than rcut: a site sees many images along it
        lat = np.array([[14.0, 0.0, 0.0], [0.0, 13.0, 0.0], [0.5, 0.0, 2.2]])
        n = 40
    frac = rng.random((n, 3))
    pos = frac @ lat
    species = rng.integers(1, 4, n)
    sites = np.arange(0, n, 3)
    hp = syn.Hyper(alpha_max=[4, 4, 4], l_max=4, basis="poly3gauss")
    ctx = Context(hp)
    _, a = built(ctx, pos, lat, species, sites)
    rows = brute_force(pos, lat, sites, 5.0)
    off = np.concatenate([[0], np.cumsum(a["n_neigh"])])
    for i, (j, d) in enumerate(rows):
        r0, r1 = off[i], off[i + 1]
        assert r1 - r0 == len(j) + 1
        assert a["neigh_atom"][r0] == sites[i] and a["rjs"][r0] == 0.0
        r = np.sqrt((d * d).sum(-1))
        th, ph = np.arccos(np.clip(d[:, 2] / r, -1, 1)), np.arctan2(d[:, 1], d[:, 0])
        sl = slice(r0 + 1, r1)
        o1 = canonical([r1 - r0 - 1], a["neigh_atom"][sl], a["rjs"][sl], a["thetas"][sl], a["phis"][sl])
        o2 = canonical([len(j)], j, r, th, ph)
        np.testing.assert_array_equal(a["neigh_atom"][sl][o1], j[o2])
        np.testing.assert_allclose(a["rjs"][sl][o1], r[o2], rtol=0, atol=1e-11)
        np.testing.assert_allclose(a["thetas"][sl][o1], th[o2], rtol=0, atol=1e-9)
        np.testing.assert_allclose(a["phis"][sl][o1], ph[o2], rtol=0, atol=1e-9)


def test_species_multiplicity_follows_the_reference_mask_loop():
    """Atoms of several species: mask(k2, s) is set from the neighbour's first
    multiplicity(central atom) species (src/soap_turbo.f90:2203-2211)."""
    rng = np.random.default_rng(13)
    n, L = 60, 9.0
    pos = rng.random((n, 3)) * L
    table = np.array([[1, 0], [2, 0], [3, 0], [1, 2], [2, 3], [3, 1]], np.int32)
    atom_species = table[rng.integers(0, len(table), n)]
    mult = (atom_species > 0).sum(1).astype(np.int32)
    sites = np.arange(n)
    hp = syn.Hyper(alpha_max=[4, 4, 4], l_max=3, basis="poly3gauss")
    ctx = Context(hp)
    _, a = built(ctx, pos, np.eye(3) * L, atom_species, sites, atom_mult=mult)
    off = np.concatenate([[0], np.cumsum(a["n_neigh"])])
    expect = np.zeros_like(a["mask"])
    for i in range(n):
        for k in range(off[i], off[i + 1]):
            j = a["neigh_atom"][k]
            for i2 in range(mult[sites[i]]):
                sp = atom_species[j, i2]
                if sp > 0:
                    expect[sp - 1, k] = 1
    np.testing.assert_array_equal(a["mask"], expect)
    np.testing.assert_array_equal(a["species"], atom_species[sites])
    np.testing.assert_array_equal(a["species_multiplicity"], mult[sites])


def test_descriptor_and_vjp_from_the_built_list():
    w = syn.config(2, seed=21, scale=0.25)
    st = w.structures[0]
    ctx = Context(w.hyper)
    b, _ = built(ctx, st.positions, np.eye(3) * st.box, st.species + 1, w.nl.site_atom)
    s_built = ctx.descriptor(b).cpu().numpy()
    G = torch.as_tensor(np.random.default_rng(1).standard_normal((ctx.n_soap, w.nl.n_sites))).cuda()
    p_built = ctx.contract(b, torch.as_tensor(s_built).cuda(), G).cpu().numpy()
    ref = ctx.batch(w.nl)
    s_np = ctx.descriptor(ref).cpu().numpy()
    p_np = ctx.contract(ref, torch.as_tensor(s_np).cuda(), G).cpu().numpy()
    assert site_rel_err(s_built, s_np) <= 1e-9
    assert np.abs(p_built - p_np).max() <= 1e-9 * np.abs(p_np).max()


def test_bad_inputs_are_reported():
    w = syn.config(1, seed=6)
    st = w.structures[0]
    ctx = Context(w.hyper)
    with pytest.raises(_lib.SoapError) as e:
        built(ctx, st.positions, np.eye(3) * st.box, st.species + 1, [0, 1, st.positions.shape[0]])
    assert e.value.code == 8
    pos = st.positions.copy()
    pos[5, 1] = np.nan
    with pytest.raises(_lib.SoapError) as e:
        built(ctx, pos, np.eye(3) * st.box, st.species + 1, [0, 1])
    assert e.value.code == 8
    with pytest.raises(_lib.SoapError) as e:  # about 4000 neighbours per site at rcut = 20
        built(ctx, st.positions, np.eye(3) * st.box, st.species + 1, [0], rcut=20.0)
    assert e.value.code == 1
    with pytest.raises(_lib.SoapError) as e:
        built(ctx, st.positions, np.zeros((3, 3)), st.species + 1, [0])
    assert e.value.code == 1
    # the context still works after the refusals
    _, a = built(ctx, st.positions, np.eye(3) * st.box, st.species + 1, w.nl.site_atom)
    compare(a, w.nl)
