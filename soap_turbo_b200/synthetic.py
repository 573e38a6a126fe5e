"""Seeded synthetic structures and CSR neighbour lists in get_soap's input format.

No public dataset is involved: the workloads are random periodic cubes with the
shapes of the benchmark configurations (atom counts, densities, minimum
distances, species mole fractions).  The neighbour list is what the callers of
soap_turbo's ``get_soap`` (src/soap_turbo.f90:139-169) hand it:

* one CSR row per central site, the site itself first with ``rjs = 0`` and
  ``theta = phi = 0``;
* every periodic image of every atom within ``rcut`` of the site;
* ``theta = acos(dz/r)``, ``phi = atan2(dy, dx)`` of ``r_j - r_i``, the
  convention of the Cartesian rotation in src/soap_turbo.f90:869-876;
* ``mask(k, s)`` true when neighbour ``k`` is of species ``s``, as
  ``assign_species_multiplicity`` builds it (src/soap_turbo.f90:2188-2214) for
  species multiplicity 1.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Structure:
    positions: np.ndarray  # (n_atoms, 3) in [0, L)
    box: float             # cube side, Angstrom
    species: np.ndarray    # (n_atoms,) 0-based species index


@dataclasses.dataclass
class NeighbourList:
    """CSR neighbour list in the layout get_soap takes."""

    n_sites: int
    n_neigh: np.ndarray      # (n_sites,) int32
    rjs: np.ndarray          # (n_pairs,) float64
    thetas: np.ndarray       # (n_pairs,) float64
    phis: np.ndarray         # (n_pairs,) float64
    mask: np.ndarray         # (n_species, n_pairs) uint8 == Fortran mask(n_pairs, n_species)
    species: np.ndarray      # (n_sites, max_mult) int32, 1-based == Fortran species(max_mult, n_sites)
    species_multiplicity: np.ndarray  # (n_sites,) int32
    site_atom: np.ndarray    # (n_sites,) atom index of each site
    neigh_atom: np.ndarray   # (n_pairs,) atom index of each neighbour
    disp: np.ndarray         # (n_pairs, 3) displacement r_j - r_i (image included)

    @property
    def n_pairs(self) -> int:
        return int(self.rjs.shape[0])


def random_structure(n_atoms: int, *, density: float | None = None, box: float | None = None,
                     d_min: float = 0.0, fractions=(1.0,), seed: int = 0) -> Structure:
    """Uniform random periodic cube, rejection-sampled to a minimum image
    distance ``d_min``; species drawn with the given mole fractions."""
    rng = np.random.default_rng(seed)
    if box is None:
        box = (n_atoms / density) ** (1.0 / 3.0)
    pos = rng.random((n_atoms, 3)) * box
    if d_min > 0.0 and n_atoms > 1:
        from scipy.spatial import cKDTree
        for _ in range(10000):
            tree = cKDTree(pos, boxsize=box)
            pairs = tree.query_pairs(d_min, output_type="ndarray")
            if pairs.shape[0] == 0:
                break
            bad = np.unique(np.max(pairs, axis=1))
            pos[bad] = rng.random((bad.shape[0], 3)) * box
        else:  # pragma: no cover - only with absurd densities
            raise RuntimeError("could not reach the minimum distance")
    fr = np.asarray(fractions, dtype=np.float64)
    fr = fr / fr.sum()
    species = rng.choice(len(fr), size=n_atoms, p=fr).astype(np.int32)
    return Structure(pos, float(box), species)


def _pairs_all_images(pos, box, sites, rcut):
    """(site_idx, atom_idx, displacement) for every image within rcut."""
    nimg = int(math.ceil(rcut / box))
    rng_ = np.arange(-nimg, nimg + 1)
    shifts = np.stack(np.meshgrid(rng_, rng_, rng_, indexing="ij"), -1).reshape(-1, 3) * box
    out_i, out_j, out_d = [], [], []
    for si, a in enumerate(sites):
        d = pos[None, :, :] + shifts[:, None, :] - pos[a][None, None, :]
        r2 = np.einsum("sjc,sjc->sj", d, d)
        s_idx, j_idx = np.nonzero(r2 < rcut * rcut)
        keep = ~((j_idx == a) & np.all(shifts[s_idx] == 0.0, axis=1))
        out_i.append(np.full(int(keep.sum()), si))
        out_j.append(j_idx[keep])
        out_d.append(d[s_idx[keep], j_idx[keep]])
    return np.concatenate(out_i), np.concatenate(out_j), np.concatenate(out_d)


def _pairs_min_image(pos, box, sites, rcut):
    from scipy.spatial import cKDTree
    tree = cKDTree(pos, boxsize=box)
    pairs = tree.query_pairs(rcut, output_type="ndarray")
    i = np.concatenate([pairs[:, 0], pairs[:, 1]])
    j = np.concatenate([pairs[:, 1], pairs[:, 0]])
    d = pos[j] - pos[i]
    d -= box * np.round(d / box)
    is_site = np.full(pos.shape[0], -1, dtype=np.int64)
    is_site[sites] = np.arange(len(sites))
    sel = is_site[i] >= 0
    return is_site[i[sel]], j[sel], d[sel]


def neighbour_list(struct: Structure, rcut: float, n_species: int, central_species=None) -> NeighbourList:
    """CSR list for the sites of ``central_species`` (0-based species index;
    None = every atom), neighbours of every species within ``rcut``."""
    pos, box = struct.positions, struct.box
    if central_species is None:
        sites = np.arange(pos.shape[0])
    else:
        sites = np.nonzero(struct.species == central_species)[0]
    if box >= 2.0 * rcut:
        si, nj, d = _pairs_min_image(pos, box, sites, rcut)
    else:
        si, nj, d = _pairs_all_images(pos, box, sites, rcut)
    r = np.sqrt(np.einsum("pc,pc->p", d, d))
    order = np.lexsort((r, nj, si))
    si, nj, d, r = si[order], nj[order], d[order], r[order]
    counts = np.bincount(si, minlength=len(sites))
    n_sites = len(sites)
    n_pairs = n_sites + si.shape[0]
    # interleave: self pair first in each row
    row_start = np.concatenate([[0], np.cumsum(counts + 1)[:-1]])
    self_pos = row_start
    other_pos = np.ones(n_pairs, dtype=bool)
    other_pos[self_pos] = False
    rjs = np.zeros(n_pairs)
    thetas = np.zeros(n_pairs)
    phis = np.zeros(n_pairs)
    neigh_atom = np.empty(n_pairs, dtype=np.int64)
    disp = np.zeros((n_pairs, 3))
    neigh_atom[self_pos] = sites
    rjs[other_pos] = r
    disp[other_pos] = d
    neigh_atom[other_pos] = nj
    with np.errstate(invalid="ignore", divide="ignore"):
        ct = np.clip(d[:, 2] / r, -1.0, 1.0)
    thetas[other_pos] = np.arccos(ct)
    phis[other_pos] = np.arctan2(d[:, 1], d[:, 0])
    mask = np.zeros((n_species, n_pairs), dtype=np.uint8)
    mask[struct.species[neigh_atom], np.arange(n_pairs)] = 1
    species = (struct.species[sites] + 1).astype(np.int32).reshape(n_sites, 1)
    return NeighbourList(
        n_sites=n_sites,
        n_neigh=(counts + 1).astype(np.int32),
        rjs=rjs, thetas=thetas, phis=phis, mask=mask,
        species=species,
        species_multiplicity=np.ones(n_sites, dtype=np.int32),
        site_atom=sites.astype(np.int64),
        neigh_atom=neigh_atom,
        disp=disp,
    )


def concatenate(lists) -> NeighbourList:
    """Concatenate independent structures' lists into one CSR batch."""
    return NeighbourList(
        n_sites=sum(nl.n_sites for nl in lists),
        n_neigh=np.concatenate([nl.n_neigh for nl in lists]),
        rjs=np.concatenate([nl.rjs for nl in lists]),
        thetas=np.concatenate([nl.thetas for nl in lists]),
        phis=np.concatenate([nl.phis for nl in lists]),
        mask=np.concatenate([nl.mask for nl in lists], axis=1),
        species=np.concatenate([nl.species for nl in lists]),
        species_multiplicity=np.concatenate([nl.species_multiplicity for nl in lists]),
        site_atom=np.concatenate([nl.site_atom for nl in lists]),
        neigh_atom=np.concatenate([nl.neigh_atom for nl in lists]),
        disp=np.concatenate([nl.disp for nl in lists]),
    )


# --------------------------------------------------------------------------
# Hyperparameters and the benchmark configurations
# --------------------------------------------------------------------------
@dataclasses.dataclass
class Hyper:
    """Per-species hyperparameters of get_soap (src/soap_turbo.f90:150-162)."""

    alpha_max: list
    l_max: int = 8
    rcut_hard: float | list = 5.0
    rcut_soft: float | list = 4.5
    nf: float | list = 4.0
    global_scaling: float | list = 1.0
    atom_sigma_r: float | list = 0.5
    atom_sigma_r_scaling: float | list = 0.0
    atom_sigma_t: float | list = 0.5
    atom_sigma_t_scaling: float | list = 0.0
    amplitude_scaling: float | list = 1.0
    central_weight: float | list = 1.0
    radial_enhancement: int = 0
    basis: str = "poly3"
    scaling_mode: str = "polynomial"
    compress_mode: str = "None"

    @property
    def n_species(self) -> int:
        return len(self.alpha_max)

    def arr(self, name: str) -> np.ndarray:
        v = getattr(self, name)
        if np.isscalar(v):
            v = [v] * self.n_species
        return np.ascontiguousarray(v, dtype=np.float64)

    @property
    def n_max(self) -> int:
        return int(sum(self.alpha_max))


@dataclasses.dataclass
class Workload:
    name: str
    hyper: Hyper
    nl: NeighbourList
    structures: list


def config(idx: int, seed: int = 1234, scale: float = 1.0) -> Workload:
    """The benchmark configurations 1..5; ``scale`` < 1 shrinks the atom count
    (same density, shapes and hyperparameters) for quick parity runs."""
    if idx in (1, 4):
        n = 64 if idx == 1 else 32768
        n = max(8, int(round(n * scale)))
        if idx == 1 and scale == 1.0:
            st = random_structure(64, box=8.0, d_min=1.2, seed=seed)
        else:
            st = random_structure(n, density=0.125 if idx == 1 else 0.11, d_min=1.2, seed=seed)
        hp = Hyper(alpha_max=[8], basis="poly3")
        nl = neighbour_list(st, 5.0, 1)
        return Workload(f"config{idx}", hp, nl, [st])
    if idx in (2, 5):
        n = 4096 if idx == 2 else 262144
        n = max(16, int(round(n * scale)))
        st = random_structure(n, density=0.10, d_min=0.9, fractions=(0.4, 0.4, 0.2), seed=seed)
        hp = Hyper(alpha_max=[8, 8, 8], basis="poly3gauss", compress_mode="trivial")
        nl = neighbour_list(st, 5.0, 3, central_species=1)
        return Workload(f"config{idx}", hp, nl, [st])
    if idx == 3:
        rng = np.random.default_rng(seed)
        n_struct = max(1, int(round(512 * scale)))
        lists, structs = [], []
        for t in range(n_struct):
            na = int(math.floor(math.exp(rng.uniform(math.log(16), math.log(2048)))))
            rho = rng.uniform(0.06, 0.14)
            st = random_structure(na, density=rho, d_min=0.9, fractions=(0.4, 0.4, 0.2),
                                  seed=seed * 1000 + t)
            structs.append(st)
            lists.append(neighbour_list(st, 5.0, 3, central_species=1))
        hp = Hyper(alpha_max=[8, 8, 8], basis="poly3gauss", compress_mode="trivial")
        return Workload("config3", hp, concatenate(lists), structs)
    raise ValueError(idx)


def trivial_compress_indices(alpha_max, l_max):
    """Python statement of get_compress_indices' trivial branch
    (src/soap_turbo_compress.f90:86-119): 1-based P_i, P_j, P_el."""
    n_species = len(alpha_max)
    pivot = [1]
    for i in range(n_species - 1):
        pivot.append(pivot[i] + alpha_max[i])
    n_max = sum(alpha_max)
    P_i, P_j = [], []
    k = 1
    counter = 0
    for n in range(1, n_max + 1):
        for m in range(n, n_max + 1):
            for _ in range(l_max + 1):
                if n in pivot or m in pivot:
                    counter += 1
                    P_i.append(counter)
                    P_j.append(k)
                k += 1
    return (np.asarray(P_i, dtype=np.int32), np.asarray(P_j, dtype=np.int32),
            np.ones(counter, dtype=np.float64))
