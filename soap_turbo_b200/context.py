"""Context API of libsoapb200.so on device memory.

A ``Context`` holds one descriptor definition (hyperparameters, basis
matrices, compression map) on one GPU.  Batches are CSR neighbour lists held
in device memory; torch tensors provide the device allocations and streams
(plumbing only -- every computation is a libsoapb200 kernel).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib


def _f64(v, n):
    v = np.atleast_1d(np.asarray(v, dtype=np.float64))
    if v.shape[0] == 1 and n > 1:
        v = np.repeat(v, n)
    return np.ascontiguousarray(v)


class DeviceBatch:
    """A neighbour list resident on the GPU (the ``soapb_batch`` the kernels read)."""

    def __init__(self, nl, device="cuda"):
        dev = torch.device(device)
        self.n_sites = int(nl.n_sites)
        self.n_pairs = int(nl.n_pairs)
        self.n_neigh = torch.as_tensor(np.ascontiguousarray(nl.n_neigh, dtype=np.int32)).to(dev)
        sp = np.ascontiguousarray(nl.species, dtype=np.int32)  # (n_sites, max_mult) C == Fortran (max_mult, n_sites)
        self.max_mult = int(sp.shape[1])
        self.species = torch.as_tensor(sp).to(dev)
        self.species_multiplicity = torch.as_tensor(
            np.ascontiguousarray(nl.species_multiplicity, dtype=np.int32)).to(dev)
        self.mask = torch.as_tensor(np.ascontiguousarray(nl.mask, dtype=np.uint8)).to(dev)
        self.rjs = torch.as_tensor(np.ascontiguousarray(nl.rjs, dtype=np.float64)).to(dev)
        self.thetas = torch.as_tensor(np.ascontiguousarray(nl.thetas, dtype=np.float64)).to(dev)
        self.phis = torch.as_tensor(np.ascontiguousarray(nl.phis, dtype=np.float64)).to(dev)
        self._c = _lib.Batch(self.n_sites, self.n_pairs, self.max_mult, self.n_neigh.data_ptr(),
                             self.species.data_ptr(), self.species_multiplicity.data_ptr(),
                             self.mask.data_ptr(), self.rjs.data_ptr(), self.thetas.data_ptr(),
                             self.phis.data_ptr())

    @property
    def c(self):
        return C.byref(self._c)

    def input_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (
            self.n_neigh, self.species, self.species_multiplicity, self.mask, self.rjs,
            self.thetas, self.phis))


class _DeviceView:
    """A device array owned by the library, seen through __cuda_array_interface__."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr or 0), False), "version": 2}


class BuiltBatch:
    """The neighbour list soapb_build_neighbors built in a context's buffers:
    usable as a batch of that context until its next build."""

    def __init__(self, c_batch, neigh_atom_ptr, n_species):
        self._c = c_batch
        self.n_sites = int(c_batch.n_sites)
        self.n_pairs = int(c_batch.n_atom_pairs)
        self.max_mult = int(c_batch.max_species_multiplicity)
        self._neigh_atom = neigh_atom_ptr
        self._n_species = n_species

    @property
    def c(self):
        return C.byref(self._c)

    def arrays(self) -> dict:
        """Host copies of the list, in synthetic.NeighbourList's layout."""
        b, ns, npair = self._c, self.n_sites, self.n_pairs

        def get(ptr, shape, ts, dt):
            if int(np.prod(shape)) == 0:
                return np.zeros(shape, dtype=dt)
            return torch.as_tensor(_DeviceView(ptr, shape, ts), device="cuda").cpu().numpy().copy()
        return {
            "n_neigh": get(b.n_neigh, (ns,), "<i4", np.int32),
            "rjs": get(b.rjs, (npair,), "<f8", np.float64),
            "thetas": get(b.thetas, (npair,), "<f8", np.float64),
            "phis": get(b.phis, (npair,), "<f8", np.float64),
            "mask": get(b.mask, (self._n_species, npair), "|u1", np.uint8),
            "species": get(b.species, (ns, self.max_mult), "<i4", np.int32),
            "species_multiplicity": get(b.species_multiplicity, (ns,), "<i4", np.int32),
            "neigh_atom": get(self._neigh_atom, (npair,), "<i4", np.int32),
        }


class Context:
    def __init__(self, hyper, *, legacy_filter_seed=True, compress=None, device=None):
        """``hyper``: a synthetic.Hyper-like object (alpha_max, l_max, per-species
        arrays, radial_enhancement, basis, scaling_mode, compress_mode)."""
        self._lib = _lib.load()
        self.hyper = hyper
        n = len(hyper.alpha_max)
        keep = {}
        keep["alpha"] = np.ascontiguousarray(hyper.alpha_max, dtype=np.int32)
        names = ("rcut_hard", "rcut_soft", "nf", "global_scaling", "atom_sigma_r",
                 "atom_sigma_r_scaling", "atom_sigma_t", "atom_sigma_t_scaling",
                 "amplitude_scaling", "central_weight")
        for nm in names:
            keep[nm] = _f64(getattr(hyper, nm), n)
        mode = getattr(hyper, "compress_mode", "None")
        if compress is None and mode not in (None, "", "None"):
            # trivial or a Darby mode "nu_R_nu_S"; others raise, as the reference stops
            from .descriptor import get_compress_indices
            _, _, P_i, P_j, P_el = get_compress_indices(mode, hyper.alpha_max, hyper.l_max)
            compress = (P_i, P_j, P_el)
        h = _lib.Hyper()
        h.n_species = n
        h.l_max = int(hyper.l_max)
        h.basis = _lib.BASIS[hyper.basis]
        h.scaling_mode = 0 if hyper.scaling_mode == "polynomial" else 1
        h.radial_enhancement = int(hyper.radial_enhancement)
        h.legacy_filter_seed = int(bool(legacy_filter_seed))
        h.alpha_max = keep["alpha"].ctypes.data_as(_lib.i32p)
        for nm in names:
            setattr(h, nm, keep[nm].ctypes.data_as(_lib.f64p))
        if compress is not None:
            P_i, P_j, P_el = (np.ascontiguousarray(compress[0], dtype=np.int32),
                              np.ascontiguousarray(compress[1], dtype=np.int32),
                              np.ascontiguousarray(compress[2], dtype=np.float64))
            keep.update(P_i=P_i, P_j=P_j, P_el=P_el)
            h.compress = 1
            h.P_nonzero = P_i.shape[0]
            h.P_i = P_i.ctypes.data_as(_lib.i32p)
            h.P_j = P_j.ctypes.data_as(_lib.i32p)
            h.P_el = P_el.ctypes.data_as(_lib.f64p)
        ptr = C.c_void_p()
        dev = -1 if device is None else int(device)
        _lib.check(self._lib.soapb_create(C.byref(h), dev, C.byref(ptr)))
        self._h = ptr
        self.n_max = int(sum(hyper.alpha_max))
        ns = C.c_int32(0)
        _lib.check(self._lib.soapb_n_soap(self._h, C.byref(ns)))
        self.n_soap = ns.value
        self.set_stream(torch.cuda.current_stream())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.soapb_destroy(h)
            self._h = None

    # ---------------------------------------------------------------- setup
    def set_stream(self, stream):
        self.stream = stream
        _lib.check(self._lib.soapb_set_stream(self._h, C.c_void_p(stream.cuda_stream)))

    def set_threads_per_site(self, threads: int):
        _lib.check(self._lib.soapb_set_threads_per_site(self._h, int(threads)))

    def set_radial_tables(self, enable: bool):
        """soapb_set_radial_tables: the pair kernel's tabulated FP32 radial
        expansion (True, when its check passed) or the FP64 expansion (False)."""
        _lib.check(self._lib.soapb_set_radial_tables(self._h, int(bool(enable))))

    def set_tensor_cores(self, enable: bool):
        """soapb_set_tensor_cores: the site kernels' contractions on the tensor
        cores (True, the default) or on the CUDA cores (False)."""
        _lib.check(self._lib.soapb_set_tensor_cores(self._h, int(bool(enable))))

    def radial_tables(self):
        """(in use, largest relative error of the tables; -1 when not tabulated)."""
        use, err = C.c_int32(0), C.c_double(0.0)
        _lib.check(self._lib.soapb_radial_tables(self._h, C.byref(use), C.byref(err)))
        return bool(use.value), float(err.value)

    def basis(self):
        W = np.zeros((self.n_max, self.n_max), order="F")
        S = np.zeros((self.n_max, self.n_max), order="F")
        _lib.check(self._lib.soapb_get_basis(self._h, W.ctypes.data_as(_lib.f64p),
                                             S.ctypes.data_as(_lib.f64p)))
        return W, S

    def set_basis(self, W, S):
        W = np.asfortranarray(W, dtype=np.float64)
        S = np.asfortranarray(S, dtype=np.float64)
        _lib.check(self._lib.soapb_set_basis(self._h, W.ctypes.data_as(_lib.f64p),
                                             S.ctypes.data_as(_lib.f64p)))

    @property
    def launch_count(self) -> int:
        v = C.c_int64(0)
        _lib.check(self._lib.soapb_launch_count(self._h, C.byref(v)))
        return v.value

    def build_neighbors(self, positions, lattice, atom_species, sites, atom_mult=None,
                        rcut=0.0) -> BuiltBatch:
        """soapb_build_neighbors: the CSR neighbour list of one periodic
        structure, built on the GPU.  positions: (n_atoms, 3) float64 CUDA
        tensor; lattice: 3x3 host array, rows = cell vectors; atom_species:
        (n_atoms, max_mult) int32 CUDA tensor of 1-based species (0 beyond an
        atom's multiplicity); sites: (n_sites,) int32 CUDA tensor of atom
        indices; atom_mult: (n_atoms,) int32 (default: the non-zero entries)."""
        pos = positions.contiguous()
        sp = atom_species.to(torch.int32).contiguous()
        if sp.dim() == 1:
            sp = sp.reshape(-1, 1)
        if atom_mult is None:
            atom_mult = (sp > 0).sum(dim=1).to(torch.int32)
        am = atom_mult.to(torch.int32).contiguous()
        st = sites.to(torch.int32).contiguous()
        lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(9)
        out = _lib.Batch()
        na = C.c_void_p()
        _lib.check(self._lib.soapb_build_neighbors(
            self._h, int(pos.shape[0]), C.c_void_p(pos.data_ptr()), lat.ctypes.data_as(_lib.f64p),
            C.c_void_p(sp.data_ptr()), int(sp.shape[1]), C.c_void_p(am.data_ptr()),
            int(st.shape[0]), C.c_void_p(st.data_ptr()), float(rcut), C.byref(out), C.byref(na)))
        return BuiltBatch(out, na.value, len(self.hyper.alpha_max))

    def kernel_timing(self, capacity: int):
        """soapb_kernel_timing: time the next `capacity` kernel launches with
        CUDA events on the context's stream (0 switches timing off)."""
        _lib.check(self._lib.soapb_kernel_timing(self._h, int(capacity)))

    def kernel_times(self) -> dict:
        """soapb_kernel_times: {kernel: (launches, total device ms)} of the
        launches timed since the last read, plus "dropped"."""
        cnt = (C.c_int64 * 4)()
        tot = (C.c_double * 4)()
        drop = C.c_int64(0)
        _lib.check(self._lib.soapb_kernel_times(self._h, cnt, tot, C.byref(drop)))
        out = {k: (int(cnt[i]), float(tot[i])) for i, k in enumerate(_lib.KERNEL_KINDS)}
        out["dropped"] = int(drop.value)
        return out

    def check_inputs(self):
        bad = C.c_int64(-1)
        _lib.check(self._lib.soapb_check_inputs(self._h, C.byref(bad)))

    # ---------------------------------------------------------------- compute
    def batch(self, nl) -> DeviceBatch:
        return DeviceBatch(nl, device=torch.device("cuda", torch.cuda.current_device()))

    def _new(self, shape):
        return torch.empty(shape, dtype=torch.float64, device=self.stream.device)

    def descriptor(self, b: DeviceBatch, out=None, keep=True):
        """soap as (n_sites, n_soap) == Fortran soap(n_soap, n_sites)."""
        out = self._new((b.n_sites, self.n_soap)) if out is None else out
        _lib.check(self._lib.soapb_descriptor(self._h, b.c, C.c_void_p(out.data_ptr()), int(keep)))
        return out

    def autotune(self, b: DeviceBatch) -> dict:
        """soapb_autotune: time both site kernels on this batch in each form
        (tensor cores, CUDA cores at every CTA size) and grid cap, and keep the
        fastest; returns the choice (threads 0: the tensor-core kernel)."""
        ch = (C.c_int32 * 4)()
        _lib.check(self._lib.soapb_autotune(self._h, b.c, ch))
        return {"descriptor_threads": ch[0], "descriptor_max_ctas": ch[1],
                "contract_threads": ch[2], "contract_max_ctas": ch[3],
                "descriptor_tensor_cores": ch[0] == 0, "contract_tensor_cores": ch[2] == 0}

    def descriptor_noalloc(self, b: DeviceBatch, out=None):
        """soapb_descriptor_noalloc: the descriptor with its scratch in the
        library's static device array (no device allocation in the call)."""
        out = self._new((b.n_sites, self.n_soap)) if out is None else out
        _lib.check(self._lib.soapb_descriptor_noalloc(self._h, b.c, C.c_void_p(out.data_ptr())))
        return out

    def contract(self, b: DeviceBatch, soap, G, sgn=1.0, g_layout=_lib.G_SITE_FASTEST, out=None):
        """pair forces (n_pairs, 3) == Fortran pair(3, n_pairs).  G is the
        reference's G(n_sites, n_soap) given as a (n_soap, n_sites) tensor
        (g_layout 0), or (n_sites, n_soap) with g_layout 1."""
        out = self._new((b.n_pairs, 3)) if out is None else out
        _lib.check(self._lib.soapb_contract(self._h, b.c, C.c_void_p(soap.data_ptr()),
                                            C.c_void_p(G.data_ptr()), int(g_layout), float(sgn),
                                            C.c_void_p(out.data_ptr())))
        return out

    def descriptor_and_vjp(self, b: DeviceBatch, G, sgn=1.0, g_layout=_lib.G_SITE_FASTEST,
                           soap=None, pair=None):
        soap = self._new((b.n_sites, self.n_soap)) if soap is None else soap
        pair = self._new((b.n_pairs, 3)) if pair is None else pair
        _lib.check(self._lib.soapb_descriptor_and_vjp(self._h, b.c, C.c_void_p(G.data_ptr()),
                                                      int(g_layout), float(sgn),
                                                      C.c_void_p(soap.data_ptr()),
                                                      C.c_void_p(pair.data_ptr())))
        return soap, pair

    def descriptor_fp64(self, b: DeviceBatch, cart=False):
        soap = self._new((b.n_sites, self.n_soap))
        cart_t = self._new((b.n_pairs, self.n_soap, 3)) if cart else None
        _lib.check(self._lib.soapb_descriptor_fp64(
            self._h, b.c, C.c_void_p(soap.data_ptr()),
            C.c_void_p(cart_t.data_ptr()) if cart_t is not None else None))
        return soap, cart_t

    def central_hessian(self, b: DeviceBatch, vecs, soap=None, out=None):
        """soapb_central_hessian: vecs (n_sites, n_vec, n_soap) == Fortran
        vecs(n_soap, n_vec, n_sites); returns hess (n_pairs, n_vec, 3, 3) ==
        Fortran hess(3, 3, n_vec, n_pairs), element [k, v, b, a].  soap: the
        normalised descriptor the weights were formed against (None: the FP64
        one the call computes)."""
        n_vec = int(vecs.shape[1])
        out = self._new((b.n_pairs, n_vec, 3, 3)) if out is None else out
        _lib.check(self._lib.soapb_central_hessian(
            self._h, b.c, C.c_void_p(soap.data_ptr()) if soap is not None else None, n_vec,
            C.c_void_p(vecs.data_ptr()), C.c_void_p(out.data_ptr())))
        return out

    def contract_cart_der(self, b: DeviceBatch, cart, G, sgn=1.0, g_layout=_lib.G_SITE_FASTEST,
                          out=None):
        out = self._new((b.n_pairs, 3)) if out is None else out
        _lib.check(self._lib.soapb_contract_cart_der(self._h, b.c, C.c_void_p(cart.data_ptr()),
                                                     C.c_void_p(G.data_ptr()), int(g_layout),
                                                     float(sgn), C.c_void_p(out.data_ptr())))
        return out
