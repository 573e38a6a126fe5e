// soapb_neigh.cu -- neighbour lists of periodic structures on the device, in
// the CSR layout get_soap takes (src/soap_turbo.f90:139-169): one row per
// central site, the site itself first (r = 0, theta = phi = 0), then every
// periodic image of every atom within rcut, with theta = acos(dz / r) and
// phi = atan2(dy, dx) of the displacement, and the species mask of
// assign_species_multiplicity (src/soap_turbo.f90:2188-2214).
//
// Atoms are binned into a cell list over the (possibly triclinic) cell: cells
// are at least rcut wide along each axis, and a site visits the cells within
// R = ceil(rcut * n_cells / plane_spacing) of its own along each axis, with the
// lattice translation each wrap implies (so small cells, where R cells reach
// around the box, visit several images of the same atoms).  Two passes: count,
// scan the counts into CSR offsets, then fill.  One warp per site; the fill
// pass gathers the site's row in shared memory and sorts it by (neighbour
// atom, distance) so the order depends on nothing but the inputs.
#include "soapb_scan.cuh"

namespace soapb {

namespace {

constexpr int kNbWarps = 4;      // warps (sites) per CTA of the count kernel
constexpr int kNbFillWarps = 2;  // warps (sites) per CTA of the fill kernel (its rows sit in shared memory)
constexpr int kNbShift = 512;    // image components are stored as n + kNbShift in 10 bits
static_assert(kNbMaxReach + 1 + 2 * kNbMaxWrap < kNbShift, "image translations must fit 10 bits");

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Displacement of atom j's image n (integer lattice vector) from atom i:
// (r_j + n . lattice) - r_i.  Both passes call this, so they agree bit for bit.
__device__ __forceinline__ void image_disp(const NbGeom &g, const double *pos, int i, int j, int nx, int ny,
                                           int nz, double &dx, double &dy, double &dz) {
  const double tx = nx * g.lat[0] + ny * g.lat[3] + nz * g.lat[6];
  const double ty = nx * g.lat[1] + ny * g.lat[4] + nz * g.lat[7];
  const double tz = nx * g.lat[2] + ny * g.lat[5] + nz * g.lat[8];
  dx = (pos[3 * j] + tx) - pos[3 * i];
  dy = (pos[3 * j + 1] + ty) - pos[3 * i + 1];
  dz = (pos[3 * j + 2] + tz) - pos[3 * i + 2];
}

// ---- per atom: its cell and the lattice translation that wraps it into the cell
// (image translations then stay within +-(kNbMaxReach + 1 + 2 kNbMaxWrap) <
// kNbShift, the packing range of the fill pass; farther atoms, and non-finite
// positions, are reported and put in cell 0)
__global__ void k_nb_bin(NbGeom g, const double *pos, int4 *atom_cell, int *cell_count,
                         unsigned long long *err) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= g.n_atoms) return;
  const double x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
  int c[3], w[3];
  bool bad = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double s = x * g.inv[d] + y * g.inv[3 + d] + z * g.inv[6 + d];
    const double f = floor(s);
    if (!(fabs(f) <= (double)kNbMaxWrap)) {
      bad = true;
      w[d] = 0;
      c[d] = 0;
    } else {
      w[d] = (int)f;
      c[d] = min(g.nc[d] - 1, max(0, (int)((s - f) * g.nc[d])));
    }
  }
  if (bad) atomicMax(err, kErrTop - kErrWrap);
  const int cell = (c[0] * g.nc[1] + c[1]) * g.nc[2] + c[2];
  atom_cell[a] = make_int4(cell, w[0], w[1], w[2]);
  atomicAdd(&cell_count[cell], 1);
}

// ---- per atom: its slot in its cell (the order inside a cell is arbitrary)
__global__ void k_nb_place(NbGeom g, const int4 *atom_cell, const int *cell_start, int *cell_fill,
                           int *cell_atoms) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= g.n_atoms) return;
  const int cell = atom_cell[a].x;
  cell_atoms[cell_start[cell] + atomicAdd(&cell_fill[cell], 1)] = a;
}

// Visits every candidate image of a site's stencil: visit(j, nx, ny, nz, ok)
// is called by all lanes of the warp together (ok false on padding lanes), so
// it may use warp collectives.
template <typename Visit>
__device__ __forceinline__ void for_each_neighbour(const NbGeom &g, const double *pos, const int4 *atom_cell,
                                                   const int *cell_start, const int *cell_atoms, int a,
                                                   Visit visit) {
  const int lane = threadIdx.x & 31;
  const int4 ca = atom_cell[a];
  const int cell = ca.x;
  const int cz = cell % g.nc[2], cy = (cell / g.nc[2]) % g.nc[1], cx = cell / (g.nc[2] * g.nc[1]);
  for (int ox = -g.R[0]; ox <= g.R[0]; ++ox) {
    const int X = cx + ox, wx = floor_div(X, g.nc[0]);
    const int qx = X - wx * g.nc[0];
    for (int oy = -g.R[1]; oy <= g.R[1]; ++oy) {
      const int Y = cy + oy, wy = floor_div(Y, g.nc[1]);
      const int qy = Y - wy * g.nc[1];
      for (int oz = -g.R[2]; oz <= g.R[2]; ++oz) {
        const int Z = cz + oz, wz = floor_div(Z, g.nc[2]);
        const int qz = Z - wz * g.nc[2];
        const int q = (qx * g.nc[1] + qy) * g.nc[2] + qz;
        const int t0 = cell_start[q], t1 = cell_start[q + 1];
        for (int t = t0; t < t1; t += 32) {
          const int tt = t + lane;
          int j = 0, nx = 0, ny = 0, nz = 0;
          bool ok = false;
          if (tt < t1) {
            j = cell_atoms[tt];
            const int4 cj = atom_cell[j];
            // the image of j in cell (X, Y, Z): translation (w - w_j + w_a) lattice vectors
            nx = wx - cj.y + ca.y;
            ny = wy - cj.z + ca.z;
            nz = wz - cj.w + ca.w;
            double dx, dy, dz;
            image_disp(g, pos, a, j, nx, ny, nz, dx, dy, dz);
            ok = dx * dx + dy * dy + dz * dz < g.rcut2 && !(j == a && nx == 0 && ny == 0 && nz == 0);
          }
          visit(j, nx, ny, nz, ok);
        }
      }
    }
  }
}

// ---- pass 1: neighbours of each site (the row length is one more: the site itself)
__global__ void __launch_bounds__(32 * kNbWarps) k_nb_count(NbGeom g, const double *pos, const int *sites,
                                                            const int4 *atom_cell, const int *cell_start,
                                                            const int *cell_atoms, int *counts,
                                                            unsigned long long *err) {
  const int w = blockIdx.x * kNbWarps + (threadIdx.x >> 5);
  if (w >= g.n_sites) return;
  const int a = sites[w];
  if (a < 0 || a >= g.n_atoms) {
    if ((threadIdx.x & 31) == 0) {
      counts[w] = 1;
      atomicMax(err, kErrTop - (unsigned long long)w);  // site index out of range
    }
    return;
  }
  int cnt = 0;
  for_each_neighbour(g, pos, atom_cell, cell_start, cell_atoms, a,
                     [&](int, int, int, int, bool ok) { cnt += __popc(__ballot_sync(0xffffffffu, ok)); });
  if ((threadIdx.x & 31) == 0) counts[w] = 1 + cnt;
}

// The species bits of neighbour j in the row of central atom a, as
// assign_species_multiplicity sets mask(k2, :) (src/soap_turbo.f90:2203-2211):
// the loop runs over the central atom's multiplicity, reading j's species.
__device__ __forceinline__ unsigned mask_bits(const NbGeom &g, const int *atom_species, const int *atom_mult,
                                              int a, int j) {
  unsigned bits = 0;
  const int mc = min(atom_mult[a], g.max_mult), mj = atom_mult[j];
  for (int i2 = 0; i2 < mc; ++i2) {
    const int sp = i2 < mj ? atom_species[(size_t)j * g.max_mult + i2] : 0;
    if (sp > 0 && sp <= g.n_species) bits |= 1u << (sp - 1);
  }
  return bits;
}

// ---- pass 2: each site's row, sorted by (neighbour atom, distance)
__global__ void __launch_bounds__(32 * kNbFillWarps) k_nb_fill(NbGeom g, const double *pos, const int *sites,
                                                           const int *atom_species, const int *atom_mult,
                                                           const int4 *atom_cell, const int *cell_start,
                                                           const int *cell_atoms, const int *off,
                                                           NbOut o, unsigned long long *err) {
  __shared__ unsigned long long s_key[kNbFillWarps][kNbCap];
  __shared__ unsigned s_img[kNbFillWarps][kNbCap];
  const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * kNbFillWarps + wl;
  if (w >= g.n_sites) return;
  const int a = sites[w];
  const int base = off[w], cnt = off[w + 1] - base - 1;
  if (a < 0 || a >= g.n_atoms) return;  // reported by the count pass
  if (cnt > kNbCap) {
    if (lane == 0) atomicMax(err, kErrTop - ((1ull << 32) + (unsigned long long)w));  // row too long
    return;
  }
  unsigned long long *key = s_key[wl];
  unsigned *img = s_img[wl];
  int filled = 0;
  const unsigned lt = (1u << lane) - 1u;
  for_each_neighbour(g, pos, atom_cell, cell_start, cell_atoms, a, [&](int j, int nx, int ny, int nz, bool ok) {
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      const int slot = filled + __popc(bal & lt);
      if (slot < kNbCap) {
        double dx, dy, dz;
        image_disp(g, pos, a, j, nx, ny, nz, dx, dy, dz);
        const float r = (float)sqrt(dx * dx + dy * dy + dz * dz);
        key[slot] = ((unsigned long long)(unsigned)j << 32) | __float_as_uint(r);
        img[slot] = ((unsigned)(nx + kNbShift) << 20) | ((unsigned)(ny + kNbShift) << 10) |
                    (unsigned)(nz + kNbShift);
      }
    }
    filled += __popc(bal);
  });
  // bitonic sort of the row by (atom, FP32 distance, image translation in x, y, z
  // order): every candidate differs in that triple, so the row's order does not
  // depend on the order the cell list happened to hold the atoms in (padded with
  // the largest key)
  int npow = 1;
  while (npow < cnt) npow <<= 1;
  for (int t = cnt + lane; t < npow; t += 32) {
    key[t] = ~0ull;
    img[t] = ~0u;
  }
  __syncwarp();
  for (int k = 2; k <= npow; k <<= 1)
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int t = lane; t < npow; t += 32) {
        const int p = t ^ jj;
        if (p > t) {
          const bool up = (t & k) == 0;
          const unsigned long long kt = key[t], kp = key[p];
          const bool gt = kt > kp || (kt == kp && img[t] > img[p]);
          if (gt == up) {
            key[t] = kp;
            key[p] = kt;
            const unsigned it = img[t];
            img[t] = img[p];
            img[p] = it;
          }
        }
      }
      __syncwarp();
    }
  // the site itself first, then its sorted neighbours
  for (int e = lane - 1; e < cnt; e += 32) {
    const int k = base + 1 + e;
    int j;
    double r = 0.0, th = 0.0, ph = 0.0;
    if (e < 0) {
      j = a;
    } else {
      j = (int)(key[e] >> 32);
      const unsigned im = img[e];
      const int nx = (int)(im >> 20) - kNbShift, ny = (int)((im >> 10) & 1023u) - kNbShift,
                nz = (int)(im & 1023u) - kNbShift;
      double dx, dy, dz;
      image_disp(g, pos, a, j, nx, ny, nz, dx, dy, dz);
      r = sqrt(dx * dx + dy * dy + dz * dz);
      th = acos(fmin(1.0, fmax(-1.0, dz / r)));
      ph = atan2(dy, dx);
    }
    o.rjs[k] = r;
    o.thetas[k] = th;
    o.phis[k] = ph;
    o.neigh_atom[k] = j;
    const unsigned bits = mask_bits(g, atom_species, atom_mult, a, j);
    for (int s = 0; s < g.n_species; ++s) o.mask[(size_t)s * o.n_pairs + k] = (uint8_t)((bits >> s) & 1u);
  }
  if (lane == 0) {
    o.n_neigh[w] = cnt + 1;
    o.species_mult[w] = atom_mult[a];
  }
  for (int m = lane; m < g.max_mult; m += 32) o.species[(size_t)w * g.max_mult + m] = atom_species[(size_t)a * g.max_mult + m];
}

__global__ void __launch_bounds__(256) k_nb_scan(DevBatch B, int tiles, int max_spins) {
  __shared__ int sv[kScanTile];
  prep_scan_tile<256>(B, tiles, sv, max_spins);
}

}  // namespace

cudaError_t launch_nb_bin(const NbGeom &g, const double *pos, int4 *atom_cell, int *cell_count,
                          unsigned long long *err, cudaStream_t s) {
  if (g.n_atoms > 0) k_nb_bin<<<(g.n_atoms + 255) / 256, 256, 0, s>>>(g, pos, atom_cell, cell_count, err);
  return cudaGetLastError();
}

cudaError_t launch_nb_place(const NbGeom &g, const int4 *atom_cell, const int *cell_start, int *cell_fill,
                            int *cell_atoms, cudaStream_t s) {
  if (g.n_atoms > 0) k_nb_place<<<(g.n_atoms + 255) / 256, 256, 0, s>>>(g, atom_cell, cell_start, cell_fill, cell_atoms);
  return cudaGetLastError();
}

cudaError_t launch_nb_count(const NbGeom &g, const double *pos, const int *sites, const int4 *atom_cell,
                            const int *cell_start, const int *cell_atoms, int *counts, unsigned long long *err,
                            cudaStream_t s) {
  if (g.n_sites > 0)
    k_nb_count<<<(g.n_sites + kNbWarps - 1) / kNbWarps, 32 * kNbWarps, 0, s>>>(g, pos, sites, atom_cell, cell_start,
                                                                               cell_atoms, counts, err);
  return cudaGetLastError();
}

cudaError_t launch_nb_fill(const NbGeom &g, const double *pos, const int *sites, const int *atom_species,
                           const int *atom_mult, const int4 *atom_cell, const int *cell_start, const int *cell_atoms,
                           const int *off, const NbOut &o, unsigned long long *err, cudaStream_t s) {
  if (g.n_sites > 0)
    k_nb_fill<<<(g.n_sites + kNbFillWarps - 1) / kNbFillWarps, 32 * kNbFillWarps, 0, s>>>(
        g, pos, sites, atom_species, atom_mult, atom_cell, cell_start, cell_atoms, off, o, err);
  return cudaGetLastError();
}

cudaError_t launch_scan(const int *counts, int n, int *off, unsigned long long *state, cudaStream_t s,
                        int blocks, int max_spins) {
  DevBatch B{};
  B.n_sites = n;
  B.n_pairs = -1;
  B.n_neigh = counts;
  B.off = off;
  B.err = state;
  const int tiles = prep_scan_tiles(n);
  if (blocks < 0 || blocks > tiles) blocks = tiles;
  if (blocks > 0) k_nb_scan<<<blocks, 256, 0, s>>>(B, tiles, max_spins);
  return cudaGetLastError();
}

}  // namespace soapb
