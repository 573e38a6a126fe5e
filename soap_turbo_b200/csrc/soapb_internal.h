// soapb_internal.h -- definitions shared by the host API and the kernels.
//
// DevParams is the whole descriptor definition as the kernels see it.  It is
// passed by value as a kernel argument (a few KB), so a launch needs no
// constant-memory symbol and two contexts never share state.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define SOAPB_MAX_SPECIES 8
#define SOAPB_MAX_ALPHA 16
#define SOAPB_MAX_LMAX 12
#define SOAPB_KMAX_CAP ((SOAPB_MAX_LMAX + 1) * (SOAPB_MAX_LMAX + 2) / 2)
#define SOAPB_NTAB 28 /* recursion tables, index n+4 for n = -4 .. 23 */

// Radial constants of one species, in the scaled units of the reference's
// radial kernel (rcut_hard = 1; src/soap_turbo_radial.f90:455-526).
struct RadSp {
  double inv_rcut, rs, atom_sigma, dr, sqrt_rcut, inv_sqrt_rcut;
  double q, drnf, sigma_sq0, N_gauss;
  double c;            // atom_sigma_r_scaling (scaled by nothing: dimensionless)
  double amp_scaling;  // amplitude_scaling
  double cw;           // central_weight
  double gscale;       // global_scaling
  double rcut_hard;    // unscaled
  int alpha, n_poly, nbeg, has_filter, do_central, pad;
};

// DevParams::basis of the poly3operator basis (SOAPB_BASIS_POLY3OPERATOR)
constexpr int kBasisOperator = 2;

// The tabulated radial expansion of one species (poly3 / poly3gauss with
// atom_sigma_r_scaling = 0, when every R_n(r) and dR_n/dr is a fixed function
// of r): piecewise polynomials in t in [-1, 1] on segments of r.  The
// reference's expansion branches on r -- the filter kept when r_soft - r < 4
// sigma (src/soap_turbo_radial.f90:721-769), the origin-Gaussian moment only
// for r < 4 (sigma_0 + sigma) (:875-908), the amplitude zero where h(r) <=
// 1e-10 (:589-635) -- so each branch state (keep | !gm << 1) has an interval
// of its own, chosen per pair by the same FP64 tests.
constexpr int kRadTabDeg = 7;  // polynomial degree of each segment
struct RadTab {
  double lo[4], inv_h[4];  // per branch state: interval start, segments per unit r
  int base[4], nseg[4];    // first segment in the coefficient table, segment count
};

struct DevParams {
  int n_species, l_max, k_max, n_max;
  int basis;          // 0 poly3, 1 poly3gauss, 2 poly3operator (kBasisOperator)
  int scaling_poly;   // scaling_mode == "polynomial"
  int radial_enh;     // radial_enhancement
  int legacy_seed;    // legacy_filter_seed
  int n_soap, n_kept, n_pairs, n_sites;
  double rcut_max, rcut2;
  RadSp rad[SOAPB_MAX_SPECIES];
  double sig_t[SOAPB_MAX_SPECIES], sig_t_c[SOAPB_MAX_SPECIES];
  double ra[SOAPB_NTAB], rb[SOAPB_NTAB], rc[SOAPB_NTAB], R1[SOAPB_NTAB], R2[SOAPB_NTAB];
  float preflm[SOAPB_KMAX_CAP];
  double preflm64[SOAPB_KMAX_CAP];
  // device tables (owned by the context)
  const double *Wblk;     // per species alpha x alpha, column-major, at s*AMAX2
  int wstride;            // doubles between species blocks
  const double *central;  // n_max: poly3gauss central-atom term per radial index
  const int *kept_nnl;    // n_kept: n | np << 8 | l << 16 of the kept components
  const int *pi_off;      // n_soap + 1: CSR over outputs of the compression map
  const int *pi_q;        //   kept position feeding each entry
  const float *pi_el;
  const double *pi_el64;
  const int *pj_off;      // n_kept + 1: CSR over kept components (transpose)
  const int *pj_o;        //   output index of each entry
  const float *pj_el;
  const double *pj_el64;
  const int *hl_off;      // (l_max+1)*n_max + 1: per (l, n) list of (np, q, fac)
  const int *hl_np;
  const int *hl_q;
  const float *hl_fac;
  const double *hl_fac64;
  // Per-CTA constants of the mixed kernels: two blobs copied into shared
  // memory with 16-byte loads, one for the pair and descriptor kernels
  // (blob: W blocks, then from off_rad on the descriptor's part) and one for
  // the contract kernel (blob_c, species constants at offset 0).  Offsets in
  // bytes from the start of the blob that holds the section.
  const unsigned char *blob;
  int blob_bytes;         // multiple of 16
  const unsigned char *blob_c;
  int blob_c_bytes;       // multiple of 16
  int amax_t;             // the kernel instantiation's radial block (8 or 16)
  // in blob:
  int off_W;              // n_species blocks of amax_t^2 doubles (alpha x alpha used)
  int off_kpx;            // (l_max+2)(l_max+3)/2 float: preflm to l_max + 1 (pair kernel)
  int off_rad;            // n_species RadSp
  int off_klm;            // KS int: l | m << 8
  int off_citem;          // n_citem int: c_nlm items species | k << 4 | half << 12
  int off_kept;           // n_kept int: kept_nnl
  int off_central;        // n_max double: poly3gauss central-atom term
  // in blob_c (n_species RadSp at 0):
  int off_kidx;           // KS int4: P_l^m indices of the derivative forms
  int off_kcoef;          // KS float4: their coefficients
  int off_klm_c;          // KS int: l | m << 8
  int off_nmap;           // n_max int: species | local index << 8
  int off_hitem;          // n_hitem int: H items n | l << 8
  int off_hloff;          // (l_max+1)*n_max + 1 int: per (l, n) list offsets
  int off_hl;             // packed Y-list entries np | q << 8 | (n == np) << 31, when hl_in_blob
  int n_citem, n_hitem;
  int hl_in_blob;         // the packed Y lists fit in the blob (else read from hl_packed)
  const int *hl_packed;   // global copy of the packed Y lists
  int cmap_identity;      // the compression map sends kept component q to output q, weight 1
  // tabulated radial expansion (the pair kernel's FP32 form, see RadTab):
  // coefficients [segment][k = 0..kRadTabDeg][2 amax_t] (R_n then dR_n/dr, with
  // 4 pi global_scaling folded in), monomials in t ascending
  int rtab;               // 1: the pair kernel evaluates the tables
  int tc_contract;        // 1: the contract's per-entry contraction runs on the tensor cores
  int tc_descriptor;      // 1: the descriptor's c_nlm runs on the tensor cores
  const float *rtab_coef;
  RadTab rtab_sp[SOAPB_MAX_SPECIES];
  // power spectrum on the tensor cores: P_l[n, J] for rows n (ps_mt tiles of
  // 16) and the column set J (ps_nt tiles of 8) that covers every kept (n, n')
  int ps_mt, ps_nt;
  // ... with tcgen05 (k_descriptor_tc): the l values in ps_ng groups; group g
  // stacks rows (l, n) for its l, the J rows first, into one M = 128 tile of
  // K = ps_gk[g] columns (l's block at ps_ko[l], 2(l+1) wide); B is the tile's
  // first ps_gnb[g] rows.  Row r of group g is described by the blob's
  // off_psrow table at ps_grow[g] + r: n | l << 8 | (D column of its P_l[n, J_0]) << 16.
  int ps_ng;              // 0: the mma.sync form
  int ps_nj;              // |J|
  int ps_gk[SOAPB_MAX_LMAX + 1], ps_gnb[SOAPB_MAX_LMAX + 1], ps_grows[SOAPB_MAX_LMAX + 1];
  int ps_grow[SOAPB_MAX_LMAX + 1], ps_ko[SOAPB_MAX_LMAX + 1];
  int off_psrow;          // (blob) the row tables of all groups
  int off_psj;            // (blob) 8 ps_nt int: the radial index of each column (-1 = padding)
  int off_kpos;           // (blob) n_kept int: tile position (l, row, column) | (n != n') << 31
};

// Size of RadSp padded to 16 bytes, as laid out in the constants blob.
#define SOAPB_RADSP_BYTES ((int)((sizeof(RadSp) + 15) / 16 * 16))

// Batch tables the prep kernel derives from the caller's CSR arrays.
struct DevBatch {
  int n_sites, n_pairs, max_mult;
  const int *n_neigh, *species, *species_mult;
  const uint8_t *mask;
  const double *rjs, *thetas, *phis;
  int *off;              // n_sites + 1 (prep output)
  uint8_t *bits;         // n_pairs: mask bits (prep output)
  unsigned long long *err;  // prep_err_words(n_sites) words, cleared before each prep launch:
                            // the first input error, the prep scan's state and (last
                            // word) the site kernels' work counters
  float *rad;            // (n_pairs, n_species, 2, amax_t): 4 pi R_n and its r-derivative
  float *ang;            // (n_pairs, ang_row): the pair's angular row (see soapb_mixed.cu)
  int *ticket;           // work counters of the persistent site kernels, in the last word
                         // of err (the kernels put them back to 0 when they finish)
  int site_lo, site_hi;  // the sites a site-kernel launch processes (all: 0, n_sites)
  int *order = nullptr;  // n_sites: the order in which the persistent site kernels take the
                         // sites, heaviest rows first (written by the pair kernel's scan when
                         // one scan tile covers the batch), or null: index order
};

// Kernel launchers (soapb_mixed.cu, soapb_fp64.cu)
namespace soapb {
struct LaunchCfg {
  int threads;           // threads per site CTA
  cudaStream_t stream;
  int max_ctas;          // persistent grid cap (0 = from the occupancy)
};
cudaError_t launch_prep(const DevParams &P, const DevBatch &B, cudaStream_t s);
// sites per tile of the CSR offset scan (soapb_scan.cuh)
constexpr int kScanTileSites = 2048;
// 64-bit words of DevBatch::err for a batch of n_sites; the launcher's caller
// clears them before each prep launch
int prep_err_words(int n_sites);
// The error code in err[0]: a bad pair's index, a value >= 2^33 for CSR and
// scan failures, or all ones when the launch found no error.
unsigned long long prep_error_code(unsigned long long word);
// The pair rows of pairs [pair_lo, pair_hi) (pair_hi < 0: all), with the CSR
// offset scan of the whole batch when scan is set (one launch per batch must).
cudaError_t launch_pair(const DevParams &P, const DevBatch &B, cudaStream_t s, int do_der, int pair_lo = 0,
                        int pair_hi = -1, bool scan = true);
int ang_row_floats(const DevParams &P);
size_t keep_floats_per_site(const DevParams &P);
cudaError_t launch_descriptor(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                              double *soap, float *keep_c, double *keep_norm, int keep);
cudaError_t launch_contract(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                            const double *soap, const double *G, int g_layout, double sgn,
                            const float *keep_c, const double *keep_norm, double *pair);
size_t descriptor_smem(const DevParams &P, int threads);
// Device address and size of the static scratch array (soapb_noalloc.cu);
// `device` must be current.
cudaError_t noalloc_scratch(int device, unsigned char **addr, size_t *bytes);
size_t contract_smem(const DevParams &P, int threads);
size_t contract_tc_smem(const DevParams &P);  // dynamic shared memory of the tensor-core contract

// Error codes reported through an error word (kErrTop - code under atomicMax,
// so the smallest code wins; 0 = none): a pair or site index below 2^32, else
constexpr unsigned long long kErrCsr = 1ull << 33;        // n_neigh negative or sum != n_pairs
constexpr unsigned long long kErrScan = (1ull << 33) + 1;  // the scan's look-back wait gave up
constexpr unsigned long long kErrWrap = (1ull << 33) + 2;  // an atom far outside the cell
constexpr unsigned long long kErrTc = (1ull << 33) + 3;    // a wait for tensor-core MMAs gave up
constexpr unsigned long long kErrTop = 1ull << 34;

// Neighbour-list builder (soapb_neigh.cu)
constexpr int kNbCap = 1024;  // neighbours within rcut of one site the fill pass can sort
constexpr int kNbMaxWrap = 200;  // |lattice translation| that wraps an atom into the cell
constexpr int kNbMaxReach = 100; // cells a site may visit on each side
struct NbGeom {
  double lat[9];   // cell vectors a, b, c as rows (Cartesian)
  double inv[9];   // inverse: fractional s = r . inv (row vectors)
  int nc[3];       // cells along each axis (each at least rcut wide)
  int R[3];        // cells visited on each side of a site's own
  double rcut2;
  int n_atoms, n_sites, max_mult, n_species;
};
struct NbOut {     // get_soap's inputs, plus the atom behind every pair
  int n_pairs;
  double *rjs, *thetas, *phis;
  uint8_t *mask;   // (n_species, n_pairs)
  int *neigh_atom, *n_neigh, *species, *species_mult;
};
cudaError_t launch_nb_bin(const NbGeom &g, const double *pos, int4 *atom_cell, int *cell_count,
                          unsigned long long *err, cudaStream_t s);
cudaError_t launch_nb_place(const NbGeom &g, const int4 *atom_cell, const int *cell_start, int *cell_fill,
                            int *cell_atoms, cudaStream_t s);
cudaError_t launch_nb_count(const NbGeom &g, const double *pos, const int *sites, const int4 *atom_cell,
                            const int *cell_start, const int *cell_atoms, int *counts, unsigned long long *err,
                            cudaStream_t s);
cudaError_t launch_nb_fill(const NbGeom &g, const double *pos, const int *sites, const int *atom_species,
                           const int *atom_mult, const int4 *atom_cell, const int *cell_start, const int *cell_atoms,
                           const int *off, const NbOut &o, unsigned long long *err, cudaStream_t s);
// Exclusive scan of n counts into off (n + 1 entries); state: prep_err_words(n)
// words cleared beforehand.  blocks < 0: one block per tile (the scan); fewer
// blocks and a smaller max_spins serve the self-test of the bounded wait.
cudaError_t launch_scan(const int *counts, int n, int *off, unsigned long long *state, cudaStream_t s,
                        int blocks = -1, int max_spins = 1 << 20);

// Plain FP64 staged path
struct Fp64Work {
  double *rad, *rad_der;   // (n_pairs, n_max)
  double *ang;             // 4 x (n_pairs, k_max) complex
  double *cnk;             // (n_sites, n_max, k_max) complex
  double *soap_unnorm;     // (n_sites, n_soap)
  double *norm;            // n_sites
};
// soap_acc (may be null): the caller's soap, accumulated into before the norm
// (compressed get_soap); self_init (may be null, with cart): the caller's self
// columns of soap_cart_der, (3, n_soap) per site, which the self column
// accumulates into.  soap may be the same array as soap_acc.
cudaError_t launch_fp64_descriptor(const DevParams &P, const DevBatch &B, cudaStream_t s,
                                   const Fp64Work &w, int do_der, double *soap, double *cart,
                                   int *launches, const double *soap_acc = nullptr,
                                   const double *self_init = nullptr);
size_t fp64_cart_smem(const DevParams &P);  // dynamic shared memory of the soap_cart_der kernel
cudaError_t launch_fp64_contract(const DevParams &P, const DevBatch &B, cudaStream_t s,
                                 const double *cart, const double *G, int g_layout, double sgn,
                                 double *pair, int *launches);
// Central-atom Hessian (soapb_hessian.cu), on the state launch_fp64_descriptor
// left with do_der: second radial derivatives into rad_der2 (n_pairs, n_max),
// per-pair geometry records into geo (n_pairs * hess_geo_doubles) and good
// (n_pairs ints), then hess (n_pairs, n_vec, 3, 3) = 9 n_vec doubles per pair,
// cleared first.  scratch: grid * hess_scratch_doubles doubles; ticket: one int.
size_t hess_scratch_doubles(const DevParams &P, int n_vec);
size_t hess_geo_doubles(const DevParams &P);
size_t hess_smem_bytes(const DevParams &P, int n_vec);  // dynamic shared memory of k64_hess
int hess_grid(const DevParams &P, int n_vec);
cudaError_t launch_hessian(const DevParams &P, const DevBatch &B, cudaStream_t s, const Fp64Work &w,
                           double *rad_der2, double *geo, int *good, const double *soap, int n_vec,
                           const double *vecs, double *hess, double *scratch, int grid, int *ticket, int *launches);
}  // namespace soapb
