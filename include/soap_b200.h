/*
 * soap_b200.h -- C ABI of libsoapb200.so, a B200 (sm_100a) implementation of
 * soap_turbo's SOAP descriptor path: get_soap, its Cartesian derivatives and
 * the soap_contract force vector-Jacobian product.
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the reference's argument lists and host
 *     arrays (soapb_get_soap, soapb_soap_contract, ...).  They keep module
 *     state the way the reference's Fortran module does (basis cache, the
 *     contract state), on the current CUDA device.  A Fortran iso_c_binding
 *     module binds exactly these (soap_turbo_b200/fortran/).
 *
 *  2. A context API on device pointers and a caller-chosen CUDA stream, for
 *     callers that keep their neighbour lists on the GPU.  No call of this
 *     layer synchronises the stream.
 *
 * Layouts are the reference's Fortran column-major layouts:
 *   soap(n_soap, n_sites)             soap[i*n_soap + s]
 *   soap_cart_der(3, n_soap, n_pairs) cart[(k*n_soap + s)*3 + c]
 *   G(n_sites, n_soap)                G[s*n_sites + i]
 *   pair(3, n_pairs)                  pair[k*3 + c]
 *   mask(n_pairs, n_species)          mask[s*n_pairs + k]  (one byte, 0/1)
 *   species(max_mult, n_sites)        species[i*max_mult + m] (1-based)
 *   W, S (n_max, n_max)               W[col*n_max + row]
 *
 * Every function returns SOAPB_OK (0) or one of the status codes below;
 * soapb_last_error() gives the message of the last failure on this thread.
 */
#ifndef SOAP_B200_H
#define SOAP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum {
  SOAPB_OK = 0,
  SOAPB_ERR_ARGUMENT = 1,        /* bad size, null pointer, unsupported value            */
  SOAPB_ERR_ALPHA_TOO_LARGE = 2, /* alpha_max above the basis' limit: poly3 > 10,
                                    poly3gauss > 11 (src/soap_turbo_radial.f90:144-153,
                                    210-219)                                            */
  SOAPB_ERR_CONTRACT_STATE = 3,  /* soap_contract without a preceding get_soap with
                                    contract (src/soap_turbo.f90:1744-1747)             */
  SOAPB_ERR_COMPRESS_MODE = 4,   /* compress_mode not understood
                                    (src/soap_turbo_compress.f90:305-306)               */
  SOAPB_ERR_BASIS = 5,           /* basis other than poly3 / poly3gauss / poly3operator,
                                    or the Hessian asked of poly3operator                */
  SOAPB_ERR_CUDA = 6,            /* CUDA runtime failure                                 */
  SOAPB_ERR_NO_DEVICE = 7,       /* no usable sm_100 device                              */
  SOAPB_ERR_INPUT = 8,           /* non-finite or negative distance, bad CSR, bad mask   */
  SOAPB_ERR_BASIS_MATRIX = 9,    /* overlap matrix not positive definite                 */
  SOAPB_ERR_HESSIAN_STATE = 10   /* get_soap_central_hessian without a matching get_soap
                                    (src/soap_turbo.f90:1206-1227)                       */
};

/* poly3operator (src/soap_turbo_radial.f90:1549-2141): poly3's W with a
 * piecewise-cubic atom density in place of the Gaussian; alpha_max 1..11; no
 * second radial derivatives (no central-atom Hessian). */
enum { SOAPB_BASIS_POLY3 = 0, SOAPB_BASIS_POLY3GAUSS = 1, SOAPB_BASIS_POLY3OPERATOR = 2 };
enum { SOAPB_SCALING_POLYNOMIAL = 0, SOAPB_SCALING_NONE = 1 };
/* Arithmetic of the descriptor + VJP path. */
enum {
  SOAPB_PREC_MIXED = 0, /* FP32 pair/contraction arithmetic; FP64 radial integrals,
                           W-transform and angular prefactors (the default)         */
  SOAPB_PREC_FP64 = 1   /* plain FP64, staged like the reference (materialises
                           soap_cart_der, then contracts)                            */
};
/* Layout of the upstream gradient G given to the contract calls. */
enum {
  SOAPB_G_SITE_FASTEST = 0, /* the reference's G(n_sites, n_soap)  */
  SOAPB_G_SOAP_FASTEST = 1  /* G(n_soap, n_sites), soap's own layout */
};

const char *soapb_last_error(void);
const char *soapb_version(void);

/* ============================================================ drop-in layer */

/* get_soap (src/soap_turbo.f90:139-169).  Same arguments in the same order,
 * as plain pointers plus the extents Fortran would carry in the descriptors:
 * max_species_multiplicity = size(species,1), n_soap = size(soap,1).
 * basis: "poly3" | "poly3gauss" | "poly3operator"; scaling_mode: "polynomial" | other
 * (poly3operator with another scaling mode: amplitude 1, which the reference
 * leaves unset).
 * soap and soap_cart_der are intent(inout) as in the reference: with
 * compress_soap the descriptor is added into the caller's soap before the norm
 * is taken (src/soap_turbo.f90:798-802), without it soap is overwritten; the
 * neighbour columns of soap_cart_der are overwritten and each site's self
 * column is accumulated into (:888-892).  The reference's callers pass both
 * zeroed.
 * do_derivatives && !contract: soap_cart_der (3, n_soap, n_atom_pairs) is
 * written, computed in FP64 as the reference does; otherwise it may be NULL.
 * do_derivatives && contract: the state for soapb_soap_contract is kept.
 * do_timing prints per-phase GPU times, as the reference's do_timing does.
 * Host arrays may be pageable (staged through the library's page-locked
 * buffers) or page-locked; a page-locked soap that the GPU can address (mapped,
 * as every page-locked allocation is on a 64-bit host with unified addressing)
 * is written by the site kernel in place while the call runs. */
int soapb_get_soap(int32_t n_sites, const int32_t *n_neigh, int32_t n_species,
                   const int32_t *species, int32_t max_species_multiplicity,
                   const int32_t *species_multiplicity, int32_t n_atom_pairs,
                   const uint8_t *mask, const double *rjs, const double *thetas,
                   const double *phis, const int32_t *alpha_max, int32_t l_max,
                   const double *rcut_hard, const double *rcut_soft, const double *nf,
                   const double *global_scaling, const double *atom_sigma_r,
                   const double *atom_sigma_r_scaling, const double *atom_sigma_t,
                   const double *atom_sigma_t_scaling, const double *amplitude_scaling,
                   int32_t radial_enhancement, const double *central_weight,
                   const char *basis, const char *scaling_mode, int32_t do_timing,
                   int32_t do_derivatives, int32_t compress_soap,
                   int32_t compress_P_nonzero, const int32_t *compress_P_i,
                   const int32_t *compress_P_j, const double *compress_P_el,
                   double *soap, int32_t n_soap, double *soap_cart_der, int32_t contract);

/* soap_contract (src/soap_turbo.f90:1723-1730): pair(1:3,k) =
 * sgn * sum_s G(i,s) * d soap(s,i) / d r_k, for the batch of the last
 * soapb_get_soap called with do_derivatives and contract.  G is
 * G(n_sites, n_soap) (site fastest), soap the normalised descriptor that call
 * returned.  The extents must match that call.  A page-locked pair that the
 * GPU can address is written by the contract kernel in place. */
int soapb_soap_contract(const double *soap, const double *G, double sgn, double *pair,
                        int32_t n_sites, int32_t n_soap, int32_t n_atom_pairs);

/* Module flag legacy_filter_seed (src/soap_turbo_radial.f90:67); default 1. */
int soapb_set_legacy_filter_seed(int32_t legacy);
int soapb_get_legacy_filter_seed(int32_t *legacy);

/* Module flag soap_hessian_enabled (src/soap_turbo.f90:76); default 0.  With
 * it set, soapb_get_soap called with do_derivatives records the batch for
 * soapb_get_soap_central_hessian; it then needs legacy_filter_seed = 0 (else
 * soapb_get_soap returns SOAPB_ERR_ARGUMENT, as the reference's radial kernel
 * stops, src/soap_turbo_radial.f90:318-323). */
int soapb_set_soap_hessian_enabled(int32_t enabled);
int soapb_get_soap_hessian_enabled(int32_t *enabled);

/* get_soap_central_hessian (src/soap_turbo.f90:1151-1160), same arguments plus
 * n_soap = size(soap,1):
 *   hess(3, 3, n_vec, n_atom_pairs)  hess[((k*n_vec + v)*3 + b)*3 + a]
 *     = sum_d vecs(d, v, i) d^2 soap(d, i) / dr_ia dr_jb
 * for pair k = (site i, neighbour j), a of the central atom and b of the
 * neighbour; the self pair's block is minus the sum of the others.
 *   vecs(n_soap, n_vec, n_sites)     vecs[(i*n_vec + v)*n_soap + d]
 *   soap                             the normalised descriptor get_soap returned
 * It must follow a soapb_get_soap on the same batch with do_derivatives and
 * soap_hessian_enabled set (else SOAPB_ERR_HESSIAN_STATE, as the reference
 * stops).  The descriptor definition, species and neighbour geometry are the
 * ones that get_soap call kept on the device (the reference reads its kept
 * buffers the same way); the geometry, cutoff, sigma and compression arguments
 * here are accepted for the reference's argument list and not read again.
 * Computed in FP64. */
int soapb_get_soap_central_hessian(int32_t n_sites, const int32_t *n_neigh, int32_t n_atom_pairs,
                                   int32_t n_species, const uint8_t *mask, const double *rjs,
                                   const double *thetas, const double *phis, int32_t l_max,
                                   const double *rcut_hard, const double *atom_sigma_t,
                                   const double *atom_sigma_t_scaling, int32_t compress_soap,
                                   int32_t compress_P_nonzero, const int32_t *compress_P_i,
                                   const int32_t *compress_P_j, const double *compress_P_el,
                                   const double *soap, int32_t n_soap, int32_t n_vec, const double *vecs,
                                   double *hess);

/* Arithmetic of the drop-in layer (SOAPB_PREC_*); default mixed. */
int soapb_set_precision(int32_t precision);

/* Replace the drop-in layer's basis matrices with caller-supplied ones (the
 * same W and S the caller feeds another implementation); n_max x n_max,
 * block diagonal.  Kept until the basis definition changes. */
int soapb_set_basis_matrices(int32_t n_max, const double *W, const double *S);

/* get_compress_indices (src/soap_turbo_compress.f90:44).  what_to_do =
 * "get_dim" fills dim and P_nonzero only; "set_indices" also fills P_i, P_j
 * (1-based) and P_el, each of capacity P_nonzero.  Modes: "trivial"
 * ("Trivial", :86-119) and Darby's "nu_R_nu_S" with nu_R, nu_S in 0..2
 * ("0_0" .. "2_2", :120-303; every species must have the same alpha_max,
 * else SOAPB_ERR_COMPRESS_MODE).  Other modes return SOAPB_ERR_COMPRESS_MODE. */
int soapb_get_compress_indices(const char *compress_mode, int32_t n_species,
                               const int32_t *alpha_max, int32_t l_max, int32_t *dim,
                               int32_t *P_nonzero, int32_t *P_i, int32_t *P_j, double *P_el,
                               const char *what_to_do);

/* Overlap S and W = S^{-1/2} of one species' basis, alpha x alpha, computed
 * in extended precision (get_orthonormalization_matrix_poly3[gauss],
 * src/soap_turbo_radial.f90:1023-1219). */
int soapb_orthonormalization_matrix(int32_t basis, int32_t alpha_max, double atom_sigma_r,
                                    double rcut_hard, double *S, double *W);

/* ============================================================ context layer */

typedef struct soapb_context soapb_context;

/* One descriptor definition: the per-species and scalar hyperparameters of
 * get_soap plus the compression map.  Arrays are host pointers of length
 * n_species (P_* of length P_nonzero) and are copied. */
typedef struct {
  int32_t n_species;
  int32_t l_max;
  int32_t basis;              /* SOAPB_BASIS_*   */
  int32_t scaling_mode;       /* SOAPB_SCALING_* */
  int32_t radial_enhancement; /* 0, 1 or 2       */
  int32_t legacy_filter_seed; /* 1 = reference default */
  const int32_t *alpha_max;
  const double *rcut_hard, *rcut_soft, *nf, *global_scaling;
  const double *atom_sigma_r, *atom_sigma_r_scaling;
  const double *atom_sigma_t, *atom_sigma_t_scaling;
  const double *amplitude_scaling, *central_weight;
  int32_t compress;           /* 0: uncompressed */
  int32_t P_nonzero;
  const int32_t *P_i, *P_j;   /* 1-based */
  const double *P_el;
} soapb_hyper;

/* One batch of sites: the CSR neighbour list, all DEVICE pointers. */
typedef struct {
  int32_t n_sites;
  int32_t n_atom_pairs;
  int32_t max_species_multiplicity;
  const int32_t *n_neigh;              /* n_sites */
  const int32_t *species;              /* (max_mult, n_sites), 1-based */
  const int32_t *species_multiplicity; /* n_sites */
  const uint8_t *mask;                 /* (n_pairs, n_species) */
  const double *rjs, *thetas, *phis;   /* n_pairs */
} soapb_batch;

/* Creates a context on `device` (-1: the current device) and builds W, S. */
int soapb_create(const soapb_hyper *hyper, int32_t device, soapb_context **out);
int soapb_destroy(soapb_context *ctx);
/* Caller-supplied basis matrices (host, n_max x n_max, block diagonal). */
int soapb_set_basis(soapb_context *ctx, const double *W, const double *S);
int soapb_get_basis(const soapb_context *ctx, double *W, double *S);
/* n_soap of the definition (compressed length when compressing). */
int soapb_n_soap(const soapb_context *ctx, int32_t *n_soap);
/* Work on this cudaStream_t from now on (0 = legacy default stream). */
int soapb_set_stream(soapb_context *ctx, void *stream);
/* Work tuning: threads per site CTA (64, 128 or 256) for both site kernels;
 * 0 returns to the autotuner's choice, or 128 before any autotuning. */
int soapb_set_threads_per_site(soapb_context *ctx, int32_t threads);
/* Autotuner: times the descriptor and the contract on this batch in each form
 * -- the tensor-core kernels (when allowed, see soapb_set_tensor_cores) and the
 * CUDA-core kernels at every CTA size (64, 128, 256 threads per site) -- and
 * each persistent grid cap (the occupancy limit, 2 and 1 CTAs per SM), and
 * keeps the fastest per kernel in the context.  choice (4, may be NULL)
 * receives {descriptor threads, descriptor grid cap, contract threads,
 * contract grid cap}: threads 0 means the tensor-core kernel, a grid cap of 0
 * the occupancy limit.  A set-up call: it allocates and frees work buffers,
 * synchronises the context's stream and discards the state kept for
 * soapb_contract.  Results are bit-reproducible for a fixed choice; another
 * CTA size changes the summation grouping within FP32 rounding. */
int soapb_autotune(soapb_context *ctx, const soapb_batch *batch, int32_t *choice);

/* Radial expansion of the mixed path.  With atom_sigma_r_scaling = 0 (poly3,
 * poly3gauss), every R_n(r) and dR_n/dr is a fixed function of r per species:
 * soapb_create fits piecewise polynomials to the FP64 expansion (segments of at
 * most 0.05 rcut_hard, degree 7, split at the reference's branch points in r,
 * src/soap_turbo_radial.f90:589-635, 721-769, 875-908) and checks them in FP32
 * against it; when the largest error relative to each function's largest value
 * is at most 5e-7 the pair kernel evaluates the tables in FP32 instead of
 * running the FP64 expansion per pair.  soapb_radial_tables reports whether
 * the tables are in use and that error (-1: not tabulated: sigma scaling,
 * poly3operator, or the check failed); soapb_set_radial_tables(ctx, 0) makes
 * the pair kernel use the FP64 expansion (1: the tables when they passed).  A
 * change discards the state kept for soapb_contract. */
int soapb_set_radial_tables(soapb_context *ctx, int32_t enable);
int soapb_radial_tables(const soapb_context *ctx, int32_t *in_use, double *max_err);

/* Tensor cores (tcgen05, 3xTF32 with FP32 accumulation in tensor memory) for
 * the site kernels' contractions where the definition has them (every
 * alpha_max <= 8 and l_max <= 8): 1 (the default) or 0 (the CUDA-core forms).
 * Results agree within FP32 rounding; each form is bitwise reproducible.  The
 * call replaces the form soapb_autotune chose; a later soapb_autotune chooses
 * again (among the tensor-core and CUDA-core kernels when enable is 1). */
int soapb_set_tensor_cores(soapb_context *ctx, int32_t enable);

/* Descriptor of one batch: d_soap (n_soap, n_sites), normalised.  With
 * keep_for_contract, the expansion coefficients c_nlm and norms stay in the
 * context for soapb_contract on the same batch. */
int soapb_descriptor(soapb_context *ctx, const soapb_batch *batch, double *d_soap,
                     int32_t keep_for_contract);

/* Size of the static scratch array behind soapb_descriptor_noalloc (64 MiB).
 * Every GPU that loads the library holds it until the process exits. */
#define SOAPB_NOALLOC_SCRATCH_BYTES (64u << 20)

/* soapb_descriptor (without keep_for_contract) that allocates nothing: no
 * cudaMalloc, cudaFree or allocating library routine, on any call.  It has no
 * counterpart in the reference.  It is for callers that cannot allow a device
 * allocation while they run -- codes that reserve the GPU's memory in their
 * own pool at start-up, and codes whose step must not synchronise the device,
 * which an allocation may do.  The batch's scratch (CSR offsets, mask bits,
 * pair rows) lives in one static device array of SOAPB_NOALLOC_SCRATCH_BYTES
 * instead of buffers that grow on demand; the context's constant tables,
 * allocated once by soapb_create, are read as by soapb_descriptor.
 *  - The context's device must be current.  The first call on a device looks
 *    up the array's address (a one-time set-up, kept for the process).  CUDA
 *    loads a library's device code lazily by default, so that first call is
 *    also when the 64 MiB are committed on the device: make it at start-up,
 *    before reserving a memory pool and before any stream capture.  After a
 *    cudaDeviceReset the array has a new address, which the kept one does not
 *    follow: do not call this entry point again in that process.
 *  - A batch needing more scratch than the array holds is rejected with
 *    SOAPB_ERR_ARGUMENT and a message giving both sizes.  The need is about
 *    (2 n_species amax + row) * 4 bytes per atom pair, with amax = 8 and a
 *    96-float row when every alpha_max <= 8 and l_max <= 8 (577 bytes per pair
 *    for 3 species: about 110 thousand pairs), else amax = 16 and a 128-float
 *    row.
 *  - All calls share the array and it keeps the last call's contents; calls
 *    whose work overlaps on the GPU (other streams, host threads or contexts
 *    on the same device) race on it: serialise them.
 *  - soapb_check_inputs on the context reports the call's input errors (a
 *    non-finite or negative pair input, a bad CSR), read from the array's
 *    error word, until another call of this entry point on the device. */
int soapb_descriptor_noalloc(soapb_context *ctx, const soapb_batch *batch, double *d_soap);

/* Force VJP on the batch of the last soapb_descriptor(keep_for_contract = 1):
 * d_pair (3, n_pairs) = sgn * G . d soap / d r, never forming soap_cart_der.
 * It reads the pair expansions and c_nlm that descriptor call kept, as the
 * reference's soap_contract reads the state its get_soap kept. */
int soapb_contract(soapb_context *ctx, const soapb_batch *batch, const double *d_soap,
                   const double *d_G, int32_t g_layout, double sgn, double *d_pair);

/* Descriptor and force VJP in one call, for an upstream gradient known up
 * front (e.g. a linear model): same outputs as the two calls above. */
int soapb_descriptor_and_vjp(soapb_context *ctx, const soapb_batch *batch, const double *d_G,
                             int32_t g_layout, double sgn, double *d_soap, double *d_pair);

/* Plain FP64 form, staged like the reference: radial, angular, c_nlm, power
 * spectrum, then (when d_cart is not NULL) soap_cart_der (3, n_soap, n_pairs)
 * with the self column minus the sum of the others. */
int soapb_descriptor_fp64(soapb_context *ctx, const soapb_batch *batch, double *d_soap,
                          double *d_cart);

/* Central-atom Hessian contracted with weight vectors (the context form of
 * soapb_get_soap_central_hessian): d_vecs (n_soap, n_vec, n_sites), d_hess
 * (3, 3, n_vec, n_pairs), layouts as there.  FP64; it recomputes the FP64
 * expansion state of the batch, so it needs no earlier call.  d_soap is the
 * normalised descriptor the weights were formed against (NULL: the FP64 one
 * this call computes).  Needs legacy_filter_seed = 0 (SOAPB_ERR_ARGUMENT).  More weight
 * vectors than the kernel's shared memory holds at once (about 90 for the benchmark
 * definition) are done in chunks, with two strided device copies per chunk. */
int soapb_central_hessian(soapb_context *ctx, const soapb_batch *batch, const double *d_soap,
                          int32_t n_vec, const double *d_vecs, double *d_hess);

/* pair = sgn * G . soap_cart_der over a materialised soap_cart_der. */
int soapb_contract_cart_der(soapb_context *ctx, const soapb_batch *batch, const double *d_cart,
                            const double *d_G, int32_t g_layout, double sgn, double *d_pair);

/* Status of the device-side input checks of the last call on this context
 * that checked its inputs (waits for the stream): SOAPB_OK or SOAPB_ERR_INPUT,
 * with the first bad pair index in *bad_pair (or -1). */
int soapb_check_inputs(soapb_context *ctx, int64_t *bad_pair);

/* Neighbour list of one periodic structure, built on the device in the
 * layout get_soap takes -- the step before get_soap, which soap_turbo leaves
 * to its callers; the species and mask follow its assign_species_multiplicity
 * (src/soap_turbo.f90:2099-2221, mask lines 2188-2214, whose loop runs over
 * the central atom's multiplicity).
 *   d_positions (3, n_atoms)       Cartesian, Angstrom (x fastest)
 *   lattice     (3, 3) on the host the cell vectors a, b, c: lattice[3*i + k]
 *                                  = component k of vector i; periodic along all three
 *   d_atom_species (max_mult, n_atoms)  1-based species of each atom, 0 beyond its
 *                                  multiplicity; d_atom_mult (n_atoms)
 *   d_sites (n_sites)              0-based atom index of each central site
 *   rcut                           <= 0: the context's largest rcut_hard
 * Each row holds the site itself first (rjs = 0, theta = phi = 0), then every
 * periodic image of every atom closer than rcut, ordered by atom index, then
 * distance (rounded to FP32), then lattice translation -- an order that
 * depends on the inputs only; theta = acos(dz/r), phi = atan2(dy, dx) of
 * r_image - r_site.
 * `batch` receives device pointers into buffers the context owns, valid until
 * the next call (use it with soapb_descriptor and friends); d_neigh_atom (may
 * be NULL) receives the atom index of every pair.  The call waits for the
 * context's stream (the pair count sizes the outputs).  Errors: a site index
 * out of range or a non-finite position (SOAPB_ERR_INPUT), more than 1024
 * neighbours of one site or an rcut reaching more than 100 cells along an
 * axis (SOAPB_ERR_ARGUMENT). */
int soapb_build_neighbors(soapb_context *ctx, int32_t n_atoms, const double *d_positions,
                          const double *lattice, const int32_t *d_atom_species, int32_t max_mult,
                          const int32_t *d_atom_mult, int32_t n_sites, const int32_t *d_sites,
                          double rcut, soapb_batch *batch, const int32_t **d_neigh_atom);

/* Self-test of the bounded wait in the CSR offset scan (no counterpart in the
 * reference): one tile of a two-tile scan runs while its predecessor's state is
 * prepared on the host -- published (publish_predecessor = 1: the wait ends at
 * once) or never published (0: the wait gives up after max_spins spins).
 * Returns the status the scan left: SOAPB_OK, or SOAPB_ERR_CUDA for a wait
 * that gave up; *last_offset (may be NULL) receives the scan's total, 4096
 * with the predecessor published.  Allocates and frees small device buffers on
 * the current device and synchronises it. */
int soapb_selftest_scan_wait(int32_t max_spins, int32_t publish_predecessor, int64_t *last_offset);

/* Number of kernel launches issued by this context since creation. */
int soapb_launch_count(const soapb_context *ctx, int64_t *count);

/* Device timing per kernel, the context-layer form of get_soap's do_timing
 * (src/soap_turbo.f90:139-169 argument do_timing, whose cpu_time table the
 * drop-in layer prints as GPU times).  soapb_kernel_timing(ctx, capacity)
 * brackets each of the next `capacity` launches of the kernels below with CUDA
 * events on the context's stream (0 switches timing off); it is a set-up call
 * (it creates events) and must not be made during stream capture, and no timed
 * call may be captured.  soapb_kernel_times waits for the last timed launch,
 * returns per kernel kind the number of timed launches and their summed device
 * milliseconds (count[4], total_ms[4], indexed by SOAPB_KERNEL_*), the number
 * of launches the full ring could not time (dropped, may be NULL), and empties
 * the ring. */
enum {
  SOAPB_KERNEL_PREP = 0,       /* CSR offsets, mask bits, input checks     */
  SOAPB_KERNEL_PAIR = 1,       /* FP64 radial and angular rows per pair    */
  SOAPB_KERNEL_DESCRIPTOR = 2, /* c_nlm, power spectrum, norm per site     */
  SOAPB_KERNEL_CONTRACT = 3,   /* force VJP per site                       */
  SOAPB_KERNEL_KINDS = 4
};
int soapb_kernel_timing(soapb_context *ctx, int32_t capacity);
int soapb_kernel_times(soapb_context *ctx, int64_t *count, double *total_ms, int64_t *dropped);

#ifdef __cplusplus
}
#endif

#endif /* SOAP_B200_H */
