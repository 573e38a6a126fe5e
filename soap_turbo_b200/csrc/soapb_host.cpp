// soapb_host.cpp -- host side of libsoapb200.so: argument checks, the basis
// matrices, the compression and adjoint index tables, device memory, and the
// two API layers declared in include/soap_b200.h.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/soap_b200.h"
#include "soapb_device.cuh"
#include "soapb_internal.h"

using namespace soapb;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(SOAPB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CU(call)                                                   \
  do {                                                             \
    cudaError_t _e = (call);                                       \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);            \
  } while (0)

// ---------------------------------------------------------------- basis
// Overlap of the primitive poly3 functions (src/soap_turbo_radial.f90:1041-1047)
void overlap_poly3(int a, double *S) {
  for (int i = 1; i <= a; ++i) {
    S[(i - 1) * a + (i - 1)] = 1.0;
    for (int j = i + 1; j <= a; ++j) {
      const double v = std::sqrt((double)(5 + 2 * i) * (double)(5 + 2 * j)) / (double)(5 + i + j);
      S[(j - 1) * a + (i - 1)] = v;
      S[(i - 1) * a + (j - 1)] = v;
    }
  }
}

// poly3 functions plus the origin Gaussian; the Gaussian-polynomial overlaps
// come from the recursion of src/soap_turbo_radial.f90:1145-1172.
void overlap_poly3gauss(int a, double sigma_in, double rcut_in, double *S) {
  overlap_poly3(a - 1, S);  // fills an (a-1)x(a-1) block with stride a-1; re-stride below
  std::vector<double> tmp(S, S + (size_t)(a - 1) * (a - 1));
  for (int j = 0; j < a; ++j)
    for (int i = 0; i < a; ++i) S[j * a + i] = (i < a - 1 && j < a - 1) ? tmp[j * (a - 1) + i] : 0.0;
  const double pi = std::acos(-1.0), sq2 = std::sqrt(2.0);
  const double sig = sigma_in / rcut_in, rc = 1.0, s2 = sig * sig;
  double I_n = 0.0, N_n = 1.0;
  double N_np1 = std::sqrt(rc / 1.0);
  double I_np1 = std::sqrt(pi / 2.0) * sig * std::erf(rc / sq2 / sig) / N_np1;
  double C2 = s2 / rc;
  for (int n = -1; n <= a - 1; ++n) {
    C2 = C2 * rc;
    const double N_np2 = std::sqrt(rc / (double)(2 * n + 5));
    const double I_np2 = s2 * (double)(n + 1) * N_n / N_np2 * I_n + N_np1 * rc / N_np2 * I_np1 - C2 / N_np2;
    if (n > 0) {
      const double v = I_np2 * sq2 / std::sqrt(sig) / std::pow(pi, 0.25);
      S[(n - 1) * a + (a - 1)] = v;
      S[(a - 1) * a + (n - 1)] = v;
    }
    N_n = N_np1;
    N_np1 = N_np2;
    I_n = I_np1;
    I_np1 = I_np2;
  }
  S[(a - 1) * a + (a - 1)] = 1.0;
}

// W = S^{-1/2}, the inverse principal square root of the SPD overlap matrix.
// The reference builds it with dgesvd + dpotrf/dpotri in FP64
// (src/soap_turbo_radial.f90:1052-1087); S is ill-conditioned (cond ~1e13 at
// alpha = 8), so this does a cyclic Jacobi eigendecomposition in long double
// and forms V diag(lambda^{-1/2}) V^T there.
int inverse_sqrt(int a, const double *S, double *W) {
  std::vector<long double> A((size_t)a * a), V((size_t)a * a, 0.0L);
  for (int i = 0; i < a * a; ++i) A[i] = S[i];
  for (int i = 0; i < a; ++i) V[i * a + i] = 1.0L;
  for (int sweep = 0; sweep < 100; ++sweep) {
    long double off = 0.0L;
    for (int p = 0; p < a; ++p)
      for (int q = p + 1; q < a; ++q) off += A[q * a + p] * A[q * a + p];
    if (off < 1.0e-70L) break;
    for (int p = 0; p < a; ++p)
      for (int q = p + 1; q < a; ++q) {
        const long double apq = A[q * a + p];
        if (apq == 0.0L) continue;
        const long double theta = (A[q * a + q] - A[p * a + p]) / (2.0L * apq);
        const long double t = (theta >= 0 ? 1.0L : -1.0L) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0L));
        const long double c = 1.0L / std::sqrt(t * t + 1.0L), s = t * c;
        for (int k = 0; k < a; ++k) {
          const long double akp = A[p * a + k], akq = A[q * a + k];
          A[p * a + k] = c * akp - s * akq;
          A[q * a + k] = s * akp + c * akq;
        }
        for (int k = 0; k < a; ++k) {
          const long double apk = A[k * a + p], aqk = A[k * a + q];
          A[k * a + p] = c * apk - s * aqk;
          A[k * a + q] = s * apk + c * aqk;
        }
        for (int k = 0; k < a; ++k) {
          const long double vkp = V[p * a + k], vkq = V[q * a + k];
          V[p * a + k] = c * vkp - s * vkq;
          V[q * a + k] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<long double> d(a);
  for (int i = 0; i < a; ++i) {
    if (!(A[i * a + i] > 0.0L)) return 1;
    d[i] = 1.0L / std::sqrt(A[i * a + i]);
  }
  for (int i = 0; i < a; ++i)
    for (int j = 0; j < a; ++j) {
      long double acc = 0.0L;
      for (int k = 0; k < a; ++k) acc += V[k * a + i] * d[k] * V[k * a + j];
      W[j * a + i] = (double)acc;
    }
  return 0;
}

// get_preflm (src/soap_turbo_functions.f90:215-241)
void preflm(int lmax, double *out) {
  int k = 0;
  for (int l = 0; l <= lmax; ++l) {
    const double ppi = std::sqrt((double)(2 * l + 1) / 4.0 / std::acos(-1.0));
    double fact2 = 1.0;
    for (int i = 1; i <= l; ++i) fact2 *= (double)i;
    double fact1 = fact2;
    for (int m = 0; m <= l; ++m) {
      if (m > 0) {
        fact1 = fact1 / (double)(l + 1 - m);
        fact2 = fact2 * (double)(l + m);
      }
      out[k++] = ppi * std::sqrt(fact1 / fact2);
    }
  }
}

// ---------------------------------------------------------------- device memory
struct DBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return SOAPB_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (bytes == 0) return SOAPB_OK;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    cap = bytes;
    return SOAPB_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <typename T>
  T *as() const { return (T *)p; }
};

// Grow-only pinned host memory: the staging area through which the drop-in
// layer moves caller arrays that live in pageable memory.  Each of the two
// areas is held to kStageCap bytes; arrays of larger calls are handed to
// the CUDA runtime's own pageable copies instead.
constexpr size_t kStageCap = size_t(256) << 20;
struct HBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return SOAPB_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    if (bytes == 0) return SOAPB_OK;
    cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc");
    cap = bytes;
    return SOAPB_OK;
  }
  template <typename T>
  T *as() const { return (T *)p; }
};

// Whether the copy engines can use a caller's array directly: page-locked
// host memory (cudaHostAlloc'd or registered), and also device or managed
// memory, which must not reach the host-side staging copies (the runtime's
// copy then either handles it or reports the misuse).  Only ordinary pageable
// host memory is staged.
// The device address of host memory the GPU can write directly (page-locked
// and mapped), or null.
void *mapped_host(const void *ptr) {
  if (!ptr) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

bool is_pinned(const void *ptr) {
  if (!ptr) return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type != cudaMemoryTypeUnregistered;
}

// Host copies between a caller's pageable array and the pinned staging area,
// split over up to 8 OpenMP threads (at most the caller's OMP_NUM_THREADS) in
// slices of at least 256 KB: one thread's memcpy runs well below what a
// host-device copy moves.
int copy_threads(size_t bytes) {
  const size_t slices = (bytes + (1u << 18) - 1) >> 18;
  return (int)std::max<size_t>(1, std::min<size_t>({slices, 8, (size_t)omp_get_max_threads()}));
}
void par_copy(void *dst, const void *src, size_t bytes) {
  const int nt = copy_threads(bytes);
  if (nt <= 1) {
    if (bytes) std::memcpy(dst, src, bytes);
    return;
  }
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int t = 0; t < nt; ++t) {
    const size_t a = bytes * t / nt, b = bytes * (t + 1) / nt;
    std::memcpy((char *)dst + a, (const char *)src + a, b - a);
  }
}
// Whether `bytes` bytes of host memory are all zero bits (8-byte aligned,
// length a multiple of 8), read by up to 8 threads.
bool host_all_zero(const void *p, size_t bytes) {
  const uint64_t *w = (const uint64_t *)p;
  const size_t n = bytes / 8;
  const int nt = copy_threads(bytes);
  int nonzero = 0;
#pragma omp parallel for num_threads(nt) schedule(static) reduction(| : nonzero)
  for (int t = 0; t < nt; ++t) {
    const size_t a = n * t / nt, b = n * (t + 1) / nt;
    uint64_t acc = 0;
    for (size_t i = a; i < b; i += 512) {  // blocks of 4 KB, so that a non-zero block ends the scan early
      const size_t e = std::min(b, i + 512);
      for (size_t j = i; j < e; ++j) acc |= w[j];
      if (acc) break;
    }
    nonzero |= acc != 0;
  }
  return !nonzero;
}
// rows of `width` bytes, `rows` of them, at the given pitches
void par_copy2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows) {
  const int nt = std::min<int>(copy_threads(width * rows), (int)std::max<size_t>(rows, 1));
  if (nt <= 1) {
    for (size_t r = 0; r < rows; ++r) std::memcpy((char *)dst + r * dpitch, (const char *)src + r * spitch, width);
    return;
  }
#pragma omp parallel for num_threads(nt) schedule(static)
  for (long long r = 0; r < (long long)rows; ++r)
    std::memcpy((char *)dst + r * dpitch, (const char *)src + r * spitch, width);
}

}  // namespace

// ====================================================================== context
struct soapb_context {
  int device = 0;
  // definition
  int n_species = 0, l_max = 0, basis = 0, scaling = 0, radial_enh = 0, legacy = 1;
  std::vector<int> alpha;
  std::vector<double> rcut_hard, rcut_soft, nf, gscale, sig_r, sig_r_c, sig_t, sig_t_c, amp_sc, cw;
  int compress = 0;
  std::vector<int> P_i, P_j;
  std::vector<double> P_el;
  int n_max = 0, n_soap = 0, n_kept = 0;
  std::vector<double> W, S;  // n_max x n_max
  DevParams P{};
  // device tables
  DBuf tables;
  // arena
  DBuf off, bits, err, keep_c, keep_norm, rad, ang;
  DBuf f64_rad, f64_rad_der, f64_ang, f64_cnk, f64_soap_un, f64_norm;
  // central-atom Hessian: second radial derivatives, pair geometry records and
  // flags, per-CTA scratch, the descriptor it recomputes, its work counter
  DBuf hs_rad_der2, hs_geo, hs_good, hs_scratch, hs_soap, hs_ticket, hs_vchunk, hs_hchunk;
  // neighbour-list builder: cell list, counts and the batch it hands out
  DBuf nb_acell, nb_ccount, nb_cstart, nb_cfill, nb_catoms, nb_counts, nb_off, nb_state;
  DBuf nb_rjs, nb_th, nb_ph, nb_mask, nb_natom, nb_nneigh, nb_species, nb_smult;
  cudaStream_t stream = 0;
  int threads = 0;   // threads per site CTA chosen by the caller (0 = tuned or default)
  int max_ctas = 0;
  // the autotuner's choice per site kernel: CTA size and persistent grid cap
  int tune_td = 0, tune_cd = 0, tune_tc = 0, tune_cc = 0;
  int64_t launches = 0;
  int keep_valid = 0, keep_sites = 0, keep_pairs = 0;
  DBuf order;           // the last whole-batch descriptor call's site order
  int order_sites = -1; // its batch's site count (-1: none)
  // the error word of the last call that checked inputs: the context's own
  // (err), or the static scratch array's after soapb_descriptor_noalloc
  unsigned long long *last_err = nullptr;
  // the pair kernel's radial tables: fitted and within tolerance (rtab_ok),
  // their largest relative error, and whether the caller allows them
  int rtab_ok = 0, rtab_enable = 1;
  double rtab_err = 0.0;
  // the site kernels' contractions on the tensor cores (where instantiated):
  // allowed by the caller, and the autotuner's choice per kernel
  int tc_enable = 0, tune_tcd = 1, tune_tcc = 1;
  // device timing of the kernels (soapb_kernel_timing): an event pair around
  // each timed launch, tkind[i] the kernel of pair i, tn pairs recorded so far
  std::vector<cudaEvent_t> tev;
  std::vector<int> tkind;
  int tn = 0;
  int64_t tdropped = 0;

  void timing_release() {
    for (cudaEvent_t e : tev) cudaEventDestroy(e);
    tev.clear();
    tkind.clear();
    tn = 0;
    tdropped = 0;
  }

  ~soapb_context() {
    timing_release();
    for (DBuf *b : {&tables, &off, &bits, &err, &keep_c, &keep_norm, &order, &rad, &ang, &f64_rad, &f64_rad_der,
                    &f64_ang, &f64_cnk, &f64_soap_un, &f64_norm, &hs_rad_der2, &hs_geo, &hs_good, &hs_scratch, &hs_soap,
                    &hs_ticket, &hs_vchunk, &hs_hchunk, &nb_acell, &nb_ccount, &nb_cstart,
                    &nb_cfill, &nb_catoms, &nb_counts, &nb_off, &nb_state, &nb_rjs, &nb_th, &nb_ph,
                    &nb_mask, &nb_natom, &nb_nneigh, &nb_species, &nb_smult})
      b->release();
  }
};

namespace {

int basis_limit_check(int basis, int alpha) {
  if (alpha < 1) return fail(SOAPB_ERR_ARGUMENT, "alpha_max must be >= 1");
  if (basis == SOAPB_BASIS_POLY3 && alpha > 10)
    return fail(SOAPB_ERR_ALPHA_TOO_LARGE,
                "ERROR: Due to numerical instabilities in the basis construction for the poly3 "
                "basis, alpha_max > 10 is refused (recommended: <= 7)");
  if (basis == SOAPB_BASIS_POLY3GAUSS && alpha > 11)
    return fail(SOAPB_ERR_ALPHA_TOO_LARGE,
                "ERROR: Due to numerical instabilities in the basis construction for the "
                "poly3gauss basis, alpha_max > 11 is refused (recommended: <= 8)");
  // poly3operator takes poly3's W from the tables for alpha_max = 1..11
  // (src/soap_turbo_radial.f90:1235-1535, called at src/soap_turbo.f90:380-381)
  if (basis == SOAPB_BASIS_POLY3OPERATOR && alpha > 11)
    return fail(SOAPB_ERR_ALPHA_TOO_LARGE, "Bad value of alpha_max (poly3operator: 1..11)");
  if (alpha > SOAPB_MAX_ALPHA) return fail(SOAPB_ERR_ARGUMENT, "alpha_max above %d", SOAPB_MAX_ALPHA);
  return SOAPB_OK;
}

int species_basis(int basis, int alpha, double sig, double rcut, double *S, double *W) {
  if (basis == SOAPB_BASIS_POLY3 || basis == SOAPB_BASIS_POLY3OPERATOR) overlap_poly3(alpha, S);
  else overlap_poly3gauss(alpha, sig, rcut, S);
  if (inverse_sqrt(alpha, S, W)) return fail(SOAPB_ERR_BASIS_MATRIX, "overlap matrix not positive definite");
  return SOAPB_OK;
}

int u_index(int n, int np, int l, int N, int L) {  // uncompressed component, 0-based, n <= np
  return (n * N - n * (n - 1) / 2 + (np - n)) * (L + 1) + l;
}

// ---------------------------------------------------------------- radial tables
// The pair kernel's FP32 radial expansion for atom_sigma_r_scaling = 0: per
// species, each branch interval of r (see RadTab) is cut into segments of at
// most 0.05 rcut_hard, and on each segment every R_n and dR_n/dr (4 pi
// global_scaling folded in) is interpolated at the kRadTabDeg + 1 Chebyshev
// nodes from the FP64 expansion itself (radial_entry, run here on the host) and
// stored as monomials in t in [-1, 1].  The tables are then checked against
// the FP64 expansion at 16 points inside every segment, evaluated in FP32 as
// the kernel does; the largest error relative to each function's largest
// value decides whether the kernel uses them (max_err <= kRadTabTol).
constexpr double kRadTabTol = 5.0e-7;
constexpr double kRadTabWidth = 0.05;  // segment width, in units of rcut_hard

template <int AMAX>
void radial_fp64(const DevParams &P, const RadSp &S, const double *W, double r, double *f) {
  double val[AMAX], der[AMAX];
  radial_entry<AMAX, false>(P, S, W, r, false, true, val, der);
  const double g4 = 4.0 * std::acos(-1.0) * S.gscale;
  for (int n = 0; n < AMAX; ++n) {
    f[n] = n < S.alpha ? g4 * val[n] : 0.0;
    f[AMAX + n] = n < S.alpha ? g4 * der[n] : 0.0;
  }
}

template <int AMAX>
int fit_radial_tables(const soapb_context *c, const DevParams &P, std::vector<float> &coef, RadTab *tabs,
                      double *max_err) {
  constexpr int D = kRadTabDeg, NF = 2 * AMAX, SEG = (D + 1) * NF;
  const double pi = std::acos(-1.0);
  *max_err = 0.0;
  coef.clear();
  if (c->basis != SOAPB_BASIS_POLY3 && c->basis != SOAPB_BASIS_POLY3GAUSS) return 0;
  for (int s = 0; s < c->n_species; ++s)
    if (c->sig_r_c[s] != 0.0 || c->alpha[s] > AMAX) return 0;
  // T_k(x) as monomials: tk[k][j]
  double tk[D + 1][D + 1] = {};
  tk[0][0] = 1.0;
  if (D >= 1) tk[1][1] = 1.0;
  for (int k = 2; k <= D; ++k)
    for (int j = 0; j <= k; ++j) tk[k][j] = (j > 0 ? 2.0 * tk[k - 1][j - 1] : 0.0) - tk[k - 2][j];
  int nseg_total = 0;
  for (int s = 0; s < c->n_species; ++s) {
    const RadSp &S = P.rad[s];
    const int a = c->alpha[s], b = S.nbeg, N = c->n_max;
    std::vector<double> W((size_t)a * a);
    for (int j = 0; j < a; ++j)
      for (int i = 0; i < a; ++i) W[(size_t)j * a + i] = c->W[(size_t)(b + j) * N + (b + i)];
    const double rc = c->rcut_hard[s];
    // branch points in r: the filter switch, the Gaussian-moment cut, the amplitude's zero
    std::vector<double> bp = {0.0};
    double end = rc;
    if (P.scaling_poly && S.amp_scaling != 0.0 && radial_branch(P, S, rc * (1.0 - 1e-15)) < 0) {
      double lo = 0.5 * rc, hi = rc;  // the first r with h(r) <= 1e-10
      for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        (radial_branch(P, S, mid) < 0 ? hi : lo) = mid;
      }
      end = hi;
    }
    if (S.has_filter) bp.push_back((S.rs - 4.0 * S.atom_sigma) * rc);
    if (P.basis == 1) bp.push_back(8.0 * S.atom_sigma * rc);
    bp.push_back(end);
    std::sort(bp.begin(), bp.end());
    RadTab T{};
    bool seen[4] = {false, false, false, false};
    std::vector<double> fmax(NF, 0.0), emax(NF, 0.0);
    for (size_t i = 0; i + 1 < bp.size(); ++i) {
      const double lo = std::max(bp[i], 0.0), hi = std::min(bp[i + 1], end);
      if (!(hi > lo)) continue;
      const int st = radial_branch(P, S, 0.5 * (lo + hi));
      if (st < 0) continue;
      if (seen[st]) return 0;  // a branch state in two intervals: not tabulated
      seen[st] = true;
      const int ns = std::max(1, (int)std::ceil((hi - lo) / (kRadTabWidth * rc) - 1e-9));
      const double h = (hi - lo) / ns;
      T.lo[st] = lo;
      T.inv_h[st] = 1.0 / h;
      T.base[st] = nseg_total;
      T.nseg[st] = ns;
      for (int g = 0; g < ns; ++g) {
        const double mid = lo + (g + 0.5) * h, half = 0.5 * h;
        double fv[D + 1][NF];
        for (int j = 0; j <= D; ++j) {
          const double x = std::cos(pi * (j + 0.5) / (D + 1));
          radial_fp64<AMAX>(P, S, W.data(), mid + half * x, fv[j]);
        }
        std::vector<double> mono((size_t)(D + 1) * NF, 0.0);
        for (int f = 0; f < NF; ++f)
          for (int k = 0; k <= D; ++k) {
            double ck = 0.0;
            for (int j = 0; j <= D; ++j) ck += fv[j][f] * std::cos(pi * k * (j + 0.5) / (D + 1));
            ck *= (k == 0 ? 1.0 : 2.0) / (D + 1);
            for (int q = 0; q <= k; ++q) mono[(size_t)q * NF + f] += ck * tk[k][q];
          }
        const size_t o = coef.size();
        coef.resize(o + SEG);
        for (int q = 0; q < SEG; ++q) coef[o + q] = (float)mono[q];
        // the check: 16 points inside the segment, FP32 Horner as on the device
        for (int j = 0; j < 16; ++j) {
          const double t = -0.995 + 1.99 * j / 15.0;
          double ref[NF];
          radial_fp64<AMAX>(P, S, W.data(), mid + half * t, ref);
          const float tf = (float)t;
          for (int f = 0; f < NF; ++f) {
            float acc = coef[o + (size_t)D * NF + f];
            for (int k = D - 1; k >= 0; --k) acc = std::fma(acc, tf, coef[o + (size_t)k * NF + f]);
            fmax[f] = std::max(fmax[f], std::fabs(ref[f]));
            emax[f] = std::max(emax[f], std::fabs((double)acc - ref[f]));
          }
        }
        ++nseg_total;
      }
    }
    for (int f = 0; f < NF; ++f)
      if (fmax[f] > 0.0) *max_err = std::max(*max_err, emax[f] / fmax[f]);
    // a state no interval has is never reached; it still names a segment that
    // exists, so that no read could leave the table
    if (nseg_total == 0) return 0;
    for (int st = 0; st < 4; ++st)
      if (!seen[st]) {
        T.lo[st] = 0.0;
        T.inv_h[st] = 0.0;
        T.base[st] = nseg_total - 1;
        T.nseg[st] = 1;
      }
    tabs[s] = T;
  }
  return *max_err <= kRadTabTol ? 1 : 0;
}

// Builds DevParams and the device tables from the context's definition.
int build_tables(soapb_context *c) {
  DevParams &P = c->P;
  std::memset(&P, 0, sizeof(P));
  const int N = c->n_max, L = c->l_max, K = (L + 1) * (L + 2) / 2;
  P.n_species = c->n_species;
  P.l_max = L;
  P.k_max = K;
  P.n_max = N;
  P.basis = c->basis;
  P.scaling_poly = c->scaling == SOAPB_SCALING_POLYNOMIAL;
  P.radial_enh = c->radial_enh;
  P.legacy_seed = c->legacy;
  double rcut_max = 0.0;
  for (int s = 0; s < c->n_species; ++s) rcut_max = std::max(rcut_max, c->rcut_hard[s]);
  P.rcut_max = rcut_max;
  P.rcut2 = rcut_max * rcut_max;
  const double pi = std::acos(-1.0);
  int nbeg = 0, amax = 0;
  for (int s = 0; s < c->n_species; ++s) {
    RadSp &R = P.rad[s];
    R.inv_rcut = 1.0 / c->rcut_hard[s];
    R.rs = c->rcut_soft[s] * R.inv_rcut;
    R.atom_sigma = c->sig_r[s] * R.inv_rcut;
    R.dr = 1.0 - R.rs;
    R.sqrt_rcut = std::sqrt(c->rcut_hard[s]);
    R.inv_sqrt_rcut = 1.0 / R.sqrt_rcut;
    R.sigma_sq0 = R.atom_sigma * R.atom_sigma;
    R.N_gauss = std::sqrt(2.0 / R.atom_sigma) / std::pow(pi, 0.25);
    R.has_filter = R.dr > 0.0;
    if (R.has_filter) {
      R.drnf = R.dr / c->nf[s];
      R.q = R.drnf * R.drnf;
    }
    R.c = c->sig_r_c[s];
    R.amp_scaling = c->amp_sc[s];
    R.cw = c->cw[s];
    R.gscale = c->gscale[s];
    // poly3operator selects its pairs by the soft and buffer zones alone, with no
    // r < rcut_hard test of its own (src/soap_turbo_radial.f90:1637-1645, 1858-1872)
    R.rcut_hard = c->basis == SOAPB_BASIS_POLY3OPERATOR ? HUGE_VAL : c->rcut_hard[s];
    R.alpha = c->alpha[s];
    R.n_poly = c->basis == SOAPB_BASIS_POLY3GAUSS ? c->alpha[s] - 1 : c->alpha[s];
    R.nbeg = nbeg;
    // poly3operator always expands the central atom, weighted by central_weight
    // (src/soap_turbo.f90:534-539)
    R.do_central = c->basis == SOAPB_BASIS_POLY3GAUSS ? 0
                   : (c->basis == SOAPB_BASIS_POLY3OPERATOR ? 1 : (c->cw[s] != 0.0));
    nbeg += c->alpha[s];
    amax = std::max(amax, c->alpha[s]);
    P.sig_t[s] = c->sig_t[s];
    P.sig_t_c[s] = c->sig_t_c[s];
  }
  // alpha recursion tables (src/soap_turbo_radial.f90:503-526), index n+4
  double Nv[SOAPB_NTAB + 8];
  auto NV = [&](int n) -> double & { return Nv[n + 4]; };
  NV(-3) = 1.0;
  for (int n = -2; n <= SOAPB_NTAB; ++n) NV(n) = std::sqrt(1.0 / (double)(2 * n + 5));
  for (int n = -1; n < SOAPB_NTAB - 4; ++n) {
    P.ra[n + 4] = (double)(n + 1) * NV(n - 2) / NV(n);
    P.rb[n + 4] = NV(n - 1) / NV(n);
    P.rc[n + 4] = 1.0 / NV(n);
  }
  P.ra[3] = 0.0;
  for (int n = 1; n < SOAPB_NTAB - 4; ++n) {
    P.R1[n + 4] = NV(n + 1) / NV(n);
    P.R2[n + 4] = NV(n + 2) / NV(n);
  }
  std::vector<double> pf(K);
  preflm(L, pf.data());
  for (int k = 0; k < K; ++k) {
    P.preflm[k] = (float)pf[k];
    P.preflm64[k] = pf[k];
  }

  // compression: kept components and the two CSR maps
  const int n_unc = N * (N + 1) / 2 * (L + 1);
  std::vector<int> Pi, Pj;
  std::vector<double> Pel;
  if (c->compress) {
    Pi = c->P_i;
    Pj = c->P_j;
    Pel = c->P_el;
    int mx = 0;
    for (size_t t = 0; t < Pi.size(); ++t) {
      if (Pi[t] < 1 || Pj[t] < 1 || Pj[t] > n_unc)
        return fail(SOAPB_ERR_ARGUMENT, "compression index out of range at entry %zu", t);
      mx = std::max(mx, Pi[t]);
    }
    c->n_soap = mx;
  } else {
    Pi.resize(n_unc);
    Pj.resize(n_unc);
    Pel.assign(n_unc, 1.0);
    for (int u = 0; u < n_unc; ++u) Pi[u] = Pj[u] = u + 1;
    c->n_soap = n_unc;
  }
  std::vector<int> qof(n_unc, -1);
  for (size_t t = 0; t < Pj.size(); ++t) qof[Pj[t] - 1] = 0;
  std::vector<int> kept_nnl;
  {
    int q = 0;
    for (int n = 0; n < N; ++n)
      for (int np = n; np < N; ++np)
        for (int l = 0; l <= L; ++l) {
          const int u = u_index(n, np, l, N, L);
          if (qof[u] < 0) continue;
          qof[u] = q++;
          kept_nnl.push_back(n | (np << 8) | (l << 16));
        }
    c->n_kept = q;
  }
  const int ns = c->n_soap, nk = c->n_kept, nz = (int)Pi.size();
  std::vector<int> pi_off(ns + 1, 0), pi_q(nz);
  std::vector<float> pi_el(nz);
  std::vector<double> pi_el64(nz);
  for (int t = 0; t < nz; ++t) pi_off[Pi[t]]++;
  for (int o = 0; o < ns; ++o) pi_off[o + 1] += pi_off[o];
  {
    std::vector<int> fill(pi_off.begin(), pi_off.end() - 1);
    for (int t = 0; t < nz; ++t) {
      const int o = Pi[t] - 1, pos = fill[o]++;
      pi_q[pos] = qof[Pj[t] - 1];
      pi_el[pos] = (float)Pel[t];
      pi_el64[pos] = Pel[t];
    }
  }
  std::vector<int> pj_off(nk + 1, 0), pj_o(nz);
  std::vector<float> pj_el(nz);
  std::vector<double> pj_el64(nz);
  for (int t = 0; t < nz; ++t) pj_off[qof[Pj[t] - 1] + 1]++;
  for (int q = 0; q < nk; ++q) pj_off[q + 1] += pj_off[q];
  {
    std::vector<int> fill(pj_off.begin(), pj_off.end() - 1);
    for (int t = 0; t < nz; ++t) {
      const int q = qof[Pj[t] - 1], pos = fill[q]++;
      pj_o[pos] = Pi[t] - 1;
      pj_el[pos] = (float)Pel[t];
      pj_el64[pos] = Pel[t];
    }
  }
  // Y(n, np, l) lists for H (src/soap_turbo.f90:1800-1835)
  std::vector<int> hl_off((L + 1) * N + 1, 0), hl_np, hl_q;
  std::vector<float> hl_fac;
  std::vector<double> hl_fac64;
  for (int l = 0; l <= L; ++l)
    for (int n = 0; n < N; ++n) {
      for (int np = 0; np < N; ++np) {
        const int u = u_index(std::min(n, np), std::max(n, np), l, N, L);
        if (qof[u] < 0) continue;
        hl_np.push_back(np);
        hl_q.push_back(qof[u]);
        const double fac = (n == np) ? 2.0 : std::sqrt(2.0);
        hl_fac.push_back((float)fac);
        hl_fac64.push_back(fac);
      }
      hl_off[l * N + n + 1] = (int)hl_np.size();
    }
  std::vector<int> hl_packed;
  // poly3gauss central-atom term (src/soap_turbo.f90:646-662)
  std::vector<double> central(N, 0.0);
  if (c->basis == SOAPB_BASIS_POLY3GAUSS) {
    for (int s = 0; s < c->n_species; ++s) {
      if (c->cw[s] == 0.0) continue;
      double amplitude = 1.0;
      if (c->radial_enh == 1) amplitude = std::sqrt(2.0 / pi) * c->sig_r[s] / c->rcut_hard[s];
      else if (c->radial_enh == 2) amplitude = std::pow(c->sig_r[s], 2) / std::pow(c->rcut_hard[s], 2);
      const double fac = amplitude * c->cw[s] * std::sqrt(4.0 * pi) * std::pow(pi, 0.25) *
                         std::sqrt(c->sig_r[s] / 2.0) * std::pow(c->rcut_hard[s], 3) /
                         std::pow(c->sig_t[s], 2) / c->sig_r[s];
      const int b = P.rad[s].nbeg, a = c->alpha[s];
      for (int n = 0; n < a; ++n) {
        double ws = 0.0;
        for (int m = 0; m < a; ++m) ws += c->W[(size_t)(b + m) * N + (b + n)] * c->S[(size_t)(b + a - 1) * N + (b + m)];
        central[b + n] = fac * ws;
      }
    }
  }
  // W blocks, alpha_s x alpha_s each, stride amax^2
  const int wstride = amax * amax;
  std::vector<double> Wblk((size_t)c->n_species * wstride, 0.0);
  for (int s = 0; s < c->n_species; ++s) {
    const int b = P.rad[s].nbeg, a = c->alpha[s];
    for (int j = 0; j < a; ++j)
      for (int i = 0; i < a; ++i) Wblk[(size_t)s * wstride + j * a + i] = c->W[(size_t)(b + j) * N + (b + i)];
  }
  // one device allocation for every table
  struct Piece { const void *src; size_t bytes; size_t off; };
  std::vector<Piece> pcs;
  size_t total = 0;
  auto add = [&](const void *src, size_t bytes) {
    total = (total + 255) / 256 * 256;
    pcs.push_back({src, bytes, total});
    total += bytes;
    return pcs.size() - 1;
  };
  const size_t iW = add(Wblk.data(), Wblk.size() * 8), iC = add(central.data(), central.size() * 8);
  const size_t iK = add(kept_nnl.data(), kept_nnl.size() * 4);
  const size_t iPo = add(pi_off.data(), pi_off.size() * 4), iPq = add(pi_q.data(), pi_q.size() * 4);
  const size_t iPe = add(pi_el.data(), pi_el.size() * 4), iPe64 = add(pi_el64.data(), pi_el64.size() * 8);
  const size_t iJo = add(pj_off.data(), pj_off.size() * 4), iJq = add(pj_o.data(), pj_o.size() * 4);
  const size_t iJe = add(pj_el.data(), pj_el.size() * 4), iJe64 = add(pj_el64.data(), pj_el64.size() * 8);
  const size_t iHo = add(hl_off.data(), hl_off.size() * 4), iHn = add(hl_np.data(), hl_np.size() * 4);
  const size_t iHq = add(hl_q.data(), hl_q.size() * 4), iHf = add(hl_fac.data(), hl_fac.size() * 4);
  const size_t iHf64 = add(hl_fac64.data(), hl_fac64.size() * 8);
  // ---- per-CTA constants of the mixed kernels (one blob, copied to shared memory)
  const int amax_t = (amax <= 8 && L <= 8) ? 8 : 16;
  const int KS = K | 1;
  std::vector<unsigned char> blob, blob_c;
  auto put_in = [](std::vector<unsigned char> &b, const void *src, size_t bytes) {
    const size_t o = b.size();
    b.resize((o + bytes + 15) / 16 * 16, 0);
    if (bytes) std::memcpy(b.data() + o, src, bytes);
    return (int)o;
  };
  auto put = [&](const void *src, size_t bytes) { return put_in(blob, src, bytes); };
  auto put_c = [&](const void *src, size_t bytes) { return put_in(blob_c, src, bytes); };
  {
    std::vector<double> Wt((size_t)c->n_species * amax_t * amax_t, 0.0);
    for (int s = 0; s < c->n_species; ++s) {
      const int b = P.rad[s].nbeg, a = c->alpha[s];
      for (int j = 0; j < a; ++j)
        for (int i = 0; i < a; ++i) Wt[(size_t)s * amax_t * amax_t + j * a + i] = c->W[(size_t)(b + j) * N + (b + i)];
    }
    P.off_W = put(Wt.data(), Wt.size() * 8);
    // preflm to l_max + 1: the pair kernel stores preflm_k P_k in the rows
    const int KX = (L + 2) * (L + 3) / 2;
    std::vector<double> pfx(KX);
    preflm(L + 1, pfx.data());
    std::vector<float> kpx(pfx.begin(), pfx.end());
    P.off_kpx = put(kpx.data(), kpx.size() * 4);
    std::vector<unsigned char> rs((size_t)c->n_species * SOAPB_RADSP_BYTES, 0);
    for (int s = 0; s < c->n_species; ++s) std::memcpy(rs.data() + (size_t)s * SOAPB_RADSP_BYTES, &P.rad[s], sizeof(RadSp));
    P.off_rad = put(rs.data(), rs.size());
    put_c(rs.data(), rs.size());  // at offset 0 of the contract's blob
    std::vector<int4> kidx(KS, make_int4(0, 0, 0, 0));
    std::vector<float4> kcoef(KS, make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<int> klm(KS, 0);
    for (int l = 0; l <= L; ++l)
      for (int m = 0; m <= l; ++m) {
        const int kk = l * (l + 1) / 2 + m;
        klm[kk] = l | (m << 8);
        // sin(t) dP/dx and -m P/sin(t) from P_l^{m-1}, P_l^{m+1}, P_{l+1}^{m-1}, P_{l+1}^{m+1}
        // (src/soap_turbo_angular.f90:194-246); the rows hold preflm_j P_j, so
        // each coefficient carries preflm_kk / preflm_j of the value it scales
        int4 ix = make_int4(kk, kk, kk, kk);
        double cx = 0.0, cy = 0.0, cz = 0.0, cq = 0.0;
        if (m == 0) {
          if (l > 0) {
            ix.x = ix.y = l * (l + 1) / 2 + 1;
            cx = cy = -0.5;
          }
        } else {
          ix.x = kk - 1;
          cx = 0.5 * (double)((l + m) * (l - m + 1));
          if (m != l) {
            ix.y = kk + 1;
            cy = -0.5;
          }
          ix.z = (l + 1) * (l + 2) / 2 + m - 1;
          cz = 0.5 * (double)((l - m + 1) * (l - m + 2));
          ix.w = (l + 1) * (l + 2) / 2 + m + 1;
          cq = 0.5;
        }
        const float4 cf = make_float4((float)(cx * pfx[kk] / pfx[ix.x]), (float)(cy * pfx[kk] / pfx[ix.y]),
                                      (float)(cz * pfx[kk] / pfx[ix.z]), (float)(cq * pfx[kk] / pfx[ix.w]));
        kidx[kk] = ix;
        kcoef[kk] = cf;
      }
    P.off_kidx = put_c(kidx.data(), kidx.size() * 16);
    P.off_kcoef = put_c(kcoef.data(), kcoef.size() * 16);
    P.off_klm = put(klm.data(), klm.size() * 4);
    P.off_klm_c = put_c(klm.data(), klm.size() * 4);
    std::vector<int> nmap(N);
    for (int s = 0; s < c->n_species; ++s)
      for (int n = 0; n < c->alpha[s]; ++n) nmap[P.rad[s].nbeg + n] = s | (n << 8);
    P.off_nmap = put_c(nmap.data(), nmap.size() * 4);
    std::vector<int> citem;
    for (int s = 0; s < c->n_species; ++s)
      for (int kk = 0; kk < K; ++kk)
        for (int half = 0; half < 2; ++half)
          if (half * (amax_t / 2) < c->alpha[s]) citem.push_back(s | (kk << 4) | (half << 12));
    P.n_citem = (int)citem.size();
    P.off_citem = put(citem.data(), citem.size() * 4);
    // H items (n, l, m0): m = m0 .. m0 + 2 (the contract kernel's kHM) of one
    // (n, l) Y list, which costs the list's length per m; empty lists give no
    // item.  Heaviest first, so that a strided assignment over the CTA's
    // threads balances.
    constexpr int kHM = 3;
    std::vector<std::pair<long, int>> hw;
    for (int l = 0; l <= L; ++l)
      for (int n = 0; n < N; ++n) {
        const long len = hl_off[l * N + n + 1] - hl_off[l * N + n];
        if (len == 0) continue;
        for (int m0 = 0; m0 <= l; m0 += kHM)
          hw.push_back({-len * std::min(kHM, l + 1 - m0), n | (l << 8) | (m0 << 16)});
      }
    std::stable_sort(hw.begin(), hw.end());
    std::vector<int> hitem;
    for (auto &p : hw) hitem.push_back(p.second);
    P.n_hitem = (int)hitem.size();
    P.off_hitem = put_c(hitem.data(), hitem.size() * 4);
    P.off_kept = put(kept_nnl.data(), kept_nnl.size() * 4);
    P.off_central = put(central.data(), central.size() * 8);
    P.off_hloff = put_c(hl_off.data(), hl_off.size() * 4);
    // Y lists packed as np | q << 8 | (n == np) << 31
    if (nk >= 65536) return fail(SOAPB_ERR_ARGUMENT, "more than 65535 kept components");
    hl_packed.resize(hl_np.size());
    for (int l = 0; l <= L; ++l)
      for (int n = 0; n < N; ++n)
        for (int t = hl_off[l * N + n]; t < hl_off[l * N + n + 1]; ++t)
          hl_packed[t] = (int)((unsigned)hl_np[t] | ((unsigned)hl_q[t] << 8) | ((n == hl_np[t]) ? 0x80000000u : 0u));
    P.hl_in_blob = hl_packed.size() * 4 <= 16384;
    P.off_hl = P.hl_in_blob ? put_c(hl_packed.data(), hl_packed.size() * 4) : 0;
    // power spectrum tiles: a column set J covering every kept (n, n') (greedy
    // vertex cover; the species pivots for the trivial map, all n when nothing
    // is compressed); each kept component reads P_l[row][J position]
    {
      std::vector<char> inJ(N, 0), covered(nk, 0);
      for (;;) {
        std::vector<int> deg(N, 0);
        for (int q = 0; q < nk; ++q) {
          if (covered[q]) continue;
          const int n = kept_nnl[q] & 0xff, np = (kept_nnl[q] >> 8) & 0xff;
          deg[n]++;
          if (np != n) deg[np]++;
        }
        const int best = (int)(std::max_element(deg.begin(), deg.end()) - deg.begin());
        if (deg[best] == 0) break;
        inJ[best] = 1;
        for (int q = 0; q < nk; ++q) {
          const int n = kept_nnl[q] & 0xff, np = (kept_nnl[q] >> 8) & 0xff;
          if (n == best || np == best) covered[q] = 1;
        }
      }
      std::vector<int> J, jpos(N, -1);
      for (int n = 0; n < N; ++n)
        if (inJ[n]) {
          jpos[n] = (int)J.size();
          J.push_back(n);
        }
      P.ps_mt = (N + 15) / 16;
      P.ps_nt = std::max(1, ((int)J.size() + 7) / 8);
      J.resize(8 * P.ps_nt, -1);
      const int MR = 16 * P.ps_mt, JP = 8 * P.ps_nt;
      std::vector<int> kpos(nk);
      for (int q = 0; q < nk; ++q) {
        const int n = kept_nnl[q] & 0xff, np = (kept_nnl[q] >> 8) & 0xff, l = kept_nnl[q] >> 16;
        const int row = jpos[np] >= 0 ? n : np, col = jpos[np] >= 0 ? jpos[np] : jpos[n];
        kpos[q] = (int)((unsigned)((l * MR + row) * JP + col) | (n != np ? 0x80000000u : 0u));
      }
      // the tile buffer (l_max+1) x MR x JP lives in shared memory: beyond
      // 64 KB the kernels keep the CUDA-core form of the power spectrum
      if ((size_t)(L + 1) * MR * JP * sizeof(float) > 65536) P.ps_mt = P.ps_nt = 0;
      P.off_psj = put(J.data(), J.size() * 4);
      P.off_kpos = put(kpos.data(), kpos.size() * 4);
      // the tcgen05 form's l groups: as many consecutive l per group as fit in
      // 128 rows (l, n), 128 B rows (l, J) and K <= 32 columns (each l's block
      // 2(l+1) wide, rounded up to 4)
      const int nJ = (int)std::count_if(J.begin(), J.end(), [](int v) { return v >= 0; });
      P.ps_nj = nJ;
      P.ps_ng = 0;
      std::vector<int> psrow;
      constexpr int kPsTcK = 32;
      bool ok = P.ps_mt > 0 && nJ > 0;
      for (int l = 0; ok && l <= L;) {
        const int g = P.ps_ng, l0 = l;
        int k = 0, cnt = 0;
        while (l <= L) {
          const int w = (2 * (l + 1) + 3) / 4 * 4;
          if ((k + w + 7) / 8 * 8 > kPsTcK || (cnt + 1) * N > 128 || (cnt + 1) * nJ > 128) break;
          P.ps_ko[l] = k;
          k += w;
          ++cnt;
          ++l;
        }
        if (cnt == 0) {
          ok = false;
          break;
        }
        P.ps_gk[g] = (k + 7) / 8 * 8;
        P.ps_gnb[g] = std::max(16, (cnt * nJ + 15) / 16 * 16);
        P.ps_grows[g] = cnt * N;
        P.ps_grow[g] = (int)psrow.size();
        for (int li = l0; li < l0 + cnt; ++li)  // the J rows first, so that B is the tile's head
          for (int jc = 0; jc < nJ; ++jc) psrow.push_back(J[jc] | (li << 8) | (((li - l0) * nJ) << 16));
        for (int li = l0; li < l0 + cnt; ++li)
          for (int n = 0; n < N; ++n)
            if (jpos[n] < 0) psrow.push_back(n | (li << 8) | (((li - l0) * nJ) << 16));
        ++P.ps_ng;
      }
      if (!ok) P.ps_ng = 0;
      P.off_psrow = put(psrow.data(), psrow.size() * 4);
    }
    // one-to-one compression: output q is kept component q with weight 1
    bool ident = (ns == nk) && (nz == nk);
    for (int o = 0; ident && o < ns; ++o)
      ident = (pi_off[o + 1] - pi_off[o] == 1) && pi_q[pi_off[o]] == o && Pel[0] == Pel[0] &&
              pi_el64[pi_off[o]] == 1.0;
    P.cmap_identity = ident ? 1 : 0;
  }
  P.amax_t = amax_t;
  std::vector<float> rtab;
  c->rtab_ok = amax_t == 8 ? fit_radial_tables<8>(c, P, rtab, P.rtab_sp, &c->rtab_err)
                           : fit_radial_tables<16>(c, P, rtab, P.rtab_sp, &c->rtab_err);
  P.rtab = c->rtab_ok && c->rtab_enable;
  P.tc_contract = c->tc_enable && c->tune_tcc;
  P.tc_descriptor = c->tc_enable && c->tune_tcd;
  const size_t iRt = add(rtab.data(), rtab.size() * 4);
  P.blob_bytes = (int)blob.size();
  P.blob_c_bytes = (int)blob_c.size();
  const size_t iBlob = add(blob.data(), blob.size());
  const size_t iBlobC = add(blob_c.data(), blob_c.size());
  const size_t iHp = add(hl_packed.data(), hl_packed.size() * 4);
  int rc = c->tables.ensure(total + 256);
  if (rc) return rc;
  std::vector<unsigned char> host(total + 256, 0);
  for (auto &p : pcs)
    if (p.bytes) std::memcpy(host.data() + p.off, p.src, p.bytes);
  CU(cudaMemcpy(c->tables.p, host.data(), total, cudaMemcpyHostToDevice));
  auto at = [&](size_t i) { return (void *)((char *)c->tables.p + pcs[i].off); };
  P.Wblk = (const double *)at(iW);
  P.wstride = wstride;
  P.central = (const double *)at(iC);
  P.kept_nnl = (const int *)at(iK);
  P.pi_off = (const int *)at(iPo);
  P.pi_q = (const int *)at(iPq);
  P.pi_el = (const float *)at(iPe);
  P.pi_el64 = (const double *)at(iPe64);
  P.pj_off = (const int *)at(iJo);
  P.pj_o = (const int *)at(iJq);
  P.pj_el = (const float *)at(iJe);
  P.pj_el64 = (const double *)at(iJe64);
  P.hl_off = (const int *)at(iHo);
  P.hl_np = (const int *)at(iHn);
  P.hl_q = (const int *)at(iHq);
  P.hl_fac = (const float *)at(iHf);
  P.hl_fac64 = (const double *)at(iHf64);
  P.blob = (const unsigned char *)at(iBlob);
  P.blob_c = (const unsigned char *)at(iBlobC);
  P.hl_packed = (const int *)at(iHp);
  P.rtab_coef = (const float *)at(iRt);
  P.n_soap = c->n_soap;
  P.n_kept = c->n_kept;
  return SOAPB_OK;
}

int init_context(soapb_context *c, const soapb_hyper *h) {
  if (!h) return fail(SOAPB_ERR_ARGUMENT, "null hyperparameters");
  if (h->n_species < 1 || h->n_species > SOAPB_MAX_SPECIES)
    return fail(SOAPB_ERR_ARGUMENT, "n_species must be in 1..%d", SOAPB_MAX_SPECIES);
  if (h->l_max < 0 || h->l_max > SOAPB_MAX_LMAX)
    return fail(SOAPB_ERR_ARGUMENT, "l_max must be in 0..%d", SOAPB_MAX_LMAX);
  if (h->basis != SOAPB_BASIS_POLY3 && h->basis != SOAPB_BASIS_POLY3GAUSS && h->basis != SOAPB_BASIS_POLY3OPERATOR)
    return fail(SOAPB_ERR_BASIS, "basis must be poly3, poly3gauss or poly3operator");
  if (h->radial_enhancement < 0 || h->radial_enhancement > 2)
    return fail(SOAPB_ERR_ARGUMENT, "radial_enhancement must be 0, 1 or 2");
  const double *arrs[] = {h->rcut_hard, h->rcut_soft, h->nf, h->global_scaling, h->atom_sigma_r,
                          h->atom_sigma_r_scaling, h->atom_sigma_t, h->atom_sigma_t_scaling,
                          h->amplitude_scaling, h->central_weight};
  if (!h->alpha_max) return fail(SOAPB_ERR_ARGUMENT, "null alpha_max");
  for (const double *a : arrs)
    if (!a) return fail(SOAPB_ERR_ARGUMENT, "null per-species hyperparameter array");
  const int ns = h->n_species;
  c->n_species = ns;
  c->l_max = h->l_max;
  c->basis = h->basis;
  c->scaling = h->scaling_mode;
  c->radial_enh = h->radial_enhancement;
  c->legacy = h->legacy_filter_seed ? 1 : 0;
  c->alpha.assign(h->alpha_max, h->alpha_max + ns);
  auto cp = [&](std::vector<double> &v, const double *a) { v.assign(a, a + ns); };
  cp(c->rcut_hard, h->rcut_hard);
  cp(c->rcut_soft, h->rcut_soft);
  cp(c->nf, h->nf);
  cp(c->gscale, h->global_scaling);
  cp(c->sig_r, h->atom_sigma_r);
  cp(c->sig_r_c, h->atom_sigma_r_scaling);
  cp(c->sig_t, h->atom_sigma_t);
  cp(c->sig_t_c, h->atom_sigma_t_scaling);
  cp(c->amp_sc, h->amplitude_scaling);
  cp(c->cw, h->central_weight);
  int n_max = 0;
  for (int s = 0; s < ns; ++s) {
    int rc = basis_limit_check(h->basis, c->alpha[s]);
    if (rc) return rc;
    if (!(c->rcut_hard[s] > 0.0) || !(c->sig_r[s] > 0.0) || !(c->sig_t[s] > 0.0) || !(c->nf[s] > 0.0))
      return fail(SOAPB_ERR_ARGUMENT, "rcut_hard, atom_sigma_r, atom_sigma_t and nf must be > 0");
    if (c->rcut_soft[s] > c->rcut_hard[s])
      return fail(SOAPB_ERR_ARGUMENT, "rcut_soft must not exceed rcut_hard");
    n_max += c->alpha[s];
  }
  if (n_max > 255) return fail(SOAPB_ERR_ARGUMENT, "sum of alpha_max above 255");
  c->n_max = n_max;
  c->compress = h->compress ? 1 : 0;
  if (c->compress) {
    if (h->P_nonzero < 1 || !h->P_i || !h->P_j || !h->P_el)
      return fail(SOAPB_ERR_ARGUMENT, "compression map missing");
    c->P_i.assign(h->P_i, h->P_i + h->P_nonzero);
    c->P_j.assign(h->P_j, h->P_j + h->P_nonzero);
    c->P_el.assign(h->P_el, h->P_el + h->P_nonzero);
  }
  // basis matrices, block diagonal over species (src/soap_turbo.f90:356-387)
  c->W.assign((size_t)n_max * n_max, 0.0);
  c->S.assign((size_t)n_max * n_max, 0.0);
  int b = 0;
  for (int s = 0; s < ns; ++s) {
    const int a = c->alpha[s];
    std::vector<double> Ss((size_t)a * a), Ws((size_t)a * a);
    int rc = species_basis(h->basis, a, c->sig_r[s], c->rcut_hard[s], Ss.data(), Ws.data());
    if (rc) return rc;
    for (int j = 0; j < a; ++j)
      for (int i = 0; i < a; ++i) {
        c->W[(size_t)(b + j) * n_max + b + i] = Ws[j * a + i];
        c->S[(size_t)(b + j) * n_max + b + i] = Ss[j * a + i];
      }
    b += a;
  }
  return build_tables(c);
}

int ensure_batch(soapb_context *c, const soapb_batch *b, DevBatch &B) {
  if (!b) return fail(SOAPB_ERR_ARGUMENT, "null batch");
  if (b->n_sites < 0 || b->n_atom_pairs < 0) return fail(SOAPB_ERR_ARGUMENT, "negative batch size");
  if (b->n_sites > 0 && (!b->n_neigh || !b->species_multiplicity || !b->species))
    return fail(SOAPB_ERR_ARGUMENT, "null site arrays");
  if (b->n_atom_pairs > 0 && (!b->mask || !b->rjs || !b->thetas || !b->phis))
    return fail(SOAPB_ERR_ARGUMENT, "null pair arrays");
  int rc;
  if ((rc = c->off.ensure(sizeof(int) * ((size_t)b->n_sites + 1)))) return rc;
  if ((rc = c->bits.ensure((size_t)b->n_atom_pairs + 16))) return rc;
  if ((rc = c->err.ensure(8 * (size_t)prep_err_words(b->n_sites)))) return rc;
  if ((rc = c->rad.ensure(sizeof(float) * 2 * (size_t)c->P.amax_t * c->n_species * ((size_t)b->n_atom_pairs + 1))))
    return rc;
  if ((rc = c->ang.ensure(sizeof(float) * (size_t)ang_row_floats(c->P) * ((size_t)b->n_atom_pairs + 128))))
    return rc;
  B.n_sites = b->n_sites;
  B.n_pairs = b->n_atom_pairs;
  B.max_mult = b->max_species_multiplicity;
  B.n_neigh = b->n_neigh;
  B.species = b->species;
  B.species_mult = b->species_multiplicity;
  B.mask = b->mask;
  B.rjs = b->rjs;
  B.thetas = b->thetas;
  B.phis = b->phis;
  B.off = c->off.as<int>();
  B.bits = c->bits.as<uint8_t>();
  B.err = c->err.as<unsigned long long>();
  B.rad = c->rad.as<float>();
  B.ang = c->ang.as<float>();
  B.ticket = (int *)(B.err + prep_err_words(b->n_sites) - 1);
  B.site_lo = 0;
  B.site_hi = b->n_sites;
  c->last_err = B.err;
  return SOAPB_OK;
}

// Clears the error word, the scan state and the work counters before a prep
// launch (the FP64 path's k_prep, or the mixed path's k_pair): one memset.
int clear_prep_state(soapb_context *c, const DevBatch &B) {
  CU(cudaMemsetAsync(B.err, 0, 8 * (size_t)prep_err_words(B.n_sites), c->stream));
  return SOAPB_OK;
}

// Brackets one kernel launch with the timing events when timing is on; a
// launch beyond the ring's capacity is counted as dropped.
struct TimedLaunch {
  soapb_context *c;
  int slot = -1;
  TimedLaunch(soapb_context *ctx, int kind) : c(ctx) {
    if (c->tev.empty()) return;
    if (2 * (size_t)c->tn + 1 >= c->tev.size()) {
      ++c->tdropped;
      return;
    }
    slot = c->tn++;
    c->tkind[slot] = kind;
    cudaEventRecord(c->tev[2 * (size_t)slot], c->stream);
  }
  ~TimedLaunch() {
    if (slot >= 0) cudaEventRecord(c->tev[2 * (size_t)slot + 1], c->stream);
  }
};

int run_prep(soapb_context *c, DevBatch &B) {
  int rc = clear_prep_state(c, B);
  if (rc) return rc;
  DevParams P = c->P;
  P.n_pairs = B.n_pairs;
  P.n_sites = B.n_sites;
  {
    TimedLaunch tl(c, SOAPB_KERNEL_PREP);
    CU(launch_prep(P, B, c->stream));
  }
  c->launches += 1;
  return SOAPB_OK;
}

int pick_threads(const soapb_context *c) {
  if (c->threads == 64 || c->threads == 128 || c->threads == 256) return c->threads;
  return 128;
}

// Launch configuration of a site kernel: the caller's CTA size if set, else
// the autotuner's choice for that kernel, else 128 threads on the occupancy grid.
LaunchCfg site_cfg(const soapb_context *c, bool contract) {
  if (c->threads) return LaunchCfg{pick_threads(c), c->stream, c->max_ctas};
  const int t = contract ? c->tune_tc : c->tune_td;
  if (t) return LaunchCfg{t, c->stream, contract ? c->tune_cc : c->tune_cd};
  return LaunchCfg{128, c->stream, c->max_ctas};
}

// Status of the inputs from the prep error word a launch left (see soapb_scan.cuh).
int input_status(unsigned long long w, int64_t *bad_pair) {
  if (bad_pair) *bad_pair = -1;
  const unsigned long long v = prep_error_code(w);
  if (v == ~0ull) return SOAPB_OK;
  if (v == (1ull << 33)) return fail(SOAPB_ERR_INPUT, "n_neigh is negative or does not sum to n_atom_pairs");
  if (v == kErrTc) return fail(SOAPB_ERR_CUDA, "a site kernel gave up waiting for its tensor-core MMAs");
  if (v > (1ull << 33)) return fail(SOAPB_ERR_CUDA, "the CSR offset scan gave up waiting for a preceding tile");
  if (bad_pair) *bad_pair = (int64_t)v;
  return fail(SOAPB_ERR_INPUT, "non-finite or negative pair input at pair %llu", v);
}

// Site chunks for the drop-in layer's overlap of copies with the site kernels:
// the site kernel runs once per chunk [bounds[i], bounds[i + 1]); before(i) runs
// before chunk i's launches (to make the stream wait for its inputs) and
// after(i) after them (to start the copy of its outputs).  With site_off (the
// host's CSR offsets) the descriptor's pair kernel runs per chunk too, on the
// chunk's pairs [site_off[bounds[i]], site_off[bounds[i + 1]]), so that a
// chunk's pair inputs may arrive while earlier chunks compute.
struct SiteChunks {
  int n = 1;
  const int *bounds = nullptr;
  const long long *site_off = nullptr;
  std::function<int(int)> before, after;
  // when set: whether chunk i adds into d_soap (asked after before(i)),
  // instead of the call's accumulate
  std::function<bool(int)> acc_of;
};

// accumulate: d_soap holds the caller's soap on entry and the descriptor is
// added into it before the norm is taken (the reference's compressed get_soap,
// src/soap_turbo.f90:798-802); else d_soap is overwritten.
int ctx_descriptor(soapb_context *c, const soapb_batch *b, double *d_soap, int keep,
                   const SiteChunks *ch = nullptr, bool accumulate = false) {
  DevBatch B{};
  int rc = ensure_batch(c, b, B);
  if (rc) return rc;
  if (b->n_sites > 0 && !d_soap) return fail(SOAPB_ERR_ARGUMENT, "null soap output");
  if ((rc = clear_prep_state(c, B))) return rc;
  DevParams P = c->P;
  P.n_pairs = B.n_pairs;
  P.n_sites = B.n_sites;
  if (keep) {
    if ((rc = c->keep_c.ensure(sizeof(float) * keep_floats_per_site(P) * ((size_t)b->n_sites + 1)))) return rc;
    if ((rc = c->keep_norm.ensure(sizeof(double) * ((size_t)b->n_sites + 1)))) return rc;
  }
  LaunchCfg cfg = site_cfg(c, false);
  // the pair kernel also scans n_neigh into the CSR offsets, packs the mask
  // and checks the inputs (its first launch scans, when it runs per chunk)
  const bool pair_chunks = ch && ch->site_off && b->n_sites > 0;
  // a batch one scan tile covers, run whole: the scan orders its sites
  // heaviest first for the site kernels (and the contract that follows)
  c->order_sites = -1;
  if (!ch && b->n_sites > 0 && b->n_sites <= kScanTileSites) {
    if ((rc = c->order.ensure(sizeof(int) * (size_t)b->n_sites))) return rc;
    B.order = c->order.as<int>();
  }
  if (!pair_chunks && (b->n_atom_pairs > 0 || b->n_sites > 0)) {
    TimedLaunch tl(c, SOAPB_KERNEL_PAIR);
    CU(launch_pair(P, B, c->stream, keep));
    c->launches += 1;
  }
  const int nch = (ch && b->n_sites > 0) ? ch->n : 1;
  for (int i = 0; i < nch && b->n_sites > 0; ++i) {
    B.site_lo = ch ? ch->bounds[i] : 0;
    B.site_hi = ch ? ch->bounds[i + 1] : b->n_sites;
    if (ch && ch->before && (rc = ch->before(i))) return rc;
    if (pair_chunks) {
      const long long p0 = ch->site_off[B.site_lo], p1 = ch->site_off[B.site_hi];
      if (p0 < 0 || p0 > p1 || p1 > b->n_atom_pairs) return fail(SOAPB_ERR_ARGUMENT, "bad chunk pair range");
      TimedLaunch tl(c, SOAPB_KERNEL_PAIR);
      CU(launch_pair(P, B, c->stream, keep, (int)p0, (int)p1, i == 0));
      c->launches += 1;
    }
    {
      TimedLaunch tl(c, SOAPB_KERNEL_DESCRIPTOR);
      const bool acc = (ch && ch->acc_of) ? ch->acc_of(i) : accumulate;
      CU(launch_descriptor(P, B, cfg, d_soap, keep ? c->keep_c.as<float>() : nullptr,
                           keep ? c->keep_norm.as<double>() : nullptr, (keep ? 1 : 0) | (acc ? 2 : 0)));
    }
    c->launches += 1;
    if (ch && ch->after && (rc = ch->after(i))) return rc;
  }
  c->keep_valid = keep;
  c->keep_sites = b->n_sites;
  c->keep_pairs = b->n_atom_pairs;
  if (B.order) c->order_sites = b->n_sites;
  return SOAPB_OK;
}

int ctx_contract(soapb_context *c, const soapb_batch *b, const double *d_soap, const double *d_G,
                 int g_layout, double sgn, double *d_pair, const SiteChunks *ch = nullptr) {
  if (!c->keep_valid || c->keep_sites != b->n_sites || c->keep_pairs != b->n_atom_pairs)
    return fail(SOAPB_ERR_CONTRACT_STATE,
                "ERROR: soap_contract needs get_soap called with contract = .true. first");
  if (g_layout != 0 && g_layout != 1) return fail(SOAPB_ERR_ARGUMENT, "bad g_layout");
  if (b->n_sites > 0 && (!d_soap || !d_G || !d_pair)) return fail(SOAPB_ERR_ARGUMENT, "null pointer");
  DevBatch B{};
  int rc = ensure_batch(c, b, B);
  if (rc) return rc;
  DevParams P = c->P;
  P.n_pairs = B.n_pairs;
  P.n_sites = B.n_sites;
  LaunchCfg cfg = site_cfg(c, true);
  // the descriptor call's site order (a permutation of the batch's sites)
  if (!ch && c->order_sites == b->n_sites && b->n_sites > 0) B.order = c->order.as<int>();
  const int nch = (ch && b->n_sites > 0) ? ch->n : 1;
  for (int i = 0; i < nch && b->n_sites > 0; ++i) {
    B.site_lo = ch ? ch->bounds[i] : 0;
    B.site_hi = ch ? ch->bounds[i + 1] : b->n_sites;
    if (ch && ch->before && (rc = ch->before(i))) return rc;
    {
      TimedLaunch tl(c, SOAPB_KERNEL_CONTRACT);
      CU(launch_contract(P, B, cfg, d_soap, d_G, g_layout, sgn, c->keep_c.as<float>(),
                         c->keep_norm.as<double>(), d_pair));
    }
    c->launches += 1;
    if (ch && ch->after && (rc = ch->after(i))) return rc;
  }
  return SOAPB_OK;
}

// accumulate: as for ctx_descriptor; d_self_init (may be null, with d_cart):
// the caller's self columns of soap_cart_der, (3, n_soap) per site.
int ctx_fp64(soapb_context *c, const soapb_batch *b, double *d_soap, double *d_cart, bool accumulate = false,
             const double *d_self_init = nullptr) {
  DevBatch B{};
  int rc = ensure_batch(c, b, B);
  if (rc) return rc;
  if ((rc = run_prep(c, B))) return rc;
  DevParams P = c->P;
  P.n_pairs = B.n_pairs;
  P.n_sites = B.n_sites;
  const size_t np = (size_t)b->n_atom_pairs + 1, ns = (size_t)b->n_sites + 1;
  const int do_der = d_cart != nullptr;
  if ((rc = c->f64_rad.ensure(8 * np * c->n_max))) return rc;
  if ((rc = c->f64_rad_der.ensure(8 * np * c->n_max))) return rc;
  if ((rc = c->f64_ang.ensure(16 * np * P.k_max * (do_der ? 4 : 1)))) return rc;
  if ((rc = c->f64_cnk.ensure(16 * ns * c->n_max * P.k_max))) return rc;
  if ((rc = c->f64_soap_un.ensure(8 * ns * c->n_soap))) return rc;
  if ((rc = c->f64_norm.ensure(8 * ns))) return rc;
  Fp64Work w{c->f64_rad.as<double>(), c->f64_rad_der.as<double>(), c->f64_ang.as<double>(),
             c->f64_cnk.as<double>(), c->f64_soap_un.as<double>(), c->f64_norm.as<double>()};
  int nl = 0;
  CU(launch_fp64_descriptor(P, B, c->stream, w, do_der, d_soap, d_cart, &nl, accumulate ? d_soap : nullptr,
                            d_self_init));
  c->launches += nl;
  return SOAPB_OK;
}

// get_soap_central_hessian (src/soap_turbo.f90:1151-1700) on one batch: the
// FP64 descriptor path with derivatives rebuilds the expansion state, then the
// second radial derivatives and the Hessian kernel.  d_soap (the normalised
// descriptor the caller holds) may be null: the recomputed one is used.
int ctx_hessian(soapb_context *c, const soapb_batch *b, const double *d_soap, int n_vec, const double *d_vecs,
                double *d_hess) {
  if (c->basis == SOAPB_BASIS_POLY3OPERATOR)
    return fail(SOAPB_ERR_BASIS,
                "ERROR: soap_turbo: the central-atom Hessian needs second radial derivatives, which the "
                "poly3operator basis does not provide. Use poly3 or poly3gauss.");
  if (c->legacy)
    return fail(SOAPB_ERR_ARGUMENT,
                "ERROR: the second radial derivatives need legacy_filter_seed = .false.; with the legacy "
                "seed the filter integrals are not the ones the recursion differentiates");
  if (n_vec < 0) return fail(SOAPB_ERR_ARGUMENT, "n_vec must be >= 0");
  DevBatch B{};
  int rc = ensure_batch(c, b, B);
  if (rc) return rc;
  if (n_vec == 0) return SOAPB_OK;
  if (b->n_sites > 0 && !d_vecs) return fail(SOAPB_ERR_ARGUMENT, "null vecs");
  // The kernel keeps per-warp k-sums for every weight vector in shared memory:
  // more vectors than fit are done in chunks (each vector's block depends on
  // that vector alone, so the chunking changes no bits).
  int chunk = n_vec;
  {
    int dev = 0, smem_max = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    while (chunk > 1 && hess_smem_bytes(c->P, chunk) > (size_t)smem_max) --chunk;
    if (hess_smem_bytes(c->P, chunk) > (size_t)smem_max)
      return fail(SOAPB_ERR_ARGUMENT, "the Hessian kernel needs more shared memory than the device has");
  }
  if (b->n_atom_pairs > 0 && !d_hess) return fail(SOAPB_ERR_ARGUMENT, "null hess");
  if ((rc = run_prep(c, B))) return rc;
  DevParams P = c->P;
  P.n_pairs = B.n_pairs;
  P.n_sites = B.n_sites;
  const size_t np = (size_t)b->n_atom_pairs + 1, ns = (size_t)b->n_sites + 1;
  if ((rc = c->f64_rad.ensure(8 * np * c->n_max))) return rc;
  if ((rc = c->f64_rad_der.ensure(8 * np * c->n_max))) return rc;
  if ((rc = c->f64_ang.ensure(16 * np * P.k_max * 4))) return rc;
  if ((rc = c->f64_cnk.ensure(16 * ns * c->n_max * P.k_max))) return rc;
  if ((rc = c->f64_soap_un.ensure(8 * ns * c->n_soap))) return rc;
  if ((rc = c->f64_norm.ensure(8 * ns))) return rc;
  if ((rc = c->hs_rad_der2.ensure(8 * np * c->n_max))) return rc;
  if ((rc = c->hs_geo.ensure(8 * np * hess_geo_doubles(P)))) return rc;
  if ((rc = c->hs_good.ensure(4 * np))) return rc;
  if ((rc = c->hs_soap.ensure(8 * ns * c->n_soap))) return rc;
  if ((rc = c->hs_ticket.ensure(16))) return rc;
  const int grid = std::max(1, std::min(hess_grid(P, chunk), b->n_sites));
  if ((rc = c->hs_scratch.ensure(8 * (size_t)grid * hess_scratch_doubles(P, chunk)))) return rc;
  const size_t nsv = (size_t)c->n_soap, npair = (size_t)b->n_atom_pairs, nsite = (size_t)b->n_sites;
  if (chunk < n_vec) {
    if ((rc = c->hs_vchunk.ensure(8 * (nsite * chunk * nsv + 1)))) return rc;
    if ((rc = c->hs_hchunk.ensure(8 * (npair * chunk * 9 + 1)))) return rc;
  }
  Fp64Work w{c->f64_rad.as<double>(), c->f64_rad_der.as<double>(), c->f64_ang.as<double>(),
             c->f64_cnk.as<double>(), c->f64_soap_un.as<double>(), c->f64_norm.as<double>()};
  int nl = 0;
  CU(launch_fp64_descriptor(P, B, c->stream, w, 1, c->hs_soap.as<double>(), nullptr, &nl));
  for (int v0 = 0; v0 < n_vec; v0 += chunk) {
    const int nc = std::min(chunk, n_vec - v0);
    const double *vecs = d_vecs;
    double *hess = d_hess;
    if (chunk < n_vec) {  // the chunk's vectors gathered, its blocks scattered back
      vecs = c->hs_vchunk.as<double>();
      hess = c->hs_hchunk.as<double>();
      if (nsite > 0)
        CU(cudaMemcpy2DAsync(c->hs_vchunk.p, 8 * nc * nsv, d_vecs + (size_t)v0 * nsv, 8 * (size_t)n_vec * nsv,
                             8 * nc * nsv, nsite, cudaMemcpyDeviceToDevice, c->stream));
    }
    CU(launch_hessian(P, B, c->stream, w, c->hs_rad_der2.as<double>(), c->hs_geo.as<double>(),
                      c->hs_good.as<int>(), d_soap ? d_soap : c->hs_soap.as<double>(), nc, vecs, hess,
                      c->hs_scratch.as<double>(), grid, c->hs_ticket.as<int>(), &nl));
    if (chunk < n_vec && npair > 0)
      CU(cudaMemcpy2DAsync(d_hess + (size_t)v0 * 9, 72 * (size_t)n_vec, c->hs_hchunk.p, 72 * (size_t)nc,
                           72 * (size_t)nc, npair, cudaMemcpyDeviceToDevice, c->stream));
  }
  c->launches += nl;
  return SOAPB_OK;
}

int ctx_contract_cart(soapb_context *c, const soapb_batch *b, const double *d_cart, const double *d_G,
                      int g_layout, double sgn, double *d_pair) {
  DevBatch B{};
  int rc = ensure_batch(c, b, B);
  if (rc) return rc;
  DevParams P = c->P;
  P.n_pairs = B.n_pairs;
  P.n_sites = B.n_sites;
  int nl = 0;
  CU(launch_fp64_contract(P, B, c->stream, d_cart, d_G, g_layout, sgn, d_pair, &nl));
  c->launches += nl;
  return SOAPB_OK;
}

int check_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(SOAPB_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  if (prop.major != 10)
    return fail(SOAPB_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", dev,
                prop.major, prop.minor);
  return SOAPB_OK;
}

}  // namespace

// ================================================================ context layer
extern "C" {

const char *soapb_last_error(void) { return g_last_error.c_str(); }
const char *soapb_version(void) { return "soap_b200 0.1 (sm_100a)"; }

int soapb_create(const soapb_hyper *hyper, int32_t device, soapb_context **out) {
  if (!out) return fail(SOAPB_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  int rc = check_device();
  if (rc) return rc;
  if (device >= 0) CU(cudaSetDevice(device));
  auto *c = new soapb_context();
  cudaGetDevice(&c->device);
  rc = init_context(c, hyper);
  if (rc) {
    delete c;
    return rc;
  }
  *out = c;
  return SOAPB_OK;
}

int soapb_destroy(soapb_context *ctx) {
  delete ctx;
  return SOAPB_OK;
}

int soapb_set_basis(soapb_context *c, const double *W, const double *S) {
  if (!c || !W || !S) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  c->W.assign(W, W + (size_t)c->n_max * c->n_max);
  c->S.assign(S, S + (size_t)c->n_max * c->n_max);
  return build_tables(c);
}

int soapb_get_basis(const soapb_context *c, double *W, double *S) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  if (W) std::memcpy(W, c->W.data(), c->W.size() * 8);
  if (S) std::memcpy(S, c->S.data(), c->S.size() * 8);
  return SOAPB_OK;
}

int soapb_n_soap(const soapb_context *c, int32_t *n_soap) {
  if (!c || !n_soap) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  *n_soap = c->n_soap;
  return SOAPB_OK;
}

int soapb_set_stream(soapb_context *c, void *stream) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  c->stream = (cudaStream_t)stream;
  return SOAPB_OK;
}

int soapb_set_threads_per_site(soapb_context *c, int32_t threads) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  if (threads != 0 && threads != 64 && threads != 128 && threads != 256)
    return fail(SOAPB_ERR_ARGUMENT, "threads per site must be 0, 64, 128 or 256");
  c->threads = threads;
  return SOAPB_OK;
}

int soapb_set_radial_tables(soapb_context *c, int32_t enable) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  c->rtab_enable = enable ? 1 : 0;
  c->P.rtab = c->rtab_ok && c->rtab_enable;
  c->keep_valid = 0;  // the kept pair rows came from the other form
  return SOAPB_OK;
}

int soapb_set_tensor_cores(soapb_context *c, int32_t enable) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  c->tc_enable = enable ? 1 : 0;
  // an explicit choice replaces the autotuner's choice of form
  c->tune_tcd = c->tune_tcc = 1;
  c->P.tc_contract = c->tc_enable && c->tune_tcc;
  c->P.tc_descriptor = c->tc_enable && c->tune_tcd;
  return SOAPB_OK;
}

int soapb_radial_tables(const soapb_context *c, int32_t *in_use, double *max_err) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  if (in_use) *in_use = c->P.rtab;
  if (max_err) *max_err = c->rtab_ok ? c->rtab_err : -1.0;
  return SOAPB_OK;
}

int soapb_descriptor(soapb_context *c, const soapb_batch *b, double *d_soap, int32_t keep) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  return ctx_descriptor(c, b, d_soap, keep);
}

int soapb_contract(soapb_context *c, const soapb_batch *b, const double *d_soap, const double *d_G,
                   int32_t g_layout, double sgn, double *d_pair) {
  if (!c || !b) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  return ctx_contract(c, b, d_soap, d_G, g_layout, sgn, d_pair);
}

int soapb_descriptor_and_vjp(soapb_context *c, const soapb_batch *b, const double *d_G,
                             int32_t g_layout, double sgn, double *d_soap, double *d_pair) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  int rc = ctx_descriptor(c, b, d_soap, 1);
  if (rc) return rc;
  return ctx_contract(c, b, d_soap, d_G, g_layout, sgn, d_pair);
}

// The descriptor with its per-call scratch carved out of the static array of
// soapb_noalloc.cu instead of the context's growable buffers: no device memory
// is allocated or freed here.  The kernels are soapb_descriptor's; the pair
// kernel writes every row the site kernel reads and the prep kernel every
// offset and mask byte, so only the work counters need clearing.
int soapb_descriptor_noalloc(soapb_context *c, const soapb_batch *b, double *d_soap) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  if (!b) return fail(SOAPB_ERR_ARGUMENT, "null batch");
  if (b->n_sites < 0 || b->n_atom_pairs < 0) return fail(SOAPB_ERR_ARGUMENT, "negative batch size");
  if (b->n_sites > 0 && (!b->n_neigh || !b->species_multiplicity || !b->species))
    return fail(SOAPB_ERR_ARGUMENT, "null site arrays");
  if (b->n_atom_pairs > 0 && (!b->mask || !b->rjs || !b->thetas || !b->phis))
    return fail(SOAPB_ERR_ARGUMENT, "null pair arrays");
  if (b->n_sites > 0 && !d_soap) return fail(SOAPB_ERR_ARGUMENT, "null soap output");
  int dev = -1;
  CU(cudaGetDevice(&dev));
  if (dev != c->device)
    return fail(SOAPB_ERR_ARGUMENT, "the context's device %d must be current (device %d is)", c->device, dev);
  // sections of the scratch, each 256-byte aligned
  const size_t np = (size_t)b->n_atom_pairs, ns = (size_t)b->n_sites;
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t o_off = 0;
  const size_t o_bits = o_off + up(sizeof(int) * (ns + 1));
  const size_t o_err = o_bits + up(np + 16);
  const size_t o_rad = o_err + up(8 * (size_t)prep_err_words(b->n_sites));
  const size_t o_ang = o_rad + up(sizeof(float) * 2 * (size_t)c->P.amax_t * c->n_species * (np + 1));
  const size_t need = o_ang + up(sizeof(float) * (size_t)ang_row_floats(c->P) * (np + 128));
  if (need > (size_t)SOAPB_NOALLOC_SCRATCH_BYTES)
    return fail(SOAPB_ERR_ARGUMENT,
                "batch of %d sites and %d pairs needs %zu bytes of scratch; the allocation-free "
                "descriptor holds %zu bytes (use soapb_descriptor, or split the batch)",
                b->n_sites, b->n_atom_pairs, need, (size_t)SOAPB_NOALLOC_SCRATCH_BYTES);
  unsigned char *base = nullptr;
  size_t cap = 0;
  CU(noalloc_scratch(dev, &base, &cap));
  if (need > cap) return fail(SOAPB_ERR_ARGUMENT, "scratch array smaller than expected");
  DevBatch B{};
  B.n_sites = b->n_sites;
  B.n_pairs = b->n_atom_pairs;
  B.max_mult = b->max_species_multiplicity;
  B.n_neigh = b->n_neigh;
  B.species = b->species;
  B.species_mult = b->species_multiplicity;
  B.mask = b->mask;
  B.rjs = b->rjs;
  B.thetas = b->thetas;
  B.phis = b->phis;
  B.off = (int *)(base + o_off);
  B.bits = (uint8_t *)(base + o_bits);
  B.err = (unsigned long long *)(base + o_err);
  B.ticket = (int *)(B.err + prep_err_words(b->n_sites) - 1);
  B.site_lo = 0;
  B.site_hi = b->n_sites;
  B.rad = (float *)(base + o_rad);
  B.ang = (float *)(base + o_ang);
  int rc = clear_prep_state(c, B);
  if (rc) return rc;
  // soapb_check_inputs reports this call's input errors from the array's word
  c->last_err = B.err;
  DevParams P = c->P;
  P.n_pairs = B.n_pairs;
  P.n_sites = B.n_sites;
  LaunchCfg cfg = site_cfg(c, false);
  if (b->n_atom_pairs > 0 || b->n_sites > 0) {
    TimedLaunch tl(c, SOAPB_KERNEL_PAIR);
    CU(launch_pair(P, B, c->stream, 0));
    c->launches += 1;
  }
  if (b->n_sites > 0) {
    TimedLaunch tl(c, SOAPB_KERNEL_DESCRIPTOR);
    CU(launch_descriptor(P, B, cfg, d_soap, nullptr, nullptr, 0));
    c->launches += 1;
  }
  return SOAPB_OK;
}

int soapb_descriptor_fp64(soapb_context *c, const soapb_batch *b, double *d_soap, double *d_cart) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  return ctx_fp64(c, b, d_soap, d_cart);
}

int soapb_central_hessian(soapb_context *c, const soapb_batch *b, const double *d_soap, int32_t n_vec,
                          const double *d_vecs, double *d_hess) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  return ctx_hessian(c, b, d_soap, n_vec, d_vecs, d_hess);
}

int soapb_contract_cart_der(soapb_context *c, const soapb_batch *b, const double *d_cart,
                            const double *d_G, int32_t g_layout, double sgn, double *d_pair) {
  if (!c || !b) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  return ctx_contract_cart(c, b, d_cart, d_G, g_layout, sgn, d_pair);
}

int soapb_check_inputs(soapb_context *c, int64_t *bad_pair) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  if (bad_pair) *bad_pair = -1;
  if (!c->last_err) return SOAPB_OK;
  unsigned long long w = 0;
  CU(cudaMemcpyAsync(&w, c->last_err, sizeof w, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return input_status(w, bad_pair);
}

int soapb_build_neighbors(soapb_context *c, int32_t n_atoms, const double *d_positions, const double *lattice,
                          const int32_t *d_atom_species, int32_t max_mult, const int32_t *d_atom_mult,
                          int32_t n_sites, const int32_t *d_sites, double rcut, soapb_batch *out,
                          const int32_t **d_neigh_atom) {
  if (!c || !lattice || !out) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  if (n_atoms < 1 || n_sites < 0 || max_mult < 1) return fail(SOAPB_ERR_ARGUMENT, "bad sizes");
  if (!d_positions || !d_atom_species || !d_atom_mult || (n_sites > 0 && !d_sites))
    return fail(SOAPB_ERR_ARGUMENT, "null device array");
  if (!(rcut > 0.0)) rcut = c->P.rcut_max;
  NbGeom g{};
  for (int t = 0; t < 9; ++t) g.lat[t] = lattice[t];
  // inverse of the row-vector cell matrix, the cell's volume and plane spacings
  const double *A = g.lat;
  const double cof[9] = {A[4] * A[8] - A[5] * A[7], A[5] * A[6] - A[3] * A[8], A[3] * A[7] - A[4] * A[6],
                         A[2] * A[7] - A[1] * A[8], A[0] * A[8] - A[2] * A[6], A[1] * A[6] - A[0] * A[7],
                         A[1] * A[5] - A[2] * A[4], A[2] * A[3] - A[0] * A[5], A[0] * A[4] - A[1] * A[3]};
  const double det = A[0] * cof[0] + A[1] * cof[1] + A[2] * cof[2];
  double lmax = 0.0;
  for (int t = 0; t < 9; ++t) lmax = std::max(lmax, std::fabs(A[t]));
  if (!(std::fabs(det) > 1e-12 * lmax * lmax * lmax)) return fail(SOAPB_ERR_ARGUMENT, "singular cell");
  for (int r = 0; r < 3; ++r)
    for (int col = 0; col < 3; ++col) g.inv[r * 3 + col] = cof[col * 3 + r] / det;
  for (int d = 0; d < 3; ++d) {
    // plane spacing along axis d: |det| / |a_e x a_f|, the norm of row d of the cofactors
    const double *cr = cof + 3 * d;
    const double width = std::fabs(det) / std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    g.nc[d] = (int)std::max(1.0, std::min(1024.0, std::floor(width / rcut)));
    g.R[d] = (int)std::ceil(rcut * g.nc[d] / width);
    if (g.R[d] > kNbMaxReach)
      return fail(SOAPB_ERR_ARGUMENT, "rcut = %g reaches more than %d cells along a cell axis", rcut, kNbMaxReach);
  }
  // no more cells than atoms need: coarser cells only widen the stencil's reach by nothing
  while ((long)g.nc[0] * g.nc[1] * g.nc[2] > std::max(64L, 2L * n_atoms)) {
    const int d = (g.nc[0] >= g.nc[1] && g.nc[0] >= g.nc[2]) ? 0 : (g.nc[1] >= g.nc[2] ? 1 : 2);
    g.nc[d] = (g.nc[d] + 1) / 2;
  }
  for (int d = 0; d < 3; ++d) {
    const double *cr = cof + 3 * d;
    const double width = std::fabs(det) / std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    g.R[d] = (int)std::ceil(rcut * g.nc[d] / width);
  }
  g.rcut2 = rcut * rcut;
  g.n_atoms = n_atoms;
  g.n_sites = n_sites;
  g.max_mult = max_mult;
  g.n_species = c->n_species;
  const int n_cells = g.nc[0] * g.nc[1] * g.nc[2];
  const size_t w_cells = (size_t)prep_err_words(n_cells), w_sites = (size_t)prep_err_words(n_sites);
  int rc;
  if ((rc = c->nb_acell.ensure(sizeof(int4) * (size_t)n_atoms)) ||
      (rc = c->nb_ccount.ensure(sizeof(int) * ((size_t)n_cells + 1))) ||
      (rc = c->nb_cstart.ensure(sizeof(int) * ((size_t)n_cells + 1))) ||
      (rc = c->nb_cfill.ensure(sizeof(int) * (size_t)n_cells)) ||
      (rc = c->nb_catoms.ensure(sizeof(int) * (size_t)n_atoms)) ||
      (rc = c->nb_counts.ensure(sizeof(int) * ((size_t)n_sites + 1))) ||
      (rc = c->nb_off.ensure(sizeof(int) * ((size_t)n_sites + 1))) ||
      (rc = c->nb_state.ensure(8 * (1 + w_cells + w_sites))))
    return rc;
  unsigned long long *st = c->nb_state.as<unsigned long long>();
  cudaStream_t s = c->stream;
  CU(cudaMemsetAsync(c->nb_ccount.p, 0, sizeof(int) * ((size_t)n_cells + 1), s));
  CU(cudaMemsetAsync(c->nb_cfill.p, 0, sizeof(int) * (size_t)n_cells, s));
  CU(cudaMemsetAsync(st, 0, 8 * (1 + w_cells + w_sites), s));
  int4 *acell = c->nb_acell.as<int4>();
  int *cstart = c->nb_cstart.as<int>(), *catoms = c->nb_catoms.as<int>();
  CU(launch_nb_bin(g, d_positions, acell, c->nb_ccount.as<int>(), st, s));
  CU(launch_scan(c->nb_ccount.as<int>(), n_cells, cstart, st + 1, s));
  CU(launch_nb_place(g, acell, cstart, c->nb_cfill.as<int>(), catoms, s));
  CU(launch_nb_count(g, d_positions, d_sites, acell, cstart, catoms, c->nb_counts.as<int>(), st, s));
  CU(launch_scan(c->nb_counts.as<int>(), n_sites, c->nb_off.as<int>(), st + 1 + w_cells, s));
  c->launches += 4 + (n_sites > 0);
  int total = 0;
  if (n_sites > 0) CU(cudaMemcpyAsync(&total, c->nb_off.as<int>() + n_sites, sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (total < 0) return fail(SOAPB_ERR_ARGUMENT, "more than 2^31 pairs");
  const size_t np = (size_t)total;
  if ((rc = c->nb_rjs.ensure(8 * (np + 1))) || (rc = c->nb_th.ensure(8 * (np + 1))) ||
      (rc = c->nb_ph.ensure(8 * (np + 1))) || (rc = c->nb_mask.ensure((size_t)c->n_species * np + 16)) ||
      (rc = c->nb_natom.ensure(4 * (np + 1))) || (rc = c->nb_nneigh.ensure(4 * ((size_t)n_sites + 1))) ||
      (rc = c->nb_species.ensure(4 * ((size_t)max_mult * n_sites + 1))) ||
      (rc = c->nb_smult.ensure(4 * ((size_t)n_sites + 1))))
    return rc;
  NbOut o{};
  o.n_pairs = total;
  o.rjs = c->nb_rjs.as<double>();
  o.thetas = c->nb_th.as<double>();
  o.phis = c->nb_ph.as<double>();
  o.mask = c->nb_mask.as<uint8_t>();
  o.neigh_atom = c->nb_natom.as<int>();
  o.n_neigh = c->nb_nneigh.as<int>();
  o.species = c->nb_species.as<int>();
  o.species_mult = c->nb_smult.as<int>();
  CU(launch_nb_fill(g, d_positions, d_sites, d_atom_species, d_atom_mult, acell, cstart, catoms,
                    c->nb_off.as<int>(), o, st, s));
  c->launches += (n_sites > 0);
  unsigned long long w[3] = {0, 0, 0};
  CU(cudaMemcpyAsync(&w[0], st, 8, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(&w[1], st + 1, 8, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(&w[2], st + 1 + w_cells, 8, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (w[1] || w[2]) return fail(SOAPB_ERR_CUDA, "the neighbour-list scan gave up waiting for a preceding tile");
  if (w[0]) {
    const unsigned long long code = kErrTop - w[0];
    if (code == kErrWrap)
      return fail(SOAPB_ERR_INPUT, "an atom position is not finite or lies more than %d cells outside the cell",
                  kNbMaxWrap);
    if (code < (1ull << 32)) return fail(SOAPB_ERR_INPUT, "sites(%llu) is not an atom index", code + 1);
    return fail(SOAPB_ERR_ARGUMENT, "site %llu has more than %d neighbours within rcut = %g",
                code - (1ull << 32) + 1, kNbCap, rcut);
  }
  out->n_sites = n_sites;
  out->n_atom_pairs = total;
  out->max_species_multiplicity = max_mult;
  out->n_neigh = o.n_neigh;
  out->species = o.species;
  out->species_multiplicity = o.species_mult;
  out->mask = o.mask;
  out->rjs = o.rjs;
  out->thetas = o.thetas;
  out->phis = o.phis;
  if (d_neigh_atom) *d_neigh_atom = o.neigh_atom;
  return SOAPB_OK;
}

// Self-test of the scan's bounded look-back wait (the wait of soapb_scan.cuh):
// a two-tile scan of 2 x 2048 unit counts of which only tile 1 runs, its tile
// index and its predecessor's state prepared on the host.  With the
// predecessor published the wait ends at once; without it the wait gives up
// after max_spins spins and the scan reports it.  Small device buffers are
// allocated and freed here; the current device is used.
int soapb_selftest_scan_wait(int32_t max_spins, int32_t publish_predecessor, int64_t *last_offset) {
  if (max_spins < 0) return fail(SOAPB_ERR_ARGUMENT, "negative max_spins");
  int rc = check_device();
  if (rc) return rc;
  const int n = 2 * kScanTileSites, words = prep_err_words(n);
  std::vector<int> ones((size_t)n, 1);
  std::vector<unsigned long long> state((size_t)words, 0ull);
  state[1] = 1;  // the tile counter: the one block launched takes tile 1
  if (publish_predecessor) state[2] = (2ull << 32) | (unsigned)kScanTileSites;  // tile 0's inclusive prefix
  DBuf counts, off, st;
  auto done = [&](int r) {
    counts.release();
    off.release();
    st.release();
    return r;
  };
  if ((rc = counts.ensure(4 * (size_t)n)) || (rc = off.ensure(4 * ((size_t)n + 1))) ||
      (rc = st.ensure(8 * (size_t)words)))
    return done(rc);
  cudaError_t e = cudaMemcpy(counts.p, ones.data(), 4 * (size_t)n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(st.p, state.data(), 8 * (size_t)words, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = launch_scan(counts.as<int>(), n, off.as<int>(), st.as<unsigned long long>(), 0, 1, max_spins);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int last = 0;
  unsigned long long w = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&last, off.as<int>() + n, 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&w, st.p, 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return done(cuda_fail(e, "scan self-test"));
  if (last_offset) *last_offset = last;
  return done(input_status(w, nullptr));
}

int soapb_launch_count(const soapb_context *c, int64_t *count) {
  if (!c || !count) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  *count = c->launches;
  return SOAPB_OK;
}

int soapb_kernel_timing(soapb_context *c, int32_t capacity) {
  if (!c) return fail(SOAPB_ERR_ARGUMENT, "null context");
  if (capacity < 0 || capacity > (1 << 20)) return fail(SOAPB_ERR_ARGUMENT, "timing capacity out of range");
  c->timing_release();
  if (capacity == 0) return SOAPB_OK;
  c->tev.resize(2 * (size_t)capacity + 2, nullptr);
  c->tkind.assign((size_t)capacity + 1, 0);
  for (cudaEvent_t &e : c->tev) {
    const cudaError_t st = cudaEventCreate(&e);
    if (st != cudaSuccess) {
      e = nullptr;
      c->timing_release();
      return cuda_fail(st, "cudaEventCreate");
    }
  }
  return SOAPB_OK;
}

int soapb_kernel_times(soapb_context *c, int64_t *count, double *total_ms, int64_t *dropped) {
  if (!c || !count || !total_ms) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  for (int k = 0; k < SOAPB_KERNEL_KINDS; ++k) {
    count[k] = 0;
    total_ms[k] = 0.0;
  }
  if (dropped) *dropped = c->tdropped;
  if (c->tn > 0) CU(cudaEventSynchronize(c->tev[2 * (size_t)c->tn - 1]));
  for (int i = 0; i < c->tn; ++i) {
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, c->tev[2 * (size_t)i], c->tev[2 * (size_t)i + 1]));
    count[c->tkind[i]] += 1;
    total_ms[c->tkind[i]] += ms;
  }
  c->tn = 0;
  c->tdropped = 0;
  return SOAPB_OK;
}

int soapb_autotune(soapb_context *c, const soapb_batch *b, int32_t *choice) {
  if (!c || !b) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  if (b->n_sites < 1) return fail(SOAPB_ERR_ARGUMENT, "autotuning needs a non-empty batch");
  int dev = 0, sms = 0;
  CU(cudaGetDevice(&dev));
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // work buffers of the timed calls (G = 0: the kernels' work does not depend on values)
  struct Tmp {
    DBuf b;
    ~Tmp() { b.release(); }
  } t_soap, t_G, t_pair;
  DBuf &soap = t_soap.b, &G = t_G.b, &pair = t_pair.b;
  int rc;
  if ((rc = soap.ensure(sizeof(double) * (size_t)b->n_sites * c->n_soap)) ||
      (rc = G.ensure(sizeof(double) * (size_t)b->n_sites * c->n_soap)) ||
      (rc = pair.ensure(sizeof(double) * 3 * ((size_t)b->n_atom_pairs + 1))))
    return rc;
  CU(cudaMemsetAsync(G.p, 0, sizeof(double) * (size_t)b->n_sites * c->n_soap, c->stream));
  const int saved_threads = c->threads, saved_ctas = c->max_ctas;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  // candidates: the tensor-core kernels (one CTA size) when the caller allows
  // them, then the CUDA-core kernels at each CTA size; each with three grid caps
  const int tcand[4] = {0, 64, 128, 256};  // 0: the tensor-core kernel
  const int ccand[3] = {0, 2 * sms, sms};
  const int saved_tcd = c->tune_tcd, saved_tcc = c->tune_tcc;
  float best_d = 1e30f, best_c = 1e30f;
  int td = 128, cd = 0, tc = 128, cc = 0;
  rc = SOAPB_OK;
  for (int it = c->tc_enable ? 0 : 1; it < 4 && !rc; ++it)
    for (int ic = 0; ic < 3 && !rc; ++ic) {
      c->threads = tcand[it] ? tcand[it] : 128;
      c->max_ctas = ccand[ic];
      c->tune_tcd = c->tune_tcc = tcand[it] == 0;
      c->P.tc_descriptor = c->P.tc_contract = tcand[it] == 0;
      float md = 1e30f, mc = 1e30f;
      for (int rep = 0; rep < 4 && !rc; ++rep) {
        float t1 = 0.f, t2 = 0.f;
        if (cudaEventRecord(e0, c->stream) != cudaSuccess) { rc = fail(SOAPB_ERR_CUDA, "event"); break; }
        if ((rc = ctx_descriptor(c, b, soap.as<double>(), 1))) break;
        if (cudaEventRecord(e1, c->stream) != cudaSuccess) { rc = fail(SOAPB_ERR_CUDA, "event"); break; }
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t1, e0, e1) != cudaSuccess) {
          rc = fail(SOAPB_ERR_CUDA, "event timing");
          break;
        }
        cudaEventRecord(e0, c->stream);
        if ((rc = ctx_contract(c, b, soap.as<double>(), G.as<double>(), 0, 1.0, pair.as<double>()))) break;
        cudaEventRecord(e1, c->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t2, e0, e1) != cudaSuccess) {
          rc = fail(SOAPB_ERR_CUDA, "event timing");
          break;
        }
        if (rep > 0) {  // the first call of a configuration is a warm-up
          md = std::min(md, t1);
          mc = std::min(mc, t2);
        }
      }
      if (!rc && md < best_d) { best_d = md; td = tcand[it]; cd = ccand[ic]; }
      if (!rc && mc < best_c) { best_c = mc; tc = tcand[it]; cc = ccand[ic]; }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->threads = saved_threads;
  c->max_ctas = saved_ctas;
  c->keep_valid = 0;  // the timed calls replaced the kept state
  if (rc) {
    c->tune_tcd = saved_tcd;
    c->tune_tcc = saved_tcc;
    c->P.tc_descriptor = c->tc_enable && c->tune_tcd;
    c->P.tc_contract = c->tc_enable && c->tune_tcc;
    return rc;
  }
  c->tune_tcd = td == 0;
  c->tune_tcc = tc == 0;
  c->P.tc_descriptor = c->tc_enable && c->tune_tcd;
  c->P.tc_contract = c->tc_enable && c->tune_tcc;
  c->tune_td = td ? td : 128;
  c->tune_cd = cd;
  c->tune_tc = tc ? tc : 128;
  c->tune_cc = cc;
  if (choice) {
    choice[0] = td;
    choice[1] = cd;
    choice[2] = tc;
    choice[3] = cc;
  }
  return SOAPB_OK;
}

int soapb_orthonormalization_matrix(int32_t basis, int32_t alpha_max, double atom_sigma_r,
                                    double rcut_hard, double *S, double *W) {
  if (!S || !W) return fail(SOAPB_ERR_ARGUMENT, "null output");
  if (basis != SOAPB_BASIS_POLY3 && basis != SOAPB_BASIS_POLY3GAUSS)
    return fail(SOAPB_ERR_BASIS, "basis must be poly3 or poly3gauss");
  int rc = basis_limit_check(basis, alpha_max);
  if (rc) return rc;
  return species_basis(basis, alpha_max, atom_sigma_r, rcut_hard, S, W);
}

namespace {

// get_compress_indices, the compression recipes of James Darby
// (src/soap_turbo_compress.f90:120-303): nu_R (radially sensitive) and nu_S
// (species sensitive) correlation indices in 0..2.  Every species must have
// the same alpha (:134-141).  The combined index runs over (species, n); for
// each uncompressed component (i <= j, l), numbered ind in that order, the
// reference numbers the non-zero entries through a dense (compressed x
// uncompressed) lookup that is only ever read in column ind, so the number
// assigned is simply the next one, and a second entry (the skipped symmetric
// term of the general recipe) exists iff i != j and its compressed index
// differs.  P_el is zeroed first and accumulated, as in the reference.
int darby_indices(const char *mode, int nu_R, int nu_S, int n_species, const int32_t *alpha_max, int l_max,
                  bool set, int32_t *dim, int32_t *P_nonzero, int32_t *P_i, int32_t *P_j, double *P_el) {
  for (int i = 0; i < n_species; ++i)
    if (alpha_max[i] != alpha_max[0])
      return fail(SOAPB_ERR_COMPRESS_MODE,
                  "ERROR: compress_mode=%s requires all species to have the same number of radial "
                  "basis functions!",
                  mode);
  const int A = alpha_max[0], NS = n_species * A, L1 = l_max + 1;
  const bool sym = nu_R % 2 == 0 && nu_S % 2 == 0;
  const int N1 = nu_R > 0 ? A : 1, N2 = nu_R == 2 ? A : 1;
  const int S1 = nu_S > 0 ? n_species : 1, S2 = nu_S == 2 ? n_species : 1;
  const long n_comp = sym ? (long)N1 * S1 * (N1 * S1 + 1) / 2 * L1 : (long)N1 * S1 * N2 * S2 * L1;
  if (n_comp > INT32_MAX) return fail(SOAPB_ERR_ARGUMENT, "compressed dimension too large");
  const int cap = *P_nonzero;
  if (set)
    for (int t = 0; t < cap; ++t) {
      P_i[t] = 0;
      P_j[t] = 0;
      P_el[t] = 0.0;
    }
  long counter = 0, ind = 0;
  auto put = [&](long comp, double el) {  // the next entry number, 1-based
    ++counter;
    if (set) {
      if (counter > cap) return false;
      P_el[counter - 1] += el;
      P_i[counter - 1] = (int32_t)(comp + 1);
      P_j[counter - 1] = (int32_t)(ind + 1);
    }
    return true;
  };
  const double r2 = std::sqrt(2.0), ir2 = 1.0 / std::sqrt(2.0);
  for (int i = 0; i < NS; ++i) {
    const int si = i / A, ni = i % A;
    for (int j = i; j < NS; ++j) {
      const int sj = j / A, nj = j % A;
      for (int l = 0; l <= l_max; ++l) {
        bool ok;
        if (sym) {
          int ic = (si % S1) * N1 + ni % N1, jc = (sj % S2) * N2 + nj % N2;
          if (jc < ic) std::swap(ic, jc);
          const long comp = ((long)ic * (2 * N1 * S1 + 1 - ic) * L1) / 2 + (long)(jc - ic) * L1 + l;
          ok = put(comp, (i != j && ic == jc) ? r2 : 1.0);
        } else {
          const int ic = (si % S1) * N1 + ni % N1, jc = (sj % S2) * N2 + nj % N2;
          const int ic2 = (sj % S1) * N1 + nj % N1, jc2 = (si % S2) * N2 + ni % N2;
          const long comp = ((long)ic * S2 * N2 + jc) * L1 + l;
          const long comp2 = ((long)ic2 * S2 * N2 + jc2) * L1 + l;
          if (i == j) ok = put(comp, 1.0);
          else if (comp == comp2) ok = put(comp, r2);
          else ok = put(comp, ir2) && put(comp2, ir2);
        }
        if (!ok) return fail(SOAPB_ERR_ARGUMENT, "index arrays too short");
        ++ind;
      }
    }
  }
  *dim = (int32_t)n_comp;
  *P_nonzero = (int32_t)counter;
  return SOAPB_OK;
}

}  // namespace

int soapb_get_compress_indices(const char *compress_mode, int32_t n_species, const int32_t *alpha_max,
                               int32_t l_max, int32_t *dim, int32_t *P_nonzero, int32_t *P_i,
                               int32_t *P_j, double *P_el, const char *what_to_do) {
  if (!compress_mode || !alpha_max || !dim || !P_nonzero || !what_to_do)
    return fail(SOAPB_ERR_ARGUMENT, "null argument");
  bool set;
  if (!std::strcmp(what_to_do, "get_dim")) set = false;
  else if (!std::strcmp(what_to_do, "set_indices")) set = true;
  else return fail(SOAPB_ERR_ARGUMENT, "ERROR: incorrect what_to_do in get_compress_indices() subroutine!");
  if (n_species < 1) return fail(SOAPB_ERR_ARGUMENT, "n_species must be >= 1");
  if (set && (!P_i || !P_j || !P_el)) return fail(SOAPB_ERR_ARGUMENT, "null index arrays");
  const bool darby = std::strlen(compress_mode) == 3 && compress_mode[1] == '_' &&
                     compress_mode[0] >= '0' && compress_mode[0] <= '2' && compress_mode[2] >= '0' &&
                     compress_mode[2] <= '2';
  if (darby) return darby_indices(compress_mode, compress_mode[0] - '0', compress_mode[2] - '0', n_species,
                                  alpha_max, l_max, set, dim, P_nonzero, P_i, P_j, P_el);
  if (std::strcmp(compress_mode, "trivial") && std::strcmp(compress_mode, "Trivial"))
    return fail(SOAPB_ERR_COMPRESS_MODE, "ERROR: I don't understand compress_mode = %s", compress_mode);
  // trivial recipe (src/soap_turbo_compress.f90:86-119)
  std::vector<int> pivot(n_species);
  pivot[0] = 1;
  int n_max = alpha_max[0];
  for (int i = 0; i < n_species - 1; ++i) {
    pivot[i + 1] = pivot[i] + alpha_max[i];
    n_max += alpha_max[i + 1];
  }
  int counter = 0, k = 1;
  for (int n = 1; n <= n_max; ++n)
    for (int m = n; m <= n_max; ++m)
      for (int l = 0; l <= l_max; ++l) {
        bool hit = false;
        for (int s = 0; s < n_species; ++s) hit = hit || n == pivot[s] || m == pivot[s];
        if (hit) {
          ++counter;
          if (set) {
            if (counter > *P_nonzero) return fail(SOAPB_ERR_ARGUMENT, "index arrays too short");
            P_i[counter - 1] = counter;
            P_j[counter - 1] = k;
            P_el[counter - 1] = 1.0;
          }
        }
        ++k;
      }
  *dim = counter;
  *P_nonzero = counter;
  return SOAPB_OK;
}

}  // extern "C"

// ================================================================== drop-in layer
namespace {

struct DropIn {
  std::mutex mu;
  soapb_context *ctx = nullptr;
  int legacy = 1;
  int precision = SOAPB_PREC_MIXED;
  std::vector<double> user_W, user_S;  // caller-supplied basis, if any
  bool warned_poly3 = false, warned_gauss = false;
  // device copies of the last batch
  DBuf n_neigh, species, species_mult, mask, rjs, thetas, phis, soap, G, pair, cart, cart_self, vecs, hess;
  std::vector<double> self_host;  // the caller's self columns of soap_cart_der, gathered
  soapb_batch batch{};
  int ct_ready = 0, ct_fp64 = 0, ct_n_sites = 0, ct_n_pairs = 0, ct_n_soap = 0;
  // soap_hessian_enabled and what get_soap_central_hessian checks against
  // (src/soap_turbo.f90:76, 93-95)
  int hessian_enabled = 0;
  int hs_ready = 0, hs_n_sites = 0, hs_n_pairs = 0, hs_l_max = -1, hs_n_soap = 0;
  cudaStream_t stream = nullptr;
  // overlap of host copies with the site kernels (mixed path): the sites go in
  // chunks, each chunk's outputs copied back (and, in soap_contract, its inputs
  // copied in) on their own streams while the next chunk computes
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> evs;
  std::vector<int> chunk;                  // site chunk bounds of the last get_soap
  std::vector<int> cchunk;                 // and of soap_contract
  std::vector<long long> host_off;         // its CSR offsets
  HBuf st_in, st_out;                      // pinned staging of pageable caller arrays
  unsigned long long *err_host = nullptr;  // pinned copy of the prep error word
};

// Site chunks of the drop-in calls, at most 8, of at least min_sites sites.
// In get_soap each chunk's pair and site kernels run one after the other on
// the compute stream, and a small chunk runs them well below the GPU's rate
// (its grids fill few SMs), so the chunks are about 512 sites, or at least
// 4096 when the site kernel writes the soap rows into the caller's page-locked
// array (its pace is then the host link's).  In soap_contract the copies in set the pace and
// every chunk's kernels but the last run behind them: its chunks are about 384
// sites, and the last is half the size of the others, to shorten what remains
// after the last copy in.
void plan_chunks(std::vector<int> &bounds, int n_sites, bool contract, int min_sites) {
  const int n = std::max(1, std::min(8, n_sites / min_sites));
  const bool short_last = contract && n > 1;
  const long long weight_sum = short_last ? 2LL * n - 1 : n;
  bounds.resize(n + 1);
  for (int i = 0; i < n; ++i)
    bounds[i] = (int)((long long)n_sites * (short_last ? 2LL * i : i) / weight_sum);
  bounds[n] = n_sites;
}

int dropin_streams(DropIn &d, int n_events) {
  if (!d.copy_in) CU(cudaStreamCreateWithFlags(&d.copy_in, cudaStreamNonBlocking));
  if (!d.copy_out) CU(cudaStreamCreateWithFlags(&d.copy_out, cudaStreamNonBlocking));
  if (!d.err_host) CU(cudaMallocHost((void **)&d.err_host, sizeof(unsigned long long)));
  while ((int)d.evs.size() < n_events) {
    cudaEvent_t e;
    CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    d.evs.push_back(e);
  }
  return SOAPB_OK;
}

DropIn &dropin() {
  static DropIn d;
  return d;
}

bool same_definition(const soapb_context *c, const soapb_hyper &h, int legacy) {
  if (!c) return false;
  if (c->n_species != h.n_species || c->l_max != h.l_max || c->basis != h.basis ||
      c->scaling != h.scaling_mode || c->radial_enh != h.radial_enhancement || c->legacy != legacy ||
      c->compress != (h.compress ? 1 : 0))
    return false;
  const int ns = h.n_species;
  if (std::memcmp(c->alpha.data(), h.alpha_max, 4 * ns)) return false;
  const std::vector<double> *v[] = {&c->rcut_hard, &c->rcut_soft, &c->nf, &c->gscale, &c->sig_r,
                                    &c->sig_r_c, &c->sig_t, &c->sig_t_c, &c->amp_sc, &c->cw};
  const double *a[] = {h.rcut_hard, h.rcut_soft, h.nf, h.global_scaling, h.atom_sigma_r,
                       h.atom_sigma_r_scaling, h.atom_sigma_t, h.atom_sigma_t_scaling,
                       h.amplitude_scaling, h.central_weight};
  for (int i = 0; i < 10; ++i)
    if (std::memcmp(v[i]->data(), a[i], 8 * ns)) return false;
  if (c->compress) {
    if ((int)c->P_i.size() != h.P_nonzero) return false;
    if (std::memcmp(c->P_i.data(), h.P_i, 4 * h.P_nonzero) ||
        std::memcmp(c->P_j.data(), h.P_j, 4 * h.P_nonzero) ||
        std::memcmp(c->P_el.data(), h.P_el, 8 * h.P_nonzero))
      return false;
  }
  return true;
}

template <typename T>
int upload(DBuf &b, const T *src, size_t n, cudaStream_t s) {
  int rc = b.ensure(sizeof(T) * (n + 1));
  if (rc) return rc;
  if (n) CU(cudaMemcpyAsync(b.p, src, sizeof(T) * n, cudaMemcpyHostToDevice, s));
  return SOAPB_OK;
}

// Where each of get_soap's inputs is read from: the caller's array when it is
// page-locked, else a region of the pinned staging area st_in (then filled
// with host copies, chunk by chunk, just before its asynchronous copy).
struct GetSoapIn {
  const int32_t *n_neigh, *species, *species_mult;
  const uint8_t *mask;
  const double *rjs, *thetas, *phis;
  bool pin_nn, pin_sp, pin_sm, pin_mask, pin_pair;  // pin_pair: rjs, thetas and phis
  uint8_t *st_nn = nullptr, *st_sp = nullptr, *st_sm = nullptr, *st_mask = nullptr, *st_r = nullptr,
          *st_t = nullptr, *st_f = nullptr;
  // the caller's soap, copied in chunk by chunk when the descriptor is added
  // into it (compressed get_soap), through st_soap when it is staged
  const double *soap = nullptr;
  int n_soap = 0;
  bool acc = false;
  uint8_t *st_soap = nullptr;
};

size_t align16(size_t x) { return (x + 15) / 16 * 16; }

// Lays out st_in for the pageable inputs of one get_soap call.
int plan_get_soap_staging(DropIn &d, GetSoapIn &in, int n_sites, int max_mult, int n_species, int n_pairs) {
  const size_t b_nn = in.pin_nn ? 0 : align16(4 * (size_t)n_sites);
  const size_t b_sp = in.pin_sp ? 0 : align16(4 * (size_t)n_sites * max_mult);
  const size_t b_sm = in.pin_sm ? 0 : align16(4 * (size_t)n_sites);
  const size_t b_mask = in.pin_mask ? 0 : align16((size_t)n_pairs * n_species);
  const size_t b_p = in.pin_pair ? 0 : align16(8 * (size_t)n_pairs);
  const size_t total = b_nn + b_sp + b_sm + b_mask + 3 * b_p;
  if (total == 0 || total > kStageCap) return SOAPB_OK;  // above the cap: the runtime's copies
  int rc = d.st_in.ensure(total);
  if (rc) return rc;
  uint8_t *q = d.st_in.as<uint8_t>();
  if (b_nn) in.st_nn = q, q += b_nn;
  if (b_sp) in.st_sp = q, q += b_sp;
  if (b_sm) in.st_sm = q, q += b_sm;
  if (b_mask) in.st_mask = q, q += b_mask;
  if (b_p) {
    in.st_r = q, q += b_p;
    in.st_t = q, q += b_p;
    in.st_f = q;
  }
  return SOAPB_OK;
}

// One host-to-device copy on copy_in from a caller array, through its staging
// region when it is pageable (the copy of the same byte range into staging
// comes first, on the host).
int h2d_in(void *dev, const void *host, uint8_t *stage, size_t bytes, cudaStream_t st) {
  if (!bytes) return SOAPB_OK;
  const void *src = host;
  if (stage) {
    par_copy(stage, host, bytes);
    src = stage;
  }
  CU(cudaMemcpyAsync(dev, src, bytes, cudaMemcpyHostToDevice, st));
  return SOAPB_OK;
}

// get_soap's per-site inputs on the copy-in stream, after the work already
// queued on the compute stream (which may still read the previous call's).
int copy_in_sites(DropIn &d, const GetSoapIn &in, int n_sites, int max_mult) {
  CU(cudaEventRecord(d.evs[0], d.stream));
  CU(cudaStreamWaitEvent(d.copy_in, d.evs[0], 0));
  int rc;
  if ((rc = h2d_in(d.n_neigh.p, in.n_neigh, in.st_nn, 4 * (size_t)n_sites, d.copy_in))) return rc;
  if ((rc = h2d_in(d.species.p, in.species, in.st_sp, 4 * (size_t)n_sites * max_mult, d.copy_in))) return rc;
  if ((rc = h2d_in(d.species_mult.p, in.species_mult, in.st_sm, 4 * (size_t)n_sites, d.copy_in))) return rc;
  return SOAPB_OK;
}

// Chunk i's pair rows of mask, rjs, thetas and phis on the copy-in stream;
// evs[i] then marks the chunk's inputs (and the per-site ones) as present.
int copy_in_pairs(DropIn &d, const GetSoapIn &in, int i, int n_species, int n_pairs) {
  const size_t p0 = (size_t)d.host_off[d.chunk[i]], p1 = (size_t)d.host_off[d.chunk[i + 1]];
  if (p1 > p0) {
    // mask(n_pairs, n_species) column-major: the chunk's rows of every column
    const uint8_t *msrc = in.mask + p0;
    if (in.st_mask) {
      par_copy2d(in.st_mask + p0, (size_t)n_pairs, in.mask + p0, (size_t)n_pairs, p1 - p0, (size_t)n_species);
      msrc = in.st_mask + p0;
    }
    CU(cudaMemcpy2DAsync(d.mask.as<uint8_t>() + p0, (size_t)n_pairs, msrc, (size_t)n_pairs, p1 - p0,
                         (size_t)n_species, cudaMemcpyHostToDevice, d.copy_in));
    const size_t b0 = 8 * p0, nb = 8 * (p1 - p0);
    int rc;
    if ((rc = h2d_in(d.rjs.as<uint8_t>() + b0, (const uint8_t *)in.rjs + b0, in.st_r ? in.st_r + b0 : nullptr, nb,
                     d.copy_in)))
      return rc;
    if ((rc = h2d_in(d.thetas.as<uint8_t>() + b0, (const uint8_t *)in.thetas + b0, in.st_t ? in.st_t + b0 : nullptr,
                     nb, d.copy_in)))
      return rc;
    if ((rc = h2d_in(d.phis.as<uint8_t>() + b0, (const uint8_t *)in.phis + b0, in.st_f ? in.st_f + b0 : nullptr, nb,
                     d.copy_in)))
      return rc;
  }
  if (in.acc) {
    // the chunk's rows of the caller's soap, which the descriptor adds into;
    // rows that are all zero (the usual call: the reference's callers pass
    // soap zeroed) are cleared on the device instead of copied, which saves
    // their share of the host link
    const size_t b0 = 8 * (size_t)d.chunk[i] * in.n_soap, nb = 8 * (size_t)(d.chunk[i + 1] - d.chunk[i]) * in.n_soap;
    if (host_all_zero((const uint8_t *)in.soap + b0, nb)) {
      CU(cudaMemsetAsync(d.soap.as<uint8_t>() + b0, 0, nb, d.copy_in));
    } else {
      int rc;
      if ((rc = h2d_in(d.soap.as<uint8_t>() + b0, (const uint8_t *)in.soap + b0,
                       in.st_soap ? in.st_soap + b0 : nullptr, nb, d.copy_in)))
        return rc;
    }
  }
  CU(cudaEventRecord(d.evs[i], d.copy_in));
  return SOAPB_OK;
}

}  // namespace

extern "C" {

int soapb_set_legacy_filter_seed(int32_t legacy) {
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  d.legacy = legacy ? 1 : 0;
  return SOAPB_OK;
}

int soapb_get_legacy_filter_seed(int32_t *legacy) {
  if (!legacy) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  *legacy = d.legacy;
  return SOAPB_OK;
}

int soapb_set_soap_hessian_enabled(int32_t enabled) {
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  d.hessian_enabled = enabled ? 1 : 0;
  return SOAPB_OK;
}

int soapb_get_soap_hessian_enabled(int32_t *enabled) {
  if (!enabled) return fail(SOAPB_ERR_ARGUMENT, "null argument");
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  *enabled = d.hessian_enabled;
  return SOAPB_OK;
}

int soapb_set_precision(int32_t precision) {
  if (precision != SOAPB_PREC_MIXED && precision != SOAPB_PREC_FP64)
    return fail(SOAPB_ERR_ARGUMENT, "precision must be SOAPB_PREC_MIXED or SOAPB_PREC_FP64");
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  d.precision = precision;
  return SOAPB_OK;
}

int soapb_set_basis_matrices(int32_t n_max, const double *W, const double *S) {
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  if (n_max <= 0 || !W || !S) {
    d.user_W.clear();
    d.user_S.clear();
  } else {
    d.user_W.assign(W, W + (size_t)n_max * n_max);
    d.user_S.assign(S, S + (size_t)n_max * n_max);
  }
  if (d.ctx && !d.user_W.empty() && (int)d.user_W.size() == d.ctx->n_max * d.ctx->n_max) {
    int rc = soapb_set_basis(d.ctx, d.user_W.data(), d.user_S.data());
    if (rc) return rc;
  }
  return SOAPB_OK;
}

int soapb_get_soap(int32_t n_sites, const int32_t *n_neigh, int32_t n_species, const int32_t *species,
                   int32_t max_species_multiplicity, const int32_t *species_multiplicity,
                   int32_t n_atom_pairs, const uint8_t *mask, const double *rjs, const double *thetas,
                   const double *phis, const int32_t *alpha_max, int32_t l_max, const double *rcut_hard,
                   const double *rcut_soft, const double *nf, const double *global_scaling,
                   const double *atom_sigma_r, const double *atom_sigma_r_scaling,
                   const double *atom_sigma_t, const double *atom_sigma_t_scaling,
                   const double *amplitude_scaling, int32_t radial_enhancement,
                   const double *central_weight, const char *basis, const char *scaling_mode,
                   int32_t do_timing, int32_t do_derivatives, int32_t compress_soap,
                   int32_t compress_P_nonzero, const int32_t *compress_P_i,
                   const int32_t *compress_P_j, const double *compress_P_el, double *soap,
                   int32_t n_soap, double *soap_cart_der, int32_t contract) {
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  d.ct_ready = 0;
  d.hs_ready = 0;
  // the second derivatives only come with the first ones, and only with the
  // corrected filter seed (src/soap_turbo.f90:228; src/soap_turbo_radial.f90:318-323)
  const bool do_hessian = d.hessian_enabled && do_derivatives;
  if (do_hessian && d.legacy)
    return fail(SOAPB_ERR_ARGUMENT,
                "ERROR: soap_hessian_enabled needs legacy_filter_seed = .false. (the second radial "
                "derivatives are taken with the corrected filter seed)");
  if (!basis || !scaling_mode) return fail(SOAPB_ERR_ARGUMENT, "null basis or scaling_mode");
  int b;
  if (!std::strcmp(basis, "poly3")) b = SOAPB_BASIS_POLY3;
  else if (!std::strcmp(basis, "poly3gauss")) b = SOAPB_BASIS_POLY3GAUSS;
  else if (!std::strcmp(basis, "poly3operator")) b = SOAPB_BASIS_POLY3OPERATOR;
  else return fail(SOAPB_ERR_BASIS, "basis \"%s\" is not supported (poly3, poly3gauss, poly3operator)", basis);
  if (do_hessian && b == SOAPB_BASIS_POLY3OPERATOR)  // src/soap_turbo.f90:485-489
    return fail(SOAPB_ERR_BASIS,
                "ERROR: soap_turbo: the central-atom Hessian needs second radial derivatives, which the "
                "poly3operator basis does not provide. Use poly3 or poly3gauss.");
  if (n_sites < 0 || n_atom_pairs < 0) return fail(SOAPB_ERR_ARGUMENT, "negative sizes");
  if (n_sites > 0 && !n_neigh) return fail(SOAPB_ERR_ARGUMENT, "null n_neigh");
  // CSR check on the host: the kernels trust the offsets
  long long total = 0;
  d.host_off.resize((size_t)n_sites + 1);
  for (int i = 0; i < n_sites; ++i) {
    if (n_neigh[i] < 0) return fail(SOAPB_ERR_INPUT, "n_neigh(%d) is negative", i + 1);
    d.host_off[i] = total;
    total += n_neigh[i];
  }
  d.host_off[n_sites] = total;
  if (total != n_atom_pairs)
    return fail(SOAPB_ERR_INPUT, "sum(n_neigh) = %lld but n_atom_pairs = %d", total, n_atom_pairs);
  for (int i = 0; i < n_sites; ++i)
    if (species_multiplicity[i] > max_species_multiplicity || species_multiplicity[i] < 0)
      return fail(SOAPB_ERR_INPUT, "species_multiplicity(%d) out of range", i + 1);
  for (int s = 0; s < n_species && s < SOAPB_MAX_SPECIES; ++s) {
    if (b == SOAPB_BASIS_POLY3 && alpha_max[s] > 7 && alpha_max[s] <= 10 && !d.warned_poly3) {
      d.warned_poly3 = true;
      std::fprintf(stderr,
                   "WARNING: Due to numerical instabilities in the basis construction for the poly3 "
                   "basis, it is strongly recommended not to exceed alpha_max = 7.\n");
    }
    if (b == SOAPB_BASIS_POLY3GAUSS && alpha_max[s] > 8 && alpha_max[s] <= 11 && !d.warned_gauss) {
      d.warned_gauss = true;
      std::fprintf(stderr,
                   "WARNING: Due to numerical instabilities in the basis construction for the "
                   "poly3gauss basis, it is strongly recommended not to exceed alpha_max = 8.\n");
    }
  }
  soapb_hyper h{};
  h.n_species = n_species;
  h.l_max = l_max;
  h.basis = b;
  h.scaling_mode = std::strcmp(scaling_mode, "polynomial") ? SOAPB_SCALING_NONE : SOAPB_SCALING_POLYNOMIAL;
  h.radial_enhancement = radial_enhancement;
  h.legacy_filter_seed = d.legacy;
  h.alpha_max = alpha_max;
  h.rcut_hard = rcut_hard;
  h.rcut_soft = rcut_soft;
  h.nf = nf;
  h.global_scaling = global_scaling;
  h.atom_sigma_r = atom_sigma_r;
  h.atom_sigma_r_scaling = atom_sigma_r_scaling;
  h.atom_sigma_t = atom_sigma_t;
  h.atom_sigma_t_scaling = atom_sigma_t_scaling;
  h.amplitude_scaling = amplitude_scaling;
  h.central_weight = central_weight;
  h.compress = compress_soap;
  h.P_nonzero = compress_P_nonzero;
  h.P_i = compress_P_i;
  h.P_j = compress_P_j;
  h.P_el = compress_P_el;
  int rc;
  if (!same_definition(d.ctx, h, d.legacy)) {
    // the reference recomputes its basis when the definition changes (:289-388)
    soapb_context *nc = nullptr;
    rc = soapb_create(&h, -1, &nc);
    if (rc) return rc;
    if (d.ctx) soapb_destroy(d.ctx);
    d.ctx = nc;
    if (!d.stream) CU(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
    d.ctx->stream = d.stream;
    if (!d.user_W.empty() && (int)d.user_W.size() == nc->n_max * nc->n_max)
      if ((rc = soapb_set_basis(nc, d.user_W.data(), d.user_S.data()))) return rc;
  }
  soapb_context *c = d.ctx;
  if (n_soap != c->n_soap)
    return fail(SOAPB_ERR_ARGUMENT, "size(soap,1) = %d but the descriptor has n_soap = %d", n_soap, c->n_soap);
  if (n_sites > 0 && !soap) return fail(SOAPB_ERR_ARGUMENT, "null soap");
  const bool want_cart = do_derivatives && !contract;
  if (want_cart && n_atom_pairs > 0 && !soap_cart_der)
    return fail(SOAPB_ERR_ARGUMENT, "soap_cart_der is needed when do_derivatives and not contract");
  const bool fp64 = d.precision == SOAPB_PREC_FP64 || want_cart;
  cudaStream_t s = d.stream;
  cudaEvent_t ev[4];
  if (do_timing)
    for (auto &e : ev) cudaEventCreate(&e);
  if (do_timing) cudaEventRecord(ev[0], s);
  // The mixed path without do_timing runs in site chunks: chunk i's pair
  // inputs come in on copy_in (evs[i]), its pair and site kernels run on the
  // compute stream once they are there, and its soap rows go out on copy_out
  // (evs[nch + i]) while later chunks compute.  Caller arrays in pageable
  // memory pass through the pinned staging areas: a chunk's inputs are copied
  // into st_in on the host just before their asynchronous copy (so the host
  // fills chunk i + 1 while chunk i computes), and the soap rows land in
  // st_out, from where each chunk is copied out once its copy has arrived
  // (evs[2 nch + 1 + i]) while later ones are still in flight.  Otherwise
  // everything is copied in on the compute stream first.
  const bool chunked = !fp64 && !do_timing && n_sites > 0;
  int nch = 1;
  GetSoapIn in{n_neigh, species, species_multiplicity, mask, rjs, thetas, phis, is_pinned(n_neigh),
               is_pinned(species), is_pinned(species_multiplicity), is_pinned(mask),
               is_pinned(rjs) && is_pinned(thetas) && is_pinned(phis)};
  // soap in page-locked memory the GPU can address: the site kernel writes
  // its rows there directly, so they cross the host link while later sites
  // compute, instead of in copies after each chunk's kernels
  double *soap_dev = chunked ? (double *)mapped_host(soap) : nullptr;
  const bool soap_staged = chunked && !soap_dev && !is_pinned(soap) && 8 * (size_t)n_sites * n_soap <= kStageCap;
  // The reference adds the compressed descriptor into the caller's soap
  // (src/soap_turbo.f90:798-802; its callers pass it zeroed) and overwrites an
  // uncompressed one; the caller's values therefore come in when compressing.
  const bool accumulate = compress_soap != 0 && n_sites > 0;
  in.soap = soap;
  in.n_soap = n_soap;
  in.acc = accumulate && !soap_dev;
  if (chunked) {
    // written in place, soap rows take the host link at the rate the site
    // kernel produces them, and a chunk's kernels start and end with the link
    // idle: chunks of at least 4096 sites (the chunking then only overlaps
    // the inputs of large batches with their kernels)
    plan_chunks(d.chunk, n_sites, false, soap_dev ? 4096 : 512);
    nch = (int)d.chunk.size() - 1;
    if ((rc = dropin_streams(d, 3 * nch + 1))) return rc;
    if ((rc = d.n_neigh.ensure(4 * ((size_t)n_sites + 1)))) return rc;
    if ((rc = d.species.ensure(4 * ((size_t)n_sites * max_species_multiplicity + 1)))) return rc;
    if ((rc = d.species_mult.ensure(4 * ((size_t)n_sites + 1)))) return rc;
    if ((rc = d.mask.ensure((size_t)n_atom_pairs * n_species + 1))) return rc;
    if ((rc = d.rjs.ensure(8 * ((size_t)n_atom_pairs + 1)))) return rc;
    if ((rc = d.thetas.ensure(8 * ((size_t)n_atom_pairs + 1)))) return rc;
    if ((rc = d.phis.ensure(8 * ((size_t)n_atom_pairs + 1)))) return rc;
    if ((rc = d.soap.ensure(8 * ((size_t)n_sites * n_soap + 1)))) return rc;
    if ((rc = plan_get_soap_staging(d, in, n_sites, max_species_multiplicity, n_species, n_atom_pairs))) return rc;
    if (soap_staged && (rc = d.st_out.ensure(8 * (size_t)n_sites * n_soap))) return rc;
    // staged soap rows come in through the output staging area: chunk i's rows
    // are copied out of it only after its kernels, which wait for its copy in
    if (soap_staged) in.st_soap = d.st_out.as<uint8_t>();
    const int copied = copy_in_sites(d, in, n_sites, max_species_multiplicity);
    if (copied) {
      cudaStreamSynchronize(d.copy_in);  // no copy from the caller's arrays outlives the call
      return copied;
    }
  } else {
    if ((rc = upload(d.n_neigh, n_neigh, n_sites, s))) return rc;
    if ((rc = upload(d.species, species, (size_t)n_sites * max_species_multiplicity, s))) return rc;
    if ((rc = upload(d.species_mult, species_multiplicity, n_sites, s))) return rc;
    if ((rc = upload(d.mask, mask, (size_t)n_atom_pairs * n_species, s))) return rc;
    if ((rc = upload(d.rjs, rjs, n_atom_pairs, s))) return rc;
    if ((rc = upload(d.thetas, thetas, n_atom_pairs, s))) return rc;
    if ((rc = upload(d.phis, phis, n_atom_pairs, s))) return rc;
    if ((rc = d.soap.ensure(8 * ((size_t)n_sites * n_soap + 1)))) return rc;
    if (accumulate) {
      const size_t nb = 8 * (size_t)n_sites * n_soap;
      if (host_all_zero(soap, nb)) CU(cudaMemsetAsync(d.soap.p, 0, nb, s));
      else CU(cudaMemcpyAsync(d.soap.p, soap, nb, cudaMemcpyHostToDevice, s));
    }
  }
  soapb_batch &bt = d.batch;
  bt.n_sites = n_sites;
  bt.n_atom_pairs = n_atom_pairs;
  bt.max_species_multiplicity = max_species_multiplicity;
  bt.n_neigh = d.n_neigh.as<int32_t>();
  bt.species = d.species.as<int32_t>();
  bt.species_multiplicity = d.species_mult.as<int32_t>();
  bt.mask = d.mask.as<uint8_t>();
  bt.rjs = d.rjs.as<double>();
  bt.thetas = d.thetas.as<double>();
  bt.phis = d.phis.as<double>();
  if (do_timing) cudaEventRecord(ev[1], s);
  const bool keep_cart = fp64 && do_derivatives;  // FP64 contract works on soap_cart_der
  bool soap_copied = false;
  if (fp64) {
    if (keep_cart && (rc = d.cart.ensure(8 * ((size_t)n_atom_pairs * n_soap * 3 + 1)))) return rc;
    // The self column of soap_cart_der is accumulated into (:888-892): the
    // caller's self columns come in, gathered into (3, n_soap) per site.
    const double *self_init = nullptr;
    if (want_cart && n_atom_pairs > 0) {
      const size_t w3 = 3 * (size_t)n_soap;
      d.self_host.resize(w3 * (size_t)n_sites);
      double *dst = d.self_host.data();
      const long long *off = d.host_off.data();
#pragma omp parallel for schedule(static) num_threads(copy_threads(8 * w3 * (size_t)n_sites))
      for (int i = 0; i < n_sites; ++i) {
        if (off[i + 1] > off[i]) std::memcpy(dst + w3 * i, soap_cart_der + w3 * (size_t)off[i], 8 * w3);
        else std::memset(dst + w3 * i, 0, 8 * w3);
      }
      if ((rc = upload(d.cart_self, dst, w3 * (size_t)n_sites, s))) return rc;
      self_init = d.cart_self.as<double>();
    }
    rc = ctx_fp64(c, &bt, d.soap.as<double>(), keep_cart ? d.cart.as<double>() : nullptr, accumulate, self_init);
  } else if (chunked) {
    SiteChunks ch;
    ch.n = nch;
    ch.bounds = d.chunk.data();
    ch.site_off = d.host_off.data();
    ch.before = [&](int i) -> int {
      const int r2 = copy_in_pairs(d, in, i, n_species, n_atom_pairs);
      if (r2) return r2;
      CU(cudaStreamWaitEvent(s, d.evs[i], 0));
      return SOAPB_OK;
    };
    double *soap_dst = soap_staged ? d.st_out.as<double>() : soap;
    // with soap_dev, a chunk whose caller rows are all zero (the usual call)
    // is written without reading them; any other is added into in place.  The
    // host scans a chunk's rows after its pair kernel is queued, while the
    // GPU copies its inputs and runs that kernel.
    if (soap_dev)
      ch.acc_of = [&](int i) {
        const size_t b0 = 8 * (size_t)d.chunk[i] * n_soap, nb = 8 * (size_t)(d.chunk[i + 1] - d.chunk[i]) * n_soap;
        return accumulate && !host_all_zero((const uint8_t *)soap + b0, nb);
      };
    ch.after = [&](int i) -> int {
      if (soap_dev) return SOAPB_OK;
      const size_t lo = (size_t)d.chunk[i], hi = (size_t)d.chunk[i + 1];
      CU(cudaEventRecord(d.evs[nch + i], s));
      CU(cudaStreamWaitEvent(d.copy_out, d.evs[nch + i], 0));
      CU(cudaMemcpyAsync(soap_dst + lo * n_soap, d.soap.as<double>() + lo * n_soap, 8 * (hi - lo) * n_soap,
                         cudaMemcpyDeviceToHost, d.copy_out));
      if (soap_staged) CU(cudaEventRecord(d.evs[2 * nch + 1 + i], d.copy_out));
      return SOAPB_OK;
    };
    rc = ctx_descriptor(c, &bt, soap_dev ? soap_dev : d.soap.as<double>(), do_derivatives && contract, &ch,
                        accumulate);
    // the staged soap rows, chunk by chunk as their copies arrive
    for (int i = 0; rc == 0 && soap_staged && i < nch; ++i) {
      const cudaError_t e = cudaEventSynchronize(d.evs[2 * nch + 1 + i]);
      if (e != cudaSuccess) {
        rc = cuda_fail(e, "cudaEventSynchronize");
        break;
      }
      const size_t lo = (size_t)d.chunk[i], hi = (size_t)d.chunk[i + 1];
      par_copy(soap + lo * n_soap, soap_dst + lo * n_soap, 8 * (hi - lo) * n_soap);
    }
    soap_copied = true;
  } else {
    rc = ctx_descriptor(c, &bt, d.soap.as<double>(), do_derivatives && contract, nullptr, accumulate);
  }
  if (rc) {
    if (chunked) {  // no copy from or into the caller's arrays outlives the call
      cudaStreamSynchronize(d.copy_in);
      cudaStreamSynchronize(d.copy_out);
    }
    return rc;
  }
  if (do_timing) cudaEventRecord(ev[2], s);
  if (n_sites > 0 && !soap_copied)
    CU(cudaMemcpyAsync(soap, d.soap.p, 8 * (size_t)n_sites * n_soap, cudaMemcpyDeviceToHost, s));
  if (want_cart && n_atom_pairs > 0)
    CU(cudaMemcpyAsync(soap_cart_der, d.cart.p, 8 * (size_t)n_atom_pairs * n_soap * 3,
                       cudaMemcpyDeviceToHost, s));
  if (do_timing) cudaEventRecord(ev[3], s);
  // the prep error word comes back with the same wait.  The compute stream
  // has waited for every chunk's copies in; made to wait for the last soap
  // rows on copy_out as well, its synchronisation covers all three streams
  // (each is synchronised if the join cannot be made).
  if ((rc = dropin_streams(d, 0))) return rc;
  bool joined = false;
  if (chunked) {
    cudaEvent_t ej = d.evs[2 * nch];
    joined = cudaEventRecord(ej, d.copy_out) == cudaSuccess && cudaStreamWaitEvent(s, ej, 0) == cudaSuccess;
  }
  *d.err_host = 0;
  if (c->err.p) CU(cudaMemcpyAsync(d.err_host, c->err.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  const cudaError_t es = cudaStreamSynchronize(s);
  const cudaError_t ei = (chunked && !joined) ? cudaStreamSynchronize(d.copy_in) : cudaSuccess;
  const cudaError_t eo = (chunked && !joined) ? cudaStreamSynchronize(d.copy_out) : cudaSuccess;
  CU(es);
  CU(ei);
  CU(eo);
  if ((rc = input_status(*d.err_host, nullptr))) return rc;
  if (do_timing) {
    float t01, t12, t23;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    cudaEventElapsedTime(&t23, ev[2], ev[3]);
    std::printf("                                       |\n");
    std::printf("SOAP timings (GPU, %s):              |\n", fp64 ? "FP64" : "mixed");
    std::printf("  *) Host to device copies: %8.3f ms |\n", t01);
    std::printf("  *) Descriptor kernels:    %8.3f ms |\n", t12);
    std::printf("  *) Device to host copies: %8.3f ms |\n", t23);
    std::fflush(stdout);
    for (auto &e : ev) cudaEventDestroy(e);
  }
  if (do_hessian) {
    d.hs_ready = 1;
    d.hs_n_sites = n_sites;
    d.hs_n_pairs = n_atom_pairs;
    d.hs_l_max = l_max;
    d.hs_n_soap = n_soap;
  }
  if (do_derivatives && contract) {
    d.ct_ready = 1;
    d.ct_fp64 = fp64;
    d.ct_n_sites = n_sites;
    d.ct_n_pairs = n_atom_pairs;
    d.ct_n_soap = n_soap;
  }
  return SOAPB_OK;
}

int soapb_soap_contract(const double *soap, const double *G, double sgn, double *pair, int32_t n_sites,
                        int32_t n_soap, int32_t n_atom_pairs) {
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  if (!d.ct_ready || !d.ctx)
    return fail(SOAPB_ERR_CONTRACT_STATE, "ERROR: soap_contract needs get_soap called with contract = .true. first");
  if (n_sites != d.ct_n_sites || n_soap != d.ct_n_soap || n_atom_pairs != d.ct_n_pairs)
    return fail(SOAPB_ERR_ARGUMENT, "extents differ from the last get_soap call");
  if (n_sites > 0 && (!soap || !G || !pair)) return fail(SOAPB_ERR_ARGUMENT, "null pointer");
  cudaStream_t s = d.stream;
  int rc;
  if ((rc = d.pair.ensure(8 * (3 * (size_t)n_atom_pairs + 1)))) return rc;
  if (d.ct_fp64) {
    if ((rc = upload(d.soap, soap, (size_t)n_sites * n_soap, s))) return rc;
    if ((rc = upload(d.G, G, (size_t)n_sites * n_soap, s))) return rc;
    if ((rc = soapb_contract_cart_der(d.ctx, &d.batch, d.cart.as<double>(), d.G.as<double>(),
                                      SOAPB_G_SITE_FASTEST, sgn, d.pair.as<double>())))
      return rc;
    if (n_atom_pairs > 0)
      CU(cudaMemcpyAsync(pair, d.pair.p, 24 * (size_t)n_atom_pairs, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return SOAPB_OK;
  }
  // per site chunk: soap rows and G columns in on copy_in (evs[i]), the
  // contract on the compute stream once they are there, the chunk's pair
  // forces out on copy_out.  Pageable caller arrays pass through the pinned
  // staging areas as in get_soap: a chunk's soap rows and G columns are copied
  // into st_in on the host just before their asynchronous copy, and the pair
  // forces land in st_out, copied out chunk by chunk as they arrive
  // (evs[2 nch + 1 + i]).
  if ((rc = d.soap.ensure(8 * ((size_t)n_sites * n_soap + 1)))) return rc;
  if ((rc = d.G.ensure(8 * ((size_t)n_sites * n_soap + 1)))) return rc;
  if ((int)d.cchunk.size() < 2 || d.cchunk.back() != n_sites) plan_chunks(d.cchunk, n_sites, true, 384);
  const int nch = (int)d.cchunk.size() - 1;
  if ((rc = dropin_streams(d, 3 * nch + 1))) return rc;
  const size_t b_rows = align16(8 * (size_t)n_sites * n_soap);
  const bool big = 2 * b_rows > kStageCap;  // above the cap: the runtime's copies
  const bool st_soap = !big && !is_pinned(soap), st_G = !big && !is_pinned(G);
  // pair in page-locked memory the GPU can address: the contract writes the
  // forces there directly, so no copy out follows the last chunk
  double *pair_mapped = (double *)mapped_host(pair);
  const bool st_pair = !pair_mapped && !is_pinned(pair) && 24 * (size_t)n_atom_pairs <= kStageCap;
  if ((st_soap || st_G) && (rc = d.st_in.ensure((st_soap ? b_rows : 0) + (st_G ? b_rows : 0)))) return rc;
  if (st_pair && (rc = d.st_out.ensure(24 * (size_t)n_atom_pairs))) return rc;
  double *sg_soap = st_soap ? d.st_in.as<double>() : nullptr;
  double *sg_G = st_G ? (double *)(d.st_in.as<uint8_t>() + (st_soap ? b_rows : 0)) : nullptr;
  double *pair_dst = st_pair ? d.st_out.as<double>() : pair;
  double *dS = d.soap.as<double>(), *dG = d.G.as<double>(), *dP = pair_mapped ? pair_mapped : d.pair.as<double>();
  CU(cudaEventRecord(d.evs[0], s));  // the copies in must not overwrite what earlier work still reads
  CU(cudaStreamWaitEvent(d.copy_in, d.evs[0], 0));
  SiteChunks ch;
  ch.n = nch;
  ch.bounds = d.cchunk.data();
  ch.before = [&](int i) -> int {
    const size_t lo = (size_t)d.cchunk[i], hi = (size_t)d.cchunk[i + 1];
    const int r2 = h2d_in(dS + lo * n_soap, soap + lo * n_soap, sg_soap ? (uint8_t *)(sg_soap + lo * n_soap) : nullptr,
                          8 * (hi - lo) * n_soap, d.copy_in);
    if (r2) return r2;
    // G(n_sites, n_soap): the chunk's sites of every column
    const double *gsrc = G + lo;
    if (sg_G) {
      par_copy2d(sg_G + lo, 8 * (size_t)n_sites, G + lo, 8 * (size_t)n_sites, 8 * (hi - lo), (size_t)n_soap);
      gsrc = sg_G + lo;
    }
    CU(cudaMemcpy2DAsync(dG + lo, 8 * (size_t)n_sites, gsrc, 8 * (size_t)n_sites, 8 * (hi - lo), n_soap,
                         cudaMemcpyHostToDevice, d.copy_in));
    CU(cudaEventRecord(d.evs[i], d.copy_in));
    CU(cudaStreamWaitEvent(s, d.evs[i], 0));
    return SOAPB_OK;
  };
  ch.after = [&](int i) -> int {
    if (pair_mapped) return SOAPB_OK;
    const long long p0 = d.host_off[d.cchunk[i]], p1 = d.host_off[d.cchunk[i + 1]];
    CU(cudaEventRecord(d.evs[nch + i], s));
    CU(cudaStreamWaitEvent(d.copy_out, d.evs[nch + i], 0));
    if (p1 > p0)
      CU(cudaMemcpyAsync(pair_dst + 3 * p0, dP + 3 * p0, 24 * (size_t)(p1 - p0), cudaMemcpyDeviceToHost,
                         d.copy_out));
    if (st_pair) CU(cudaEventRecord(d.evs[2 * nch + 1 + i], d.copy_out));
    return SOAPB_OK;
  };
  rc = ctx_contract(d.ctx, &d.batch, dS, dG, SOAPB_G_SITE_FASTEST, sgn, dP, &ch);
  // the staged pair forces, chunk by chunk as their copies arrive
  for (int i = 0; rc == 0 && st_pair && n_sites > 0 && i < nch; ++i) {
    const cudaError_t e = cudaEventSynchronize(d.evs[2 * nch + 1 + i]);
    if (e != cudaSuccess) {
      rc = cuda_fail(e, "cudaEventSynchronize");
      break;
    }
    const long long p0 = d.host_off[d.cchunk[i]], p1 = d.host_off[d.cchunk[i + 1]];
    par_copy(pair + 3 * p0, pair_dst + 3 * p0, 24 * (size_t)(p1 - p0));
  }
  // whatever ran, no copy may still be in flight when this returns.  The
  // compute stream has waited for every chunk's copies in; made to wait for the
  // last pair forces out as well, its synchronisation covers all three streams.
  if (rc == 0) {
    cudaEvent_t ej = d.evs[2 * nch];
    if (cudaEventRecord(ej, d.copy_out) == cudaSuccess && cudaStreamWaitEvent(s, ej, 0) == cudaSuccess) {
      CU(cudaStreamSynchronize(s));
      return SOAPB_OK;
    }
  }
  const cudaError_t e1 = cudaStreamSynchronize(d.copy_in), e2 = cudaStreamSynchronize(s),
                    e3 = cudaStreamSynchronize(d.copy_out);
  if (rc) return rc;
  CU(e1);
  CU(e2);
  CU(e3);
  return SOAPB_OK;
}

int soapb_get_soap_central_hessian(int32_t n_sites, const int32_t *n_neigh, int32_t n_atom_pairs,
                                   int32_t n_species, const uint8_t *mask, const double *rjs,
                                   const double *thetas, const double *phis, int32_t l_max,
                                   const double *rcut_hard, const double *atom_sigma_t,
                                   const double *atom_sigma_t_scaling, int32_t compress_soap,
                                   int32_t compress_P_nonzero, const int32_t *compress_P_i,
                                   const int32_t *compress_P_j, const double *compress_P_el,
                                   const double *soap, int32_t n_soap, int32_t n_vec, const double *vecs,
                                   double *hess) {
  (void)n_neigh; (void)n_species; (void)mask; (void)rjs; (void)thetas; (void)phis; (void)rcut_hard;
  (void)atom_sigma_t; (void)atom_sigma_t_scaling; (void)compress_soap; (void)compress_P_nonzero;
  (void)compress_P_i; (void)compress_P_j; (void)compress_P_el;
  DropIn &d = dropin();
  std::lock_guard<std::mutex> g(d.mu);
  // state check (src/soap_turbo.f90:1206-1227)
  if (!d.hs_ready || !d.ctx)
    return fail(SOAPB_ERR_HESSIAN_STATE,
                "ERROR: get_soap_central_hessian was called without a matching get_soap. Set "
                "soap_hessian_enabled = .true. and call get_soap with do_derivatives = .true. first.");
  if (n_sites != d.hs_n_sites || n_atom_pairs != d.hs_n_pairs || l_max != d.hs_l_max || n_soap != d.hs_n_soap)
    return fail(SOAPB_ERR_HESSIAN_STATE,
                "ERROR: get_soap_central_hessian was called on a different batch than the get_soap that "
                "filled the buffers it reads.");
  if (n_vec < 0) return fail(SOAPB_ERR_ARGUMENT, "n_vec must be >= 0");
  if (n_vec == 0 || n_atom_pairs == 0) return SOAPB_OK;
  if (!soap || !vecs || !hess) return fail(SOAPB_ERR_ARGUMENT, "null pointer");
  cudaStream_t s = d.stream;
  int rc;
  const size_t nsv = (size_t)n_sites * n_soap;
  const size_t b_soap = align16(8 * nsv), b_vecs = align16(8 * nsv * n_vec);
  const size_t b_hess = 72 * (size_t)n_vec * n_atom_pairs;
  // pageable soap and vecs go through the pinned staging area (the host fills
  // vecs' region while soap's copy runs), pageable hess comes back through it
  const bool st_soap = !is_pinned(soap) && b_soap + b_vecs <= kStageCap;
  const bool st_vecs = !is_pinned(vecs) && b_soap + b_vecs <= kStageCap;
  const bool st_hess = !is_pinned(hess) && b_hess <= kStageCap;
  if ((st_soap || st_vecs) && (rc = d.st_in.ensure(b_soap + b_vecs))) return rc;
  if (st_hess && (rc = d.st_out.ensure(b_hess))) return rc;
  if ((rc = d.soap.ensure(8 * (nsv + 1)))) return rc;
  if ((rc = d.vecs.ensure(8 * (nsv * n_vec + 1)))) return rc;
  if ((rc = d.hess.ensure(8 * (9 * (size_t)n_vec * n_atom_pairs + 1)))) return rc;
  if ((rc = h2d_in(d.soap.p, soap, st_soap ? d.st_in.as<uint8_t>() : nullptr, 8 * nsv, s))) return rc;
  if ((rc = h2d_in(d.vecs.p, vecs, st_vecs ? d.st_in.as<uint8_t>() + b_soap : nullptr, 8 * nsv * n_vec, s))) {
    cudaStreamSynchronize(s);
    return rc;
  }
  if ((rc = ctx_hessian(d.ctx, &d.batch, d.soap.as<double>(), n_vec, d.vecs.as<double>(), d.hess.as<double>()))) {
    cudaStreamSynchronize(s);
    return rc;
  }
  CU(cudaMemcpyAsync(st_hess ? d.st_out.p : (void *)hess, d.hess.p, b_hess, cudaMemcpyDeviceToHost, s));
  if ((rc = dropin_streams(d, 0))) return rc;
  *d.err_host = 0;
  if (d.ctx->err.p)
    CU(cudaMemcpyAsync(d.err_host, d.ctx->err.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (st_hess) par_copy(hess, d.st_out.p, b_hess);
  return input_status(*d.err_host, nullptr);
}

}  // extern "C"
