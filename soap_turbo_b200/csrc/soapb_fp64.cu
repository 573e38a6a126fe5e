// soapb_fp64.cu -- the plain FP64 form of the descriptor path, staged like the
// reference (src/soap_turbo.f90:491-909): radial and angular expansions of
// every pair to global memory, c_nlm per site, power spectrum, then the
// spherical derivatives, normalisation derivative and Cartesian rotation into
// a materialised soap_cart_der (3, n_soap, n_pairs), and a contraction of
// that array with G.  It serves callers that read soap_cart_der itself
// (get_soap with do_derivatives and contract = .false.) and is the FP64
// baseline the mixed-precision adjoint path is measured against.  Kernels are
// coalesced and do no redundant zeroing, but keep the reference's structure.
#include "soapb_device.cuh"

namespace soapb {

constexpr double kFourPi64 = 12.566370614359172954;

// ---- radial, one thread per pair, every species block (:491-544)
template <int AMAX, bool OP>
__global__ void k64_radial(const DevParams P, const DevBatch B, int do_der, double *rad,
                           double *rad_der) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= B.n_pairs) return;
  // site-local index: binary search of the CSR offsets
  int lo = 0, hi = B.n_sites;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (B.off[mid] <= k) lo = mid; else hi = mid;
  }
  const bool is_self = (B.off[lo] == k);
  const double r = B.rjs[k];
  const unsigned bits = B.bits[k];
  double *ro = rad + (size_t)k * P.n_max, *rdo = rad_der + (size_t)k * P.n_max;
  unsigned todo = 0u;
  for (int s = 0; s < P.n_species; ++s) {
    const RadSp &S = P.rad[s];
    const bool ok = ((bits >> s) & 1u) && r < S.rcut_hard && (!is_self || S.do_central);
    if (ok) todo |= 1u << s;
    else
      for (int n = 0; n < S.alpha; ++n) {
        ro[S.nbeg + n] = 0.0;
        if (do_der) rdo[S.nbeg + n] = 0.0;
      }
  }
  // one expansion call per valid species; lanes of different species share it
  while (todo) {
    const int s = __ffs(todo) - 1;
    todo &= todo - 1u;
    const RadSp &S = P.rad[s];
    double val[AMAX], der[AMAX];
    radial_entry<AMAX, OP>(P, S, P.Wblk + (size_t)s * P.wstride, r, is_self, do_der != 0, val, der);
    for (int n = 0; n < S.alpha; ++n) {
      ro[S.nbeg + n] = val[n] * S.gscale;
      if (do_der) rdo[S.nbeg + n] = der[n] * S.gscale;
    }
  }
}

// ---- angular, one thread per pair (src/soap_turbo_angular.f90:549-607)
template <int LC>
__global__ void k64_angular(const DevParams P, const DevBatch B, int do_der, double2 *ang) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= B.n_pairs) return;
  const int K = P.k_max;
  const size_t plane = (size_t)B.n_pairs * K;
  double2 *A = ang + (size_t)k * K;
  const double r = B.rjs[k];
  const unsigned bits = B.bits[k];
  if (!(r < P.rcut_max) || bits == 0u) {
    for (int kk = 0; kk < K; ++kk) {
      A[kk] = make_double2(0.0, 0.0);
      if (do_der) {
        A[plane + kk] = make_double2(0.0, 0.0);
        A[2 * plane + kk] = make_double2(0.0, 0.0);
        A[3 * plane + kk] = make_double2(0.0, 0.0);
      }
    }
    return;
  }
  AngScalars<LC> S;
  angular_scalars<LC>(P, __ffs(bits) - 1, r, B.thetas[k], B.phis[k], do_der != 0, S);
  double plm[(LC + 2) * (LC + 3) / 2];
  plm_array<LC + 1, double>(P.l_max + 1, S.x, S.sq, plm);
  for (int l = 0; l <= P.l_max; ++l) {
    for (int m = 0; m <= l; ++m) {
      const int kk = l * (l + 1) / 2 + m;
      const double e_re = S.il[l] * S.er[m], e_im = S.il[l] * S.ei[m];
      const double u = S.amp * P.preflm64[kk];
      const double v = u * plm[kk];
      A[kk] = make_double2(v * e_re, v * e_im);
      if (do_der) {
        const double er_re = S.ild[l] * S.er[m], er_im = S.ild[l] * S.ei[m];
        A[plane + kk] = make_double2(v * er_re - S.sig_fac * v * e_re, v * er_im - S.sig_fac * v * e_im);
        double dms, dvs;
        if (m == 0) {
          dms = (l == 0) ? 0.0 : -0.5 * plm[l * (l + 1) / 2 + 1];
          dvs = 0.0;
        } else {
          dms = 0.5 * (double)(l + m) * (double)(l - m + 1) * plm[kk - 1];
          dvs = 0.5 * (double)(l - m + 1) * (double)(l - m + 2) * plm[(l + 1) * (l + 2) / 2 + m - 1] +
                0.5 * plm[(l + 1) * (l + 2) / 2 + m + 1];
        }
        if (m != l) dms = dms + -0.5 * plm[kk + 1];
        const double w = u * dvs;
        A[2 * plane + kk] = make_double2(-(w * e_im), w * e_re);
        const double w2 = u * dms;
        A[3 * plane + kk] = make_double2(w2 * e_re, w2 * e_im);
      }
    }
  }
}

// ---- the same with the associated Legendre rows streamed: P_l^m of rows l - 1,
// l and l + 1 only (the recursion of get_plm_array, src/soap_turbo_angular.f90:
// 108-160), every loop unrolled so that they stay in registers, and each (l, m)
// written as soon as rows l and l + 1 exist (the derivative forms need
// P_{l+1}^{m+-1}, :181-248).  With derivatives the CTA is four warps over the
// same 32 pairs, warp w writing plane w (the expansion, its radial, azimuthal
// and polar derivative), so that a pair's four planes are formed at once;
// without, one warp writes the expansion.  Same arithmetic as k64_angular.
template <int LC>
__global__ void __launch_bounds__(128, 4) k64_angular2(const DevParams P, const DevBatch B, int do_der, double2 *ang) {
  const int pl = do_der ? (int)(threadIdx.x >> 5) : 0;  // warp-uniform
  const int k = blockIdx.x * 32 + (threadIdx.x & 31);
  if (k >= B.n_pairs) return;
  const int K = P.k_max, L = P.l_max;
  const size_t plane = (size_t)B.n_pairs * K;
  double2 *A = ang + pl * plane + (size_t)k * K;
  const double r = B.rjs[k];
  const unsigned bits = B.bits[k];
  if (!(r < P.rcut_max) || bits == 0u) {
    for (int kk = 0; kk < K; ++kk) A[kk] = make_double2(0.0, 0.0);
    return;
  }
  AngScalars<LC> S;
  angular_scalars<LC>(P, __ffs(bits) - 1, r, B.thetas[k], B.phis[k], pl == 1, S);
  const double x = S.x, sq = S.sq, x2 = x * x;
  // rows: pc (l), pn (l + 1); m <= l + 1 <= LC + 1
  double pc[LC + 2], pn[LC + 2];
#pragma unroll
  for (int m = 0; m < LC + 2; ++m) pc[m] = pn[m] = 0.0;
  pc[0] = 1.0;        // l = 0
  pn[0] = x;          // l = 1
  pn[1] = -sq;
#pragma unroll
  for (int l = 0; l <= LC; ++l) {
    if (l > L) break;
#pragma unroll
    for (int m = 0; m <= l; ++m) {
      const int kk = l * (l + 1) / 2 + m;
      const double e_re = S.il[l] * S.er[m], e_im = S.il[l] * S.ei[m];
      const double u = S.amp * P.preflm64[kk];
      const double v = u * pc[m];
      if (pl == 0) {
        A[kk] = make_double2(v * e_re, v * e_im);
      } else if (pl == 1) {
        const double er_re = S.ild[l] * S.er[m], er_im = S.ild[l] * S.ei[m];
        A[kk] = make_double2(v * er_re - S.sig_fac * v * e_re, v * er_im - S.sig_fac * v * e_im);
      } else if (pl == 2) {
        const double dvs =
            (m == 0) ? 0.0 : 0.5 * (double)(l - m + 1) * (double)(l - m + 2) * pn[m - 1] + 0.5 * pn[m + 1];
        const double w = u * dvs;
        A[kk] = make_double2(-(w * e_im), w * e_re);
      } else {
        double dms;
        if (m == 0) dms = (l == 0) ? 0.0 : -0.5 * pc[1];
        else dms = 0.5 * (double)(l + m) * (double)(l - m + 1) * pc[m - 1];
        if (m != l) dms = dms + -0.5 * pc[m + 1];
        const double w2 = u * dms;
        A[kk] = make_double2(w2 * e_re, w2 * e_im);
      }
    }
    // advance: row l + 2 from rows l + 1 (pn) and l (pc)
    const int l2 = l + 2;
    double nn[LC + 2];
#pragma unroll
    for (int m = 0; m < LC + 2; ++m) nn[m] = 0.0;
    if (l2 == 2) {
      nn[0] = 1.5 * x2 - 0.5;
      nn[1] = -3.0 * x * sq;
      nn[2] = 3.0 - 3.0 * x2;
    } else if (l2 <= LC + 1) {
#pragma unroll
      for (int m = 0; m <= l2 - 2 && m < LC + 2; ++m) {
        const double aa = (double)(2 * l2 - 1) / (double)(l2 - m);
        const double bb = (double)(l2 - 1 + m) / (double)(l2 - m);
        nn[m] = aa * x * pn[m] - bb * pc[m];
      }
      if (l2 - 1 < LC + 2) nn[l2 - 1] = x * (double)(2 * l2 - 1) * pn[l2 - 1];
      if (l2 < LC + 2) nn[l2] = -(double)(2 * l2 - 1) * sq * pn[l2 - 1];
    }
#pragma unroll
    for (int m = 0; m < LC + 2; ++m) {
      pc[m] = pn[m];
      pn[m] = nn[m];
    }
  }
}

// ---- c_nlm, one CTA per site, threads over (n, k) (src/soap_turbo.f90:626-664).
// The site's pairs go in chunks of kCnkChunk whose radial values and angular
// plane are staged in shared memory with coalesced loads; each thread then sums
// its (n, k) items over the chunk's pairs in CSR order.
constexpr int kCnkChunk = 32;
__global__ void __launch_bounds__(256) k64_cnk(const DevParams P, const DevBatch B, const double *rad,
                                               const double2 *ang, double2 *cnk) {
  extern __shared__ double csm[];
  const int site = blockIdx.x;
  const int K = P.k_max, N = P.n_max;
  const int p0 = B.off[site], p1 = min(B.off[site + 1], B.n_pairs);
  double *sR = csm;                          // kCnkChunk x N
  double2 *sA = (double2 *)(csm + kCnkChunk * N);  // kCnkChunk x K
  constexpr int IT = 8;                      // items per thread (N K <= 8 * 256)
  double cr[IT], ci[IT];
#pragma unroll
  for (int j = 0; j < IT; ++j) cr[j] = ci[j] = 0.0;
  for (int c0 = p0; c0 < p1; c0 += kCnkChunk) {
    const int np_ = min(kCnkChunk, p1 - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < np_ * N; t += blockDim.x) sR[t] = rad[(size_t)c0 * N + t];
    for (int t = threadIdx.x; t < np_ * K; t += blockDim.x) sA[t] = ang[(size_t)c0 * K + t];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < IT; ++j) {
      const int it = threadIdx.x + j * blockDim.x;
      if (it >= N * K) break;
      const int n = it / K, kk = it - n * K;
      for (int q = 0; q < np_; ++q) {
        const double fr = kFourPi64 * sR[q * N + n];
        const double2 a = sA[q * K + kk];
        cr[j] = cr[j] + fr * a.x;
        ci[j] = ci[j] + fr * a.y;
      }
    }
  }
  double2 *c = cnk + (size_t)site * N * K;
#pragma unroll
  for (int j = 0; j < IT; ++j) {
    const int it = threadIdx.x + j * blockDim.x;
    if (it >= N * K) break;
    const int n = it / K, kk = it - n * K;
    double r = cr[j];
    if (P.basis == 1 && kk == 0) {
      for (int mm = 0; mm < B.species_mult[site]; ++mm) {
        const int s = B.species[(size_t)site * B.max_mult + mm] - 1;
        if (s >= 0 && s < P.n_species && n >= P.rad[s].nbeg && n < P.rad[s].nbeg + P.rad[s].alpha)
          r += P.central[n];
      }
    }
    c[it] = make_double2(r, ci[j]);
  }
}

// The CSR-order item loop of the form above for definitions with N K > 8 x 256.
__global__ void k64_cnk_wide(const DevParams P, const DevBatch B, const double *rad, const double2 *ang,
                             double2 *cnk) {
  const int site = blockIdx.x;
  const int K = P.k_max, N = P.n_max;
  const int p0 = B.off[site], p1 = min(B.off[site + 1], B.n_pairs);
  double2 *c = cnk + (size_t)site * N * K;
  for (int it = threadIdx.x; it < N * K; it += blockDim.x) {
    const int n = it / K, kk = it - n * K;
    double cr = 0.0, ci = 0.0;
    for (int k = p0; k < p1; ++k) {
      const double fr = kFourPi64 * rad[(size_t)k * N + n];
      const double2 a = ang[(size_t)k * K + kk];
      cr = cr + fr * a.x;
      ci = ci + fr * a.y;
    }
    if (P.basis == 1 && kk == 0) {
      for (int mm = 0; mm < B.species_mult[site]; ++mm) {
        const int s = B.species[(size_t)site * B.max_mult + mm] - 1;
        if (s >= 0 && s < P.n_species && n >= P.rad[s].nbeg && n < P.rad[s].nbeg + P.rad[s].alpha)
          cr += P.central[n];
      }
    }
    c[it] = make_double2(cr, ci);
  }
}

// ---- power spectrum + compression + norm, one CTA per site (:750-813).
// soap_acc (may be null): the caller's soap, added before the norm is taken, as
// the reference adds the compressed descriptor into soap (:798-802).
__global__ void k64_soap(const DevParams P, const DevBatch B, const double2 *cnk, const double *soap_acc,
                         double *soap_un, double *norm) {
  extern __shared__ double sp[];  // n_kept
  __shared__ double red[32];
  const int site = blockIdx.x;
  const int K = P.k_max;
  const double2 *c = cnk + (size_t)site * P.n_max * K;
  for (int q = threadIdx.x; q < P.n_kept; q += blockDim.x) {
    const int code = P.kept_nnl[q];
    const int n = code & 0xff, np = (code >> 8) & 0xff, l = code >> 16;
    double acc = 0.0;
    const double base = (n == np) ? 1.0 : sqrt(2.0);
    for (int m = 0; m <= l; ++m) {
      const int kk = l * (l + 1) / 2 + m;
      const double2 a = c[(size_t)n * K + kk], b = c[(size_t)np * K + kk];
      const double mult = base * ((m > 0) ? 2.0 : 1.0);
      acc = acc + mult * (a.x * b.x + a.y * b.y);
    }
    sp[q] = acc;
  }
  __syncthreads();
  double part = 0.0;
  double *out = soap_un + (size_t)site * P.n_soap;
  const double *in = soap_acc ? soap_acc + (size_t)site * P.n_soap : nullptr;
  for (int o = threadIdx.x; o < P.n_soap; o += blockDim.x) {
    double v = in ? in[o] : 0.0;
    for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) v = v + P.pi_el64[t] * sp[P.pi_q[t]];
    out[o] = v;
    part += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    double nr = sqrt(t);
    if (nr < 1.0e-5) nr = 1.0;
    norm[site] = nr;
  }
}

// Fixed-order sum of three values over the CTA (warp shuffles, then warp 0).
template <int NT>
__device__ __forceinline__ void cta_sum3(double &a, double &b, double &c, double (*red)[NT / 32]) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = a;
    red[1][threadIdx.x >> 5] = b;
    red[2][threadIdx.x >> 5] = c;
  }
  __syncthreads();
  a = b = c = 0.0;
  for (int w = 0; w < NT / 32; ++w) {
    a += red[0][w];
    b += red[1][w];
    c += red[2][w];
  }
}

// Shared memory of k64_cart_site, in doubles.  STAGED: the site's c_nlm, soap
// row and self column are in shared memory too (else they are read and summed
// in global memory, for definitions whose rows do not fit).
struct CartSmem {
  int C, A, PQ, sd, sv, dc, self, total;
};
__host__ __device__ inline CartSmem cart_smem(const DevParams &P, bool staged) {
  CartSmem L;
  const int N = P.n_max, K = P.k_max, L1 = P.l_max + 1;
  int o = 0;
  L.A = o;    o += 8 * K;                // the pair's four angular planes
  L.PQ = o;   o += 4 * N * L1;           // P, Q, Qa, Qo (n, l)
  L.sd = o;   o += 3 * P.n_kept;         // kept components' spherical derivatives
  L.dc = o;   o += 3 * P.n_soap;         // compressed derivatives, then the Cartesian column
  L.C = L.sv = L.self = -1;
  if (staged) {
    o = (o + 1) & ~1;                    // c_nlm is read as double2: an even offset
    L.C = o;    o += 2 * N * K;          // the site's c_nlm
    L.sv = o;   o += P.n_soap;           // the site's unnormalised soap row
    L.self = o; o += 3 * P.n_soap;       // the self column, summed over the pairs
  }
  L.total = o;
  return L;
}

// ---- spherical derivatives, normalisation derivative and Cartesian rotation
// into soap_cart_der (src/soap_turbo.f90:837-895, 1927-2075): one CTA per site,
// which walks the site's pairs in CSR order with the site's c_nlm and soap row
// in shared memory, writes each neighbour column with coalesced stores, and
// sums the self column (minus every other column, :888-892) in shared memory,
// written once at the end.  self_init (may be null): the caller's self
// columns on entry, which the reference's subtraction accumulates into.
template <int NT, bool STAGED>
__global__ void __launch_bounds__(NT) k64_cart_site(const DevParams P, const DevBatch B, const double *rad,
                                                    const double *rad_der, const double2 *ang,
                                                    const double2 *cnk, const double *soap_un,
                                                    const double *norm, const double *self_init,
                                                    double *cart) {
  extern __shared__ double sm[];
  __shared__ double red[3][NT / 32];
  const int site = blockIdx.x;
  const int p0 = B.off[site], p1 = min(B.off[site + 1], B.n_pairs);
  if (p1 <= p0) return;
  const int N = P.n_max, K = P.k_max, L1 = P.l_max + 1, ns = P.n_soap, w3 = 3 * ns;
  const size_t plane = (size_t)B.n_pairs * K;
  const CartSmem Ly = cart_smem(P, STAGED);
  const double2 *c = cnk + (size_t)site * N * K;
  const double *sv_g = soap_un + (size_t)site * ns;
  // without staging, the self column is summed in place in global memory (each
  // element always by the same thread)
  double *sSelf = STAGED ? sm + Ly.self : cart + (size_t)p0 * w3;
  const double2 *sC = STAGED ? (const double2 *)(sm + Ly.C) : c;
  const double *sv = STAGED ? sm + Ly.sv : sv_g;
  double2 *sA = (double2 *)(sm + Ly.A);
  double *sPQ = sm + Ly.PQ, *sd = sm + Ly.sd, *sdc = sm + Ly.dc;
  if (STAGED) {
    for (int t = threadIdx.x; t < N * K; t += NT) ((double2 *)(sm + Ly.C))[t] = c[t];
    for (int o = threadIdx.x; o < ns; o += NT) (sm + Ly.sv)[o] = sv_g[o];
  }
  const double *si = self_init ? self_init + (size_t)site * w3 : nullptr;
  for (int t = threadIdx.x; t < w3; t += NT) sSelf[t] = si ? si[t] : 0.0;
  const double nr = norm[site];
  const double inv_p = 1.0 / nr, inv_p3 = 1.0 / (nr * nr * nr);
  const double *Pp = sPQ, *Q = sPQ + N * L1, *Qa = sPQ + 2 * N * L1, *Qo = sPQ + 3 * N * L1;

  for (int k = p0 + 1; k < p1; ++k) {
    __syncthreads();  // the previous pair's readers of sA, sPQ, sd and sdc are done
    for (int t = threadIdx.x; t < 4 * K; t += NT) {
      const int pl = t / K, kk = t - pl * K;
      sA[t] = ang[pl * plane + (size_t)k * K + kk];
    }
    __syncthreads();
    // P, Q, Qa, Qo(n, l) = sum_m w_m Re(X_lm conj c_nlm) for X = A, dA/dr, dA/dphi, dA/dtheta
    for (int it = threadIdx.x; it < N * L1; it += NT) {
      const int n = it / L1, l = it - n * L1;
      double ap = 0, aq = 0, aa = 0, ao = 0;
      for (int m = 0; m <= l; ++m) {
        const int kk = l * (l + 1) / 2 + m;
        const double w = (m == 0) ? 1.0 : 2.0;
        const double2 cc = sC[n * K + kk];
        const double2 a0 = sA[kk], a1 = sA[K + kk], a2 = sA[2 * K + kk], a3 = sA[3 * K + kk];
        ap = ap + w * (a0.x * cc.x + a0.y * cc.y);
        aq = aq + w * (a1.x * cc.x + a1.y * cc.y);
        aa = aa + w * (a2.x * cc.x + a2.y * cc.y);
        ao = ao + w * (a3.x * cc.x + a3.y * cc.y);
      }
      sPQ[it] = ap;
      sPQ[N * L1 + it] = aq;
      sPQ[2 * N * L1 + it] = aa;
      sPQ[3 * N * L1 + it] = ao;
    }
    __syncthreads();
    const double *R = rad + (size_t)k * N, *Rd = rad_der + (size_t)k * N;
    for (int q = threadIdx.x; q < P.n_kept; q += NT) {
      const int code = P.kept_nnl[q];
      const int n = code & 0xff, np = (code >> 8) & 0xff, l = code >> 16;
      const double pre = kFourPi64 * ((n == np) ? 1.0 : sqrt(2.0));
      const double rn = R[n], rdn = Rd[n], rnp = R[np], rdnp = Rd[np];
      sd[3 * q + 0] = pre * (rdn * Pp[np * L1 + l] + rn * Q[np * L1 + l] + rdnp * Pp[n * L1 + l] + rnp * Q[n * L1 + l]);
      sd[3 * q + 1] = pre * (rn * Qa[np * L1 + l] + rnp * Qa[n * L1 + l]);
      sd[3 * q + 2] = pre * (rn * Qo[np * L1 + l] + rnp * Qo[n * L1 + l]);
    }
    __syncthreads();
    double dr = 0, da = 0, dp = 0;
    for (int o = threadIdx.x; o < ns; o += NT) {
      double vr = 0, va = 0, vp = 0;
      for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) {
        const double el = P.pi_el64[t];
        const int q = P.pi_q[t];
        vr = vr + el * sd[3 * q];
        va = va + el * sd[3 * q + 1];
        vp = vp + el * sd[3 * q + 2];
      }
      sdc[3 * o] = vr;
      sdc[3 * o + 1] = va;
      sdc[3 * o + 2] = vp;
      dr += sv[o] * vr;
      da += sv[o] * va;
      dp += sv[o] * vp;
    }
    cta_sum3<NT>(dr, da, dp, red);
    double st, ct, sf, cf;
    sincos(B.thetas[k], &st, &ct);
    sincos(B.phis[k], &sf, &cf);
    const double ir = 1.0 / B.rjs[k];
    const double cx = st * cf, cy = st * sf, cz = ct;
    const double px = -ct * cf * ir, py = -ct * sf * ir, pz = st * ir;
    const double ax = -sf * ir, ay = cf * ir;
    // each thread turns its own components o into the Cartesian column in place
    for (int o = threadIdx.x; o < ns; o += NT) {
      const double s = sv[o];
      const double vr = sdc[3 * o] * inv_p - s * inv_p3 * dr;
      const double va = sdc[3 * o + 1] * inv_p - s * inv_p3 * da;
      const double vo = sdc[3 * o + 2] * inv_p - s * inv_p3 * dp;
      sdc[3 * o + 0] = cx * vr + px * vo + ax * va;
      sdc[3 * o + 1] = cy * vr + py * vo + ay * va;
      sdc[3 * o + 2] = cz * vr + pz * vo;
    }
    __syncthreads();
    double *out = cart + (size_t)k * w3;
    for (int t = threadIdx.x; t < w3; t += NT) {
      const double v = sdc[t];
      out[t] = v;
      sSelf[t] = sSelf[t] - v;
    }
  }
  if (STAGED) {
    __syncthreads();
    double *out = cart + (size_t)p0 * w3;
    for (int t = threadIdx.x; t < w3; t += NT) out[t] = sSelf[t];
  }
}

// ---- the same, for n_soap <= OPT * NT (OPT = 3): each thread keeps the compressed
// spherical derivatives of its components o = tid, tid + NT, .. in registers,
// formed directly from P, Q, Qa, Qo and the pair's radial values (no kept- or
// output-sized arrays in shared memory), so that three CTAs fit an SM; the
// pair's angles are turned into the rotation once per CTA.  Shared memory: the
// site's c_nlm, soap row and self column, the pair's angular planes, radial
// values and P, Q, Qa, Qo.
struct Cart2Smem {
  int C, sv, self, A, R, PQ, rot, total;
};
__host__ __device__ inline Cart2Smem cart2_smem(const DevParams &P) {
  Cart2Smem L;
  const int N = P.n_max, K = P.k_max, L1 = P.l_max + 1;
  int o = 0;
  L.C = o;    o += 2 * N * K;
  L.sv = o;   o += P.n_soap;
  L.self = o; o += 3 * P.n_soap;
  L.A = o;    o += 8 * K;
  L.R = o;    o += 2 * N;
  L.PQ = o;   o += 4 * N * L1;
  L.rot = o;  o += 8;
  L.total = o;
  return L;
}

template <int NT, int OPT>
__global__ void __launch_bounds__(NT, 3) k64_cart_site2(const DevParams P, const DevBatch B, const double *rad,
                                                     const double *rad_der, const double2 *ang,
                                                     const double2 *cnk, const double *soap_un,
                                                     const double *norm, const double *self_init,
                                                     double *cart) {
  extern __shared__ double sm[];
  __shared__ double red[3][NT / 32];
  const int site = blockIdx.x;
  const int p0 = B.off[site], p1 = min(B.off[site + 1], B.n_pairs);
  if (p1 <= p0) return;
  const int N = P.n_max, K = P.k_max, L1 = P.l_max + 1, ns = P.n_soap, w3 = 3 * ns;
  const size_t plane = (size_t)B.n_pairs * K;
  const Cart2Smem Ly = cart2_smem(P);
  double2 *sC = (double2 *)(sm + Ly.C);
  double2 *sA = (double2 *)(sm + Ly.A);
  double *sv = sm + Ly.sv, *sSelf = sm + Ly.self, *sR = sm + Ly.R, *sPQ = sm + Ly.PQ, *sRot = sm + Ly.rot;
  const double2 *c = cnk + (size_t)site * N * K;
  for (int t = threadIdx.x; t < N * K; t += NT) sC[t] = c[t];
  for (int o = threadIdx.x; o < ns; o += NT) sv[o] = soap_un[(size_t)site * ns + o];
  const double *si = self_init ? self_init + (size_t)site * w3 : nullptr;
  for (int t = threadIdx.x; t < w3; t += NT) sSelf[t] = si ? si[t] : 0.0;
  const double nr = norm[site];
  const double inv_p = 1.0 / nr, inv_p3 = 1.0 / (nr * nr * nr);
  const double *Pp = sPQ, *Q = sPQ + N * L1, *Qa = sPQ + 2 * N * L1, *Qo = sPQ + 3 * N * L1;
  // this thread's kept components (the compression map is one-to-one here or
  // read through its CSR below)
  int code[OPT];
#pragma unroll
  for (int j = 0; j < OPT; ++j) {
    const int o = threadIdx.x + j * NT;
    code[j] = (o < ns && P.cmap_identity) ? P.kept_nnl[o] : 0;
  }

  for (int k = p0 + 1; k < p1; ++k) {
    __syncthreads();  // the previous pair's readers of sA, sR, sPQ and sRot are done
    for (int t = threadIdx.x; t < 4 * K; t += NT) {
      const int pl = t / K, kk = t - pl * K;
      sA[t] = ang[pl * plane + (size_t)k * K + kk];
    }
    for (int t = threadIdx.x; t < 2 * N; t += NT) sR[t] = t < N ? rad[(size_t)k * N + t] : rad_der[(size_t)k * N + t - N];
    if (threadIdx.x == NT - 1) {
      double st, ct, sf, cf;
      sincos(B.thetas[k], &st, &ct);
      sincos(B.phis[k], &sf, &cf);
      const double ir = 1.0 / B.rjs[k];
      sRot[0] = st * cf; sRot[1] = st * sf; sRot[2] = ct;           // cx cy cz
      sRot[3] = -ct * cf * ir; sRot[4] = -ct * sf * ir; sRot[5] = st * ir;  // px py pz
      sRot[6] = -sf * ir; sRot[7] = cf * ir;                        // ax ay
    }
    __syncthreads();
    // P, Q, Qa, Qo(n, l) = sum_m w_m Re(X_lm conj c_nlm) for X = A, dA/dr, dA/dphi, dA/dtheta
    for (int it = threadIdx.x; it < N * L1; it += NT) {
      const int n = it / L1, l = it - n * L1;
      double ap = 0, aq = 0, aa = 0, ao = 0;
      for (int m = 0; m <= l; ++m) {
        const int kk = l * (l + 1) / 2 + m;
        const double w = (m == 0) ? 1.0 : 2.0;
        const double2 cc = sC[n * K + kk];
        const double2 a0 = sA[kk], a1 = sA[K + kk], a2 = sA[2 * K + kk], a3 = sA[3 * K + kk];
        ap = ap + w * (a0.x * cc.x + a0.y * cc.y);
        aq = aq + w * (a1.x * cc.x + a1.y * cc.y);
        aa = aa + w * (a2.x * cc.x + a2.y * cc.y);
        ao = ao + w * (a3.x * cc.x + a3.y * cc.y);
      }
      sPQ[it] = ap;
      sPQ[N * L1 + it] = aq;
      sPQ[2 * N * L1 + it] = aa;
      sPQ[3 * N * L1 + it] = ao;
    }
    __syncthreads();
    // the compressed spherical derivatives of this thread's components (:1999-2066)
    double vr[OPT], va[OPT], vp[OPT];
    double dr = 0, da = 0, dp = 0;
#pragma unroll
    for (int j = 0; j < OPT; ++j) {
      const int o = threadIdx.x + j * NT;
      vr[j] = va[j] = vp[j] = 0.0;
      if (o >= ns) continue;
      if (P.cmap_identity) {
        const int n = code[j] & 0xff, np = (code[j] >> 8) & 0xff, l = code[j] >> 16;
        const double pre = kFourPi64 * ((n == np) ? 1.0 : sqrt(2.0));
        const double rn = sR[n], rdn = sR[N + n], rnp = sR[np], rdnp = sR[N + np];
        vr[j] = pre * (rdn * Pp[np * L1 + l] + rn * Q[np * L1 + l] + rdnp * Pp[n * L1 + l] + rnp * Q[n * L1 + l]);
        va[j] = pre * (rn * Qa[np * L1 + l] + rnp * Qa[n * L1 + l]);
        vp[j] = pre * (rn * Qo[np * L1 + l] + rnp * Qo[n * L1 + l]);
      } else {
        for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) {
          const double el = P.pi_el64[t];
          const int cq = P.kept_nnl[P.pi_q[t]];
          const int n = cq & 0xff, np = (cq >> 8) & 0xff, l = cq >> 16;
          const double pre = kFourPi64 * ((n == np) ? 1.0 : sqrt(2.0));
          const double rn = sR[n], rdn = sR[N + n], rnp = sR[np], rdnp = sR[N + np];
          vr[j] = vr[j] + el * (pre * (rdn * Pp[np * L1 + l] + rn * Q[np * L1 + l] + rdnp * Pp[n * L1 + l] +
                                       rnp * Q[n * L1 + l]));
          va[j] = va[j] + el * (pre * (rn * Qa[np * L1 + l] + rnp * Qa[n * L1 + l]));
          vp[j] = vp[j] + el * (pre * (rn * Qo[np * L1 + l] + rnp * Qo[n * L1 + l]));
        }
      }
      dr += sv[o] * vr[j];
      da += sv[o] * va[j];
      dp += sv[o] * vp[j];
    }
    cta_sum3<NT>(dr, da, dp, red);
    const double cx = sRot[0], cy = sRot[1], cz = sRot[2], px = sRot[3], py = sRot[4], pz = sRot[5];
    const double ax = sRot[6], ay = sRot[7];
    double *out = cart + (size_t)k * w3;
#pragma unroll
    for (int j = 0; j < OPT; ++j) {
      const int o = threadIdx.x + j * NT;
      if (o >= ns) continue;
      const double s = sv[o];
      const double r_ = vr[j] * inv_p - s * inv_p3 * dr;
      const double a_ = va[j] * inv_p - s * inv_p3 * da;
      const double o_ = vp[j] * inv_p - s * inv_p3 * dp;
      const double x = cx * r_ + px * o_ + ax * a_, y = cy * r_ + py * o_ + ay * a_, z = cz * r_ + pz * o_;
      out[3 * o] = x;
      out[3 * o + 1] = y;
      out[3 * o + 2] = z;
      sSelf[3 * o] -= x;
      sSelf[3 * o + 1] -= y;
      sSelf[3 * o + 2] -= z;
    }
  }
  __syncthreads();
  double *out = cart + (size_t)p0 * w3;
  for (int t = threadIdx.x; t < w3; t += NT) out[t] = sSelf[t];
}

// ---- soap_cart_der for n_max <= 32, l_max <= 8, n_soap <= 3 x 256: the CTA
// takes its site's pairs kC3Pairs at a time.
//  * the next batch's angular planes and radial values are copied
//    asynchronously into a second buffer, and its rotations formed, while a
//    batch computes;
//  * P, Q, Qa, Qo: two warps per pair, lane n summing sum_m w_m Re(X_lm conj
//    c_nlm) over every (l, m) for two of the four planes X in registers (the
//    angular values broadcast from shared memory, c_nlm rows padded to 49 so
//    that the lanes' rows fall in distinct banks, the (n, l) rows stored with
//    an odd stride of 9 so that the lanes' stores do too);
//  * the compressed spherical derivatives, the normalisation derivative and the
//    rotation CTA-wide: thread t owns components o = t, t + 256, t + 512 (their
//    (n, n', l) offsets decoded once per site), sums the self column in its
//    registers in pair order, forms the batch's dot products with p (reduced
//    together, in a fixed order), then forms the derivatives again to write the
//    columns (cheaper than holding them: the registers would halve the CTAs
//    per SM).
__device__ __forceinline__ void cp_async_16(void *dst_smem, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_8(void *dst_smem, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
constexpr int kC3Pairs = 4;
constexpr int kC3Kp = 49;  // padded c_nlm row (double2), k_max <= 45
constexpr int kC3L1 = 9;   // P, Q rows of l_max + 1 <= 9 entries
struct Cart3Smem {
  int C, A, PQ, R, sv, rot, red, total;
};
__host__ __device__ inline Cart3Smem cart3_smem(const DevParams &P) {
  Cart3Smem L;
  const int N = P.n_max, K = P.k_max;
  // the double2 arrays first, at even offsets (16-byte aligned), then the doubles
  int o = 0;
  L.C = o;   o += 2 * N * kC3Kp;
  L.A = o;   o += 2 * kC3Pairs * 8 * K;  // two buffers: this batch, the next
  L.PQ = o;  o += kC3Pairs * 4 * N * kC3L1;
  L.R = o;   o += 2 * kC3Pairs * 2 * N;  // two buffers
  L.sv = o;  o += P.n_soap;
  L.rot = o; o += 2 * kC3Pairs * 8;      // two buffers
  L.red = o; o += 8 * 3 * kC3Pairs;
  L.total = o;
  return L;
}

template <int LC>
__global__ void __launch_bounds__(256, 2) k64_cart_site3(const DevParams P, const DevBatch B, const double *rad,
                                                         const double *rad_der, const double2 *ang,
                                                         const double2 *cnk, const double *soap_un,
                                                         const double *norm, const double *self_init,
                                                         double *cart) {
  static_assert(LC + 1 == kC3L1, "P, Q row length");
  static_assert(kC3Pairs * 2 == 256 / 32, "two warps per pair");
  constexpr int NT = 256, OPT = 3, L1 = LC + 1;
  extern __shared__ double sm[];
  const int site = blockIdx.x;
  const int p0 = B.off[site], p1 = min(B.off[site + 1], B.n_pairs);
  if (p1 <= p0) return;
  const int N = P.n_max, K = P.k_max, ns = P.n_soap, w3 = 3 * ns, L = P.l_max;
  const size_t plane = (size_t)B.n_pairs * K;
  const Cart3Smem Ly = cart3_smem(P);
  double2 *sC = (double2 *)(sm + Ly.C);
  double2 *sA = (double2 *)(sm + Ly.A);
  double *sPQ = sm + Ly.PQ, *sR = sm + Ly.R, *sv = sm + Ly.sv, *sRot = sm + Ly.rot, *sRed = sm + Ly.red;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double2 *c = cnk + (size_t)site * N * K;
  for (int t = tid; t < N * K; t += NT) {
    const int n = t / K, kk = t - n * K;
    sC[n * kC3Kp + kk] = c[t];
  }
  for (int o = tid; o < ns; o += NT) sv[o] = soap_un[(size_t)site * ns + o];
  const double nr = norm[site];
  const double inv_p = 1.0 / nr, inv_p3 = 1.0 / (nr * nr * nr);
  // this thread's components: offsets of (n, l) and (n', l) in a pair's P, Q
  // rows, and the multiplicity prefactor (identity compression map)
  int ia[OPT], ib[OPT];
  double pre[OPT], self_[OPT][3];
  const double *si = self_init ? self_init + (size_t)site * w3 : nullptr;
#pragma unroll
  for (int j = 0; j < OPT; ++j) {
    const int o = tid + j * NT;
    const int code = (o < ns && P.cmap_identity) ? P.kept_nnl[o] : 0;
    const int n = code & 0xff, np = (code >> 8) & 0xff, l = code >> 16;
    ia[j] = n * L1 + l;
    ib[j] = np * L1 + l;
    pre[j] = kFourPi64 * ((n == np) ? 1.0 : sqrt(2.0));
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) self_[j][cc] = (o < ns && si) ? si[3 * o + cc] : 0.0;
  }
  const int NL = N * L1;
  const double *cR = sR;  // the current batch's radial values (set per batch)
  // the derivatives of component (n, n', l) of pair q; a_, b_ = n L1 + l, n' L1 + l
  auto deriv1 = [&](int q, int a_, int b_, double pf, double &vr, double &va, double &vp) {
    const double *Pp = sPQ + (size_t)(q * 4) * NL, *Q = Pp + NL, *Qa = Q + NL, *Qo = Qa + NL;
    const double *R = cR + q * 2 * N;
    const int n = a_ / L1, np = b_ / L1;
    const double rn = R[n], rdn = R[N + n], rnp = R[np], rdnp = R[N + np];
    vr = pf * (rdn * Pp[b_] + rn * Q[b_] + rdnp * Pp[a_] + rnp * Q[a_]);
    va = pf * (rn * Qa[b_] + rnp * Qa[a_]);
    vp = pf * (rn * Qo[b_] + rnp * Qo[a_]);
  };
  auto deriv = [&](int q, int j, double &vr, double &va, double &vp) {
    if (P.cmap_identity) {
      deriv1(q, ia[j], ib[j], pre[j], vr, va, vp);
      return;
    }
    const int o = tid + j * NT;
    vr = va = vp = 0.0;
    for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) {
      const double el = P.pi_el64[t];
      const int cq = P.kept_nnl[P.pi_q[t]];
      const int n = cq & 0xff, np = (cq >> 8) & 0xff, l = cq >> 16;
      double r_, a_, p_;
      deriv1(q, n * L1 + l, np * L1 + l, kFourPi64 * ((n == np) ? 1.0 : sqrt(2.0)), r_, a_, p_);
      vr = vr + el * r_;
      va = va + el * a_;
      vp = vp + el * p_;
    }
  };

  const int szA = kC3Pairs * 4 * K, szR = kC3Pairs * 2 * N;
  // a batch's angular planes and radial values, copied asynchronously into
  // buffer b while the previous batch computes, and its rotations (FP64
  // sincos), formed by the CTA's last kC3Pairs threads during that batch
  auto stage = [&](int b, int kb_) {
    const int nb_ = min(kC3Pairs, p1 - kb_);
    double2 *dA = sA + b * szA;
    double *dR = sR + b * szR;
    for (int t = tid; t < nb_ * 4 * K; t += NT) {
      const int q = t / (4 * K), r = t - q * 4 * K, pl = r / K, kk = r - pl * K;
      cp_async_16(dA + (q * 4 + pl) * K + kk, ang + pl * plane + (size_t)(kb_ + q) * K + kk);
    }
    for (int t = tid; t < nb_ * 2 * N; t += NT) {
      const int q = t / (2 * N), r = t - q * 2 * N;
      cp_async_8(dR + t, r < N ? rad + (size_t)(kb_ + q) * N + r : rad_der + (size_t)(kb_ + q) * N + r - N);
    }
    cp_async_commit();
  };
  auto rotation = [&](int b, int kb_) {
    const int j = tid - (NT - kC3Pairs);
    if (j >= 0 && j < min(kC3Pairs, p1 - kb_)) {
      const int k = kb_ + j;
      double st, ct, sf, cf;
      sincos(B.thetas[k], &st, &ct);
      sincos(B.phis[k], &sf, &cf);
      const double ir = 1.0 / B.rjs[k];
      double *rt = sRot + b * kC3Pairs * 8 + 8 * j;
      rt[0] = st * cf; rt[1] = st * sf; rt[2] = ct;
      rt[3] = -ct * cf * ir; rt[4] = -ct * sf * ir; rt[5] = st * ir;
      rt[6] = -sf * ir; rt[7] = cf * ir;
    }
  };
  if (p0 + 1 < p1) {
    stage(0, p0 + 1);
    rotation(0, p0 + 1);
  }

  int buf = 0;
  for (int kb = p0 + 1; kb < p1; kb += kC3Pairs, buf ^= 1) {
    const int nb = min(kC3Pairs, p1 - kb);
    __syncthreads();  // the previous batch's readers are done, buffer buf ^ 1 is free
    const bool more = kb + kC3Pairs < p1;
    if (more) {
      stage(buf ^ 1, kb + kC3Pairs);
      cp_async_wait_1();
    } else {
      cp_async_wait_0();
    }
    __syncthreads();
    const double2 *cA = sA + buf * szA;
    cR = sR + buf * szR;
    const double *cRot = sRot + buf * kC3Pairs * 8;
    // ---- P, Q, Qa, Qo: warp 2q + h, lane n: planes 2h, 2h + 1 of pair q
    {
      const int q = warp >> 1, h = warp & 1, n = lane;
      if (q < nb && n < N) {
        const double2 *A0 = cA + (q * 4 + 2 * h) * K, *A1 = A0 + K;
        const double2 *cn = sC + n * kC3Kp;
        double *o0 = sPQ + (size_t)(q * 4 + 2 * h) * NL + n * L1, *o1 = o0 + NL;
#pragma unroll
        for (int l = 0; l <= LC; ++l) {
          double s0 = 0.0, s1 = 0.0;
          if (l <= L) {
#pragma unroll
            for (int m = 0; m <= l; ++m) {
              const int kk = l * (l + 1) / 2 + m;
              const double w = (m == 0) ? 1.0 : 2.0;
              const double2 cc = cn[kk], a0 = A0[kk], a1 = A1[kk];
              s0 = s0 + w * (a0.x * cc.x + a0.y * cc.y);
              s1 = s1 + w * (a1.x * cc.x + a1.y * cc.y);
            }
          }
          o0[l] = s0;
          o1[l] = s1;
        }
      }
    }
    __syncthreads();
    // ---- the compressed spherical derivatives (:1999-2066): pass 1, each
    // pair's dots with p, reduced in a fixed order (warp shuffles, then the
    // eight warps in order)
#pragma unroll 1
    for (int q = 0; q < nb; ++q) {
      double d0 = 0.0, d1 = 0.0, d2 = 0.0;
#pragma unroll
      for (int j = 0; j < OPT; ++j) {
        const int o = tid + j * NT;
        if (o >= ns) continue;
        double vr, va, vp;
        deriv(q, j, vr, va, vp);
        d0 += sv[o] * vr;
        d1 += sv[o] * va;
        d2 += sv[o] * vp;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        d0 += __shfl_xor_sync(0xffffffffu, d0, off);
        d1 += __shfl_xor_sync(0xffffffffu, d1, off);
        d2 += __shfl_xor_sync(0xffffffffu, d2, off);
      }
      if (lane == 0) {
        sRed[(q * 3 + 0) * 8 + warp] = d0;
        sRed[(q * 3 + 1) * 8 + warp] = d1;
        sRed[(q * 3 + 2) * 8 + warp] = d2;
      }
    }
    if (more) rotation(buf ^ 1, kb + kC3Pairs);
    __syncthreads();
    // ---- pass 2: the Cartesian columns, and the self column in registers
#pragma unroll 1
    for (int q = 0; q < nb; ++q) {
      double dr = 0.0, da = 0.0, dp = 0.0;
#pragma unroll
      for (int w = 0; w < NT / 32; ++w) {
        dr += sRed[(q * 3 + 0) * 8 + w];
        da += sRed[(q * 3 + 1) * 8 + w];
        dp += sRed[(q * 3 + 2) * 8 + w];
      }
      const double *rt = cRot + 8 * q;
      const double cx = rt[0], cy = rt[1], cz = rt[2], px = rt[3], py = rt[4], pz = rt[5], ax = rt[6], ay = rt[7];
      double *out = cart + (size_t)(kb + q) * w3;
#pragma unroll
      for (int j = 0; j < OPT; ++j) {
        const int o = tid + j * NT;
        if (o >= ns) continue;
        double vr, va, vp;
        deriv(q, j, vr, va, vp);
        const double s = sv[o];
        const double r_ = vr * inv_p - s * inv_p3 * dr;
        const double a_ = va * inv_p - s * inv_p3 * da;
        const double o_ = vp * inv_p - s * inv_p3 * dp;
        const double x = cx * r_ + px * o_ + ax * a_, y = cy * r_ + py * o_ + ay * a_, z = cz * r_ + pz * o_;
        out[3 * o] = x;
        out[3 * o + 1] = y;
        out[3 * o + 2] = z;
        self_[j][0] -= x;
        self_[j][1] -= y;
        self_[j][2] -= z;
      }
    }
  }
  double *out = cart + (size_t)p0 * w3;
#pragma unroll
  for (int j = 0; j < OPT; ++j) {
    const int o = tid + j * NT;
    if (o < ns) {
      out[3 * o] = self_[j][0];
      out[3 * o + 1] = self_[j][1];
      out[3 * o + 2] = self_[j][2];
    }
  }
}

// ---- pair = sgn * sum_s G(i,s) soap_cart_der(:, s, k): one CTA per site with
// the site's G row in shared memory, one warp per pair; lane j takes the
// components o = j, j + 32, ... (a warp's three loads of a step cover 768
// contiguous bytes of the column).
template <int NT>
__global__ void __launch_bounds__(NT) k64_contract_site(const DevParams P, const DevBatch B, const double *cart,
                                                        const double *G, int g_layout, double sgn,
                                                        double *pair) {
  extern __shared__ double sG[];  // n_soap
  const int site = blockIdx.x;
  const int p0 = B.off[site], p1 = min(B.off[site + 1], B.n_pairs);
  const int ns = P.n_soap;
  for (int o = threadIdx.x; o < ns; o += NT)
    sG[o] = g_layout == 0 ? G[(size_t)o * B.n_sites + site] : G[(size_t)site * ns + o];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = p0 + warp; k < p1; k += NT / 32) {
    const double *ck = cart + (size_t)k * 3 * ns;
    double x = 0.0, y = 0.0, z = 0.0;
    for (int o = lane; o < ns; o += 32) {
      const double g = sG[o];
      x += g * ck[3 * o];
      y += g * ck[3 * o + 1];
      z += g * ck[3 * o + 2];
    }
    for (int s = 16; s > 0; s >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, s);
      y += __shfl_xor_sync(0xffffffffu, y, s);
      z += __shfl_xor_sync(0xffffffffu, z, s);
    }
    if (lane == 0) {
      pair[3 * (size_t)k] = sgn * x;
      pair[3 * (size_t)k + 1] = sgn * y;
      pair[3 * (size_t)k + 2] = sgn * z;
    }
  }
}

__global__ void k64_normalise(const DevParams P, const DevBatch B, const double *soap_un,
                              const double *norm, double *soap) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n = (size_t)B.n_sites * P.n_soap;
  if (t >= n) return;
  soap[t] = soap_un[t] / norm[t / P.n_soap];
}

static int max_alpha64(const DevParams &P) {
  int a = 0;
  for (int s = 0; s < P.n_species; ++s) a = a > P.rad[s].alpha ? a : P.rad[s].alpha;
  return a;
}

constexpr int kCartThreads = 256;

// The staged layout when it fits in a CTA's shared memory (227 KB on B200).
constexpr size_t kCartSmemCap = 227 * 1024;
size_t fp64_cart_smem(const DevParams &P) {
  const size_t staged = (size_t)cart_smem(P, true).total * sizeof(double);
  return staged <= kCartSmemCap ? staged : (size_t)cart_smem(P, false).total * sizeof(double);
}

cudaError_t launch_fp64_descriptor(const DevParams &P, const DevBatch &B, cudaStream_t s,
                                   const Fp64Work &w, int do_der, double *soap, double *cart,
                                   int *launches, const double *soap_acc, const double *self_init) {
  const int np = B.n_pairs, nsites = B.n_sites;
  int nl = 0;
  if (np > 0) {
    const int blocks = (np + 127) / 128;
    const bool op = P.basis == kBasisOperator;
    if (max_alpha64(P) <= 8) {
      if (op) k64_radial<8, true><<<blocks, 128, 0, s>>>(P, B, do_der, w.rad, w.rad_der);
      else k64_radial<8, false><<<blocks, 128, 0, s>>>(P, B, do_der, w.rad, w.rad_der);
    } else {
      if (op) k64_radial<16, true><<<blocks, 128, 0, s>>>(P, B, do_der, w.rad, w.rad_der);
      else k64_radial<16, false><<<blocks, 128, 0, s>>>(P, B, do_der, w.rad, w.rad_der);
    }
    if (P.l_max <= 8) k64_angular2<8><<<(np + 31) / 32, do_der ? 128 : 32, 0, s>>>(P, B, do_der, (double2 *)w.ang);
    else k64_angular<12><<<blocks, 128, 0, s>>>(P, B, do_der, (double2 *)w.ang);
    nl += 2;
  }
  if (nsites > 0) {
    if (P.n_max * P.k_max <= 8 * 256) {
      const size_t smc = (size_t)kCnkChunk * (P.n_max + 2 * P.k_max) * sizeof(double);
      cudaFuncSetAttribute(k64_cnk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc);
      k64_cnk<<<nsites, 256, smc, s>>>(P, B, w.rad, (const double2 *)w.ang, (double2 *)w.cnk);
    } else {
      k64_cnk_wide<<<nsites, 256, 0, s>>>(P, B, w.rad, (const double2 *)w.ang, (double2 *)w.cnk);
    }
    const size_t sm = (size_t)P.n_kept * sizeof(double);
    cudaFuncSetAttribute(k64_soap, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k64_soap<<<nsites, 256, sm, s>>>(P, B, (const double2 *)w.cnk, soap_acc, w.soap_unnorm, w.norm);
    nl += 2;
  }
  if (do_der && cart && np > 0 && nsites > 0) {
    const size_t sm2 = (size_t)cart2_smem(P).total * sizeof(double);
    const size_t sm3 = (size_t)cart3_smem(P).total * sizeof(double);
    if (P.n_max <= 32 && P.l_max <= 8 && P.n_soap <= 3 * 256 && sm3 <= kCartSmemCap) {
      auto kern = k64_cart_site3<8>;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm3);
      if (e != cudaSuccess) return e;
      kern<<<nsites, 256, sm3, s>>>(P, B, w.rad, w.rad_der, (const double2 *)w.ang, (const double2 *)w.cnk,
                                    w.soap_unnorm, w.norm, self_init, cart);
    } else if (P.n_soap <= 3 * kCartThreads && sm2 <= kCartSmemCap) {
      auto kern = k64_cart_site2<kCartThreads, 3>;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
      if (e != cudaSuccess) return e;
      kern<<<nsites, kCartThreads, sm2, s>>>(P, B, w.rad, w.rad_der, (const double2 *)w.ang,
                                             (const double2 *)w.cnk, w.soap_unnorm, w.norm, self_init, cart);
    } else {
      const size_t sm = fp64_cart_smem(P);
      const bool staged = sm == (size_t)cart_smem(P, true).total * sizeof(double);
      auto kern = staged ? k64_cart_site<kCartThreads, true> : k64_cart_site<kCartThreads, false>;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      if (e != cudaSuccess) return e;
      kern<<<nsites, kCartThreads, sm, s>>>(P, B, w.rad, w.rad_der, (const double2 *)w.ang,
                                            (const double2 *)w.cnk, w.soap_unnorm, w.norm, self_init, cart);
    }
    nl += 1;
  }
  if (nsites > 0) {
    const size_t n = (size_t)nsites * P.n_soap;
    k64_normalise<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, B, w.soap_unnorm, w.norm, soap);
    nl += 1;
  }
  if (launches) *launches += nl;
  return cudaGetLastError();
}

cudaError_t launch_fp64_contract(const DevParams &P, const DevBatch &B, cudaStream_t s,
                                 const double *cart, const double *G, int g_layout, double sgn,
                                 double *pair, int *launches) {
  if (B.n_pairs <= 0 || B.n_sites <= 0) return cudaSuccess;
  const size_t sm = (size_t)P.n_soap * sizeof(double);
  auto kern = k64_contract_site<256>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  kern<<<B.n_sites, 256, sm, s>>>(P, B, cart, G, g_layout, sgn, pair);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

}  // namespace soapb
