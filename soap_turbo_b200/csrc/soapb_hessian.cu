// soapb_hessian.cu -- the central-atom Hessian of soap_turbo
// (get_soap_central_hessian, src/soap_turbo.f90:1151-1700) in FP64:
//
//   hess(a, b, v, k2) = sum_d vecs(d, v, i) d^2 q_d / dr_ia dr_jb
//
// for every pair k2 = (site i, neighbour j), a of the central atom and b of
// the neighbour, the self pair's block being minus the sum of the others.
//
// k64_radial_d2 adds the second radial derivatives to the plain FP64 path's
// state (src/soap_turbo_radial.f90:838-861, 895-905, 917-956; unified filter
// seed only); k64_hgeo writes one geometry record per pair (pair_geometry,
// src/soap_turbo.f90:1537-1652); k64_hess is persistent, one CTA per site at a
// time, and follows the reference's two passes around the weight vectors' S
// matrices (see the kernel).  The angular factor Omega = C_k Q_l^m(t) w^m and
// its Cartesian gradient and Hessian are rebuilt from the record where needed
// (Q_l^m = d^m P_l / dt^m, w = (x - iy)/r), as the reference does.  Every sum
// runs in a fixed order, so results repeat bit for bit.
#include "soapb_device.cuh"

namespace soapb {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kHessThreads = 128;
constexpr int kHessS = 26;  // k-sums per weight vector in pass B
constexpr int kHessPC = 8;  // pairs per chunk of pass A
constexpr int kHessRed = kHessS + 1;  // row stride of the per-warp transpose buffer

#define CU_RET(x)                         \
  do {                                    \
    const cudaError_t e_ = (x);           \
    if (e_ != cudaSuccess) return e_;     \
  } while (0)

struct dcx {
  double re, im;
};
__device__ __forceinline__ dcx cx(double r, double i) { return dcx{r, i}; }
__device__ __forceinline__ dcx operator+(dcx a, dcx b) { return cx(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ dcx operator-(dcx a, dcx b) { return cx(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ dcx operator*(dcx a, dcx b) {
  return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ dcx operator*(double s, dcx a) { return cx(s * a.re, s * a.im); }

__device__ __forceinline__ double nv_tab(int n) { return n == -3 ? 1.0 : sqrt(1.0 / (double)(2 * n + 5)); }

// One (pair, species) radial expansion with its first and second r
// derivatives (process_block, src/soap_turbo_radial.f90:550-1002, unified
// seed), the polynomials kept whole to alpha + 4 as the reference does.
template <int AMAX>
__device__ void radial_pair_d2(const DevParams &P, const RadSp &S, const double *W, double r_in, bool is_central,
                               double *val, double *der, double *der2) {
  const double sqpi2 = 1.2533141373155002512, isq2 = 0.70710678118654752440;
  const double sq2pi = 0.79788456080286535588, sq8pi = 1.5957691216057307118;
  constexpr int NT = AMAX + 8;
  const int a = S.alpha, n_poly = S.n_poly, n_hi = n_poly + 4;
  const double c = S.c, rs = S.rs, dr = S.dr;
  const double rj = r_in * S.inv_rcut;
  double T1[NT], T2[NT], pol[NT], DT[NT], D2T[NT];  // index n + 3
#pragma unroll
  for (int t = 0; t < NT; ++t) T1[t] = T2[t] = pol[t] = DT[t] = D2T[t] = 0.0;
  const double sig = S.atom_sigma + c * rj, s2 = sig * sig;              // :560-570
  const double isig = 1.0 / sig, is2 = isig * isig, is3 = is2 * isig;
  double amp, ampd, ampd2;                                               // :589-635
  if (!P.scaling_poly) {
    amp = 1.0; ampd = 0.0; ampd2 = 0.0;
  } else if (S.amp_scaling == 0.0) {
    amp = isig; ampd = -c * is2; ampd2 = 2.0 * c * c * is3;
  } else if (S.amp_scaling == 1.0) {
    const double h = 1.0 + 2.0 * (rj * rj * rj) - 3.0 * rj * rj;
    const double hp = 6.0 * rj * rj - 6.0 * rj, hpp = 12.0 * rj - 6.0, g = isig * h;
    amp = (h <= 1.0e-10) ? 0.0 : g;
    ampd = (h <= 1.0e-10) ? 0.0 : hp * isig - c * isig * g;
    ampd2 = (h <= 1.0e-10) ? 0.0 : hpp * isig - 2.0 * c * hp * is2 + 2.0 * c * c * h * is3;
  } else {
    const double h = 1.0 + 2.0 * (rj * rj * rj) - 3.0 * rj * rj;
    if (h <= 1.0e-10) {
      amp = 0.0; ampd = 0.0; ampd2 = 0.0;
    } else {
      const double hp = 6.0 * rj * rj - 6.0 * rj, hpp = 12.0 * rj - 6.0, aa = S.amp_scaling;
      amp = isig * pow(h, aa);
      ampd = aa * pow(h, aa - 1.0) * hp * isig - c * isig * amp;
      ampd2 = (aa * (aa - 1.0) * pow(h, aa - 2.0) * hp * hp + aa * pow(h, aa - 1.0) * hpp) * isig -
              2.0 * c * aa * pow(h, aa - 1.0) * hp * is2 + 2.0 * c * c * pow(h, aa) * is3;
    }
  }
  if (S.do_central && S.cw != 1.0 && is_central) {                       // :638-646
    amp *= S.cw; ampd *= S.cw; ampd2 *= S.cw;
  }
  if (P.radial_enh == 1) {                                               // :651-670
    const double g = rj + sq2pi * sig, f = 1.0 + sq2pi * c;
    ampd2 = ampd2 * g + 2.0 * ampd * f;
    ampd = amp * f + ampd * g;
    amp = amp * g;
  } else if (P.radial_enh == 2) {
    const double g = rj * rj + s2 + sq8pi * sig * rj;
    const double f = 2.0 * rj + 2.0 * sig * c + sq8pi * sig + sq8pi * rj * c;
    const double h = 2.0 + 2.0 * c * c + 2.0 * sq8pi * c;
    ampd2 = ampd2 * g + 2.0 * ampd * f + amp * h;
    ampd = amp * f + ampd * g;
    amp = amp * g;
  }
  // inner overlap on [0, rcut_soft] (:676-698)
  const double es = exp(-0.5 * (rs - rj) * (rs - rj) * is2), e0 = exp(-0.5 * rj * rj * is2);
  double C1 = s2 * es;
  const double C2 = s2 * e0;
  T1[0] = 0.0;
  T1[1] = sqpi2 * sig * (erf((rs - rj) * isq2 * isig) + erf(rj * isq2 * isig));
  for (int n = -1; n <= n_hi; ++n) {
    if (n >= 0) C1 = C1 * dr;
    const double ra = n == -1 ? 0.0 : (double)(n + 1) * nv_tab(n - 2) / nv_tab(n);
    T1[n + 3] = s2 * ra * T1[n + 1] - nv_tab(n - 1) / nv_tab(n) * (rj - 1.0) * T1[n + 2] +
                (C1 - C2) * (1.0 / nv_tab(n));
  }
  double pref = 0.0;
  if (S.has_filter) {                                                    // :721-795
    const double q = S.q, drnf = S.drnf;
    const double iD = 1.0 / (s2 + q), sqiD = sqrt(iD);
    const double sgf = sig * drnf * sqiD, rjf = (s2 * rs + q * rj) * iD, sf2 = sgf * sgf;
    const bool keep = (rs - rj) < 4.0 * sig;
    const double isgf = 1.0 / sgf, isf2 = isgf * isgf;
    pref = keep ? exp(-0.5 * (rs - rj) * (rs - rj) * iD) : 0.0;
    double C2f = sf2 * exp(-0.5 * (rs - rjf) * (rs - rjf) * isf2);
    T2[0] = 0.0;
    T2[1] = sqpi2 * sgf * (erf((1.0 - rjf) * isq2 * isgf) - erf((rs - rjf) * isq2 * isgf));
    for (int n = -1; n <= n_hi; ++n) {
      if (n >= 0) C2f = C2f * dr;
      const double ra = n == -1 ? 0.0 : (double)(n + 1) * nv_tab(n - 2) / nv_tab(n);
      T2[n + 3] = sf2 * ra * T2[n + 1] - nv_tab(n - 1) / nv_tab(n) * (rjf - 1.0) * T2[n + 2] -
                  C2f * (1.0 / nv_tab(n));
      if (n == -1) T2[2] = T2[2] + sf2 * exp(-0.5 * (1.0 - rjf) * (1.0 - rjf) * isf2) * (1.0 / nv_tab(-1));
    }
  }
  for (int n = 1; n <= n_hi; ++n) pol[n + 3] = T1[n + 3] + pref * T2[n + 3];  // :808-812
  {                                                                      // :825-861
    const double f = 1.0 - rj;
    const double g0 = f * is2 + c * f * f * is3, g1 = -(is2 + 2.0 * c * f * is3), g2 = c * is3;
    const double is4 = is2 * is2, is5 = is4 * isig, is6 = is4 * is2;
    const double k0 = -is2, k1 = -4.0 * c * is3, k2 = (1.0 - 3.0 * c * c) * is4, k3 = 2.0 * c * is5,
                 k4 = c * c * is6;
    const double B0 = k0 + k1 * f + k2 * f * f + k3 * f * f * f + k4 * f * f * f * f;
    const double B1 = -(k1 + 2.0 * k2 * f + 3.0 * k3 * f * f + 4.0 * k4 * f * f * f);
    const double B2 = k2 + 3.0 * k3 * f + 6.0 * k4 * f * f, B3 = -(k3 + 4.0 * k4 * f), B4 = k4;
    for (int n = 1; n <= n_poly; ++n) {
      const double R1 = nv_tab(n + 1) / nv_tab(n), R2 = nv_tab(n + 2) / nv_tab(n);
      const double R3 = nv_tab(n + 3) / nv_tab(n), R4 = nv_tab(n + 4) / nv_tab(n);
      DT[n + 3] = g0 * pol[n + 3] + R1 * g1 * pol[n + 4] + R2 * g2 * pol[n + 5];
      D2T[n + 3] = B0 * pol[n + 3] + R1 * B1 * pol[n + 4] + R2 * B2 * pol[n + 5] + R3 * B3 * pol[n + 6] +
                   R4 * B4 * pol[n + 7];
    }
  }
  if (P.basis == 1) {                                                    // :875-908
    const double ss2 = S.sigma_sq0 + s2, iss = 1.0 / ss2, siss = sqrt(iss);
    const bool gm = rj < 4.0 * (S.atom_sigma + sig);
    const double ge = gm ? S.N_gauss * e0 : 0.0;
    const double M0 = gm ? exp(-0.5 * rj * rj * iss) * sqpi2 * sig * S.atom_sigma * siss *
                               (1.0 + erf(S.atom_sigma * isig * rj * isq2 * siss)) * S.N_gauss
                         : 0.0;
    pol[a + 3] = M0;
    const double sc0 = S.sigma_sq0 * s2 * iss, pp = s2 * rj * iss;
    const double M1 = sc0 * ge - pp * M0, M2 = sc0 * ge * (-rj) - pp * M1 + sc0 * M0;
    const double M3 = sc0 * ge * rj * rj - pp * M2 + 2.0 * sc0 * M1;
    const double M4 = sc0 * ge * (-rj * rj * rj) - pp * M3 + 3.0 * sc0 * M2;
    const double is4 = is2 * is2, is5 = is4 * isig, is6 = is4 * is2;
    DT[a + 3] = M1 * is2 + c * M2 * is3;
    D2T[a + 3] = -M0 * is2 - 4.0 * c * M1 * is3 + (1.0 - 3.0 * c * c) * M2 * is4 + 2.0 * c * M3 * is5 +
                 c * c * M4 * is6;
  }
  // transform from g_alpha to g_n (:911-976)
  for (int i = 0; i < a; ++i) {
    double v = 0.0, d = 0.0, d2 = 0.0;
    for (int m = 1; m <= a; ++m) {
      const double w = W[(m - 1) * a + i];
      v = v + w * pol[m + 3];
      d = d + w * (amp * DT[m + 3] + ampd * pol[m + 3]);
      d2 = d2 + w * (amp * D2T[m + 3] + 2.0 * ampd * DT[m + 3] + ampd2 * pol[m + 3]);
    }
    val[i] = amp * v * S.sqrt_rcut;
    der[i] = d * S.inv_sqrt_rcut;
    der2[i] = d2 * S.inv_sqrt_rcut * S.inv_rcut;
  }
}

// ---- second radial derivatives, one thread per pair; the values and first
// derivatives the FP64 descriptor path already holds are left as they are
template <int AMAX>
__global__ void k64_radial_d2(const DevParams P, const DevBatch B, double *rad_der2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= B.n_pairs) return;
  int lo = 0, hi = B.n_sites;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (B.off[mid] <= k) lo = mid; else hi = mid;
  }
  const bool is_self = (B.off[lo] == k);
  const double r = B.rjs[k];
  const unsigned bits = B.bits[k];
  double *r2o = rad_der2 + (size_t)k * P.n_max;
  for (int s = 0; s < P.n_species; ++s) {
    const RadSp &S = P.rad[s];
    const bool ok = ((bits >> s) & 1u) && r < S.rcut_hard && (!is_self || S.do_central);
    if (!ok) {
      for (int n = 0; n < S.alpha; ++n) r2o[S.nbeg + n] = 0.0;
      continue;
    }
    double val[AMAX], der[AMAX], der2[AMAX];
    radial_pair_d2<AMAX>(P, S, P.Wblk + (size_t)s * P.wstride, r, is_self, val, der, der2);
    for (int n = 0; n < S.alpha; ++n) r2o[S.nbeg + n] = der2[n] * S.gscale;
  }
}

// Per-pair record of the Hessian (pair_geometry, src/soap_turbo.f90:1537-1652),
// written once by k64_hgeo and read by k64_hess: offsets in doubles.
struct GeoLayout {
  int nh, invr, F, F1, F2, t, th, w, wh, Q, wp, size;
  __host__ __device__ explicit GeoLayout(int L) {
    const int L1 = L + 1, K = L1 * (L1 + 1) / 2;
    nh = 0;
    invr = 3;
    F = 4;
    F1 = F + L1;
    F2 = F1 + L1;
    t = F2 + L1;
    th = t + 3;
    w = th + 9;   // 3 complex
    wh = w + 6;   // 9 complex
    Q = wh + 18;  // K: Q_l^m(t) = d^m P_l / dt^m
    wp = Q + K;   // L + 3 complex: w^m at m + 2, w^-2 = w^-1 = 0
    size = wp + 2 * (L + 3);
    size += size & 1;
  }
};

__device__ __forceinline__ dcx ldc(const double *p) { return cx(p[0], p[1]); }
__device__ __forceinline__ void stc(double *p, dcx v) {
  p[0] = v.re;
  p[1] = v.im;
}

__device__ __forceinline__ int l_of_k(int k) {
  int l = 0;
  while ((l + 1) * (l + 2) / 2 <= k) ++l;
  return l;
}

// get_ilexp (src/soap_turbo_angular.f90:361-422) to lmax, for the F_l of the Hessian
__device__ void ilexp_to(int lmax, double x, double *out) {
  const double xcut = 1.0e-7, x2 = x * x, x4 = x2 * x2, inv_x2 = (x2 > 0.0) ? 1.0 / x2 : 0.0;
  double x2pow = x2 * x2, flm2, flm1, fact = 1.0;
  if (x > 0.0) {
    const double e2 = exp(-2.0 * x2);
    flm2 = fabs((1.0 - e2) / 2.0 / x2);
    flm1 = fabs((x2 - 1.0 + e2 * (x2 + 1.0)) / 2.0 / x4);
  } else {
    flm2 = 1.0;
    flm1 = 0.0;
  }
  for (int l = 0; l <= lmax; ++l) {
    if (l > 0) fact = fact * (2.0 * (double)l + 1.0);
    if (l == 0) {
      out[0] = (x < xcut) ? 1.0 - x2 : flm2;
    } else if (l == 1) {
      out[1] = (x2 / 1000.0 < xcut) ? (x2 - x4) / fact : flm1;
    } else {
      const double ratio = x2pow / fact;
      const double fl = (ratio * (double)l < xcut) ? ratio : fabs(flm2 - (2.0 * (double)l - 1.0) * inv_x2 * flm1);
      x2pow = x2pow * x2;
      flm2 = flm1;
      flm1 = fl;
      out[l] = fl;
    }
  }
}

// ---- pair geometry, one thread per pair: F_l and its first two r-derivatives,
// the unit vector, the gradients and Hessians of t = cos(theta) and
// w = (x - iy)/r, Q_l^m(t) and w^m.  good[k] = 0 for pairs the Hessian skips
// (beyond rcut_max, at the origin, or in no species).
__global__ void k64_hgeo(const DevParams P, const DevBatch B, double *geo, int *good) {
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  if (kk >= B.n_pairs) return;
  const int L = P.l_max;
  const GeoLayout Lg(L);
  double *g = geo + (size_t)kk * Lg.size;
  const double rr = B.rjs[kk];
  const unsigned bits = B.bits[kk];
  const bool ok = rr < P.rcut_max && rr >= 1.0e-10 && bits != 0u;
  good[kk] = ok ? 1 : 0;
  if (!ok) return;
  const int isp = __ffs(bits) - 1;
  const double invr = 1.0 / rr, invr2 = invr * invr;
  g[Lg.invr] = invr;
  const double sscal = P.sig_t_c[isp], sig = P.sig_t[isp] + sscal * rr;
  const double amp = P.rcut2 / (sig * sig), ampd = -2.0 * sscal / sig * amp;
  const double ampdd = 6.0 * sscal * sscal / (sig * sig) * amp;
  const double xarg = rr / sig, invz = 1.0 / (xarg * xarg);
  double il[SOAPB_MAX_LMAX + 3];
  ilexp_to(L + 2, xarg, il);
  const double zp = 2.0 * rr / (sig * sig) - 2.0 * rr * rr * sscal / (sig * sig * sig);
  const double zp2 = 2.0 / (sig * sig) - 8.0 * rr * sscal / (sig * sig * sig) +
                     6.0 * rr * rr * sscal * sscal / (sig * sig * sig * sig);
  for (int l = 0; l <= L; ++l) {
    const double rl = (double)l;
    const double dil = il[l + 1] + (rl * invz - 1.0) * il[l];
    const double d2il = il[l + 2] + ((double)(2 * l + 1) * invz - 2.0) * il[l + 1] +
                        (rl * (rl - 1.0) * invz * invz - 2.0 * rl * invz + 1.0) * il[l];
    const double f0 = il[l], f1 = dil * zp, f2 = d2il * zp * zp + dil * zp2;
    g[Lg.F + l] = amp * f0;
    g[Lg.F1 + l] = ampd * f0 + amp * f1;
    g[Lg.F2 + l] = ampdd * f0 + 2.0 * ampd * f1 + amp * f2;
  }
  double nh[3];
  const double sin_t = sin(B.thetas[kk]), cos_t = cos(B.thetas[kk]);
  const double sin_f = sin(B.phis[kk]), cos_f = cos(B.phis[kk]);
  nh[0] = sin_t * cos_f;
  nh[1] = sin_t * sin_f;
  nh[2] = cos_t;
  for (int q = 0; q < 3; ++q) g[Lg.nh + q] = nh[q];
  const double tt = nh[2];
  const dcx wc = cx(nh[0], -nh[1]);
  const dcx ec[3] = {cx(1.0, 0.0), cx(0.0, -1.0), cx(0.0, 0.0)};
  for (int q = 0; q < 3; ++q) {
    g[Lg.t + q] = -tt * nh[q] * invr + (q == 2 ? invr : 0.0);
    stc(g + Lg.w + 2 * q, (-nh[q] * invr) * wc + invr * ec[q]);
  }
  for (int bb = 0; bb < 3; ++bb)
    for (int aa = 0; aa < 3; ++aa) {
      double th = (3.0 * tt * nh[aa] * nh[bb]) * invr2;
      dcx wh = invr2 * ((3.0 * nh[aa] * nh[bb]) * wc - nh[bb] * ec[aa] - nh[aa] * ec[bb]);
      if (bb == 2) th = th - nh[aa] * invr2;
      if (aa == 2) th = th - nh[bb] * invr2;
      if (aa == bb) {
        th = th - tt * invr2;
        wh = wh - invr2 * wc;
      }
      g[Lg.th + bb * 3 + aa] = th;
      stc(g + Lg.wh + 2 * (bb * 3 + aa), wh);
    }
  double *Qt = g + Lg.Q;
  Qt[0] = 1.0;
  if (L >= 1) {
    Qt[1] = tt;
    Qt[2] = 1.0;
  }
  for (int ll = 2; ll <= L; ++ll) {
    const int kbb = ll * (ll + 1) / 2;
    for (int mm = 0; mm <= ll - 2; ++mm) {
      const int kq = kbb + mm;
      Qt[kq] = ((double)(2 * ll - 1) * tt * Qt[kq - ll] - (double)(ll + mm - 1) * Qt[kq - 2 * ll + 1]) /
               (double)(ll - mm);
    }
    Qt[kbb + ll - 1] = (double)(2 * ll - 1) * tt * Qt[kbb - 1];
    Qt[kbb + ll] = (double)(2 * ll - 1) * Qt[kbb - 1];
  }
  dcx wpow = cx(1.0, 0.0);
  stc(g + Lg.wp, cx(0.0, 0.0));
  stc(g + Lg.wp + 2, cx(0.0, 0.0));
  stc(g + Lg.wp + 4, wpow);
  for (int mm = 1; mm <= L; ++mm) {
    wpow = wpow * wc;
    stc(g + Lg.wp + 2 * (mm + 2), wpow);
  }
}

// Omega, dOmega and (want2) d2Omega of component kq from a pair record
// (:1620-1650); Ck the signed prefactor (-1)^m preflm.
__device__ __forceinline__ void omega_k(const double *g, const GeoLayout &Lg, int kq, int ll, int mm, double Ck,
                                        bool want2, dcx &Om, dcx *dOm, dcx *d2Om) {
  const double *Qt = g + Lg.Q;
  const double q0 = Qt[kq], q1 = (mm + 1 <= ll) ? Qt[kq + 1] : 0.0, q2 = (mm + 2 <= ll) ? Qt[kq + 2] : 0.0;
  const dcx w0 = ldc(g + Lg.wp + 2 * (mm + 2)), w1 = ldc(g + Lg.wp + 2 * (mm + 1)), w2 = ldc(g + Lg.wp + 2 * mm);
  const double *tv = g + Lg.t;
  dcx wv[3];
  for (int aa = 0; aa < 3; ++aa) wv[aa] = ldc(g + Lg.w + 2 * aa);
  Om = (Ck * q0) * w0;
  for (int aa = 0; aa < 3; ++aa) dOm[aa] = Ck * ((q1 * tv[aa]) * w0 + (q0 * (double)mm) * (w1 * wv[aa]));
  if (want2)
    for (int bb = 0; bb < 3; ++bb)
      for (int aa = 0; aa < 3; ++aa)
        d2Om[bb * 3 + aa] =
            Ck * ((q2 * tv[aa] * tv[bb]) * w0 + (q1 * g[Lg.th + bb * 3 + aa]) * w0 +
                  (q1 * (double)mm) * (w1 * (tv[aa] * wv[bb] + tv[bb] * wv[aa])) +
                  (q0 * (double)(mm * (mm - 1))) * (w2 * (wv[aa] * wv[bb])) +
                  (q0 * (double)mm) * (w1 * ldc(g + Lg.wh + 2 * (bb * 3 + aa))));
}

// One (b, a) element of the second-derivative block from the k-sums S of a
// weight vector (layout: S1, S2, S3[3], S4 upper triangle[6], S5[3], S6[3][3], S7[3]).
__device__ __forceinline__ double hv_block(const double *S, const double *nh, double invr, int aa, int bb) {
  const int lo = aa < bb ? aa : bb, hi = aa < bb ? bb : aa;
  const int tri = lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
  return -(nh[aa] * nh[bb] * S[0] + (aa == bb ? invr * S[1] : 0.0) + nh[aa] * S[2 + bb] + nh[bb] * S[2 + aa] +
           S[5 + tri] + nh[bb] * S[11 + aa] + S[14 + aa * 3 + bb]);
}

// Per-CTA global scratch of the Hessian kernel (hess_scratch_doubles)
struct HessScratch {
  double *Gacc;   // (n_max, k_max, 3) complex: G = sum_j d c_nlm / d r_j
  double *Zv;     // (n_vec + 4, n_max, k_max) complex: S_v c for every weight vector
  double *ZGv;    // (n_vec + 1, n_max, k_max, 3) complex: S_v G for the Hessian's vectors
  double *dp1;    // (n_soap, 3): d p / d r_i, unnormalised
  double *kept3;  // (3, n_kept)
  double *vk;     // (n_kept): a weight vector spread through the compression
};

__device__ HessScratch carve(double *base, const DevParams &P, int n_vec) {
  const size_t nk = (size_t)P.n_max * P.k_max;
  HessScratch h;
  h.Gacc = base;
  h.Zv = h.Gacc + 6 * nk;
  h.ZGv = h.Zv + 2 * (size_t)(n_vec + 4) * nk;
  h.dp1 = h.ZGv + 6 * (size_t)(n_vec + 1) * nk;
  h.kept3 = h.dp1 + 3 * (size_t)P.n_soap;
  h.vk = h.kept3 + 3 * (size_t)P.n_kept;
  return h;
}

// Warp-wise dot product over fixed lane strides and a fixed shuffle tree.
__device__ __forceinline__ double warp_dot(const double *x, int sx, const double *y, int sy, int n) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int t = lane; t < n; t += 32) s += x[(size_t)t * sx] * y[(size_t)t * sy];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// Weight vectors of one site: v < n_vec the caller's, v = n_vec the site's
// unnormalised p, v = n_vec + 1 + a the column a of dp1.  Of the first n_vec + 1
// the Hessian is formed; the last three give dp1 . dp_j.
__device__ __forceinline__ double weight(const double *vecs, const double *soap_i, double sv, const double *dp1,
                                         int n_vec, int ns, int site, int v, int o) {
  if (v < n_vec) return vecs[((size_t)site * n_vec + v) * ns + o];
  if (v == n_vec) return soap_i[o] * sv;
  return dp1[3 * o + (v - n_vec - 1)];
}

// ---- the Hessian, persistent, one CTA per site at a time.  Per site:
//  A  G(n,k) = sum_j d/dr_j [4 pi R_n F_l Omega_k] (:1305-1334), a fixed-order
//     sum over the site's pairs of R'_n A_j + R_n B_j, with the pairs' angular
//     factors A_j, B_j built in shared memory chunk by chunk; then
//     dp1 = d p / d r_i = -(d p / d c) G component by component of p (the
//     reference sums -dp_j over the pairs; the two agree to rounding, since
//     sum_j d c / d r_j = G);
//  Z  every weight vector v spread back through the compression into its
//     S_v(n, n', l) and applied to c_nlm (Z_v) and to G (ZG_v) (:1336-1376);
//  B  one half-warp per pair, lanes over k: Z_v and ZG_v contracted with the pair's
//     R_n, R'_n, R''_n and Omega, dOmega, d2Omega (:1378-1412) give the second
//     derivative hv and the first derivative v . dp_j (what the reference's
//     self-test rebuilds, here the value used), and from them the
//     normalisation (:1414-1484).
// Sums run in a fixed order (pairs to half-warps by index, k within a round by
// lane order through shared memory, k rounds in order, half-warps in order).
__global__ void __launch_bounds__(kHessThreads, 4) k64_hess(const DevParams P, const DevBatch B, const double *rad,
                                                         const double *rad_der, const double *rad_der2,
                                                         const double *geo, const int *good, const double2 *cnk,
                                                         const double *norm, const double *soap, int n_vec,
                                                         const double *vecs, double *hess, double *scratch,
                                                         size_t scratch_per_cta, int *ticket) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_site;
  const int N = P.n_max, K = P.k_max, ns = P.n_soap, nk = P.n_kept;
  const int nvh = n_vec + 1, nva = n_vec + 4;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, n_warps = kHessThreads / 32;
  const GeoLayout Lg(P.l_max);
  // shared: the site's dot products (3 + 4 n_vec), then a region used by pass
  // A (a chunk of kHessPC pairs: their A, B factors (K, 12) and R, R' rows) and
  // by pass B (per half-warp: the k-sums of its pair (n_vec + 4, kHessS), its
  // radial rows (3 n_max), its running hsum (n_vec, 9) and its transpose buffer)
  const int sd = 3 + 4 * n_vec + ((3 + 4 * n_vec) & 1);
  const int per_half = kHessS * nva + 3 * N + 9 * n_vec + 16 * kHessRed;  // per half-warp, pass B
  double *sdot = sm;
  double *cab = sm + sd;
  double *crr = cab + (size_t)kHessPC * K * 12;
  const int half = lane >> 4, hl = lane & 15, n_halves = 2 * n_warps;
  double *wsum = sm + sd + (size_t)(2 * warp + half) * per_half;
  double *wrad = wsum + kHessS * nva;
  double *whs = wrad + 3 * N;
  double *red = whs + 9 * n_vec;  // (16 lanes, kHessRed): the k-sums before their column sums
  const HessScratch h = carve(scratch + scratch_per_cta * blockIdx.x, P, n_vec);
  const double fourpi = 4.0 * kPi;

  for (;;) {
    __syncthreads();
    if (tid == 0) s_site = atomicAdd(ticket, 1);
    __syncthreads();
    const int site = s_site;
    if (site >= B.n_sites) break;
    const int p0 = B.off[site], p1 = min(B.off[site + 1], B.n_pairs);
    const double sv = norm[site], invs = 1.0 / sv, invs3 = invs / (sv * sv), invs5 = invs3 / (sv * sv);
    const double2 *c = cnk + (size_t)site * N * K;
    const double *soap_i = soap + (size_t)site * ns;
    // ---- A: G, threads over (n, k), the pairs in CSR order in chunks of kHessPC:
    // A(j, k, q) = 4 pi F_l nh_q Omega_k, B = 4 pi (F'_l nh_q Omega_k + F_l dOmega_kq),
    // G(n, k, q) = sum_j R'_n(j) A(j, k, q) + R_n(j) B(j, k, q) (:1320-1331)
    for (int t = tid; t < 6 * N * K; t += kHessThreads) h.Gacc[t] = 0.0;
    for (int jc = p0 + 1; jc < p1; jc += kHessPC) {
      const int nc = min(kHessPC, p1 - jc);
      __syncthreads();
      for (int t = tid; t < nc * 2 * N; t += kHessThreads) {
        const int pp = t / (2 * N), r = t - pp * 2 * N;
        crr[t] = (r < N ? rad : rad_der)[(size_t)(jc + pp) * N + (r < N ? r : r - N)];
      }
      for (int t = tid; t < nc * K; t += kHessThreads) {
        const int pp = t / K, k = t - pp * K, j = jc + pp;
        double *o = cab + (size_t)t * 12;
        if (!good[j]) {
          for (int e = 0; e < 12; ++e) o[e] = 0.0;
          continue;
        }
        const double *g = geo + (size_t)j * Lg.size;
        const int l = l_of_k(k), m = k - l * (l + 1) / 2;
        dcx Om, dOm[3];
        omega_k(g, Lg, k, l, m, (m & 1) ? -P.preflm64[k] : P.preflm64[k], false, Om, dOm, nullptr);
        const double f0 = fourpi * g[Lg.F + l], f1 = fourpi * g[Lg.F1 + l];
        for (int q = 0; q < 3; ++q) {
          const double nq = g[Lg.nh + q];
          stc(o + 4 * q, (f0 * nq) * Om);
          stc(o + 4 * q + 2, (f1 * nq) * Om + f0 * dOm[q]);
        }
      }
      __syncthreads();
      // threads over (k, four radial indices): each pair's A, B are loaded once for four n
      for (int it = tid; it < ((N + 3) >> 2) * K; it += kHessThreads) {
        const int nb = it / K, k = it - nb * K, n0 = 4 * nb;
        dcx gq[4][3];
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
          for (int q = 0; q < 3; ++q)
            gq[t][q] = (n0 + t < N) ? ldc(h.Gacc + ((size_t)(n0 + t) * K + k) * 6 + 2 * q) : cx(0.0, 0.0);
        for (int pp = 0; pp < nc; ++pp) {
          const double *a = cab + ((size_t)pp * K + k) * 12;
          dcx Aq[3], Bq[3];
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            Aq[q] = ldc(a + 4 * q);
            Bq[q] = ldc(a + 4 * q + 2);
          }
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int n = min(n0 + t, N - 1);  // the tail's extra rows are not stored
            const double r0 = crr[pp * 2 * N + n], r1 = crr[pp * 2 * N + N + n];
#pragma unroll
            for (int q = 0; q < 3; ++q) gq[t][q] = gq[t][q] + r1 * Aq[q] + r0 * Bq[q];
          }
        }
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if (n0 + t < N)
#pragma unroll
            for (int q = 0; q < 3; ++q) stc(h.Gacc + ((size_t)(n0 + t) * K + k) * 6 + 2 * q, gq[t][q]);
      }
    }
    __syncthreads();
    // dp1 in the kept components, then through the compression map
    for (int q = tid; q < nk; q += kHessThreads) {
      const int code = P.kept_nnl[q];
      const int n = code & 0xff, np = (code >> 8) & 0xff, l = code >> 16;
      const double base = (n == np) ? 1.0 : sqrt(2.0);
      double d[3] = {0.0, 0.0, 0.0};
      for (int m = 0; m <= l; ++m) {
        const int k = l * (l + 1) / 2 + m;
        const double w = base * ((m > 0) ? 2.0 : 1.0);
        const double2 a = c[(size_t)n * K + k], b = c[(size_t)np * K + k];
        const double *ga = h.Gacc + ((size_t)n * K + k) * 6, *gb = h.Gacc + ((size_t)np * K + k) * 6;
        for (int e = 0; e < 3; ++e)
          d[e] = d[e] - w * (ga[2 * e] * b.x + ga[2 * e + 1] * b.y + a.x * gb[2 * e] + a.y * gb[2 * e + 1]);
      }
      for (int e = 0; e < 3; ++e) h.kept3[(size_t)e * nk + q] = d[e];
    }
    __syncthreads();
    for (int o = tid; o < ns; o += kHessThreads) {
      double d0 = 0.0, d1 = 0.0, d2 = 0.0;
      for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) {
        const double e = P.pi_el64[t];
        const int q = P.pi_q[t];
        d0 = d0 + e * h.kept3[q];
        d1 = d1 + e * h.kept3[nk + q];
        d2 = d2 + e * h.kept3[2 * nk + q];
      }
      h.dp1[3 * o] = d0;
      h.dp1[3 * o + 1] = d1;
      h.dp1[3 * o + 2] = d2;
    }
    __syncthreads();
    // the site's dot products: t1 (3), then per v wp, u1 (3)
    for (int d = warp; d < 3 + 4 * n_vec; d += n_warps) {
      double r;
      if (d < 3) r = sv * warp_dot(soap_i, 1, h.dp1 + d, 3, ns);
      else {
        const int v = (d - 3) >> 2, e = (d - 3) & 3;
        const double *wv = vecs + ((size_t)site * n_vec + v) * ns;
        r = (e == 0) ? sv * warp_dot(wv, 1, soap_i, 1, ns) : warp_dot(wv, 1, h.dp1 + (e - 1), 3, ns);
      }
      if (lane == 0) sdot[d] = r;
    }
    // ---- Z: S_v applied to c and G through the per-(l, n) lists of the kept
    // components (2 v on the diagonal, sqrt 2 v off it, np ascending)
    for (int v = 0; v < nva; ++v) {
      for (int q = tid; q < nk; q += kHessThreads) {
        double s = 0.0;
        for (int t = P.pj_off[q]; t < P.pj_off[q + 1]; ++t)
          s = s + P.pj_el64[t] * weight(vecs, soap_i, sv, h.dp1, n_vec, ns, site, v, P.pj_o[t]);
        h.vk[q] = s;
      }
      __syncthreads();
      for (int it = tid; it < N * K; it += kHessThreads) {
        const int n = it / K, k = it - n * K, l = l_of_k(k);
        dcx zc = cx(0.0, 0.0), b0[3] = {cx(0.0, 0.0), cx(0.0, 0.0), cx(0.0, 0.0)};
        for (int t = P.hl_off[l * N + n]; t < P.hl_off[l * N + n + 1]; ++t) {
          const int np = P.hl_np[t];
          const double smv = P.hl_fac64[t] * h.vk[P.hl_q[t]];
          const double2 cc = c[(size_t)np * K + k];
          zc = zc + cx(smv * cc.x, smv * cc.y);
          if (v < nvh)
            for (int q = 0; q < 3; ++q) b0[q] = b0[q] + smv * ldc(h.Gacc + ((size_t)np * K + k) * 6 + 2 * q);
        }
        stc(h.Zv + (((size_t)v * N + n) * K + k) * 2, zc);
        if (v < nvh)
          for (int q = 0; q < 3; ++q) stc(h.ZGv + ((((size_t)v * N + n) * K + k) * 3 + q) * 2, b0[q]);
      }
      __syncthreads();
    }
    // ---- B: one half-warp per pair, lanes over k (rounds of 16).  Per weight
    // vector the k-sums below give the block (:1378-1412, reassociated over k):
    //   S1 = sum w Re[(z2 - z1/r) Om]   S2 = sum w Re[z1 Om]    S3_b = sum w Re[z1 dOm_b]
    //   S4_ab = sum w Re[z0 d2Om_ab]    S5_a = sum w Re[gg1_a Om]
    //   S6_ab = sum w Re[gg0_a dOm_b]   S7_b = sum w Re[z0 dOm_b]
    //   hv(b, a) = -(n_a n_b S1 + [a = b] S2 / r + n_a S3_b + n_b S3_a + S4_ab + n_b S5_a + S6_ab)
    //   v . dp_j (b) = n_b S2 + S7_b
    // The two halves of a warp read the same Z rows (same k), for two pairs.
    for (int t = hl; t < 9 * n_vec; t += 16) whs[t] = 0.0;
    for (int jb = p0 + 1 + 2 * warp; jb < p1; jb += 2 * n_warps) {  // the same trip count for both halves
      const int j = jb + half;
      const bool pv = j < p1 && good[j];  // this half has a pair
      const double *g = geo + (size_t)(pv ? j : 0) * Lg.size;
      for (int t = hl; t < 3 * N; t += 16) {
        const int w = t / N, n = t - w * N;
        wrad[t] = pv ? (w == 0 ? rad : (w == 1 ? rad_der : rad_der2))[(size_t)j * N + n] : 0.0;
      }
      for (int t = hl; t < kHessS * nva; t += 16) wsum[t] = 0.0;
      __syncwarp();
      for (int k0 = 0; k0 < K; k0 += 16) {
        const int k = k0 + hl;
        const bool act = pv && k < K;
        const int kc = act ? k : 0;
        const int l = l_of_k(kc), m = kc - l * (l + 1) / 2;
        dcx Om = cx(0.0, 0.0), dOm[3], d2Om[9];
        for (int e = 0; e < 3; ++e) dOm[e] = Om;
        for (int e = 0; e < 9; ++e) d2Om[e] = Om;
        double wmk = 0.0, f0 = 0.0, f1 = 0.0, f2 = 0.0, invr = 0.0;
        if (act) {
          omega_k(g, Lg, kc, l, m, (m & 1) ? -P.preflm64[kc] : P.preflm64[kc], true, Om, dOm, d2Om);
          wmk = (m > 0) ? 2.0 : 1.0;
          f0 = fourpi * g[Lg.F + l];
          f1 = fourpi * g[Lg.F1 + l];
          f2 = fourpi * g[Lg.F2 + l];
          invr = g[Lg.invr];
        }
        for (int v = 0; v < nva; ++v) {
          const bool full = v < nvh;
          double *ws = wsum + v * kHessS;
          double *my = red + hl * kHessRed;
          // a-pass: R, R', R'' against Z_v
          dcx a0 = cx(0.0, 0.0), a1 = a0, a2 = a0;
          if (act) {
            const double2 *zv = (const double2 *)h.Zv + (size_t)v * N * K + k;
#pragma unroll 8
            for (int n = 0; n < N; ++n) {
              const double2 zz = zv[(size_t)n * K];
              const dcx zc = cx(zz.x, -zz.y);
              a0 = a0 + wrad[n] * zc;
              a1 = a1 + wrad[N + n] * zc;
              if (full) a2 = a2 + wrad[2 * N + n] * zc;
            }
          }
          const dcx z0 = f0 * a0, z1 = f0 * a1 + f1 * a0;
          my[1] = wmk * (z1 * Om).re;
#pragma unroll
          for (int bb = 0; bb < 3; ++bb) my[23 + bb] = wmk * (z0 * dOm[bb]).re;
          if (!full) {  // the four first-derivative sums: lanes 0..3 of each half add its 16 rows
            __syncwarp();
            if (hl < 4) {
              const int e = hl == 0 ? 1 : 22 + hl;
              double acc = 0.0;
              for (int r = 0; r < 16; ++r) acc += red[r * kHessRed + e];
              ws[e] += acc;
            }
            __syncwarp();
            continue;
          }
          {
            const dcx z2 = f0 * a2 + (2.0 * f1) * a1 + f2 * a0;
            my[0] = wmk * ((z2 - invr * z1) * Om).re;
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) my[2 + bb] = wmk * (z1 * dOm[bb]).re;
            int e = 5;
#pragma unroll
            for (int aa = 0; aa < 3; ++aa)
#pragma unroll
              for (int bb = aa; bb < 3; ++bb) my[e++] = wmk * (z0 * d2Om[bb * 3 + aa]).re;
          }
          // b-pass: R, R' against ZG_v, one Cartesian component at a time
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            dcx b0 = cx(0.0, 0.0), b1 = b0;
            if (act) {
              const double2 *zg = (const double2 *)h.ZGv + ((size_t)v * N * K + k) * 3 + q;
#pragma unroll 8
              for (int n = 0; n < N; ++n) {
                const double2 gz = zg[(size_t)n * K * 3];
                const dcx gc = cx(gz.x, -gz.y);
                b0 = b0 + wrad[n] * gc;
                b1 = b1 + wrad[N + n] * gc;
              }
            }
            const dcx gg0 = f0 * b0, gg1 = f0 * b1 + f1 * b0;
            my[11 + q] = wmk * (gg1 * Om).re;
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) my[14 + q * 3 + bb] = wmk * (gg0 * dOm[bb]).re;
          }
          // the 26 sums over the half's k: lane e adds the 16 rows of column e in order
          __syncwarp();
          for (int e = hl; e < kHessS; e += 16) {
            double acc = 0.0;
            for (int r = 0; r < 16; ++r) acc += red[r * kHessRed + e];
            ws[e] += acc;
          }
          __syncwarp();
        }
      }
      __syncwarp();
      // the normalisation (:1414-1484): t2 = p . dp_j, c12(b, a) = dp1(:, a) . dp_j(:, b),
      // u2 = w . dp_j
      if (pv) {
        const double invr = g[Lg.invr];
        const double nh[3] = {g[Lg.nh], g[Lg.nh + 1], g[Lg.nh + 2]};
        for (int t = hl; t < 9 * n_vec; t += 16) {
          const int v = t / 9, e = t - v * 9, bb = e / 3, aa = e - bb * 3;
          const double *t1 = sdot, *dv = sdot + 3 + 4 * v;
          const double wp = dv[0], *u1 = dv + 1;
          const double *Sp = wsum + n_vec * kHessS, *Sv = wsum + v * kHessS;
          const double t2b = nh[bb] * Sp[1] + Sp[23 + bb], u2b = nh[bb] * Sv[1] + Sv[23 + bb];
          const double *Sc = wsum + (n_vec + 1 + aa) * kHessS;
          const double c12 = nh[bb] * Sc[1] + Sc[23 + bb];
          const double hvv = hv_block(Sv, nh, invr, aa, bb), hvp = hv_block(Sp, nh, invr, aa, bb);
          const double hval = hvv * invs - (u1[aa] * t2b + u2b * t1[aa]) * invs3 - wp * (c12 + hvp) * invs3 +
                              3.0 * wp * t1[aa] * t2b * invs5;
          hess[((size_t)j * n_vec + v) * 9 + e] = hval;
          whs[t] += hval;
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // the self pair: minus the sum of the others (:1488-1495), half-warps in
    // order; pairs the Hessian skips keep the zero blocks the launcher cleared
    if (p1 > p0)
      for (int t = tid; t < 9 * n_vec; t += kHessThreads) {
        double s = 0.0;
        for (int w = 0; w < n_halves; ++w) s += sm[sd + (size_t)w * per_half + kHessS * nva + 3 * N + t];
        hess[((size_t)p0 * n_vec) * 9 + t] = -s;
      }
  }
}

}  // namespace

// Doubles per CTA, a multiple of 32 so that every CTA's region (and the
// complex tables in it, read with 16-byte loads) starts on a 256-byte boundary.
size_t hess_scratch_doubles(const DevParams &P, int n_vec) {
  const size_t nk = (size_t)P.n_max * P.k_max;
  const size_t n = 6 * nk + 2 * (size_t)(n_vec + 4) * nk + 6 * (size_t)(n_vec + 1) * nk + 3 * (size_t)P.n_soap +
                   4 * (size_t)P.n_kept;
  return (n + 31) / 32 * 32;
}

size_t hess_geo_doubles(const DevParams &P) { return (size_t)GeoLayout(P.l_max).size; }

size_t hess_smem_bytes(const DevParams &P, int n_vec) {
  const size_t nw = kHessThreads / 32, sd = 3 + 4 * (size_t)n_vec;
  const size_t pass_a = (size_t)kHessPC * (12 * (size_t)P.k_max + 2 * (size_t)P.n_max);
  const size_t pass_b =
      2 * nw * (kHessS * (size_t)(n_vec + 4) + 3 * (size_t)P.n_max + 9 * (size_t)n_vec + 16 * (size_t)kHessRed);
  return sizeof(double) * (sd + (sd & 1) + (pass_a > pass_b ? pass_a : pass_b));
}

int hess_grid(const DevParams &P, int n_vec) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t sm = hess_smem_bytes(P, n_vec);
  if (cudaFuncSetAttribute(k64_hess, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return sms;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k64_hess, kHessThreads, sm);
  return sms * (per_sm > 0 ? per_sm : 1);
}

cudaError_t launch_hessian(const DevParams &P, const DevBatch &B, cudaStream_t s, const Fp64Work &w,
                           double *rad_der2, double *geo, int *good, const double *soap, int n_vec,
                           const double *vecs, double *hess, double *scratch, int grid, int *ticket, int *launches) {
  CU_RET(cudaMemsetAsync(hess, 0, sizeof(double) * 9 * (size_t)n_vec * B.n_pairs, s));
  CU_RET(cudaMemsetAsync(ticket, 0, sizeof(int), s));
  if (B.n_pairs > 0) {
    const int blocks = (B.n_pairs + 127) / 128;
    int amax = 0;
    for (int sp = 0; sp < P.n_species; ++sp) amax = amax > P.rad[sp].alpha ? amax : P.rad[sp].alpha;
    if (amax <= 8) k64_radial_d2<8><<<blocks, 128, 0, s>>>(P, B, rad_der2);
    else k64_radial_d2<16><<<blocks, 128, 0, s>>>(P, B, rad_der2);
    k64_hgeo<<<blocks, 128, 0, s>>>(P, B, geo, good);
    if (launches) *launches += 2;
  }
  if (B.n_sites > 0) {
    const size_t sm = hess_smem_bytes(P, n_vec);
    CU_RET(cudaFuncSetAttribute(k64_hess, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int g = grid < B.n_sites ? grid : B.n_sites;
    k64_hess<<<g, kHessThreads, sm, s>>>(P, B, w.rad, w.rad_der, rad_der2, geo, good, (const double2 *)w.cnk,
                                        w.norm, soap, n_vec, vecs, hess, scratch, hess_scratch_doubles(P, n_vec),
                                        ticket);
    if (launches) *launches += 1;
  }
  return cudaGetLastError();
}

}  // namespace soapb
