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
// seed only); k64_hess is persistent, one CTA per site at a time, and follows
// the reference's two passes: pass A builds G (the central-atom gradient of
// the expansion) and the unnormalised central derivative dp1, the weight
// vectors are spread back through the compression into their S matrices and
// contracted with c_nlm and G (Z, ZG), and pass B contracts every pair's
// radial values and first and second derivatives against them and applies the
// normalisation.  The angular factor Omega = C_k Q_l^m(t) w^m and its Cartesian
// gradient and Hessian are rebuilt per pair (Q_l^m = d^m P_l / dt^m, w = x - iy
// over r), as the reference does.  Every reduction runs in a fixed order.
#include "soapb_device.cuh"

namespace soapb {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kHessThreads = 256;
constexpr int kHessVB = 8;  // weight vectors contracted per pass over a pair's k

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
__device__ __forceinline__ dcx conjg(dcx a) { return cx(a.re, -a.im); }

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

// Shared per-pair quantities of the Hessian kernel (pair_geometry,
// src/soap_turbo.f90:1537-1652): written by pair_setup, read by all threads.
struct PairGeo {
  int good;
  double nh[3], invr;
  double tvec[3], thes[9];
  dcx wvec[3], whes[9];
  double Fl[SOAPB_MAX_LMAX + 1], Fl1[SOAPB_MAX_LMAX + 1], Fl2[SOAPB_MAX_LMAX + 1];
  double Qt[SOAPB_KMAX_CAP];
  dcx wpow[SOAPB_MAX_LMAX + 3];  // wpow[m + 2] = w^m, w^-1 = w^-2 = 0
};

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

// The scalar part of pair_geometry, one thread: F_l and its derivatives, the
// unit vector, the gradients and Hessians of t = cos(theta) and w, Q_l^m, w^m.
__device__ void pair_setup(const DevParams &P, const DevBatch &B, int kk, bool want2, PairGeo &G) {
  G.good = 0;
  const double rr = B.rjs[kk];
  if (rr >= P.rcut_max || rr < 1.0e-10) return;
  const unsigned bits = B.bits[kk];
  if (bits == 0u) return;
  const int isp = __ffs(bits) - 1;
  G.good = 1;
  const int L = P.l_max;
  const double invr = 1.0 / rr, invr2 = invr * invr;
  G.invr = invr;
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
    G.Fl[l] = amp * f0;
    G.Fl1[l] = ampd * f0 + amp * f1;
    G.Fl2[l] = ampdd * f0 + 2.0 * ampd * f1 + amp * f2;
  }
  const double sin_t = sin(B.thetas[kk]), cos_t = cos(B.thetas[kk]);
  const double sin_f = sin(B.phis[kk]), cos_f = cos(B.phis[kk]);
  G.nh[0] = sin_t * cos_f;
  G.nh[1] = sin_t * sin_f;
  G.nh[2] = cos_t;
  const double tt = G.nh[2];
  const dcx wc = cx(G.nh[0], -G.nh[1]);
  const dcx ec[3] = {cx(1.0, 0.0), cx(0.0, -1.0), cx(0.0, 0.0)};
  for (int q = 0; q < 3; ++q) {
    G.tvec[q] = -tt * G.nh[q] * invr;
    G.wvec[q] = (-G.nh[q] * invr) * wc;
  }
  G.tvec[2] = G.tvec[2] + invr;
  for (int q = 0; q < 3; ++q) G.wvec[q] = G.wvec[q] + invr * ec[q];
  if (want2) {
    for (int bb = 0; bb < 3; ++bb)
      for (int aa = 0; aa < 3; ++aa) {
        G.thes[bb * 3 + aa] = (3.0 * tt * G.nh[aa] * G.nh[bb]) * invr2;
        G.whes[bb * 3 + aa] = invr2 * ((3.0 * G.nh[aa] * G.nh[bb]) * wc - G.nh[bb] * ec[aa] - G.nh[aa] * ec[bb]);
      }
    for (int aa = 0; aa < 3; ++aa) {
      G.thes[aa * 3 + 2] = G.thes[aa * 3 + 2] - G.nh[aa] * invr2;
      G.thes[2 * 3 + aa] = G.thes[2 * 3 + aa] - G.nh[aa] * invr2;
      G.thes[aa * 3 + aa] = G.thes[aa * 3 + aa] - tt * invr2;
      G.whes[aa * 3 + aa] = G.whes[aa * 3 + aa] - invr2 * wc;
    }
  }
  G.Qt[0] = 1.0;
  if (L >= 1) {
    G.Qt[1] = tt;
    G.Qt[2] = 1.0;
  }
  for (int ll = 2; ll <= L; ++ll) {
    const int kbb = ll * (ll + 1) / 2;
    for (int mm = 0; mm <= ll - 2; ++mm) {
      const int kq = kbb + mm;
      G.Qt[kq] = ((double)(2 * ll - 1) * tt * G.Qt[kq - ll] - (double)(ll + mm - 1) * G.Qt[kq - 2 * ll + 1]) /
                 (double)(ll - mm);
    }
    G.Qt[kbb + ll - 1] = (double)(2 * ll - 1) * tt * G.Qt[kbb - 1];
    G.Qt[kbb + ll] = (double)(2 * ll - 1) * G.Qt[kbb - 1];
  }
  G.wpow[0] = cx(0.0, 0.0);
  G.wpow[1] = cx(0.0, 0.0);
  G.wpow[2] = cx(1.0, 0.0);
  for (int mm = 1; mm <= L; ++mm) G.wpow[mm + 2] = G.wpow[mm + 1] * wc;
}

// Omega, dOmega and (want2) d2Omega of component kq (:1620-1650); Ck the signed prefactor.
__device__ __forceinline__ void omega_k(const PairGeo &G, int kq, int ll, int mm, double Ck, bool want2, dcx &Om,
                                        dcx *dOm, dcx *d2Om) {
  const double q0 = G.Qt[kq], q1 = (mm + 1 <= ll) ? G.Qt[kq + 1] : 0.0, q2 = (mm + 2 <= ll) ? G.Qt[kq + 2] : 0.0;
  const dcx w0 = G.wpow[mm + 2], w1 = G.wpow[mm + 1], w2 = G.wpow[mm];
  Om = (Ck * q0) * w0;
  for (int aa = 0; aa < 3; ++aa) dOm[aa] = Ck * ((q1 * G.tvec[aa]) * w0 + (q0 * (double)mm) * (w1 * G.wvec[aa]));
  if (want2)
    for (int bb = 0; bb < 3; ++bb)
      for (int aa = 0; aa < 3; ++aa)
        d2Om[bb * 3 + aa] =
            Ck * ((q2 * G.tvec[aa] * G.tvec[bb]) * w0 + (q1 * G.thes[bb * 3 + aa]) * w0 +
                  (q1 * (double)mm) * (w1 * (G.tvec[aa] * G.wvec[bb] + G.tvec[bb] * G.wvec[aa])) +
                  (q0 * (double)(mm * (mm - 1))) * (w2 * (G.wvec[aa] * G.wvec[bb])) +
                  (q0 * (double)mm) * (w1 * G.whes[bb * 3 + aa]));
}

// Per-CTA global scratch of the Hessian kernel (doubles), see hess_scratch_doubles
struct HessScratch {
  dcx *Gacc;      // (n_max, k_max, 3)
  dcx *Zv, *ZGv;  // (nv, n_max, k_max), (nv, n_max, k_max, 3)
  double *dp1, *dp2;  // (n_soap, 3)
  double *kept3;  // (3, n_kept): one pair's spherical derivatives of the kept components
  double *vk;     // (n_kept): a weight vector spread through the compression
};

__device__ HessScratch carve(double *base, const DevParams &P, int nv) {
  const size_t nk = (size_t)P.n_max * P.k_max;
  HessScratch h;
  h.Gacc = (dcx *)base;
  h.Zv = h.Gacc + 3 * nk;
  h.ZGv = h.Zv + (size_t)nv * nk;
  h.dp1 = (double *)(h.ZGv + 3 * (size_t)nv * nk);
  h.dp2 = h.dp1 + 3 * (size_t)P.n_soap;
  h.kept3 = h.dp2 + 3 * (size_t)P.n_soap;
  h.vk = h.kept3 + 3 * (size_t)P.n_kept;
  return h;
}

// The Cartesian, unnormalised derivative of the site's compressed p for pair
// kk (pair_dp, :1520-1534, on soap_rad/azi/pol_der, :1927-2075) into dp (n_soap, 3).
__device__ void pair_dp(const DevParams &P, const DevBatch &B, int kk, const double *rad, const double *rad_der,
                        const double2 *ang, const double2 *c, double *sPQ, double *kept3, double *dp) {
  const int N = P.n_max, K = P.k_max, L1 = P.l_max + 1, nk = P.n_kept;
  const size_t plane = (size_t)B.n_pairs * K;
  const double2 *A = ang + (size_t)kk * K;
  for (int it = threadIdx.x; it < N * L1; it += blockDim.x) {
    const int n = it / L1, l = it - n * L1;
    double ap = 0.0, aq = 0.0, aa = 0.0, ao = 0.0;
    for (int m = 0; m <= l; ++m) {
      const int k = l * (l + 1) / 2 + m;
      const double w = (m == 0) ? 1.0 : 2.0;
      const double2 cc = c[(size_t)n * K + k];
      const double2 a0 = A[k], a1 = A[plane + k], a2 = A[2 * plane + k], a3 = A[3 * plane + k];
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
  const double *Pm = sPQ, *Qm = sPQ + N * L1, *Qa = sPQ + 2 * N * L1, *Qo = sPQ + 3 * N * L1;
  for (int q = threadIdx.x; q < nk; q += blockDim.x) {
    const int code = P.kept_nnl[q];
    const int n = code & 0xff, np = (code >> 8) & 0xff, l = code >> 16;
    const double rn = rad[(size_t)kk * N + n], rdn = rad_der[(size_t)kk * N + n];
    const double rnp = rad[(size_t)kk * N + np], rdnp = rad_der[(size_t)kk * N + np];
    const double pre = 4.0 * kPi * ((n == np) ? 1.0 : sqrt(2.0));
    kept3[q] = pre * (rdn * Pm[np * L1 + l] + rn * Qm[np * L1 + l] + rdnp * Pm[n * L1 + l] + rnp * Qm[n * L1 + l]);
    kept3[nk + q] = pre * (rn * Qa[np * L1 + l] + rnp * Qa[n * L1 + l]);
    kept3[2 * nk + q] = pre * (rn * Qo[np * L1 + l] + rnp * Qo[n * L1 + l]);
  }
  __syncthreads();
  const double st = sin(B.thetas[kk]), ct = cos(B.thetas[kk]), sf = sin(B.phis[kk]), cf = cos(B.phis[kk]);
  const double ir = 1.0 / B.rjs[kk];
  const double cxr = st * cf, cyr = st * sf, czr = ct, pxr = -ct * cf * ir, pyr = -ct * sf * ir, pzr = st * ir;
  const double axr = -sf * ir, ayr = cf * ir;
  for (int o = threadIdx.x; o < P.n_soap; o += blockDim.x) {
    double dr = 0.0, da = 0.0, dpl = 0.0;
    for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) {
      const double e = P.pi_el64[t];
      const int q = P.pi_q[t];
      dr = dr + e * kept3[q];
      da = da + e * kept3[nk + q];
      dpl = dpl + e * kept3[2 * nk + q];
    }
    dp[3 * o + 0] = cxr * dr + pxr * dpl + axr * da;
    dp[3 * o + 1] = cyr * dr + pyr * dpl + ayr * da;
    dp[3 * o + 2] = czr * dr + pzr * dpl;
  }
  __syncthreads();
}

// Warp-wise dot products of length n over fixed lane strides and a fixed
// shuffle tree: x . y (both with element stride sx, sy).
__device__ __forceinline__ double warp_dot(const double *x, int sx, const double *y, int sy, int n) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int t = lane; t < n; t += 32) s += x[(size_t)t * sx] * y[(size_t)t * sy];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

__global__ void __launch_bounds__(kHessThreads) k64_hess(const DevParams P, const DevBatch B, const double *rad,
                                                         const double *rad_der, const double *rad_der2,
                                                         const double2 *ang, const double2 *cnk,
                                                         const double *norm, const double *soap, int n_vec,
                                                         const double *vecs, double *hess, double *scratch,
                                                         size_t scratch_per_cta, int *ticket) {
  extern __shared__ __align__(16) double sm[];
  __shared__ PairGeo G;
  __shared__ int s_site;
  const int N = P.n_max, K = P.k_max, L1 = P.l_max + 1, ns = P.n_soap, nv = n_vec + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, n_warps = kHessThreads / 32;
  // shared: pvec (ns), sPQ (4 N L1), per-k partial sums (K, kHessVB, 9), hv (nv, 9),
  // hsum (n_vec, 9), dots (15 + 7 n_vec)
  double *pvec = sm;
  double *sPQ = pvec + ns;
  double *part = sPQ + 4 * N * L1;
  double *hv = part + (size_t)K * kHessVB * 9;
  double *hsum = hv + 9 * nv;
  double *dots = hsum + 9 * n_vec;
  const HessScratch h = carve(scratch + scratch_per_cta * blockIdx.x, P, nv);
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
    for (int q = tid; q < ns; q += kHessThreads) pvec[q] = soap[(size_t)site * ns + q] * sv;
    // ---- pass A: G and the unnormalised central-atom derivative (:1305-1334)
    for (int t = tid; t < 3 * N * K; t += kHessThreads) h.Gacc[t] = cx(0.0, 0.0);
    for (int t = tid; t < 3 * ns; t += kHessThreads) h.dp1[t] = 0.0;
    __syncthreads();
    for (int k2 = p0 + 1; k2 < p1; ++k2) {
      if (tid == 0) pair_setup(P, B, k2, false, G);
      __syncthreads();
      if (!G.good) continue;
      pair_dp(P, B, k2, rad, rad_der, ang, c, sPQ, h.kept3, h.dp2);
      for (int t = tid; t < 3 * ns; t += kHessThreads) h.dp1[t] = h.dp1[t] - h.dp2[t];
      for (int it = tid; it < N * K; it += kHessThreads) {
        const int n = it / K, k = it - n * K;
        int l = 0;
        while ((l + 1) * (l + 2) / 2 <= k) ++l;
        const int m = k - l * (l + 1) / 2;
        dcx Om, dOm[3];
        omega_k(G, k, l, m, (m & 1) ? -P.preflm64[k] : P.preflm64[k], false, Om, dOm, nullptr);
        const double r0 = fourpi * rad[(size_t)k2 * N + n], r1 = fourpi * rad_der[(size_t)k2 * N + n];
        const double g0 = r0 * G.Fl[l], g1 = r1 * G.Fl[l] + r0 * G.Fl1[l];
        for (int q = 0; q < 3; ++q) h.Gacc[(size_t)it * 3 + q] = h.Gacc[(size_t)it * 3 + q] + (g1 * G.nh[q]) * Om + g0 * dOm[q];
      }
      __syncthreads();
    }
    // ---- the weight vectors spread back through the compression, their S
    // matrices applied to c_nlm and G (:1336-1376), through the Y lists
    for (int v = 0; v < nv; ++v) {
      const double *vin = v < n_vec ? vecs + ((size_t)site * n_vec + v) * ns : pvec;
      for (int q = tid; q < P.n_kept; q += kHessThreads) {
        double s = 0.0;
        for (int t = P.pj_off[q]; t < P.pj_off[q + 1]; ++t) s = s + P.pj_el64[t] * vin[P.pj_o[t]];
        h.vk[q] = s;
      }
      __syncthreads();
      for (int it = tid; it < N * K; it += kHessThreads) {
        const int n = it / K, k = it - n * K;
        int l = 0;
        while ((l + 1) * (l + 2) / 2 <= k) ++l;
        // S(n, np, l) from the kept component (min, max, l): 2 v on the
        // diagonal, sqrt 2 v off it; the list runs over np ascending
        dcx zc = cx(0.0, 0.0), b0[3] = {cx(0.0, 0.0), cx(0.0, 0.0), cx(0.0, 0.0)};
        for (int t = P.hl_off[l * N + n]; t < P.hl_off[l * N + n + 1]; ++t) {
          const int np = P.hl_np[t];
          const double smv = P.hl_fac64[t] * h.vk[P.hl_q[t]];
          const double2 cc = c[(size_t)np * K + k];
          zc = zc + cx(smv * cc.x, smv * cc.y);
          for (int q = 0; q < 3; ++q) b0[q] = b0[q] + smv * h.Gacc[((size_t)np * K + k) * 3 + q];
        }
        h.Zv[((size_t)v * N + n) * K + k] = zc;
        for (int q = 0; q < 3; ++q) h.ZGv[(((size_t)v * N + n) * K + k) * 3 + q] = b0[q];
      }
      __syncthreads();
    }
    // ---- pass B: per pair, the contraction and the normalisation (:1378-1486)
    for (int t = tid; t < 9 * n_vec; t += kHessThreads) hsum[t] = 0.0;
    __syncthreads();
    for (int k2 = p0 + 1; k2 < p1; ++k2) {
      if (tid == 0) pair_setup(P, B, k2, true, G);
      __syncthreads();
      if (!G.good) continue;
      pair_dp(P, B, k2, rad, rad_der, ang, c, sPQ, h.kept3, h.dp2);
      for (int vb = 0; vb < nv; vb += kHessVB) {
        const int nvb = min(kHessVB, nv - vb);
        for (int it = tid; it < K * nvb; it += kHessThreads) {
          const int k = it / nvb, v = vb + (it - (it / nvb) * nvb);
          int l = 0;
          while ((l + 1) * (l + 2) / 2 <= k) ++l;
          const int m = k - l * (l + 1) / 2;
          dcx Om, dOm[3], d2Om[9];
          omega_k(G, k, l, m, (m & 1) ? -P.preflm64[k] : P.preflm64[k], true, Om, dOm, d2Om);
          dcx a0 = cx(0.0, 0.0), a1 = a0, a2 = a0, b0[3] = {a0, a0, a0}, b1[3] = {a0, a0, a0};
          for (int n = 0; n < N; ++n) {
            const double r0 = rad[(size_t)k2 * N + n], r1 = rad_der[(size_t)k2 * N + n];
            const double r2 = rad_der2[(size_t)k2 * N + n];
            const dcx zc = conjg(h.Zv[((size_t)v * N + n) * K + k]);
            a0 = a0 + r0 * zc;
            a1 = a1 + r1 * zc;
            a2 = a2 + r2 * zc;
            for (int q = 0; q < 3; ++q) {
              const dcx gc = conjg(h.ZGv[(((size_t)v * N + n) * K + k) * 3 + q]);
              b0[q] = b0[q] + r0 * gc;
              b1[q] = b1[q] + r1 * gc;
            }
          }
          const double f0 = G.Fl[l], f1 = G.Fl1[l], f2 = G.Fl2[l], wmk = (m > 0) ? 2.0 : 1.0;
          const dcx z0 = (fourpi * f0) * a0, z1 = fourpi * (f0 * a1 + f1 * a0);
          const dcx z2 = fourpi * (f0 * a2 + (2.0 * f1) * a1 + f2 * a0);
          dcx gg0[3], gg1[3];
          for (int q = 0; q < 3; ++q) {
            gg0[q] = (fourpi * f0) * b0[q];
            gg1[q] = fourpi * (f0 * b1[q] + f1 * b0[q]);
          }
          double *pk = part + ((size_t)k * kHessVB + (v - vb)) * 9;
          for (int bb = 0; bb < 3; ++bb)
            for (int aa = 0; aa < 3; ++aa) {
              dcx tE = ((G.nh[aa] * G.nh[bb]) * (z2 - G.invr * z1)) * Om + z1 * (G.nh[aa] * dOm[bb] + G.nh[bb] * dOm[aa]) +
                       z0 * d2Om[bb * 3 + aa];
              if (aa == bb) tE = tE + G.invr * (z1 * Om);
              const dcx tD = G.nh[bb] * (gg1[aa] * Om) + gg0[aa] * dOm[bb];
              pk[bb * 3 + aa] = -wmk * (tE.re + tD.re);
            }
        }
        __syncthreads();
        // the sum over k, in k order
        for (int t = tid; t < nvb * 9; t += kHessThreads) {
          const int v = t / 9, e = t - v * 9;
          double s = 0.0;
          for (int k = 0; k < K; ++k) s = s + part[((size_t)k * kHessVB + v) * 9 + e];
          hv[(vb + v) * 9 + e] = s;
        }
        __syncthreads();
      }
      // dot products of the normalisation: t1 (3), t2 (3), c12 (9), then per v wp, u1 (3), u2 (3)
      const int n_dots = 15 + 7 * n_vec;
      for (int d = warp; d < n_dots; d += n_warps) {
        double r;
        if (d < 3) r = warp_dot(pvec, 1, h.dp1 + d, 3, ns);
        else if (d < 6) r = warp_dot(pvec, 1, h.dp2 + (d - 3), 3, ns);
        else if (d < 15) r = warp_dot(h.dp1 + (d - 6) % 3, 3, h.dp2 + (d - 6) / 3, 3, ns);  // c12[b * 3 + a]
        else {
          const int v = (d - 15) / 7, e = (d - 15) % 7;
          const double *wv = vecs + ((size_t)site * n_vec + v) * ns;
          if (e == 0) r = warp_dot(wv, 1, pvec, 1, ns);
          else if (e < 4) r = warp_dot(wv, 1, h.dp1 + (e - 1), 3, ns);
          else r = warp_dot(wv, 1, h.dp2 + (e - 4), 3, ns);
        }
        if (lane == 0) dots[d] = r;
      }
      __syncthreads();
      for (int t = tid; t < 9 * n_vec; t += kHessThreads) {
        const int v = t / 9, e = t - v * 9, bb = e / 3, aa = e - bb * 3;
        const double *t1 = dots, *t2 = dots + 3, *c12 = dots + 6, *dv = dots + 15 + 7 * v;
        const double wp = dv[0], *u1 = dv + 1, *u2 = dv + 4;
        const double hval = hv[v * 9 + e] * invs - (u1[aa] * t2[bb] + u2[bb] * t1[aa]) * invs3 -
                            wp * (c12[bb * 3 + aa] + hv[n_vec * 9 + e]) * invs3 + 3.0 * wp * t1[aa] * t2[bb] * invs5;
        hess[((size_t)k2 * n_vec + v) * 9 + e] = hval;
        hsum[t] += hval;
      }
      __syncthreads();
    }
    // the self pair: minus the sum of the others (:1488-1495); pairs outside
    // every cutoff keep the zero blocks the launcher cleared
    if (p1 > p0)
      for (int t = tid; t < 9 * n_vec; t += kHessThreads) hess[((size_t)p0 * n_vec) * 9 + t] = -hsum[t];
  }
}

}  // namespace

size_t hess_scratch_doubles(const DevParams &P, int n_vec) {
  const size_t nk = (size_t)P.n_max * P.k_max, nv = (size_t)n_vec + 1;
  return 2 * (3 * nk + nv * nk + 3 * nv * nk) + 6 * (size_t)P.n_soap + 3 * (size_t)P.n_kept + (size_t)P.n_kept + 8;
}

size_t hess_smem_bytes(const DevParams &P, int n_vec) {
  const size_t N = P.n_max, K = P.k_max, L1 = P.l_max + 1, nv = (size_t)n_vec + 1;
  return sizeof(double) * (P.n_soap + 4 * N * L1 + K * kHessVB * 9 + 9 * nv + 9 * (size_t)n_vec + 15 + 7 * (size_t)n_vec);
}

int hess_grid(const DevParams &P, int n_vec) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k64_hess, kHessThreads, hess_smem_bytes(P, n_vec));
  return sms * (per_sm > 0 ? per_sm : 1);
}

cudaError_t launch_hessian(const DevParams &P, const DevBatch &B, cudaStream_t s, const Fp64Work &w,
                           const double *rad_der2, const double *soap, int n_vec, const double *vecs, double *hess,
                           double *scratch, int grid, int *ticket, int *launches) {
  CU_RET(cudaMemsetAsync(hess, 0, sizeof(double) * 9 * (size_t)n_vec * B.n_pairs, s));
  CU_RET(cudaMemsetAsync(ticket, 0, sizeof(int), s));
  if (B.n_pairs > 0) {
    const int blocks = (B.n_pairs + 127) / 128;
    int amax = 0;
    for (int sp = 0; sp < P.n_species; ++sp) amax = amax > P.rad[sp].alpha ? amax : P.rad[sp].alpha;
    if (amax <= 8) k64_radial_d2<8><<<blocks, 128, 0, s>>>(P, B, (double *)rad_der2);
    else k64_radial_d2<16><<<blocks, 128, 0, s>>>(P, B, (double *)rad_der2);
    if (launches) *launches += 1;
  }
  if (B.n_sites > 0) {
    const size_t sm = hess_smem_bytes(P, n_vec);
    cudaError_t e = cudaFuncSetAttribute(k64_hess, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const int g = grid < B.n_sites ? grid : B.n_sites;
    k64_hess<<<g, kHessThreads, sm, s>>>(P, B, w.rad, w.rad_der, rad_der2, (const double2 *)w.ang,
                                        (const double2 *)w.cnk, w.norm, soap, n_vec, vecs, hess, scratch,
                                        hess_scratch_doubles(P, n_vec), ticket);
    if (launches) *launches += 1;
  }
  return cudaGetLastError();
}

}  // namespace soapb
