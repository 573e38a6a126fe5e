// soapb_device.cuh -- per-pair device math shared by the mixed-precision and
// the plain-FP64 kernels.
//
// radial_entry: the poly3 / poly3gauss radial expansion of one (pair, species)
// entry (src/soap_turbo_radial.f90:550-1002), in FP64.  The basis matrix W has
// norm ~1e6 and the primitive overlaps cancel against it, so this part cannot
// run in FP32 (a 3e-2 relative error at alpha = 8); it is a few hundred FP64
// operations per entry.  Instead of the reference's block buffers it streams
// over alpha: the two overlap recursions advance together, each polynomial
// value is folded into the W-transform accumulators as it appears, and the
// derivative DT(m) is formed two steps later from a three-value window.  The
// summation order of every W-transform is the reference's (m ascending, the
// origin Gaussian last).
//
// angular_scalars: the per-pair FP64 inputs of the angular expansion
// (src/soap_turbo_angular.f90:267-463, 578-589): i_l(x^2)e^{-x^2} and its
// radial derivative, e^{-i m phi} by the reference's Chebyshev recursion, the
// amplitude rcut_max^2/sigma_t^2 and cos/sin theta.
#pragma once

#include "soapb_internal.h"

namespace soapb {

// Recursion table index for alpha index n (n >= -4).
#define SOAPB_TI(n) ((n) + 4)

// ---------------------------------------------------------------- poly3operator
// The poly3operator radial expansion of one (pair, species) entry
// (get_radial_expansion_coefficients_poly3operator, src/soap_turbo_radial.f90:
// 1549-2141, helpers :2154-2557), in FP64.  The atom density is the piecewise
// cubic g(x) = 1 - 3x^2 -+ 2x^3 of x = (r - r_j)/w on [-1, 0] and [0, 1],
// w = 2 sqrt(2 ln 2) sigma(r_j); on [r_soft, r_hard] it is multiplied by the
// filter, the right piece centred at r_soft with width 2 sqrt(2 ln 2)(r_hard -
// r_soft).  Its overlaps with (1 - r)^(n+2) sqrt(2n + 5) (r_hard = 1 after
// scaling) are closed forms by repeated integration by parts: for a piece P
// of degree d between lo and hi,
//   I_n = sum_{j=1..d+1} A(n, j) [-(1 - r)^(n+2+j) P^(j-1)(r)]_lo^hi,
//   A(n, 1) = sqrt(2n + 5)/(n + 3), A(n, j) = A(n, j-1)/(n + 2 + j).
// The derivative differentiates the density in r_j (with w growing with r_j);
// the moving limits add nothing (g vanishes at x = -1, 1 and is continuous at 0).

// Taylor coefficients about r of a piece (value, slope, half the curvature, a
// sixth of the third derivative) and their r0-derivatives (g_aux, g_aux_der_array)
__device__ __forceinline__ void op_piece(double r, double r0, double w, bool right, double *c) {
  const double x = (r - r0) / w, iw = 1.0 / w;
  const double sg = right ? 1.0 : -1.0;
  c[0] = 1.0 - 3.0 * x * x + sg * 2.0 * x * x * x;
  c[1] = 6.0 * (sg * x * x - x) * iw;
  c[2] = 3.0 * (sg * 2.0 * x - 1.0) * iw * iw;
  c[3] = sg * 2.0 * iw * iw * iw;
}
__device__ __forceinline__ void op_piece_d(double r, double r0, double w, double ws, bool right, double *c) {
  const double x = (r - r0) / w, iw = 1.0 / w, iw2 = iw * iw;
  const double sg = right ? 1.0 : -1.0;  // right: (ws - 1), left: (ws + 1)
  c[0] = 6.0 * (x + (ws - sg) * x * x - sg * ws * x * x * x) * iw;
  c[1] = 6.0 * (1.0 + 2.0 * (ws - sg) * x - 3.0 * sg * ws * x * x) * iw2;
  c[2] = 6.0 * (ws - sg - 3.0 * sg * ws * x) * iw2 * iw;
  c[3] = -sg * 6.0 * ws * iw2 * iw2;
}

// Adds I_n of one piece, given -P^(j-1)(lim)(1 - lim)^(j-1) at both limits
// (ml, mh, nj terms), scaled by f, to acc[n].
template <int AMAX>
__device__ __forceinline__ void op_accumulate(int a, double lo, double hi, const double *ml, const double *mh,
                                              int nj, double f, double (&acc)[AMAX]) {
  double pl = (1.0 - lo) * (1.0 - lo), ph = (1.0 - hi) * (1.0 - hi);
  pl = pl * pl;  // (1 - lim)^(n + 3) at n = 1
  ph = ph * ph;
#pragma unroll
  for (int i = 0; i < AMAX; ++i) {
    if (i < a) {
      const int n = i + 1;
      double An = sqrt((double)(2 * n + 5)) / (double)(n + 3);
      double sh = 0.0, sl = 0.0;
      for (int j = 0; j < nj; ++j) {
        if (j > 0) An = An / (double)(n + 3 + j);
        sh += mh[j] * An;
        sl += ml[j] * An;
      }
      acc[i] += f * (sh * ph - sl * pl);
      pl *= (1.0 - lo);
      ph *= (1.0 - hi);
    }
  }
}

// Soft zone: a cubic piece given by its Taylor coefficients at the two limits
// (the table's -1, -1, -2, -6 factors turn them into derivatives with the sign).
__device__ __forceinline__ void op_soft_terms(double lim, const double *c, double *m) {
  const double q = 1.0 - lim;
  m[0] = -c[0];
  m[1] = -c[1] * q;
  m[2] = -2.0 * c[2] * q * q;
  m[3] = -6.0 * c[3] * q * q * q;
}

// Buffer zone: B = (piece) x (filter) as monomials about r = 0, degree 6; m[d] =
// -B^(d)(lim) (1 - lim)^d for d = 0..6.
__device__ __forceinline__ void op_buffer_terms(double lim, const double *B, double *m) {
  const double q = 1.0 - lim;
  double qd = 1.0;
  for (int d = 0; d < 7; ++d) {
    double v = 0.0;
    for (int p = 6; p >= d; --p) {  // Horner on the d-th derivative
      double f = 1.0;
      for (int t = p - d + 1; t <= p; ++t) f *= (double)t;
      v = v * lim + B[p] * f;
    }
    m[d] = -v * qd;
    qd *= q;
  }
}

__device__ __forceinline__ void op_product(const double *col, const double *C, double *B) {
  for (int m = 0; m < 7; ++m) B[m] = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int q = 0; q < 4; ++q) B[i + q] += col[q] * C[i];
}

template <int AMAX>
__device__ __forceinline__ void radial_entry_op(const DevParams &P, const RadSp &S, const double *__restrict__ W,
                                                double r_in, bool is_central, bool do_der, double (&val)[AMAX],
                                                double (&der)[AMAX]) {
  const double c_w = 2.3548200450309493820;  // 2 sqrt(2 ln 2)
  const double sq2pi = 0.79788456080286535588, sq8pi = 1.5957691216057307118;
  const int a = S.alpha;
  const double rs = S.rs, c = S.c;
  const double rj = r_in * S.inv_rcut, sig = S.atom_sigma + c * rj, w = c_w * sig, ws = c_w * c;
  const double filter_width = c_w * (1.0 - rs);
  double e[AMAX], ed[AMAX];
#pragma unroll
  for (int i = 0; i < AMAX; ++i) {
    e[i] = 0.0;
    ed[i] = 0.0;
  }
  // amplitude (:1699-1757); not polynomial scaling: 1 (the reference leaves it unset)
  double amp = 1.0, ampd = 0.0;
  if (P.scaling_poly) {
    if (S.amp_scaling == 0.0) {
      amp = 1.0 / sig;
      ampd = -c / (sig * sig);
    } else if (S.amp_scaling == 1.0) {
      amp = 1.0 / sig * (1.0 + 2.0 * rj * rj * rj - 3.0 * rj * rj);
      ampd = 6.0 / sig * (rj * rj - rj) - c / sig * amp;
    } else {
      const double h = 1.0 + 2.0 * rj * rj * rj - 3.0 * rj * rj;
      amp = 1.0 / sig * pow(h, S.amp_scaling);
      ampd = 6.0 * S.amp_scaling / sig * (rj * rj - rj) * pow(h, S.amp_scaling - 1.0) - c / sig * amp;
    }
  }
  if (is_central) {
    amp *= S.cw;
    ampd *= S.cw;
  }
  if (P.radial_enh == 1) {
    ampd = amp * (1.0 + sq2pi * c) + ampd * (rj + sq2pi * sig);
    amp = amp * (rj + sq2pi * sig);
  } else if (P.radial_enh == 2) {
    ampd = amp * (2.0 * rj + 2.0 * sig * c + sq8pi * sig + sq8pi * rj * c) +
           ampd * (rj * rj + sig * sig + sq8pi * sig * rj);
    amp = amp * (rj * rj + sig * sig + sq8pi * sig * rj);
  }
  double m0[7], m1[7], cc[4];
  if (rj - w < rs) {  // soft zone (:1637-1645, 1770-1846)
    const double l1 = fmax(0.0, rj - w), l2 = fmin(rj, rs), l3 = fmin(rs, rj + w);
    op_piece(l1, rj, w, false, cc); op_soft_terms(l1, cc, m0);
    op_piece(l2, rj, w, false, cc); op_soft_terms(l2, cc, m1);
    op_accumulate<AMAX>(a, l1, l2, m0, m1, 4, 1.0, e);
    op_piece(l2, rj, w, true, cc); op_soft_terms(l2, cc, m0);
    op_piece(l3, rj, w, true, cc); op_soft_terms(l3, cc, m1);
    op_accumulate<AMAX>(a, l2, l3, m0, m1, 4, 1.0, e);
    if (do_der) {
      op_piece_d(l1, rj, w, ws, false, cc); op_soft_terms(l1, cc, m0);
      op_piece_d(l2, rj, w, ws, false, cc); op_soft_terms(l2, cc, m1);
      op_accumulate<AMAX>(a, l1, l2, m0, m1, 4, 1.0, ed);
      op_piece_d(l2, rj, w, ws, true, cc); op_soft_terms(l2, cc, m0);
      op_piece_d(l3, rj, w, ws, true, cc); op_soft_terms(l3, cc, m1);
      op_accumulate<AMAX>(a, l2, l3, m0, m1, 4, 1.0, ed);
    }
  }
  if (rs < 1.0 && rj + w > rs) {  // buffer zone (:1858-2075)
    const double l1 = fmax(rs, rj - w), l2 = fmax(rj, rs), l3 = fmin(1.0, rj + w);
    double C[4], B[7];
    op_piece(0.0, rs, filter_width, true, C);
    for (int pc = 0; pc < (do_der ? 4 : 2); ++pc) {
      const bool right = pc & 1, dv = pc >= 2;
      if (dv) op_piece_d(-rj, 0.0, w, ws, right, cc);
      else op_piece(-rj, 0.0, w, right, cc);
      op_product(cc, C, B);
      const double lo = right ? l2 : l1, hi = right ? l3 : l2;
      op_buffer_terms(lo, B, m0);
      op_buffer_terms(hi, B, m1);
      if (dv) op_accumulate<AMAX>(a, lo, hi, m0, m1, 7, 1.0, ed);
      else op_accumulate<AMAX>(a, lo, hi, m0, m1, 7, 1.0, e);
    }
  }
  // W-transform (:2097-2100) and the change of variable (:2113-2117)
#pragma unroll
  for (int i = 0; i < AMAX; ++i) {
    val[i] = 0.0;
    der[i] = 0.0;
  }
#pragma unroll
  for (int m = 0; m < AMAX; ++m) {
    if (m < a) {
      const double *Wc = W + m * a;
      const double em = amp * e[m], dm = amp * ed[m] + ampd * e[m];
#pragma unroll
      for (int i = 0; i < AMAX; ++i)
        if (i < a) {
          val[i] = val[i] + Wc[i] * em;
          der[i] = der[i] + Wc[i] * dm;
        }
    }
  }
#pragma unroll
  for (int i = 0; i < AMAX; ++i) {
    val[i] = val[i] * S.sqrt_rcut;
    der[i] = der[i] * S.inv_sqrt_rcut;
  }
}

// OP: the poly3operator basis (a separate instantiation, so that the poly3 and
// poly3gauss kernels are compiled without its code).  The poly3 / poly3gauss
// form also runs on the host, which fits the pair kernel's radial tables to it.
template <int AMAX, bool OP = false>
__host__ __device__ __forceinline__ void radial_entry(const DevParams &P, const RadSp &S,
                                             const double *__restrict__ W, double r_in,
                                             bool is_central, bool do_der, double (&val)[AMAX],
                                             double (&der)[AMAX]) {
  if constexpr (OP) {
    radial_entry_op<AMAX>(P, S, W, r_in, is_central, do_der, val, der);
    return;
  }
  const double sqpi2 = 1.2533141373155002512, isq2 = 0.70710678118654752440;
  const double sq2pi = 0.79788456080286535588, sq8pi = 1.5957691216057307118;
  const int a = S.alpha;
  const int n_poly = S.n_poly;
  const int n_hi = n_poly + (do_der ? 2 : 0);
  const bool unified = !P.legacy_seed;
  const double c = S.c, rs = S.rs, dr = S.dr;
  const double rj = r_in * S.inv_rcut;

  const double sig = S.atom_sigma + c * rj, s2 = sig * sig;             // :560-570
  const double isig = 1.0 / sig, is2 = isig * isig, is3 = is2 * isig;

  double amp, ampd;                                                      // :589-635
  if (!P.scaling_poly) {
    amp = 1.0;
    ampd = 0.0;
  } else if (S.amp_scaling == 0.0) {
    amp = isig;
    ampd = -c * is2;
  } else {
    const double h = 1.0 + 2.0 * (rj * rj * rj) - 3.0 * rj * rj;
    const double hp = 6.0 * rj * rj - 6.0 * rj;
    if (h <= 1.0e-10) {
      amp = 0.0;
      ampd = 0.0;
    } else if (S.amp_scaling == 1.0) {
      const double g = isig * h;
      amp = g;
      ampd = hp * isig - c * isig * g;
    } else {
      const double aa = S.amp_scaling;
      amp = isig * pow(h, aa);
      ampd = aa * pow(h, aa - 1.0) * hp * isig - c * isig * amp;
    }
  }
  if (S.do_central && S.cw != 1.0 && is_central) {                      // :638-646
    amp *= S.cw;
    ampd *= S.cw;
  }
  if (P.radial_enh == 1) {                                               // :651-670
    const double g = rj + sq2pi * sig, f = 1.0 + sq2pi * c;
    ampd = amp * f + ampd * g;
    amp = amp * g;
  } else if (P.radial_enh == 2) {
    const double g = rj * rj + s2 + sq8pi * sig * rj;
    const double f = 2.0 * rj + 2.0 * sig * c + sq8pi * sig + sq8pi * rj * c;
    ampd = amp * f + ampd * g;
    amp = amp * g;
  }

  // Overlap with the atom Gaussian on [0, rcut_soft], seeded by erf (:676-686)
  const double es = exp(-0.5 * (rs - rj) * (rs - rj) * is2);
  const double e0 = exp(-0.5 * rj * rj * is2);
  double C1 = s2 * es;
  const double C2 = s2 * e0;
  double t1m2 = 0.0;
  double t1m1 = sqpi2 * sig * (erf((rs - rj) * isq2 * isig) + erf(rj * isq2 * isig));  // inv_Nm2 = 1

  // Gaussian filter on [rcut_soft, rcut_hard] (:721-769)
  const bool filt = S.has_filter != 0;
  double pref = 0.0, sf2 = 0.0, rjf = 0.0, isf2 = 0.0, C2f = 0.0, t2m2 = 0.0, t2m1 = 0.0;
  double iD = 0.0, sqiD = 0.0, sgf = 0.0, isgf = 0.0;
  if (filt) {
    const double q = S.q, drnf = S.drnf;
    iD = 1.0 / (s2 + q);
    sqiD = sqrt(iD);
    sgf = sig * drnf * sqiD;
    rjf = (s2 * rs + q * rj) * iD;
    sf2 = sgf * sgf;
    const bool keep = (rs - rj) < 4.0 * sig;
    isgf = 1.0 / sgf;
    isf2 = isgf * isgf;
    pref = keep ? exp(-0.5 * (rs - rj) * (rs - rj) * iD) : 0.0;
    C2f = sf2 * exp(-0.5 * (rs - rjf) * (rs - rjf) * isf2);
    t2m1 = sqpi2 * sgf * (erf((1.0 - rjf) * isq2 * isgf) - erf((rs - rjf) * isq2 * isgf));
  }

  // Derivative coefficients (legacy :701-713, :774-788; unified :825-831)
  double g0 = 0, g1 = 0, g2 = 0;           // unified
  double ca = 0, cb = 0, cc = 0;           // legacy, inner piece
  double ca2 = 0, cb2 = 0, cc2 = 0, dpref = 0;  // legacy, filter piece
  if (do_der) {
    if (unified) {
      const double f = 1.0 - rj;
      g0 = f * is2 + c * f * f * is3;
      g1 = -(is2 + 2.0 * c * f * is3);
      g2 = c * is3;
    } else {
      const double f = rj - 1.0, g = c * f * isig;
      ca = f * is2 * (g - 1.0);
      cb = is2 * (2.0 * g - 1.0);
      cc = c * is3;
      if (filt) {
        const double q = S.q;
        const double fs = rs - rj;
        dpref = pref * (fs * iD + fs * fs * iD * iD * sig * c);
        const double drjf = (2.0 * sig * rs * c + q) * iD - (s2 * rs + q * rj) * 2.0 * sig * c * iD * iD;
        const double dsgf = c * S.drnf * sqiD * (1.0 - s2 * iD);
        const double ff = rjf - 1.0, gg = dsgf * ff * isgf;
        ca2 = pref * ff * isf2 * (gg - drjf);
        cb2 = pref * isf2 * (2.0 * gg - drjf);
        cc2 = pref * dsgf * isgf * isf2;
      }
    }
  }

#pragma unroll
  for (int i = 0; i < AMAX; ++i) {
    val[i] = 0.0;
    der[i] = 0.0;
  }
  double p0 = 0, p1 = 0, p2 = 0;  // pol window (n-2, n-1, n)
  double q0 = 0, q1 = 0, q2 = 0;  // T1 window
  double z0 = 0, z1 = 0, z2 = 0;  // T2 window

#pragma unroll 1
  for (int n = -1; n <= n_hi; ++n) {                                     // :688-698, :751-770
    if (n >= 0) {
      C1 = C1 * dr;
      C2f = C2f * dr;
    }
    const double t1 = s2 * P.ra[SOAPB_TI(n)] * t1m2 - P.rb[SOAPB_TI(n)] * (rj - 1.0) * t1m1 +
                      (C1 - C2) * P.rc[SOAPB_TI(n)];
    double t2 = 0.0;
    if (filt) {
      t2 = sf2 * P.ra[SOAPB_TI(n)] * t2m2 - P.rb[SOAPB_TI(n)] * (rjf - 1.0) * t2m1 -
           C2f * P.rc[SOAPB_TI(n)];
      if (n == -1 && unified)
        t2 = t2 + sf2 * exp(-0.5 * (1.0 - rjf) * (1.0 - rjf) * isf2) * P.rc[SOAPB_TI(-1)];
    }
    t1m2 = t1m1;
    t1m1 = t1;
    t2m2 = t2m1;
    t2m1 = t2;
    if (n < 1) continue;
    const double pol = t1 + pref * t2;                                   // :808-812
    p0 = p1; p1 = p2; p2 = pol;
    q0 = q1; q1 = q2; q2 = t1;
    z0 = z1; z1 = z2; z2 = t2;
    if (n <= n_poly) {                                                   // :962-976
      const double *Wc = W + (n - 1) * a;
#pragma unroll
      for (int i = 0; i < AMAX; ++i)
        if (i < a) val[i] = val[i] + Wc[i] * pol;
    }
    if (do_der && n >= 3) {                                              // :911-942
      const int m = n - 2;
      double DT;
      if (unified) {
        DT = g0 * p0 + P.R1[SOAPB_TI(m)] * g1 * p1 + P.R2[SOAPB_TI(m)] * g2 * p2;
      } else {
        DT = ca * q0 + P.R1[SOAPB_TI(m)] * cb * q1 + P.R2[SOAPB_TI(m)] * cc * q2;
        if (filt)
          DT = DT + ca2 * z0 + P.R1[SOAPB_TI(m)] * cb2 * z1 + P.R2[SOAPB_TI(m)] * cc2 * z2 + dpref * z0;
      }
      const double dtot = amp * DT + ampd * p0;
      const double *Wc = W + (m - 1) * a;
#pragma unroll
      for (int i = 0; i < AMAX; ++i)
        if (i < a) der[i] = der[i] + Wc[i] * dtot;
    }
  }

  if (P.basis == 1) {                                                    // :875-908
    const double ss2 = S.sigma_sq0 + s2, iss = 1.0 / ss2, siss = sqrt(iss);
    const bool gm = rj < 4.0 * (S.atom_sigma + sig);
    const double ge = gm ? S.N_gauss * e0 : 0.0;
    const double M0 = gm ? exp(-0.5 * rj * rj * iss) * sqpi2 * sig * S.atom_sigma * siss *
                               (1.0 + erf(S.atom_sigma * isig * rj * isq2 * siss)) * S.N_gauss
                         : 0.0;
    const double *Wc = W + (a - 1) * a;
#pragma unroll
    for (int i = 0; i < AMAX; ++i)
      if (i < a) val[i] = val[i] + Wc[i] * M0;
    if (do_der) {
      const double sc0 = S.sigma_sq0 * s2 * iss, pp = s2 * rj * iss;
      const double M1 = sc0 * ge - pp * M0;
      const double M2 = sc0 * ge * (-rj) - pp * M1 + sc0 * M0;
      const double dtot = amp * (M1 * is2 + c * M2 * is3) + ampd * M0;
#pragma unroll
      for (int i = 0; i < AMAX; ++i)
        if (i < a) der[i] = der[i] + Wc[i] * dtot;
    }
  }

#pragma unroll
  for (int i = 0; i < AMAX; ++i) {
    val[i] = amp * val[i] * S.sqrt_rcut;
    der[i] = der[i] * S.inv_sqrt_rcut;
  }
}

// ---------------------------------------------------------------- radial tables
// The branch state of a (pair, species) entry at distance r, by the same FP64
// tests as radial_entry (sigma constant: atom_sigma_r_scaling = 0); -1 where
// the amplitude is zero (h(r) <= 1e-10), which makes R_n and dR_n/dr zero.
__host__ __device__ __forceinline__ int radial_branch(const DevParams &P, const RadSp &S, double r_in) {
  const double rj = r_in * S.inv_rcut;
  const double sig = S.atom_sigma + S.c * rj;
  if (P.scaling_poly && S.amp_scaling != 0.0) {
    const double h = 1.0 + 2.0 * (rj * rj * rj) - 3.0 * rj * rj;
    if (h <= 1.0e-10) return -1;
  }
  const bool keep = S.has_filter != 0 && (S.rs - rj) < 4.0 * sig;
  const bool gm = P.basis != 1 || rj < 4.0 * (S.atom_sigma + sig);
  return (keep ? 1 : 0) | (gm ? 0 : 2);
}

// R_n (out[0..AMAX)) and, with do_der, dR_n/dr (out[AMAX..2 AMAX)) of one entry
// from its species' table, 4 pi global_scaling included: the segment and its
// local coordinate t in FP64, the polynomial by Horner in FP32.
// The entry's segment: the offset of its coefficients in rtab_coef (floats;
// -1 where R_n and dR_n/dr are zero) and its local coordinate t in [-1, 1].
template <int AMAX>
__device__ __forceinline__ int radial_table_locate(const DevParams &P, const RadSp &S, const RadTab &T, double r,
                                                   float &t) {
  const int st = radial_branch(P, S, r);
  t = 0.f;
  if (st < 0) return -1;
  const double u = (r - T.lo[st]) * T.inv_h[st];
  int seg = (int)floor(u);
  seg = seg < 0 ? 0 : (seg >= T.nseg[st] ? T.nseg[st] - 1 : seg);
  t = (float)(2.0 * (u - (double)seg) - 1.0);
  return (T.base[st] + seg) * (kRadTabDeg + 1) * 2 * AMAX;
}

template <int AMAX>
__device__ __forceinline__ void radial_from_table(const DevParams &P, const RadSp &S, const RadTab &T,
                                                  double r, bool do_der, float (&out)[2 * AMAX]) {
  float t;
  const int cb = radial_table_locate<AMAX>(P, S, T, r, t);
  if (cb < 0) {
#pragma unroll
    for (int f = 0; f < 2 * AMAX; ++f) out[f] = 0.f;
    return;
  }
  const float4 *c4 = (const float4 *)(P.rtab_coef + cb);
  constexpr int F4 = 2 * AMAX / 4;
  const int nf4 = do_der ? F4 : F4 / 2;
#pragma unroll
  for (int j = 0; j < F4; ++j) {
    if (j < nf4) {
      float4 a = c4[kRadTabDeg * F4 + j];
#pragma unroll
      for (int k = kRadTabDeg - 1; k >= 0; --k) {
        const float4 b = c4[k * F4 + j];
        a.x = fmaf(a.x, t, b.x);
        a.y = fmaf(a.y, t, b.y);
        a.z = fmaf(a.z, t, b.z);
        a.w = fmaf(a.w, t, b.w);
      }
      out[4 * j] = a.x;
      out[4 * j + 1] = a.y;
      out[4 * j + 2] = a.z;
      out[4 * j + 3] = a.w;
    } else {
      out[4 * j] = out[4 * j + 1] = out[4 * j + 2] = out[4 * j + 3] = 0.f;
    }
  }
}

// ---------------------------------------------------------------- angular
template <int LC>
struct AngScalars {
  double il[LC + 2];   // i_l(x^2) exp(-x^2), l = 0..LC+1
  double ild[LC + 1];  // its radial derivative
  double er[LC + 1], ei[LC + 1];  // e^{-i m phi} = cos(m phi) - i sin(m phi)
  double amp;          // rcut_max^2 / sigma_t^2
  double sig_fac;      // 2 sigma_t_scaling / sigma_t
  double x, sq;        // cos(theta), sqrt(1 - x^2)
};

// get_ilexp (src/soap_turbo_angular.f90:361-422) for l = 0..lmax
template <int LC>
__device__ __forceinline__ void ilexp_array(int lmax, double x, double (&out)[LC + 2]) {
  const double xcut = 1.0e-7;
  const double x2 = x * x, x4 = x2 * x2;
  const double inv_x2 = (x2 > 0.0) ? 1.0 / x2 : 0.0;
  double x2pow = x2 * x2;
  double flm2, flm1;
  if (x > 0.0) {
    const double e2 = exp(-2.0 * x2);
    flm2 = fabs((1.0 - e2) / 2.0 / x2);
    flm1 = fabs((x2 - 1.0 + e2 * (x2 + 1.0)) / 2.0 / x4);
  } else {
    flm2 = 1.0;
    flm1 = 0.0;
  }
  double fact = 1.0;
#pragma unroll
  for (int l = 0; l < LC + 2; ++l) {
    if (l > lmax) {
      out[l] = 0.0;
      continue;
    }
    if (l > 0) fact = fact * (2.0 * (double)l + 1.0);
    if (l == 0) {
      out[0] = (x < xcut) ? 1.0 - x2 : flm2;
    } else if (l == 1) {
      out[1] = (x2 / 1000.0 < xcut) ? (x2 - x4) / fact : flm1;
    } else {
      const double ratio = x2pow / fact;
      double fl;
      if (ratio * (double)l < xcut)
        fl = ratio;
      else
        fl = fabs(flm2 - (2.0 * (double)l - 1.0) * inv_x2 * flm1);
      x2pow = x2pow * x2;
      flm2 = flm1;
      flm1 = fl;
      out[l] = fl;
    }
  }
}

template <int LC>
__device__ __forceinline__ void angular_scalars(const DevParams &P, int i_sp, double rj,
                                                double theta, double phi, bool do_der,
                                                AngScalars<LC> &A) {
  const int L = P.l_max;
  const double sig = P.sig_t[i_sp] + P.sig_t_c[i_sp] * rj;               // :579-580
  A.amp = P.rcut2 / (sig * sig);
  A.x = cos(theta);
  A.sq = sqrt(1.0 - A.x * A.x);
  ilexp_array<LC>(L + 1, rj / sig, A.il);
  // e^{-i m phi}, Chebyshev recursion of get_eimphi_conjg (:284-298)
  double cosm2 = cos(phi), sinm2 = -sin(phi);
  const double cosphi2 = 2.0 * cosm2;
  double cosm1 = 1.0, sinm1 = 0.0;
  A.er[0] = 1.0;
  A.ei[0] = 0.0;
#pragma unroll
  for (int l = 1; l <= LC; ++l) {
    const double cos0 = cosphi2 * cosm1 - cosm2, sin0 = cosphi2 * sinm1 - sinm2;
    cosm2 = cosm1;
    sinm2 = sinm1;
    cosm1 = cos0;
    sinm1 = sin0;
    A.er[l] = cos0;
    A.ei[l] = -sin0;
  }
  A.sig_fac = 0.0;
  if (do_der) {                                                          // :436-463
    const double sc = P.sig_t_c[i_sp];
    const double c1 = 2.0 * rj / (sig * sig), c2 = 1.0 - sc * rj / sig;
#pragma unroll
    for (int l = 0; l <= LC; ++l) A.ild[l] = 0.0;
    if (rj >= 1.0e-5) {
      A.ild[0] = c1 * (A.il[1] - A.il[0]) * c2;
#pragma unroll
      for (int l = 1; l <= LC; ++l)
        if (l <= L) A.ild[l] = ((-c1 - (double)(2 * l + 2) / rj) * A.il[l] + c1 * A.il[l - 1]) * c2;
    }
    A.sig_fac = 2.0 * sc / sig;                                          // :589
  }
}

// Associated Legendre P_l^m(x) for l = 0..lmax (get_plm_array,
// src/soap_turbo_angular.f90:108-160), k = l(l+1)/2 + m.  T is float or double.
template <int LC, typename T>
__device__ __forceinline__ void plm_array(int lmax, T x, T sq, T (&p)[(LC + 1) * (LC + 2) / 2]) {
  const T x2 = x * x;
#pragma unroll
  for (int k = 0; k < (LC + 1) * (LC + 2) / 2; ++k) p[k] = T(0);
  p[0] = T(1);
  if (LC >= 1) {
    p[1] = x;
    p[2] = -sq;
  }
  if (LC >= 2) {
    p[3] = T(1.5) * x2 - T(0.5);
    p[4] = T(-3) * x * sq;
    p[5] = T(3) - T(3) * x2;
  }
#pragma unroll
  for (int l = 3; l <= LC; ++l) {
    if (l > lmax) break;
#pragma unroll
    for (int m = 0; m <= l - 2; ++m) {
      const int k = l * (l + 1) / 2 + m;
      const T aa = T(2 * l - 1) / T(l - m);
      const T bb = T(l - 1 + m) / T(l - m);
      p[k] = aa * x * p[k - l] - bb * p[k - 2 * l + 1];
    }
    const int k1 = l * (l + 1) / 2 + l - 1;
    p[k1] = x * T(2 * l - 1) * p[k1 - l];
    p[k1 + 1] = -T(2 * l - 1) * sq * p[k1 - l];
  }
}

// ---------------------------------------------------------------- streamed angular stage
// The same quantities as angular_scalars, written in FP32 to `out` as each one
// appears so that only the last two terms of each recursion are live in FP64.
// The amplitude rcut_max^2 / sigma_t^2 is folded into i_l and its derivative:
//   out[o_il + l] = amp i_l, out[o_ild + l] = amp d i_l / dr (DER),
//   out[o_er + m], out[o_ei + m], out[o_amp] = amp, out[o_sf];
// cos(theta) and sqrt(1 - cos^2) are returned in x, sq.
template <int LC, bool DER>
__device__ __forceinline__ void angular_stage(const DevParams &P, int i_sp, double rj, double theta,
                                              double phi, float *out, int o_il, int o_ild, int o_er,
                                              int o_ei, int o_amp, int o_sf, double &x, double &sq) {
  // The pair kernel rounds everything below to FP32, so the quotients of the
  // reference's expressions are taken as products with one reciprocal each of
  // sigma, x^2 and r (an FP64 division is a long dependent sequence; these are
  // the kernel's critical path), which moves the FP64 values by an ulp or so.
  const int L = P.l_max;
  const double sig = P.sig_t[i_sp] + P.sig_t_c[i_sp] * rj;               // :579-580
  const double isig = 1.0 / sig;
  const double amp = P.rcut2 * (isig * isig);
  out[o_amp] = (float)amp;
  x = cos(theta);
  sq = sqrt(1.0 - x * x);
  // i_l(x^2) exp(-x^2) (src/soap_turbo_angular.f90:361-422) and its radial
  // derivative (:436-463), streamed over l
  const double xx = rj * isig;
  const double xcut = 1.0e-7;
  const double x2 = xx * xx, x4 = x2 * x2;
  const double inv_x2 = (x2 > 0.0) ? 1.0 / x2 : 0.0;
  double x2pow = x2 * x2;
  double flm2, flm1;
  if (xx > 0.0) {
    const double e2 = exp(-2.0 * x2);
    flm2 = fabs((1.0 - e2) * 0.5 * inv_x2);
    flm1 = fabs((x2 - 1.0 + e2 * (x2 + 1.0)) * 0.5 * (inv_x2 * inv_x2));
  } else {
    flm2 = 1.0;
    flm1 = 0.0;
  }
  const double sc = P.sig_t_c[i_sp];
  const double c1 = 2.0 * rj * (isig * isig), c2 = 1.0 - sc * rj * isig;
  const bool dz = !(rj >= 1.0e-5);
  const double irj = dz ? 0.0 : 1.0 / rj;  // one division for every l below
  double fact = 1.0, il_prev = 0.0, il0 = 0.0;
#pragma unroll
  for (int l = 0; l <= LC + 1; ++l) {
    if (l > L + 1) break;
    if (l > 0) fact = fact * (2.0 * (double)l + 1.0);
    double il;
    if (l == 0) {
      il = (xx < xcut) ? 1.0 - x2 : flm2;
    } else if (l == 1) {
      il = (x2 / 1000.0 < xcut) ? (x2 - x4) / fact : flm1;
    } else {
      const double ratio = x2pow / fact;
      double fl;
      if (ratio * (double)l < xcut)
        fl = ratio;
      else
        fl = fabs(flm2 - (2.0 * (double)l - 1.0) * inv_x2 * flm1);
      x2pow = x2pow * x2;
      flm2 = flm1;
      flm1 = fl;
      il = fl;
    }
    if (l <= LC) out[o_il + l] = (float)(amp * il);
    if (DER) {
      if (l == 0) il0 = il;
      if (l == 1 && L >= 0) out[o_ild + 0] = dz ? 0.f : (float)(amp * (c1 * (il - il0) * c2));
      if (l >= 1 && l <= L && l <= LC)
        out[o_ild + l] =
            dz ? 0.f : (float)(amp * (((-c1 - (double)(2 * l + 2) * irj) * il + c1 * il_prev) * c2));
    }
    il_prev = il;
  }
  if (DER) out[o_sf] = (float)(2.0 * sc * isig);                         // :589
  // e^{-i m phi}, Chebyshev recursion of get_eimphi_conjg (:284-298)
  double sphi, cphi;
  sincos(phi, &sphi, &cphi);
  double cosm2 = cphi, sinm2 = -sphi;
  const double cosphi2 = 2.0 * cosm2;
  double cosm1 = 1.0, sinm1 = 0.0;
  out[o_er] = 1.f;
  out[o_ei] = 0.f;
#pragma unroll
  for (int l = 1; l <= LC; ++l) {
    const double cos0 = cosphi2 * cosm1 - cosm2, sin0 = cosphi2 * sinm1 - sinm2;
    cosm2 = cosm1;
    sinm2 = sinm1;
    cosm1 = cos0;
    sinm1 = sin0;
    out[o_er + l] = (float)cos0;
    out[o_ei + l] = (float)(-sin0);
  }
}

// P_l^m(x) for l = 0..lmax row by row (get_plm_array,
// src/soap_turbo_angular.f90:108-160), keeping two rows in registers and
// handing each value to emit(k, value) with k = l(l+1)/2 + m.
template <int LC, typename Emit>
__device__ __forceinline__ void plm_rows(int lmax, float x, float sq, Emit emit) {
  float rm2[LC + 1], rm1[LC + 1], cur[LC + 1];
#pragma unroll
  for (int m = 0; m <= LC; ++m) rm2[m] = rm1[m] = cur[m] = 0.f;
  const float x2 = x * x;
#pragma unroll
  for (int l = 0; l <= LC; ++l) {
    if (l > lmax) break;
    if (l == 0) {
      cur[0] = 1.f;
    } else if (l == 1) {
      cur[0] = x;
      cur[1] = -sq;
    } else if (l == 2) {
      cur[0] = 1.5f * x2 - 0.5f;
      cur[1] = -3.f * x * sq;
      cur[2] = 3.f - 3.f * x2;
    } else {
#pragma unroll
      for (int m = 0; m <= LC; ++m) {
        if (m <= l - 2) {
          const float aa = (float)(2 * l - 1) / (float)(l - m);
          const float bb = (float)(l - 1 + m) / (float)(l - m);
          cur[m] = aa * x * rm1[m] - bb * rm2[m];
        }
      }
      cur[l - 1] = x * (float)(2 * l - 1) * rm1[l - 1];
      cur[l] = -(float)(2 * l - 1) * sq * rm1[l - 1];
    }
#pragma unroll
    for (int m = 0; m <= LC; ++m) {
      if (m <= l) emit(l * (l + 1) / 2 + m, cur[m]);
      rm2[m] = rm1[m];
      rm1[m] = cur[m];
    }
  }
}

}  // namespace soapb
