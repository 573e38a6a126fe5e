/*
 * soap_oracle.c -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * A plain FP64 CPU restatement of soap_turbo's descriptor path (get_soap with
 * its derivatives and the soap_contract adjoint).  Only the test suite, the
 * smoke check and the CPU-baseline leg of bench.py load this file's library;
 * the product path (libsoapb200.so) never links or calls it.
 *
 * Every routine follows the reference's arithmetic in the reference's order,
 * so that FP64 results agree with a gfortran build of the reference to a few
 * ulps.  Citations are file:line inside the reference project.
 *
 * Parity pinning: the reference ships no tests or fixtures and no Fortran
 * compiler exists on either machine of this project, so the reference itself
 * cannot be run.  The oracle is pinned by (a) the reference's own poly3tab
 * W/S tables (src/soap_turbo_radial.f90:1247-1528) against the W built here,
 * (b) the reference's documented identities (soap_contract equals
 * soap_cart_der contracted with G, src/soap_turbo.f90:1721; the self column is
 * minus the sum of the others, :888-892; the unified filter seed makes the
 * radial derivative a finite-difference-exact derivative,
 * src/soap_turbo_radial.f90:53-54; unit norm, :805-809), and (c) the scalar
 * reference functions plm_double / ilexp_double
 * (src/soap_turbo_functions.f90:44-77, 279-330) against the array routines.
 *
 * Layouts are Fortran column-major, as the reference's arguments:
 *   soap(n_soap, n_sites)              -> soap[i*n_soap + s]
 *   soap_cart_der(3, n_soap, n_pairs)  -> cart[(k*n_soap + s)*3 + c]
 *   G(n_sites, n_soap)                 -> G[s*n_sites + i]
 *   pair(3, n_pairs)                   -> pair[k*3 + c]
 *   mask(n_pairs, n_species)           -> mask[s*n_pairs + k]   (uint8)
 *   species(max_mult, n_sites)         -> species[i*max_mult + m]  (1-based)
 *   W, S (n_max, n_max)                -> W[col*n_max + row]
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_PI 3.141592653589793238462643383279502884

/* ------------------------------------------------------------------------ */
/* Arguments of get_soap (src/soap_turbo.f90:139-169), flattened.            */
/* ------------------------------------------------------------------------ */
typedef struct {
  int n_sites, n_species, n_pairs, max_mult, l_max, radial_enhancement;
  int basis;            /* 0 = poly3, 1 = poly3gauss, 2 = poly3operator */
  int scaling_poly;     /* 1 when scaling_mode == "polynomial" */
  int legacy_filter_seed;
  const int *n_neigh, *species, *species_multiplicity;
  const uint8_t *mask;
  const double *rjs, *thetas, *phis;
  const int *alpha_max;
  const double *rcut_hard, *rcut_soft, *nf, *global_scaling;
  const double *atom_sigma_r, *atom_sigma_r_scaling;
  const double *atom_sigma_t, *atom_sigma_t_scaling;
  const double *amplitude_scaling, *central_weight;
  int compress, P_nonzero;
  const int *P_i, *P_j;     /* 1-based, as the reference */
  const double *P_el;
  const double *W, *S;      /* n_max x n_max block diagonal, column-major */
} or_args;

static int kidx(int l, int m) { return l * (l + 1) / 2 + m; } /* 0-based k */

/* ------------------------------------------------------------------------ */
/* Math primitives                                                           */
/* ------------------------------------------------------------------------ */

/* get_preflm, src/soap_turbo_functions.f90:215-241 */
void or_preflm(int lmax, double *preflm) {
  int k = 0;
  for (int l = 0; l <= lmax; l++) {
    double ppi = sqrt((double)(2 * l + 1) / 4.0 / acos(-1.0));
    double fact2 = 1.0;
    for (int i = 1; i <= l; i++) fact2 *= (double)i;
    double fact1 = fact2;
    for (int m = 0; m <= l; m++) {
      if (m > 0) {
        fact1 = fact1 / (double)(l + 1 - m);
        fact2 = fact2 * (double)(l + m);
      }
      preflm[k++] = ppi * sqrt(fact1 / fact2);
    }
  }
}

/* get_plm_array, src/soap_turbo_angular.f90:108-160, with the l-recursion
 * coefficients of build_plm_tables (:55-74) evaluated inline. */
void or_plm_array(int lmax, double x, double *p) {
  double x2 = x * x, sq = sqrt(1.0 - x2);
  p[0] = 1.0;
  if (lmax < 1) return;
  p[1] = x;
  p[2] = -sq;
  if (lmax < 2) return;
  p[3] = 1.5 * x2 - 0.5;
  p[4] = -3.0 * x * sq;
  p[5] = 3.0 - 3.0 * x2;
  for (int l = 3; l <= lmax; l++) {
    int k = 0;
    for (int m = 0; m <= l - 2; m++) {
      k = kidx(l, m);
      double a = (double)(2 * l - 1) / (double)(l - m);
      double b = (double)(l - 1 + m) / (double)(l - m);
      p[k] = a * x * p[k - l] - b * p[k - 2 * l + 1];
    }
    k++;
    p[k] = x * (double)(2 * l - 1) * p[k - l];
    k++;
    p[k] = -(double)(2 * l - 1) * sq * p[k - l - 1];
  }
}

/* get_plm_array_der, src/soap_turbo_angular.f90:181-248 (tables :80-99).
 * p must hold P_l^m up to lmax+1. */
void or_plm_array_der(int lmax, const double *p, double *div_sin, double *der_mul_sin) {
  for (int l = 0; l <= lmax; l++) {
    for (int m = 0; m <= l; m++) {
      int k = kidx(l, m);
      double part1, part2;
      if (m == 0) {
        part1 = (l == 0) ? 0.0 : -0.5 * p[kidx(l, 1)];
      } else {
        part1 = 0.5 * (double)(l + m) * (double)(l - m + 1) * p[k - 1];
      }
      part2 = (m == l) ? 0.0 : -0.5 * p[k + 1];
      der_mul_sin[k] = part1 + part2;
    }
  }
  for (int l = 0; l <= lmax; l++) div_sin[kidx(l, 0)] = 0.0;
  for (int l = 0; l <= lmax; l++) {
    for (int m = 1; m <= l; m++) {
      int k = kidx(l, m);
      double part1 = 0.5 * (double)(l - m + 1) * (double)(l - m + 2) * p[kidx(l + 1, m - 1)];
      double part2 = 0.5 * p[kidx(l + 1, m + 1)];
      div_sin[k] = part1 + part2;
    }
  }
}

/* plm_double, src/soap_turbo_functions.f90:44-77 (scalar cross-check) */
double or_plm_double(int l, int m, double x) {
  double pmm = 1.0, pl2m = 0.0;
  if (m > 0) {
    double sq = sqrt(1.0 - x * x), dfact = -1.0;
    for (int i = 1; i <= m; i++) { dfact += 2.0; pmm = -pmm * dfact * sq; }
  }
  if (l == m) return pmm;
  double pmp1m = x * (2.0 * (double)m + 1.0) * pmm;
  if (l == m + 1) return pmp1m;
  for (int l2 = m + 2; l2 <= l; l2++) {
    pl2m = (x * (double)(2 * l2 - 1) * pmp1m - (double)(l2 + m - 1) * pmm) / (double)(l2 - m);
    pmm = pmp1m;
    pmp1m = pl2m;
  }
  return pl2m;
}

/* get_ilexp, src/soap_turbo_angular.f90:361-422 (semifactorials :344-356).
 * i_l(x^2) exp(-x^2) for l = 0..lmax; out needs lmax+1 entries. */
void or_ilexp_array(int lmax, double x, double *out) {
  const double xcut = 1.0e-7;
  double x2 = x * x, x4 = x2 * x2;
  double inv_x2 = (x2 > 0.0) ? 1.0 / x2 : 0.0;
  double x2pow = x2 * x2;
  double flm2, flm1;
  if (x > 0.0) {
    flm2 = fabs((1.0 - exp(-2.0 * x2)) / 2.0 / x2);
    flm1 = fabs((x2 - 1.0 + exp(-2.0 * x2) * (x2 + 1.0)) / 2.0 / x4);
  } else {
    flm2 = 1.0;
    flm1 = 0.0;
  }
  double fact = 1.0;
  for (int l = 0; l <= lmax; l++) {
    if (l > 0) fact *= (2.0 * (double)l + 1.0);
    if (l == 0) {
      out[0] = (x < xcut) ? 1.0 - x2 : flm2;
    } else if (l == 1) {
      out[1] = (x2 / 1000.0 < xcut) ? (x2 - x4) / fact : flm1;
    } else {
      double ratio = x2pow / fact, fl;
      if (ratio * (double)l < xcut) fl = ratio;
      else fl = fabs(flm2 - (2.0 * (double)l - 1.0) * inv_x2 * flm1);
      x2pow *= x2;
      flm2 = flm1;
      flm1 = fl;
      out[l] = fl;
    }
  }
}

/* ilexp_double, src/soap_turbo_functions.f90:279-330 (scalar cross-check) */
double or_ilexp_double(int l, double x) {
  const double xcut = 1.0e-7;
  double x2 = x * x, x4 = pow(x, 4.0), fact = 1.0;
  if (l == 0 && x < xcut) return 1.0 - x2;
  for (int i = 1; i <= l; i++) fact *= (2.0 * (double)i + 1.0);
  if (l == 1 && x2 / 1000.0 < xcut) return (x2 - x4) / fact;
  if (l > 1 && pow(x2, (double)l) / fact * (double)l < xcut) return pow(x2, (double)l) / fact;
  double flm2 = fabs((1.0 - exp(-2.0 * x2)) / 2.0 / x2);
  double flm1 = fabs((x2 - 1.0 + exp(-2.0 * x2) * (x2 + 1.0)) / 2.0 / x4);
  if (l == 0) return flm2;
  if (l == 1) return flm1;
  double fl = 0.0;
  for (int i = 2; i <= l; i++) {
    fl = fabs(flm2 - (2.0 * (double)i - 1.0) / x2 * flm1);
    flm2 = flm1;
    flm1 = fl;
  }
  return fl;
}

/* get_ilexp_der, src/soap_turbo_angular.f90:436-463.  il needs lmax+2
 * entries (the l = 0 term reads il[1]). */
static void or_ilexp_der(const double *il, int lmax, double rj, double sig, double scaling, double *der) {
  double c1 = 2.0 * rj / (sig * sig), c2 = 1.0 - scaling * rj / sig;
  for (int l = 0; l <= lmax; l++) der[l] = 0.0;
  if (rj < 1.0e-5) return;
  der[0] = c1 * (il[1] - il[0]);
  for (int l = 1; l <= lmax; l++)
    der[l] = (-c1 - (double)(2 * l + 2) / rj) * il[l] + c1 * il[l - 1];
  for (int l = 0; l <= lmax; l++) der[l] *= c2;
}

/* ------------------------------------------------------------------------ */
/* Orthonormalisation matrices                                               */
/* ------------------------------------------------------------------------ */

/* Overlap of the primitive poly3 functions, src/soap_turbo_radial.f90:1041-1047 */
void or_overlap_poly3(int a, double *S) {
  for (int i = 1; i <= a; i++) {
    S[(i - 1) * a + (i - 1)] = 1.0;
    for (int j = i + 1; j <= a; j++) {
      double v = sqrt((double)(5 + 2 * i) * (double)(5 + 2 * j)) / (double)(5 + i + j);
      S[(j - 1) * a + (i - 1)] = v;
      S[(i - 1) * a + (j - 1)] = v;
    }
  }
}

/* Overlap of poly3 + origin Gaussian, src/soap_turbo_radial.f90:1133-1172
 * (N_a at :82-96 with rcut = 1). */
void or_overlap_poly3gauss(int a, double sigma_in, double rcut_in, double *S) {
  for (int i = 1; i <= a - 1; i++) {
    S[(i - 1) * a + (i - 1)] = 1.0;
    for (int j = i + 1; j <= a - 1; j++) {
      double v = sqrt((double)(5 + 2 * i) * (double)(5 + 2 * j)) / (double)(5 + i + j);
      S[(j - 1) * a + (i - 1)] = v;
      S[(i - 1) * a + (j - 1)] = v;
    }
  }
  double sig = sigma_in / rcut_in, rc = 1.0, s2 = sig * sig;
  double sq2 = sqrt(2.0), pi = acos(-1.0);
  double I_n = 0.0, N_n = 1.0;
  double N_np1 = sqrt(rc / (double)(2 * (-2) + 5));
  double I_np1 = sqrt(pi / 2.0) * sig * erf(rc / sq2 / sig) / N_np1;
  double C2 = s2 / rc;
  for (int n = -1; n <= a - 1; n++) {
    C2 = C2 * rc;
    double N_np2 = sqrt(rc / (double)(2 * n + 5));
    double I_np2 = s2 * (double)(n + 1) * N_n / N_np2 * I_n + N_np1 * rc / N_np2 * I_np1 - C2 / N_np2;
    if (n > 0) {
      double v = I_np2 * sq2 / sqrt(sig) / pow(pi, 0.25);
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

/* W = S^{-1/2}.  The reference forms it as SVD -> U sqrt(sigma) V^T ->
 * Cholesky inverse (src/soap_turbo_radial.f90:1052-1087); for a symmetric
 * positive definite S that is the inverse principal square root, computed
 * here from a cyclic Jacobi eigendecomposition in long double.  Returns 0,
 * or 1 if S is not positive definite. */
int or_inverse_sqrt(int a, const double *S, double *W) {
  long double A[16 * 16], V[16 * 16];
  if (a > 16 || a < 1) return 2;
  for (int i = 0; i < a * a; i++) A[i] = S[i];
  for (int i = 0; i < a; i++)
    for (int j = 0; j < a; j++) V[j * a + i] = (i == j) ? 1.0L : 0.0L;
  for (int sweep = 0; sweep < 100; sweep++) {
    long double off = 0.0L;
    for (int p = 0; p < a; p++)
      for (int q = p + 1; q < a; q++) off += A[q * a + p] * A[q * a + p];
    if (off < 1.0e-70L) break;
    for (int p = 0; p < a; p++) {
      for (int q = p + 1; q < a; q++) {
        long double apq = A[q * a + p];
        if (apq == 0.0L) continue;
        long double app = A[p * a + p], aqq = A[q * a + q];
        long double theta = (aqq - app) / (2.0L * apq);
        long double t = (theta >= 0 ? 1.0L : -1.0L) / (fabsl(theta) + sqrtl(theta * theta + 1.0L));
        long double c = 1.0L / sqrtl(t * t + 1.0L), s = t * c;
        for (int k = 0; k < a; k++) {
          long double akp = A[p * a + k], akq = A[q * a + k];
          A[p * a + k] = c * akp - s * akq;
          A[q * a + k] = s * akp + c * akq;
        }
        for (int k = 0; k < a; k++) {
          long double apk = A[k * a + p], aqk = A[k * a + q];
          A[k * a + p] = c * apk - s * aqk;
          A[k * a + q] = s * apk + c * aqk;
        }
        for (int k = 0; k < a; k++) {
          long double vkp = V[p * a + k], vkq = V[q * a + k];
          V[p * a + k] = c * vkp - s * vkq;
          V[q * a + k] = s * vkp + c * vkq;
        }
      }
    }
  }
  long double d[16];
  for (int i = 0; i < a; i++) {
    if (!(A[i * a + i] > 0.0L)) return 1;
    d[i] = 1.0L / sqrtl(A[i * a + i]);
  }
  for (int i = 0; i < a; i++)
    for (int j = 0; j < a; j++) {
      long double s = 0.0L;
      for (int k = 0; k < a; k++) s += V[k * a + i] * d[k] * V[k * a + j];
      W[j * a + i] = (double)s;
    }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Radial expansion: radial_expansion_kernel + process_block,                */
/* src/soap_turbo_radial.f90:281-1004, one pair at a time.                   */
/* ------------------------------------------------------------------------ */
typedef struct {
  int alpha, n_poly, n_hi, with_gauss, unified, has_filter, do_der, do_der2;
  double rcut_soft, atom_sigma, c, dr, sqrt_rcut, inv_sqrt_rcut, inv_rcut;
  double q, drnf, sigma_sq0, N_gauss, inv_Nm2, amp_scaling, cw;
  int do_central, scaling_poly, radial_enhancement;
  double Nv[32], ra[32], rb[32], rc[32], R1[32], R2[32], R3[32], R4[32]; /* index n+4 */
  const double *W; int ldw;                                /* alpha x alpha block */
} or_radial_setup;

#define NI(n) ((n) + 4)

static void or_radial_init(or_radial_setup *s, int alpha, double rcut_soft_in, double rcut_hard_in,
                           double sigma_in, double sigma_scaling, double amp_scaling, double nf,
                           const double *W, int ldw, int scaling_poly, int radial_enhancement,
                           int do_der, int do_central, double central_weight, int with_gauss,
                           int legacy_seed) {
  memset(s, 0, sizeof(*s));
  s->alpha = alpha;
  s->inv_rcut = 1.0 / rcut_hard_in;                                 /* :459-464 */
  s->rcut_soft = rcut_soft_in * s->inv_rcut;
  s->atom_sigma = sigma_in * s->inv_rcut;
  s->dr = 1.0 - s->rcut_soft;
  s->sqrt_rcut = sqrt(rcut_hard_in);
  s->inv_sqrt_rcut = 1.0 / s->sqrt_rcut;
  s->sigma_sq0 = s->atom_sigma * s->atom_sigma;                     /* :467-468 */
  s->N_gauss = sqrt(2.0 / s->atom_sigma) / pow(OR_PI, 0.25);
  s->has_filter = s->dr > 0.0;                                      /* :475-481 */
  if (s->has_filter) { s->drnf = s->dr / nf; s->q = s->drnf * s->drnf; }
  s->n_poly = with_gauss ? alpha - 1 : alpha;                       /* :483-491 */
  s->n_hi = s->n_poly + (do_der ? 2 : 0);
  s->with_gauss = with_gauss;
  s->unified = !legacy_seed;
  s->do_der = do_der;
  s->c = sigma_scaling;
  s->amp_scaling = amp_scaling;
  s->cw = central_weight;
  s->do_central = do_central;
  s->scaling_poly = scaling_poly;
  s->radial_enhancement = radial_enhancement;
  s->W = W;
  s->ldw = ldw;
  s->Nv[NI(-3)] = 1.0;                                              /* :503-513 */
  for (int n = -2; n <= alpha + 4; n++) s->Nv[NI(n)] = sqrt(1.0 / (double)(2 * n + 5));
  for (int n = -1; n <= s->n_hi; n++) {
    s->ra[NI(n)] = (double)(n + 1) * s->Nv[NI(n - 2)] / s->Nv[NI(n)];
    s->rb[NI(n)] = s->Nv[NI(n - 1)] / s->Nv[NI(n)];
    s->rc[NI(n)] = 1.0 / s->Nv[NI(n)];
  }
  s->ra[NI(-1)] = 0.0;
  s->inv_Nm2 = 1.0 / s->Nv[NI(-2)];
  for (int n = 1; n <= s->n_poly; n++) {                            /* :515-519 */
    s->R1[NI(n)] = s->Nv[NI(n + 1)] / s->Nv[NI(n)];
    s->R2[NI(n)] = s->Nv[NI(n + 2)] / s->Nv[NI(n)];
  }
}

/* Second radial derivatives as well (src/soap_turbo_radial.f90:489-491,
 * 520-525): the recursions run to alpha + 4.  Only with the unified filter
 * seed (:318-328); returns -1 otherwise. */
static int or_radial_enable_der2(or_radial_setup *s) {
  if (!s->unified || !s->do_der) return -1;
  s->do_der2 = 1;
  s->n_hi = s->n_poly + 4;
  for (int n = -1; n <= s->n_hi; n++) {
    s->ra[NI(n)] = (double)(n + 1) * s->Nv[NI(n - 2)] / s->Nv[NI(n)];
    s->rb[NI(n)] = s->Nv[NI(n - 1)] / s->Nv[NI(n)];
    s->rc[NI(n)] = 1.0 / s->Nv[NI(n)];
  }
  s->ra[NI(-1)] = 0.0;
  for (int n = 1; n <= s->n_poly; n++) {
    s->R3[NI(n)] = s->Nv[NI(n + 3)] / s->Nv[NI(n)];
    s->R4[NI(n)] = s->Nv[NI(n + 4)] / s->Nv[NI(n)];
  }
  return 0;
}

/* One pair of process_block (src/soap_turbo_radial.f90:550-1002).  rj_in is
 * the unscaled distance.  Writes alpha values to out (and der if do_der). */
static void or_radial_pair(const or_radial_setup *s, double rj_in, int is_central, double *out, double *der,
                           double *der2) {
  const double pi = acos(-1.0), sq2 = sqrt(2.0), isq2 = 1.0 / sq2;
  const double sqpi2 = sqrt(pi / 2.0), sq2pi = sqrt(2.0 / pi), sq8pi = sqrt(8.0 / pi);
  const int a = s->alpha, n_hi = s->n_hi, n_poly = s->n_poly;
  const double c = s->c, rs = s->rcut_soft, dr = s->dr;
  double T1[40], T2[40], pol[40], DT[40], dtot[40], D2T[40], d2tot[40];
  double rj = rj_in * s->inv_rcut;
  for (int i = 0; i < 40; i++) { T1[i] = T2[i] = pol[i] = DT[i] = dtot[i] = D2T[i] = d2tot[i] = 0.0; }

  double sig = s->atom_sigma + c * rj, s2 = sig * sig;               /* :560-570 */
  double isig = 1.0 / sig, is2 = isig * isig, is3 = is2 * isig;

  double amp, ampd, ampd2;                                           /* :589-635 */
  if (!s->scaling_poly) {
    amp = 1.0; ampd = 0.0; ampd2 = 0.0;
  } else if (s->amp_scaling == 0.0) {
    amp = isig; ampd = -c * is2; ampd2 = 2.0 * c * c * is3;
  } else if (s->amp_scaling == 1.0) {
    double h = 1.0 + 2.0 * (rj * rj * rj) - 3.0 * rj * rj;
    double hp = 6.0 * rj * rj - 6.0 * rj, hpp = 12.0 * rj - 6.0;
    double g = isig * h;
    amp = (h <= 1.0e-10) ? 0.0 : g;
    ampd = (h <= 1.0e-10) ? 0.0 : hp * isig - c * isig * g;
    ampd2 = (h <= 1.0e-10) ? 0.0 : hpp * isig - 2.0 * c * hp * is2 + 2.0 * c * c * h * is3;
  } else {
    double h = 1.0 + 2.0 * (rj * rj * rj) - 3.0 * rj * rj;
    if (h <= 1.0e-10) { amp = 0.0; ampd = 0.0; ampd2 = 0.0; }
    else {
      double hp = 6.0 * rj * rj - 6.0 * rj, hpp = 12.0 * rj - 6.0, aa = s->amp_scaling;
      amp = isig * pow(h, aa);
      ampd = aa * pow(h, aa - 1.0) * hp * isig - c * isig * amp;
      ampd2 = (aa * (aa - 1.0) * pow(h, aa - 2.0) * hp * hp + aa * pow(h, aa - 1.0) * hpp) * isig
              - 2.0 * c * aa * pow(h, aa - 1.0) * hp * is2 + 2.0 * c * c * pow(h, aa) * is3;
    }
  }
  if (s->do_central && s->cw != 1.0 && is_central) {                 /* :638-646 */
    amp *= s->cw; ampd *= s->cw; ampd2 *= s->cw;
  }
  if (s->radial_enhancement == 1) {                                  /* :651-670 */
    double g = rj + sq2pi * sig, f = 1.0 + sq2pi * c;
    ampd2 = ampd2 * g + 2.0 * ampd * f;
    ampd = amp * f + ampd * g;
    amp = amp * g;
  } else if (s->radial_enhancement == 2) {
    double g = rj * rj + s2 + sq8pi * sig * rj;
    double f = 2.0 * rj + 2.0 * sig * c + sq8pi * sig + sq8pi * rj * c;
    double h = 2.0 + 2.0 * c * c + 2.0 * sq8pi * c;
    ampd2 = ampd2 * g + 2.0 * ampd * f + amp * h;
    ampd = amp * f + ampd * g;
    amp = amp * g;
  }

  /* inner overlap on [0, rcut_soft], :676-698 */
  double es = exp(-0.5 * (rs - rj) * (rs - rj) * is2);
  double e0 = exp(-0.5 * rj * rj * is2);
  double C1 = s2 * es, C2 = s2 * e0;
  T1[NI(-3)] = 0.0;
  T1[NI(-2)] = sqpi2 * sig * (erf((rs - rj) * isq2 * isig) + erf(rj * isq2 * isig)) * s->inv_Nm2;
  for (int n = -1; n <= n_hi; n++) {
    if (n >= 0) C1 = C1 * dr;
    T1[NI(n)] = s2 * s->ra[NI(n)] * T1[NI(n - 2)] - s->rb[NI(n)] * (rj - 1.0) * T1[NI(n - 1)]
                + (C1 - C2) * s->rc[NI(n)];
  }
  if (s->do_der && n_poly >= 1 && !s->unified) {                     /* :701-714 */
    double f = rj - 1.0, g = c * f * isig;
    double ca = f * is2 * (g - 1.0), cb = is2 * (2.0 * g - 1.0), cc = c * is3;
    for (int n = 1; n <= n_poly; n++)
      DT[NI(n)] = ca * T1[NI(n)] + s->R1[NI(n)] * cb * T1[NI(n + 1)] + s->R2[NI(n)] * cc * T1[NI(n + 2)];
  }

  double pref = 0.0;
  if (s->has_filter) {                                               /* :721-795 */
    double q = s->q, drnf = s->drnf;
    double den = s2 + q, iD = 1.0 / den, sqiD = sqrt(iD);
    double sgf = sig * drnf * sqiD;
    double rjf = (s2 * rs + q * rj) * iD;
    double sf2 = sgf * sgf;
    int keep = (rs - rj) < 4.0 * sig;
    double isgf = 1.0 / sgf, isf2 = isgf * isgf;
    pref = keep ? exp(-0.5 * (rs - rj) * (rs - rj) * iD) : 0.0;
    double C2f = sf2 * exp(-0.5 * (rs - rjf) * (rs - rjf) * isf2);
    T2[NI(-3)] = 0.0;
    T2[NI(-2)] = sqpi2 * sgf * (erf((1.0 - rjf) * isq2 * isgf) - erf((rs - rjf) * isq2 * isgf)) * s->inv_Nm2;
    for (int n = -1; n <= n_hi; n++) {
      if (n >= 0) C2f = C2f * dr;
      T2[NI(n)] = sf2 * s->ra[NI(n)] * T2[NI(n - 2)] - s->rb[NI(n)] * (rjf - 1.0) * T2[NI(n - 1)]
                  - C2f * s->rc[NI(n)];
      if (n == -1 && s->unified)
        T2[NI(-1)] = T2[NI(-1)] + sf2 * exp(-0.5 * (1.0 - rjf) * (1.0 - rjf) * isf2) * s->rc[NI(-1)];
    }
    if (s->do_der && n_poly >= 1 && !s->unified) {
      double f = rs - rj;
      double dpref = pref * (f * iD + f * f * iD * iD * sig * c);
      double drjf = (2.0 * sig * rs * c + q) * iD - (s2 * rs + q * rj) * 2.0 * sig * c * iD * iD;
      double dsgf = c * drnf * sqiD * (1.0 - s2 * iD);
      double ff = rjf - 1.0, g = dsgf * ff * isgf;
      double ca = pref * ff * isf2 * (g - drjf);
      double cb = pref * isf2 * (2.0 * g - drjf);
      double cc = pref * dsgf * isgf * isf2;
      for (int n = 1; n <= n_poly; n++)
        DT[NI(n)] = DT[NI(n)] + ca * T2[NI(n)] + s->R1[NI(n)] * cb * T2[NI(n + 1)]
                    + s->R2[NI(n)] * cc * T2[NI(n + 2)] + dpref * T2[NI(n)];
    }
  } else {
    for (int n = 1; n <= n_hi; n++) T2[NI(n)] = 0.0;
  }
  for (int n = 1; n <= n_hi; n++) pol[NI(n)] = T1[NI(n)] + pref * T2[NI(n)];   /* :808-812 */

  if (s->do_der && n_poly >= 1 && s->unified) {                      /* :825-836 */
    double f = 1.0 - rj;
    double g0 = f * is2 + c * f * f * is3;
    double g1 = -(is2 + 2.0 * c * f * is3);
    double g2 = c * is3;
    for (int n = 1; n <= n_poly; n++)
      DT[NI(n)] = g0 * pol[NI(n)] + s->R1[NI(n)] * g1 * pol[NI(n + 1)] + s->R2[NI(n)] * g2 * pol[NI(n + 2)];
    if (s->do_der2) {                                                /* :838-861 */
      double is4 = is2 * is2, is5 = is4 * isig, is6 = is4 * is2;
      double k0 = -is2, k1 = -4.0 * c * is3, k2 = (1.0 - 3.0 * c * c) * is4, k3 = 2.0 * c * is5,
             k4 = c * c * is6;
      double B0 = k0 + k1 * f + k2 * f * f + k3 * f * f * f + k4 * f * f * f * f;
      double B1 = -(k1 + 2.0 * k2 * f + 3.0 * k3 * f * f + 4.0 * k4 * f * f * f);
      double B2 = k2 + 3.0 * k3 * f + 6.0 * k4 * f * f;
      double B3 = -(k3 + 4.0 * k4 * f);
      double B4 = k4;
      for (int n = 1; n <= n_poly; n++)
        D2T[NI(n)] = B0 * pol[NI(n)] + s->R1[NI(n)] * B1 * pol[NI(n + 1)] + s->R2[NI(n)] * B2 * pol[NI(n + 2)]
                     + s->R3[NI(n)] * B3 * pol[NI(n + 3)] + s->R4[NI(n)] * B4 * pol[NI(n + 4)];
    }
  }

  if (s->with_gauss) {                                               /* :875-908 */
    double ss2 = s->sigma_sq0 + s2, iss = 1.0 / ss2, siss = sqrt(iss);
    int gm = rj < 4.0 * (s->atom_sigma + sig);
    double ge = gm ? s->N_gauss * e0 : 0.0;
    double M0 = gm ? exp(-0.5 * rj * rj * iss) * sqpi2 * sig * s->atom_sigma * siss
                     * (1.0 + erf(s->atom_sigma * isig * rj * isq2 * siss)) * s->N_gauss
                   : 0.0;
    pol[NI(a)] = M0;
    if (s->do_der) {
      double sc0 = s->sigma_sq0 * s2 * iss, pp = s2 * rj * iss;
      double M1 = sc0 * ge - pp * M0;
      double M2 = sc0 * ge * (-rj) - pp * M1 + sc0 * M0;
      DT[NI(a)] = M1 * is2 + c * M2 * is3;
      if (s->do_der2) {                                              /* :895-905 */
        double M3 = sc0 * ge * rj * rj - pp * M2 + 2.0 * sc0 * M1;
        double M4 = sc0 * ge * (-rj * rj * rj) - pp * M3 + 3.0 * sc0 * M2;
        double is4 = is2 * is2, is5 = is4 * isig, is6 = is4 * is2;
        D2T[NI(a)] = -M0 * is2 - 4.0 * c * M1 * is3 + (1.0 - 3.0 * c * c) * M2 * is4
                     + 2.0 * c * M3 * is5 + c * c * M4 * is6;
      }
    }
  }

  if (s->do_der) {                                                   /* :911-942 */
    for (int n = 1; n <= a; n++) dtot[NI(n)] = amp * DT[NI(n)] + ampd * pol[NI(n)];
    for (int n = 1; n <= a; n++) {
      double acc = s->W[0 * s->ldw + (n - 1)] * dtot[NI(1)];
      for (int m = 2; m <= a; m++) acc = acc + s->W[(m - 1) * s->ldw + (n - 1)] * dtot[NI(m)];
      der[n - 1] = acc * s->inv_sqrt_rcut;
    }
    if (s->do_der2 && der2) {                                        /* :917-956 */
      for (int n = 1; n <= a; n++)
        d2tot[NI(n)] = amp * D2T[NI(n)] + 2.0 * ampd * DT[NI(n)] + ampd2 * pol[NI(n)];
      for (int n = 1; n <= a; n++) {
        double acc = s->W[0 * s->ldw + (n - 1)] * d2tot[NI(1)];
        for (int m = 2; m <= a; m++) acc = acc + s->W[(m - 1) * s->ldw + (n - 1)] * d2tot[NI(m)];
        der2[n - 1] = acc * s->inv_sqrt_rcut * s->inv_rcut;
      }
    }
  }
  for (int n = 1; n <= a; n++) {                                     /* :962-976 */
    double acc = s->W[0 * s->ldw + (n - 1)] * pol[NI(1)];
    for (int m = 2; m <= a; m++) acc = acc + s->W[(m - 1) * s->ldw + (n - 1)] * pol[NI(m)];
    out[n - 1] = amp * acc * s->sqrt_rcut;
  }
}

/* ------------------------------------------------------------------------ */
/* poly3operator radial expansion, one pair                                  */
/* (get_radial_expansion_coefficients_poly3operator,                        */
/*  src/soap_turbo_radial.f90:1549-2141, and its helpers :2154-2557).       */
/* The atom density is the piecewise cubic g(x) = 1 - 3x^2 -+ 2x^3 on       */
/* x = (r - r_j)/w in [-1, 0] (left) and [0, 1] (right), w = 2 sqrt(2 ln 2) */
/* sigma(r_j); on [r_soft, r_hard] it is multiplied by the filter, the      */
/* right piece centred at r_soft with width 2 sqrt(2 ln 2)(r_hard - r_soft). */
/* The overlaps with (1 - r)^(n+2)/N_n (r_hard = 1 after scaling) are taken */
/* in closed form by repeated integration by parts, as the reference does. */
/* ------------------------------------------------------------------------ */

/* g_aux / g_aux_array (:2154-2217): value, first derivative, half the second,
 * a sixth of the third of the piece at r (the Taylor coefficients about r). */
static void op_gaux(double r, double r0, double w, int right, double *poly) {
  const double x = (r - r0) / w, iw = 1.0 / w;
  if (!right) {
    poly[0] = 1.0 - 3.0 * x * x - 2.0 * x * x * x;
    poly[1] = -6.0 * (x * x + x) * iw;
    poly[2] = -3.0 * (2.0 * x + 1.0) * iw * iw;
    poly[3] = -2.0 * iw * iw * iw;
  } else {
    poly[0] = 1.0 - 3.0 * x * x + 2.0 * x * x * x;
    poly[1] = 6.0 * (x * x - x) * iw;
    poly[2] = 3.0 * (2.0 * x - 1.0) * iw * iw;
    poly[3] = 2.0 * iw * iw * iw;
  }
}

/* g_aux_der_array (:2227-2267): the same four, differentiated with respect to
 * r0 where w = w0 + ws r0. */
static void op_gaux_der(double r, double r0, double w, double ws, int right, double *poly) {
  const double x = (r - r0) / w, iw = 1.0 / w, iw2 = iw * iw, iw3 = iw2 * iw, iw4 = iw3 * iw;
  if (!right) {
    poly[0] = 6.0 * (x + (ws + 1.0) * x * x + ws * x * x * x) * iw;
    poly[1] = 6.0 * (1.0 + 2.0 * (ws + 1.0) * x + 3.0 * ws * x * x) * iw2;
    poly[2] = 6.0 * (ws + 1.0 + 3.0 * ws * x) * iw3;
    poly[3] = 6.0 * ws * iw4;
  } else {
    poly[0] = 6.0 * (x + (ws - 1.0) * x * x - ws * x * x * x) * iw;
    poly[1] = 6.0 * (1.0 + 2.0 * (ws - 1.0) * x - 3.0 * ws * x * x) * iw2;
    poly[2] = 6.0 * (ws - 1.0 - 3.0 * ws * x) * iw3;
    poly[3] = -6.0 * ws * iw4;
  }
}

/* get_constant_poly_coeff (:2276-2297) with r_hard = 1: A(n, j), j = 1..7 */
static void op_coeff_A(int alpha, double *A) {
  for (int n = 1; n <= alpha; n++) {
    const double Na = sqrt(1.0 / (double)(2 * n + 5));                  /* N_a, :82-96 */
    A[(n - 1) * 7 + 0] = 1.0 / Na / (double)(n + 3);
    for (int j = 2; j <= 7; j++) A[(n - 1) * 7 + j - 1] = A[(n - 1) * 7 + j - 2] / (double)(n + 3 + j - 1);
  }
}

/* Soft-zone overlap of one piece between limits lo and hi (:1770-1797): the
 * four integration-by-parts terms at each limit, upper minus lower.
 * g4(lim) supplies the piece's four coefficients at a limit. */
static void op_soft_piece(int alpha, const double *A, double lo, double hi, const double *g_lo,
                          const double *g_hi, double *Ov) {
  static const double vect[4] = {-1.0, -1.0, -2.0, -6.0};
  double Ml[4], Mh[4], pl[32], ph[32];
  pl[0] = ph[0] = 1.0;
  for (int j = 1; j < alpha + 4; j++) { pl[j] = pl[j - 1] * (1.0 - lo); ph[j] = ph[j - 1] * (1.0 - hi); }
  for (int j = 0; j < 4; j++) { Ml[j] = pl[j] * g_lo[j] * vect[j]; Mh[j] = ph[j] * g_hi[j] * vect[j]; }
  for (int n = 1; n <= alpha; n++) {
    double sh = 0.0, sl = 0.0;
    for (int j = 0; j < 4; j++) { sh += Mh[j] * A[(n - 1) * 7 + j]; sl += Ml[j] * A[(n - 1) * 7 + j]; }
    Ov[n - 1] = sh * ph[n + 3] - sl * pl[n + 3];
  }
}

/* get_constant_poly_filter_coeff_array (:2307-2344): the monomial coefficients
 * of (atom piece) x (filter), degree 6.  col: the piece's Taylor coefficients
 * about r = 0; C: the filter's. */
static void op_product(const double *col, const double *C, double *B) {
  for (int m = 0; m < 7; m++) B[m] = 0.0;
  for (int i = 0; i < 4; i++)
    for (int q = 0; q < 4; q++) B[i + q] += col[q] * C[i];
}

/* Buffer-zone overlap of one piece between lo and hi (:1995-2021): seven
 * integration-by-parts terms, -P^(d-1)(lim) (1 - lim)^(d-1) (M_radial_monomial,
 * :2481-2500), times A(n, d) (1 - lim)^(n+3). */
static void op_buffer_piece(int alpha, const double *A, double lo, double hi, const double *B, double *Ov) {
  double Ml[7], Mh[7], pl[32], ph[32];
  const int top = alpha + 4 > 7 ? alpha + 4 : 7;
  pl[0] = ph[0] = 1.0;
  for (int j = 1; j < top; j++) { pl[j] = pl[j - 1] * (1.0 - lo); ph[j] = ph[j - 1] * (1.0 - hi); }
  for (int d = 1; d <= 7; d++) {
    double vl = 0.0, vh = 0.0;
    for (int q = d; q <= 7; q++) {
      double f = 1.0;
      for (int t = q - d + 1; t <= q - 1; t++) f *= (double)t;               /* (q-1)!/(q-d)! */
      vl += B[q - 1] * f * pow(lo, q - d);
      vh += B[q - 1] * f * pow(hi, q - d);
    }
    Ml[d - 1] = -vl * pl[d - 1];
    Mh[d - 1] = -vh * ph[d - 1];
  }
  for (int n = 1; n <= alpha; n++) {
    double sh = 0.0, sl = 0.0;
    for (int d = 0; d < 7; d++) { sh += Mh[d] * A[(n - 1) * 7 + d]; sl += Ml[d] * A[(n - 1) * 7 + d]; }
    Ov[n - 1] = sh * ph[n + 3] - sl * pl[n + 3];
  }
}

/* The amplitude of the poly3operator expansion (:1699-1757): its value and
 * r-derivative (scaled units), with the central weight and the radial
 * enhancement.  Not polynomial scaling: the reference leaves it unset; 1 here. */
static void op_amplitude(double rj, double sig, double sig_c, double amp_scaling, int scaling_poly,
                         int radial_enhancement, int is_central, double cw, double *amp, double *ampd) {
  const double pi = acos(-1.0);
  double a = 1.0, ad = 0.0;
  if (scaling_poly) {
    if (amp_scaling == 0.0) {
      a = 1.0 / sig;
      ad = -sig_c / (sig * sig);
    } else if (amp_scaling == 1.0) {
      a = 1.0 / sig * (1.0 + 2.0 * rj * rj * rj - 3.0 * rj * rj);
      ad = 6.0 / sig * (rj * rj - rj) - sig_c / sig * a;
    } else {
      const double h = 1.0 + 2.0 * rj * rj * rj - 3.0 * rj * rj;
      a = 1.0 / sig * pow(h, amp_scaling);
      ad = 6.0 * amp_scaling / sig * (rj * rj - rj) * pow(h, amp_scaling - 1.0) - sig_c / sig * a;
    }
  }
  if (is_central) { a *= cw; ad *= cw; }
  if (radial_enhancement == 1) {
    ad = a * (1.0 + sqrt(2.0 / pi) * sig_c) + ad * (rj + sqrt(2.0 / pi) * sig);
    a = a * (rj + sqrt(2.0 / pi) * sig);
  } else if (radial_enhancement == 2) {
    ad = a * (2.0 * rj + 2.0 * sig * sig_c + sqrt(8.0 / pi) * sig + sqrt(8.0 / pi) * rj * sig_c) +
         ad * (rj * rj + sig * sig + sqrt(8.0 / pi) * sig * rj);
    a = a * (rj * rj + sig * sig + sqrt(8.0 / pi) * sig * rj);
  }
  *amp = a;
  *ampd = ad;
}

/* One masked pair: out[alpha] (and der[alpha] when der != NULL), W-transformed
 * and scaled to the unscaled radius (:2097-2117); global_scaling not applied.
 * rj_in unscaled.  A pair is in the soft zone when r - w < r_soft and in the
 * buffer zone when r_soft < r_hard and r + w > r_soft (:1637-1645, 1858-1872);
 * there is no r_hard cut of its own. */
static void or_radial_op_pair(int alpha, double rcut_soft_in, double rcut_hard_in, double sigma_in,
                              double sigma_scaling, double amp_scaling, int scaling_poly, int radial_enhancement,
                              double central_weight, int is_central, const double *W, int ldw, double rj_in,
                              double *out, double *der) {
  const double c_w = 2.0 * sqrt(2.0 * log(2.0));
  const double rs = rcut_soft_in / rcut_hard_in, sig0 = sigma_in / rcut_hard_in;
  const double filter_width = c_w * (1.0 - rs);
  const double w_in = c_w * (sigma_in + sigma_scaling * rj_in);
  double A[16 * 7], e[16], ed[16], Ov[16], Ov_d[16];
  op_coeff_A(alpha, A);
  for (int n = 0; n < alpha; n++) { e[n] = 0.0; ed[n] = 0.0; }
  const double rj = rj_in / rcut_hard_in, sig = sig0 + sigma_scaling * rj, w = c_w * sig;
  const double ws = c_w * sigma_scaling;
  double amp, ampd;
  op_amplitude(rj, sig, sigma_scaling, amp_scaling, scaling_poly, radial_enhancement, is_central, central_weight,
               &amp, &ampd);
  if (rj_in - w_in < rcut_soft_in) {                                     /* soft zone, :1770-1846 */
    const double l1 = fmax(0.0, rj - w), l2 = fmin(rj, rs), l3 = fmin(rs, rj + w);
    double g1[4], g2[4], g3[4], h2[4], tmp[16];
    op_gaux(l1, rj, w, 0, g1); op_gaux(l2, rj, w, 0, g2);
    op_gaux(l2, rj, w, 1, h2); op_gaux(l3, rj, w, 1, g3);
    op_soft_piece(alpha, A, l1, l2, g1, g2, Ov);
    op_soft_piece(alpha, A, l2, l3, h2, g3, tmp);
    for (int n = 0; n < alpha; n++) { Ov[n] += tmp[n]; e[n] = amp * Ov[n]; }
    if (der) {
      op_gaux_der(l1, rj, w, ws, 0, g1); op_gaux_der(l2, rj, w, ws, 0, g2);
      op_gaux_der(l2, rj, w, ws, 1, h2); op_gaux_der(l3, rj, w, ws, 1, g3);
      op_soft_piece(alpha, A, l1, l2, g1, g2, Ov_d);
      op_soft_piece(alpha, A, l2, l3, h2, g3, tmp);
      for (int n = 0; n < alpha; n++) ed[n] = amp * (Ov_d[n] + tmp[n]) + ampd * Ov[n];
    }
  }
  if (rcut_soft_in < rcut_hard_in && rj_in + w_in > rcut_soft_in) {     /* buffer zone, :1858-2075 */
    const double l1 = fmax(rs, rj - w), l2 = fmax(rj, rs), l3 = fmin(1.0, rj + w);
    double C[4], col[4], B[7], tmp[16];
    op_gaux(0.0, rs, filter_width, 1, C);
    op_gaux(-rj, 0.0, w, 0, col);
    op_product(col, C, B);
    op_buffer_piece(alpha, A, l1, l2, B, Ov);
    op_gaux(-rj, 0.0, w, 1, col);
    op_product(col, C, B);
    op_buffer_piece(alpha, A, l2, l3, B, tmp);
    for (int n = 0; n < alpha; n++) { Ov[n] += tmp[n]; e[n] += amp * Ov[n]; }
    if (der) {
      op_gaux_der(-rj, 0.0, w, ws, 0, col);
      op_product(col, C, B);
      op_buffer_piece(alpha, A, l1, l2, B, Ov_d);
      op_gaux_der(-rj, 0.0, w, ws, 1, col);
      op_product(col, C, B);
      op_buffer_piece(alpha, A, l2, l3, B, tmp);
      for (int n = 0; n < alpha; n++) ed[n] += amp * (Ov_d[n] + tmp[n]) + ampd * Ov[n];
    }
  }
  for (int n = 1; n <= alpha; n++) {                                      /* :2097-2100, 2113-2117 */
    double v = 0.0, d = 0.0;
    for (int m = 1; m <= alpha; m++) {
      v += W[(m - 1) * ldw + (n - 1)] * e[m - 1];
      d += W[(m - 1) * ldw + (n - 1)] * ed[m - 1];
    }
    out[n - 1] = v * sqrt(rcut_hard_in);
    if (der) der[n - 1] = d / sqrt(rcut_hard_in);
  }
}

/* ------------------------------------------------------------------------ */
/* Per-call state shared by get_soap and soap_contract                       */
/* ------------------------------------------------------------------------ */
typedef struct {
  int n_sites, n_pairs, n_max, k_max, l_max, n_soap, n_soap_unc, compress, P_nonzero;
  int *k_first;
  double *rad, *rad_der, *rad_der2;               /* (n_max, n_pairs); der2 only for the Hessian */
  double *ang, *ang_r, *ang_a, *ang_p;            /* complex (k_max, n_pairs): re,im interleaved */
  double *cnk;                                    /* complex (k_max, n_max, n_sites) */
  double *sqrt_dot_p;                             /* n_sites */
  unsigned char *skip;                            /* n_soap_unc */
  const int *P_i, *P_j; const double *P_el;
  const double *rjs, *thetas, *phis; const int *n_neigh;
} or_ctx;

void or_ctx_free(or_ctx *c) {
  if (!c) return;
  free(c->k_first); free(c->rad); free(c->rad_der); free(c->rad_der2);
  free(c->ang); free(c->ang_r); free(c->ang_a); free(c->ang_p);
  free(c->cnk); free(c->sqrt_dot_p); free(c->skip);
  free(c);
}

/* The species blocks of the radial basis, src/soap_turbo.f90:256-264 */
static void species_blocks(const or_args *a, int *i_beg, int *n_max) {
  int acc = 0;
  for (int s = 0; s < a->n_species; s++) { i_beg[s] = acc; acc += a->alpha_max[s]; }
  *n_max = acc;
}

/* get_soap, src/soap_turbo.f90:139-1037.
 *   soap:          (n_soap, n_sites), normalised.  As in the reference, a
 *                  compressed soap is accumulated into (:798-802: the
 *                  caller's values are added before the norm is taken), an
 *                  uncompressed one is overwritten
 *   soap_cart_der: (3, n_soap, n_pairs) or NULL; the neighbour columns are
 *                  overwritten and the self columns accumulated into
 *                  (:888-892), as in the reference
 *   ctx_out:       when non-NULL, receives the state soap_contract needs
 *                  (the reference's contract = .true.; :1008-1035)
 * Returns n_soap, or a negative code. */
int or_get_soap2(const or_args *a, int do_derivatives, int do_der2, double *soap, double *soap_cart_der,
                 or_ctx **ctx_out);
int or_get_soap(const or_args *a, int do_derivatives, double *soap, double *soap_cart_der, or_ctx **ctx_out) {
  return or_get_soap2(a, do_derivatives, 0, soap, soap_cart_der, ctx_out);
}

/* get_soap with, when do_der2, the second radial derivatives the central-atom
 * Hessian needs (soap_hessian_enabled, src/soap_turbo.f90:76, 228, 457-522);
 * returns -2 with the legacy filter seed (src/soap_turbo_radial.f90:318-328). */
int or_get_soap2(const or_args *a, int do_derivatives, int do_der2, double *soap, double *soap_cart_der,
                 or_ctx **ctx_out) {
  const double pi = acos(-1.0);
  int i_beg[64], n_max;
  if (a->n_species > 64) return -1;
  species_blocks(a, i_beg, &n_max);
  const int l_max = a->l_max, k_max = (l_max + 1) * (l_max + 2) / 2;
  const int n_pairs = a->n_pairs, n_sites = a->n_sites;
  const int n_soap_unc = n_max * (n_max + 1) / 2 * (l_max + 1);      /* :396 */
  const int need_der = do_derivatives;
  if (do_der2 && (!do_derivatives || a->legacy_filter_seed)) return -2;
  if (do_der2 && a->basis == 2) return -3;  /* no second derivatives for poly3operator, :485-489 */

  or_ctx *c = (or_ctx *)calloc(1, sizeof(or_ctx));
  c->n_sites = n_sites; c->n_pairs = n_pairs; c->n_max = n_max; c->k_max = k_max; c->l_max = l_max;
  c->n_soap_unc = n_soap_unc;
  c->k_first = (int *)malloc(sizeof(int) * (n_sites + 1));
  c->rad = (double *)calloc((size_t)n_max * n_pairs + 1, sizeof(double));
  c->rad_der = (double *)calloc((size_t)n_max * n_pairs + 1, sizeof(double));
  if (do_der2) c->rad_der2 = (double *)calloc((size_t)n_max * n_pairs + 1, sizeof(double));
  c->ang = (double *)calloc((size_t)2 * k_max * n_pairs + 1, sizeof(double));
  if (need_der) {
    c->ang_r = (double *)calloc((size_t)2 * k_max * n_pairs + 1, sizeof(double));
    c->ang_a = (double *)calloc((size_t)2 * k_max * n_pairs + 1, sizeof(double));
    c->ang_p = (double *)calloc((size_t)2 * k_max * n_pairs + 1, sizeof(double));
  }
  c->cnk = (double *)calloc((size_t)2 * k_max * n_max * n_sites + 1, sizeof(double));
  c->sqrt_dot_p = (double *)calloc((size_t)n_sites + 1, sizeof(double));
  c->skip = (unsigned char *)calloc((size_t)n_soap_unc + 1, 1);
  c->rjs = a->rjs; c->thetas = a->thetas; c->phis = a->phis; c->n_neigh = a->n_neigh;
  int k2 = 0;
  for (int i = 0; i < n_sites; i++) { c->k_first[i] = k2; k2 += a->n_neigh[i]; }
  c->k_first[n_sites] = k2;

  /* ---- radial, per species (:491-544 -> src/soap_turbo_radial.f90:281-384) */
  for (int sp = 0; sp < a->n_species; sp++) {
    int alpha = a->alpha_max[sp];
    int with_gauss = a->basis == 1, op = a->basis == 2;
    int do_central = with_gauss ? 0 : (a->central_weight[sp] != 0.0);  /* :238-245; :232-238 */
    if (op) do_central = 1;                                              /* src/soap_turbo.f90:539 */
    or_radial_setup st;
    or_radial_init(&st, alpha, a->rcut_soft[sp], a->rcut_hard[sp], a->atom_sigma_r[sp],
                   a->atom_sigma_r_scaling[sp], a->amplitude_scaling[sp], a->nf[sp],
                   a->W + (size_t)i_beg[sp] * n_max + i_beg[sp], n_max, a->scaling_poly,
                   a->radial_enhancement, need_der, do_central, a->central_weight[sp], with_gauss,
                   a->legacy_filter_seed);
    if (do_der2) or_radial_enable_der2(&st);
    const double gsc = a->global_scaling[sp];
    #pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n_sites; i++) {
      for (int j = 0; j < a->n_neigh[i]; j++) {
        int k = c->k_first[i] + j;
        double *out = c->rad + (size_t)k * n_max + i_beg[sp];
        double *der = c->rad_der + (size_t)k * n_max + i_beg[sp];
        double *der2 = do_der2 ? c->rad_der2 + (size_t)k * n_max + i_beg[sp] : NULL;
        for (int n = 0; n < alpha; n++) { out[n] = 0.0; der[n] = 0.0; if (der2) der2[n] = 0.0; } /* :328-340 */
        if (j == 0 && !do_central) continue;                               /* :342-355 */
        if (!op && a->rjs[k] >= a->rcut_hard[sp]) continue;
        if (!a->mask[(size_t)sp * n_pairs + k]) continue;
        double o[32], d[32], d2[32];
        if (op)
          or_radial_op_pair(alpha, a->rcut_soft[sp], a->rcut_hard[sp], a->atom_sigma_r[sp],
                            a->atom_sigma_r_scaling[sp], a->amplitude_scaling[sp], a->scaling_poly,
                            a->radial_enhancement, a->central_weight[sp], j == 0,
                            a->W + (size_t)i_beg[sp] * n_max + i_beg[sp], n_max, a->rjs[k], o, d);
        else
          or_radial_pair(&st, a->rjs[k], j == 0, o, d, der2 ? d2 : NULL);
        for (int n = 0; n < alpha; n++) {
          out[n] = o[n] * gsc;                                             /* :510-511, :532-533 */
          if (need_der) der[n] = d[n] * gsc;
          if (der2) der2[n] = d2[n] * gsc;
        }
      }
    }
  }

  /* ---- angular, src/soap_turbo_angular.f90:485-617 */
  double rcut_max = 0.0;
  for (int sp = 0; sp < a->n_species; sp++) if (a->rcut_hard[sp] > rcut_max) rcut_max = a->rcut_hard[sp];
  double *preflm = (double *)malloc(sizeof(double) * k_max);
  or_preflm(l_max, preflm);
  {
    const double rcut2 = rcut_max * rcut_max;
    #pragma omp parallel for schedule(dynamic, 64)
    for (int k = 0; k < n_pairs; k++) {
      double plm[128], div_sin[128], der_mul_sin[128], il[32], ild[32];
      double pm_re[32], pm_im[32];
      double rj = a->rjs[k];
      int i_sp = -1;
      if (rj < rcut_max)
        for (int s = 0; s < a->n_species; s++) if (a->mask[(size_t)s * n_pairs + k]) { i_sp = s; break; }
      double *A = c->ang + (size_t)2 * k_max * k;
      if (i_sp < 0) {
        for (int kk = 0; kk < 2 * k_max; kk++) A[kk] = 0.0;
        if (need_der)
          for (int kk = 0; kk < 2 * k_max; kk++) {
            c->ang_r[(size_t)2 * k_max * k + kk] = 0.0;
            c->ang_a[(size_t)2 * k_max * k + kk] = 0.0;
            c->ang_p[(size_t)2 * k_max * k + kk] = 0.0;
          }
        continue;
      }
      double phi = a->phis[k], x = cos(a->thetas[k]);
      double sig = a->atom_sigma_t[i_sp] + a->atom_sigma_t_scaling[i_sp] * rj;
      double amplitude = rcut2 / (sig * sig);
      /* get_eimphi_conjg, :267-329 */
      or_ilexp_array(l_max + 1, rj / sig, il);
      double cosm2 = cos(phi), cosphi2 = 2.0 * cosm2, sinm2 = -sin(phi), cosm1 = 1.0, sinm1 = 0.0;
      pm_re[0] = 1.0; pm_im[0] = 0.0;
      for (int l = 1; l <= l_max; l++) {
        double cos0 = cosphi2 * cosm1 - cosm2, sin0 = cosphi2 * sinm1 - sinm2;
        cosm2 = cosm1; sinm2 = sinm1; cosm1 = cos0; sinm1 = sin0;
        pm_re[l] = cos0; pm_im[l] = -sin0;
      }
      if (need_der) {
        or_ilexp_der(il, l_max, rj, sig, a->atom_sigma_t_scaling[i_sp], ild);
        or_plm_array(l_max + 1, x, plm);
        or_plm_array_der(l_max, plm, div_sin, der_mul_sin);
        double sig_fac = 2.0 * a->atom_sigma_t_scaling[i_sp] / sig;
        double *Ar = c->ang_r + (size_t)2 * k_max * k, *Aa = c->ang_a + (size_t)2 * k_max * k;
        double *Ap = c->ang_p + (size_t)2 * k_max * k;
        for (int l = 0; l <= l_max; l++)
          for (int m = 0; m <= l; m++) {
            int kk = kidx(l, m);
            double e_re = il[l] * pm_re[m], e_im = il[l] * pm_im[m];        /* eimphi */
            double er_re = ild[l] * pm_re[m], er_im = ild[l] * pm_im[m];    /* eimphi_rad_der */
            double u = amplitude * preflm[kk];
            double v = u * plm[kk];
            double ec_re = v * e_re, ec_im = v * e_im;
            A[2 * kk] = ec_re; A[2 * kk + 1] = ec_im;
            Ar[2 * kk] = v * er_re - sig_fac * ec_re;
            Ar[2 * kk + 1] = v * er_im - sig_fac * ec_im;
            double w = u * div_sin[kk];
            double ez_re = w * e_re, ez_im = w * e_im;
            Aa[2 * kk] = -ez_im; Aa[2 * kk + 1] = ez_re;
            double w2 = u * der_mul_sin[kk];
            Ap[2 * kk] = w2 * e_re; Ap[2 * kk + 1] = w2 * e_im;
          }
      } else {
        or_plm_array(l_max, x, plm);
        for (int l = 0; l <= l_max; l++)
          for (int m = 0; m <= l; m++) {
            int kk = kidx(l, m);
            double e_re = il[l] * pm_re[m], e_im = il[l] * pm_im[m];
            double v = amplitude * preflm[kk] * plm[kk];
            A[2 * kk] = v * e_re; A[2 * kk + 1] = v * e_im;
          }
      }
    }
  }

  /* ---- cnk, src/soap_turbo.f90:619-664 */
  #pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n_sites; i++) {
    double *ci = c->cnk + (size_t)2 * k_max * n_max * i;
    for (int j = 0; j < a->n_neigh[i]; j++) {
      int k = c->k_first[i] + j;
      const double *A = c->ang + (size_t)2 * k_max * k;
      for (int n = 0; n < n_max; n++) {
        double fr = 4.0 * pi * c->rad[(size_t)k * n_max + n];
        double *cn = ci + (size_t)2 * k_max * n;
        for (int kk = 0; kk < k_max; kk++) {
          cn[2 * kk] = cn[2 * kk] + fr * A[2 * kk];
          cn[2 * kk + 1] = cn[2 * kk + 1] + fr * A[2 * kk + 1];
        }
      }
    }
    for (int mm = 0; mm < a->species_multiplicity[i]; mm++) {
      int sj = a->species[(size_t)i * a->max_mult + mm] - 1;
      if (sj < 0) continue;
      if (a->basis == 1 && a->central_weight[sj] != 0.0) {
        double amplitude;
        if (a->radial_enhancement == 1) amplitude = sqrt(2.0 / pi) * a->atom_sigma_r[sj] / a->rcut_hard[sj];
        else if (a->radial_enhancement == 2)
          amplitude = pow(a->atom_sigma_r[sj], 2) / pow(a->rcut_hard[sj], 2);
        else amplitude = 1.0;
        double fac = amplitude * a->central_weight[sj] * sqrt(4.0 * pi) * pow(pi, 0.25)
                     * sqrt(a->atom_sigma_r[sj] / 2.0) * pow(a->rcut_hard[sj], 3)
                     / pow(a->atom_sigma_t[sj], 2) / a->atom_sigma_r[sj];
        int b = i_beg[sj], al = a->alpha_max[sj];
        for (int n = 0; n < al; n++) {
          double ws = 0.0;
          for (int m = 0; m < al; m++)
            ws += a->W[(size_t)(b + m) * n_max + (b + n)] * a->S[(size_t)(b + al - 1) * n_max + (b + m)];
          ci[(size_t)2 * k_max * (b + n)] += fac * ws;
        }
      }
    }
  }

  /* ---- compression skip mask, :411-431 */
  int n_soap;
  if (a->compress) {
    int mx = 0;
    for (int t = 0; t < a->P_nonzero; t++) if (a->P_i[t] > mx) mx = a->P_i[t];
    n_soap = mx;
    for (int t = 0; t < n_soap_unc; t++) c->skip[t] = 1;
    for (int t = 0; t < a->P_nonzero; t++) c->skip[a->P_j[t] - 1] = 0;
  } else {
    n_soap = n_soap_unc;
  }
  c->n_soap = n_soap; c->compress = a->compress; c->P_nonzero = a->P_nonzero;
  c->P_i = a->P_i; c->P_j = a->P_j; c->P_el = a->P_el;

  /* ---- power spectrum + compression + norm, :687-813 */
  #pragma omp parallel
  {
    double *this_soap = (double *)calloc((size_t)n_soap_unc + 1, sizeof(double));
    #pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < n_sites; i++) {
      const double *ci = c->cnk + (size_t)2 * k_max * n_max * i;
      int counter = 0;
      for (int n = 0; n < n_max; n++)
        for (int np = n; np < n_max; np++)
          for (int l = 0; l <= l_max; l++) {
            int cidx = counter++;
            if (c->skip[cidx]) { this_soap[cidx] = 0.0; continue; }
            double acc = 0.0;
            for (int m = 0; m <= l; m++) {
              int kk = kidx(l, m);
              double mult = 1.0;
              if (n != np) mult *= sqrt(2.0);
              if (m > 0) mult *= 2.0;
              double unr = ci[(size_t)2 * (k_max * n + kk)], uni = ci[(size_t)2 * (k_max * n + kk) + 1];
              double upr = ci[(size_t)2 * (k_max * np + kk)], upi = ci[(size_t)2 * (k_max * np + kk) + 1];
              acc = acc + mult * (unr * upr + uni * upi);
            }
            this_soap[cidx] = acc;
          }
      double *si = soap + (size_t)n_soap * i;
      if (a->compress) {
        for (int t = 0; t < a->P_nonzero; t++)
          si[a->P_i[t] - 1] = si[a->P_i[t] - 1] + a->P_el[t] * this_soap[a->P_j[t] - 1];
      } else {
        for (int s = 0; s < n_soap; s++) si[s] = this_soap[s];
      }
      double dot = 0.0;
      for (int s = 0; s < n_soap; s++) dot += si[s] * si[s];
      c->sqrt_dot_p[i] = sqrt(dot);
      if (c->sqrt_dot_p[i] < 1.0e-5) c->sqrt_dot_p[i] = 1.0;
    }
    free(this_soap);
  }

  /* ---- spherical derivatives + Cartesian rotation, :816-902, :1927-2075 */
  if (need_der && soap_cart_der) {
    const double fourpi = 4.0 * pi, sq2 = sqrt(2.0);
    #pragma omp parallel
    {
      double *trad = (double *)calloc((size_t)n_soap_unc + 1, sizeof(double));
      double *tazi = (double *)calloc((size_t)n_soap_unc + 1, sizeof(double));
      double *tpol = (double *)calloc((size_t)n_soap_unc + 1, sizeof(double));
      double *drad = (double *)calloc((size_t)n_soap + 1, sizeof(double));
      double *dazi = (double *)calloc((size_t)n_soap + 1, sizeof(double));
      double *dpol = (double *)calloc((size_t)n_soap + 1, sizeof(double));
      double *P = (double *)malloc(sizeof(double) * n_max * (l_max + 1));
      double *Q = (double *)malloc(sizeof(double) * n_max * (l_max + 1));
      double *Qa = (double *)malloc(sizeof(double) * n_max * (l_max + 1));
      double *Qo = (double *)malloc(sizeof(double) * n_max * (l_max + 1));
      #pragma omp for schedule(dynamic, 16)
      for (int i = 0; i < n_sites; i++) {
        const double *ci = c->cnk + (size_t)2 * k_max * n_max * i;
        const double *si = soap + (size_t)n_soap * i;
        int k3 = c->k_first[i];
        double inv_p = 1.0 / c->sqrt_dot_p[i];
        double inv_p3 = 1.0 / pow(c->sqrt_dot_p[i], 3);
        double *self = soap_cart_der + (size_t)k3 * n_soap * 3;
        for (int j = 1; j < a->n_neigh[i]; j++) {
          int k2 = c->k_first[i] + j;
          const double *A = c->ang + (size_t)2 * k_max * k2, *Ar = c->ang_r + (size_t)2 * k_max * k2;
          const double *Aa = c->ang_a + (size_t)2 * k_max * k2, *Ap = c->ang_p + (size_t)2 * k_max * k2;
          for (int n = 0; n < n_max; n++)
            for (int l = 0; l <= l_max; l++) {
              double ap = 0, aq = 0, aa = 0, ao = 0;
              for (int m = 0; m <= l; m++) {
                int kk = kidx(l, m);
                double w = (m == 0) ? 1.0 : 2.0;
                double cr = ci[(size_t)2 * (k_max * n + kk)], cim = ci[(size_t)2 * (k_max * n + kk) + 1];
                ap = ap + w * (A[2 * kk] * cr + A[2 * kk + 1] * cim);
                aq = aq + w * (Ar[2 * kk] * cr + Ar[2 * kk + 1] * cim);
                aa = aa + w * (Aa[2 * kk] * cr + Aa[2 * kk + 1] * cim);
                ao = ao + w * (Ap[2 * kk] * cr + Ap[2 * kk + 1] * cim);
              }
              P[n * (l_max + 1) + l] = ap; Q[n * (l_max + 1) + l] = aq;
              Qa[n * (l_max + 1) + l] = aa; Qo[n * (l_max + 1) + l] = ao;
            }
          int counter = 0;
          for (int n = 0; n < n_max; n++) {
            double rn = c->rad[(size_t)k2 * n_max + n], rdn = c->rad_der[(size_t)k2 * n_max + n];
            for (int np = n; np < n_max; np++) {
              double rnp = c->rad[(size_t)k2 * n_max + np], rdnp = c->rad_der[(size_t)k2 * n_max + np];
              double base = (n == np) ? 1.0 : sq2, pre = fourpi * base;
              for (int l = 0; l <= l_max; l++) {
                int cidx = counter++;
                if (c->skip[cidx]) continue;
                int L1 = l_max + 1;
                trad[cidx] = pre * (rdn * P[np * L1 + l] + rn * Q[np * L1 + l] + rdnp * P[n * L1 + l] + rnp * Q[n * L1 + l]);
                tazi[cidx] = pre * (rn * Qa[np * L1 + l] + rnp * Qa[n * L1 + l]);
                tpol[cidx] = pre * (rn * Qo[np * L1 + l] + rnp * Qo[n * L1 + l]);
              }
            }
          }
          if (a->compress) {
            for (int s = 0; s < n_soap; s++) drad[s] = dazi[s] = dpol[s] = 0.0;
            for (int t = 0; t < a->P_nonzero; t++) {
              int pi_ = a->P_i[t] - 1, pj = a->P_j[t] - 1;
              drad[pi_] = drad[pi_] + a->P_el[t] * trad[pj];
              dazi[pi_] = dazi[pi_] + a->P_el[t] * tazi[pj];
              dpol[pi_] = dpol[pi_] + a->P_el[t] * tpol[pj];
            }
          } else {
            for (int s = 0; s < n_soap; s++) { drad[s] = trad[s]; dazi[s] = tazi[s]; dpol[s] = tpol[s]; }
          }
          double dot_r = 0, dot_a = 0, dot_o = 0;
          for (int s = 0; s < n_soap; s++) {
            dot_r = dot_r + si[s] * drad[s];
            dot_a = dot_a + si[s] * dazi[s];
            dot_o = dot_o + si[s] * dpol[s];
          }
          double sin_t = sin(a->thetas[k2]), cos_t = cos(a->thetas[k2]);
          double sin_f = sin(a->phis[k2]), cos_f = cos(a->phis[k2]);
          double inv_r = 1.0 / a->rjs[k2];
          double cx = sin_t * cos_f, cy = sin_t * sin_f, cz = cos_t;
          double px = -cos_t * cos_f * inv_r, py = -cos_t * sin_f * inv_r, pz = sin_t * inv_r;
          double ax = -sin_f * inv_r, ay = cos_f * inv_r;
          double *out = soap_cart_der + (size_t)k2 * n_soap * 3;
          for (int s = 0; s < n_soap; s++) {
            double sv = si[s];
            double vr = drad[s] * inv_p - sv * inv_p3 * dot_r;
            double va = dazi[s] * inv_p - sv * inv_p3 * dot_a;
            double vo = dpol[s] * inv_p - sv * inv_p3 * dot_o;
            out[3 * s + 0] = cx * vr + px * vo + ax * va;
            out[3 * s + 1] = cy * vr + py * vo + ay * va;
            out[3 * s + 2] = cz * vr + pz * vo;
          }
          for (int t = 0; t < 3 * n_soap; t++) self[t] = self[t] - out[t];
        }
      }
      free(trad); free(tazi); free(tpol); free(drad); free(dazi); free(dpol);
      free(P); free(Q); free(Qa); free(Qo);
    }
  }

  /* ---- normalise, :904-909 */
  #pragma omp parallel for schedule(static)
  for (int i = 0; i < n_sites; i++)
    for (int s = 0; s < n_soap; s++) soap[(size_t)n_soap * i + s] = soap[(size_t)n_soap * i + s] / c->sqrt_dot_p[i];

  free(preflm);
  if (ctx_out) *ctx_out = c; else or_ctx_free(c);
  return n_soap;
}

/* soap_contract, src/soap_turbo.f90:1723-1884.  ctx comes from or_get_soap
 * called with do_derivatives = 1. */
int or_soap_contract(const or_ctx *c, const double *soap, const double *G, double sgn, double *pair) {
  if (!c || !c->ang_r) return -1;
  const double fourpi = 4.0 * acos(-1.0), sq2 = sqrt(2.0);
  const int n_max = c->n_max, k_max = c->k_max, l_max = c->l_max, n_soap = c->n_soap;
  const int n_sites = c->n_sites;
  #pragma omp parallel
  {
    double *Gp = (double *)malloc(sizeof(double) * (n_soap + 1));
    double *Gu = (double *)malloc(sizeof(double) * (c->n_soap_unc + 1));
    double *Y = (double *)malloc(sizeof(double) * n_max * n_max * (l_max + 1));
    double *H = (double *)malloc(sizeof(double) * 2 * k_max * n_max);
    #pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < n_sites; i++) {
      const double *si = soap + (size_t)n_soap * i;
      const double *ci = c->cnk + (size_t)2 * k_max * n_max * i;
      double qg = 0.0;
      for (int k = 0; k < n_soap; k++) qg = qg + si[k] * G[(size_t)k * n_sites + i];
      double inv = 1.0 / c->sqrt_dot_p[i];
      for (int k = 0; k < n_soap; k++) Gp[k] = (G[(size_t)k * n_sites + i] - si[k] * qg) * inv;
      if (c->compress) {
        for (int t = 0; t < c->n_soap_unc; t++) Gu[t] = 0.0;
        for (int t = 0; t < c->P_nonzero; t++)
          Gu[c->P_j[t] - 1] = Gu[c->P_j[t] - 1] + c->P_el[t] * Gp[c->P_i[t] - 1];
      } else {
        for (int k = 0; k < n_soap; k++) Gu[k] = Gp[k];
      }
      int counter = 0;
      for (int n = 0; n < n_max; n++)
        for (int np = n; np < n_max; np++) {
          double base = (n == np) ? 1.0 : sq2;
          for (int l = 0; l <= l_max; l++) {
            int cidx = counter++;
            double x = 0.0;
            if (!c->skip[cidx]) x = Gu[cidx] * base;
            if (n == np) Y[(l * n_max + n) * n_max + n] = 2.0 * x;
            else { Y[(l * n_max + np) * n_max + n] = x; Y[(l * n_max + n) * n_max + np] = x; }
          }
        }
      for (int n = 0; n < n_max; n++)
        for (int l = 0; l <= l_max; l++)
          for (int m = 0; m <= l; m++) {
            int kk = kidx(l, m);
            double hr = 0.0, hi = 0.0;
            for (int np = 0; np < n_max; np++) {
              double y = Y[(l * n_max + np) * n_max + n];
              hr = hr + y * ci[(size_t)2 * (k_max * np + kk)];
              hi = hi + y * ci[(size_t)2 * (k_max * np + kk) + 1];
            }
            double w = (m == 0) ? 1.0 : 2.0;
            H[2 * (kk * n_max + n)] = w * hr;
            H[2 * (kk * n_max + n) + 1] = w * hi;
          }
      int k3 = c->k_first[i];
      double sx = 0, sy = 0, sz = 0;
      for (int j = 1; j < c->n_neigh[i]; j++) {
        int k2 = c->k_first[i] + j;
        const double *A = c->ang + (size_t)2 * k_max * k2, *Ar = c->ang_r + (size_t)2 * k_max * k2;
        const double *Aa = c->ang_a + (size_t)2 * k_max * k2, *Ap = c->ang_p + (size_t)2 * k_max * k2;
        double f_rad = 0, f_azi = 0, f_pol = 0;
        for (int n = 0; n < n_max; n++) {
          double sd = 0, sr = 0, sa = 0, so = 0;
          for (int kk = 0; kk < k_max; kk++) {
            double hr = H[2 * (kk * n_max + n)], hi = H[2 * (kk * n_max + n) + 1];
            sd = sd + A[2 * kk] * hr + A[2 * kk + 1] * hi;
            sr = sr + Ar[2 * kk] * hr + Ar[2 * kk + 1] * hi;
            sa = sa + Aa[2 * kk] * hr + Aa[2 * kk + 1] * hi;
            so = so + Ap[2 * kk] * hr + Ap[2 * kk + 1] * hi;
          }
          f_rad = f_rad + c->rad_der[(size_t)k2 * n_max + n] * sd + c->rad[(size_t)k2 * n_max + n] * sr;
          f_azi = f_azi + c->rad[(size_t)k2 * n_max + n] * sa;
          f_pol = f_pol + c->rad[(size_t)k2 * n_max + n] * so;
        }
        f_rad *= fourpi; f_azi *= fourpi; f_pol *= fourpi;
        double sin_t = sin(c->thetas[k2]), cos_t = cos(c->thetas[k2]);
        double sin_f = sin(c->phis[k2]), cos_f = cos(c->phis[k2]);
        double inv_r = 1.0 / c->rjs[k2];
        double px = sgn * (sin_t * cos_f * f_rad - cos_t * cos_f * inv_r * f_pol - sin_f * inv_r * f_azi);
        double py = sgn * (sin_t * sin_f * f_rad - cos_t * sin_f * inv_r * f_pol + cos_f * inv_r * f_azi);
        double pz = sgn * (cos_t * f_rad + sin_t * inv_r * f_pol);
        pair[3 * k2] = px; pair[3 * k2 + 1] = py; pair[3 * k2 + 2] = pz;
        sx = sx - px; sy = sy - py; sz = sz - pz;
      }
      if (c->n_neigh[i] > 0) { pair[3 * k3] = sx; pair[3 * k3 + 1] = sy; pair[3 * k3 + 2] = sz; }
    }
    free(Gp); free(Gu); free(Y); free(H);
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* get_soap_central_hessian, src/soap_turbo.f90:1151-1700, on the state of    */
/* or_get_soap2(do_derivatives = 1, do_der2 = 1).                            */
/* ------------------------------------------------------------------------ */
typedef double complex cplx;

/* The unnormalised, compressed spherical derivatives of site i's p for pair
 * k2 (soap_rad/azi/pol_der, src/soap_turbo.f90:1927-2075), as get_soap builds
 * them before the normalisation. */
static void hs_pair_sph(const or_args *a, const or_ctx *c, int i, int k2, double *trad, double *tazi,
                        double *tpol, double *drad, double *dazi, double *dpol, double *P, double *Q,
                        double *Qa, double *Qo) {
  const int n_max = c->n_max, k_max = c->k_max, l_max = c->l_max, L1 = l_max + 1, n_soap = c->n_soap;
  const double fourpi = 4.0 * acos(-1.0), sq2 = sqrt(2.0);
  const double *ci = c->cnk + (size_t)2 * k_max * n_max * i;
  const double *A = c->ang + (size_t)2 * k_max * k2, *Ar = c->ang_r + (size_t)2 * k_max * k2;
  const double *Aa = c->ang_a + (size_t)2 * k_max * k2, *Ap = c->ang_p + (size_t)2 * k_max * k2;
  for (int n = 0; n < n_max; n++)
    for (int l = 0; l <= l_max; l++) {
      double ap = 0, aq = 0, aa = 0, ao = 0;
      for (int m = 0; m <= l; m++) {
        int kk = kidx(l, m);
        double w = (m == 0) ? 1.0 : 2.0;
        double cr = ci[(size_t)2 * (k_max * n + kk)], cim = ci[(size_t)2 * (k_max * n + kk) + 1];
        ap = ap + w * (A[2 * kk] * cr + A[2 * kk + 1] * cim);
        aq = aq + w * (Ar[2 * kk] * cr + Ar[2 * kk + 1] * cim);
        aa = aa + w * (Aa[2 * kk] * cr + Aa[2 * kk + 1] * cim);
        ao = ao + w * (Ap[2 * kk] * cr + Ap[2 * kk + 1] * cim);
      }
      P[n * L1 + l] = ap; Q[n * L1 + l] = aq; Qa[n * L1 + l] = aa; Qo[n * L1 + l] = ao;
    }
  int counter = 0;
  for (int n = 0; n < n_max; n++) {
    double rn = c->rad[(size_t)k2 * n_max + n], rdn = c->rad_der[(size_t)k2 * n_max + n];
    for (int np = n; np < n_max; np++) {
      double rnp = c->rad[(size_t)k2 * n_max + np], rdnp = c->rad_der[(size_t)k2 * n_max + np];
      double pre = fourpi * ((n == np) ? 1.0 : sq2);
      for (int l = 0; l <= l_max; l++) {
        int cidx = counter++;
        if (c->skip[cidx]) { trad[cidx] = tazi[cidx] = tpol[cidx] = 0.0; continue; }
        trad[cidx] = pre * (rdn * P[np * L1 + l] + rn * Q[np * L1 + l] + rdnp * P[n * L1 + l] + rnp * Q[n * L1 + l]);
        tazi[cidx] = pre * (rn * Qa[np * L1 + l] + rnp * Qa[n * L1 + l]);
        tpol[cidx] = pre * (rn * Qo[np * L1 + l] + rnp * Qo[n * L1 + l]);
      }
    }
  }
  if (c->compress) {
    for (int s = 0; s < n_soap; s++) drad[s] = dazi[s] = dpol[s] = 0.0;
    for (int t = 0; t < a->P_nonzero; t++) {
      int pi_ = a->P_i[t] - 1, pj = a->P_j[t] - 1;
      drad[pi_] = drad[pi_] + a->P_el[t] * trad[pj];
      dazi[pi_] = dazi[pi_] + a->P_el[t] * tazi[pj];
      dpol[pi_] = dpol[pi_] + a->P_el[t] * tpol[pj];
    }
  } else {
    for (int s = 0; s < n_soap; s++) { drad[s] = trad[s]; dazi[s] = tazi[s]; dpol[s] = tpol[s]; }
  }
}

/* hess(a, b, v, k2) = sum_d vecs(d, v, i) d^2 q_d / dr_ia dr_jb for pair k2 =
 * (site i, neighbour j), a of the central atom and b of the neighbour; the self
 * pair's block is minus the sum of the others (:1488-1495).  Layouts (C):
 * vecs[(i * n_vec + v) * n_soap + d], hess[((k2 * n_vec + v) * 3 + b) * 3 + a].
 * selftest_err (may be NULL) receives the largest relative gap between the
 * first derivative rebuilt from the same contraction and the one from the
 * spherical derivatives (soap_hessian_selftest, :1395-1412).  Returns 0, or -1
 * without second radial derivatives in ctx. */
int or_central_hessian(const or_args *a, const or_ctx *c, const double *soap, int n_vec, const double *vecs,
                       double *hess, double *selftest_err) {
  if (!c->rad_der2 || !c->ang_r) return -1;
  const int n_sites = c->n_sites, n_max = c->n_max, k_max = c->k_max, l_max = c->l_max;
  const int n_soap = c->n_soap, n_soap_unc = c->n_soap_unc, nv = n_vec + 1, n_pairs = c->n_pairs;
  const double pi = acos(-1.0), fourpi = 4.0 * pi, sqrt2 = sqrt(2.0);
  double rcut_max = 0.0;
  for (int sp = 0; sp < a->n_species; sp++) if (a->rcut_hard[sp] > rcut_max) rcut_max = a->rcut_hard[sp];
  int *lofk = (int *)malloc(sizeof(int) * k_max), *mofk = (int *)malloc(sizeof(int) * k_max);
  double *wm = (double *)malloc(sizeof(double) * k_max), *preflm = (double *)malloc(sizeof(double) * k_max);
  double *Ck = (double *)malloc(sizeof(double) * k_max);
  for (int l = 0, k = 0; l <= l_max; l++)
    for (int m = 0; m <= l; m++, k++) { lofk[k] = l; mofk[k] = m; wm[k] = m > 0 ? 2.0 : 1.0; }
  or_preflm(l_max, preflm);
  for (int k = 0; k < k_max; k++) Ck[k] = (mofk[k] % 2 == 0) ? preflm[k] : -preflm[k];   /* :1264-1271 */
  for (size_t t = 0; t < (size_t)9 * n_vec * n_pairs; t++) hess[t] = 0.0;
  double chk_err = 0.0, chk_ref = 0.0;

  #pragma omp parallel reduction(max : chk_err, chk_ref)
  {
    cplx *Gacc = (cplx *)malloc(sizeof(cplx) * n_max * k_max * 3);
    cplx *Zv = (cplx *)malloc(sizeof(cplx) * n_max * k_max * nv);
    cplx *ZGv = (cplx *)malloc(sizeof(cplx) * n_max * k_max * 3 * nv);
    double *Smat = (double *)malloc(sizeof(double) * n_max * n_max * (l_max + 1));
    double *vunc = (double *)malloc(sizeof(double) * (n_soap_unc + 1)), *pvec = (double *)malloc(sizeof(double) * n_soap);
    double *dp1 = (double *)malloc(sizeof(double) * n_soap * 3), *dp2 = (double *)malloc(sizeof(double) * n_soap * 3);
    double *trad = (double *)malloc(sizeof(double) * (n_soap_unc + 1)), *tazi = (double *)malloc(sizeof(double) * (n_soap_unc + 1));
    double *tpol = (double *)malloc(sizeof(double) * (n_soap_unc + 1));
    double *drad = (double *)malloc(sizeof(double) * n_soap), *dazi = (double *)malloc(sizeof(double) * n_soap);
    double *dpol = (double *)malloc(sizeof(double) * n_soap);
    double *Pb = (double *)malloc(sizeof(double) * n_max * (l_max + 1) * 4);
    double *il = (double *)malloc(sizeof(double) * (l_max + 4)), *dilz = (double *)malloc(sizeof(double) * (l_max + 1));
    double *d2ilz = (double *)malloc(sizeof(double) * (l_max + 1));
    double *Fl = (double *)malloc(sizeof(double) * (l_max + 1)), *Fl1 = (double *)malloc(sizeof(double) * (l_max + 1));
    double *Fl2 = (double *)malloc(sizeof(double) * (l_max + 1)), *Qt = (double *)malloc(sizeof(double) * k_max);
    cplx *Om = (cplx *)malloc(sizeof(cplx) * k_max), *dOm = (cplx *)malloc(sizeof(cplx) * 3 * k_max);
    cplx *d2Om = (cplx *)malloc(sizeof(cplx) * 9 * k_max), *wpow = (cplx *)malloc(sizeof(cplx) * (l_max + 3));
    double *hv = (double *)malloc(sizeof(double) * 9 * nv), *hsum = (double *)malloc(sizeof(double) * 9 * (n_vec + 1));
    double *u2rec = (double *)malloc(sizeof(double) * 3 * nv);
    double nh[3], tvec[3], thes[9], rr = 0, invr = 0;
    cplx wvec[3], whes[9];

    /* F_l, Omega, dOmega and (want2) d2Omega of one pair (pair_geometry, :1537-1652) */
#define PAIR_GEOMETRY(kk, good, want2)                                                                       \
    do {                                                                                                     \
      good = 0;                                                                                              \
      rr = a->rjs[kk];                                                                                       \
      if (rr >= rcut_max || rr < 1.0e-10) break;                                                            \
      int isp = -1;                                                                                          \
      for (int q = 0; q < a->n_species; q++) if (a->mask[(size_t)q * n_pairs + (kk)]) { isp = q; break; }    \
      if (isp < 0) break;                                                                                    \
      good = 1;                                                                                              \
      invr = 1.0 / rr;                                                                                       \
      const double invr2 = invr * invr;                                                                      \
      const double sscal = a->atom_sigma_t_scaling[isp], sig = a->atom_sigma_t[isp] + sscal * rr;           \
      const double amp = rcut_max * rcut_max / (sig * sig), ampd = -2.0 * sscal / sig * amp;                 \
      const double ampdd = 6.0 * sscal * sscal / (sig * sig) * amp;                                          \
      const double xarg = rr / sig, zz = xarg * xarg, invz = 1.0 / zz;                                      \
      or_ilexp_array(l_max + 2, xarg, il);                                                                   \
      for (int l = 0; l <= l_max; l++) {                                                                     \
        const double rl = (double)l;                                                                         \
        dilz[l] = il[l + 1] + (rl * invz - 1.0) * il[l];                                                     \
        d2ilz[l] = il[l + 2] + ((double)(2 * l + 1) * invz - 2.0) * il[l + 1]                               \
                   + (rl * (rl - 1.0) * invz * invz - 2.0 * rl * invz + 1.0) * il[l];                        \
      }                                                                                                      \
      const double zp = 2.0 * rr / (sig * sig) - 2.0 * rr * rr * sscal / (sig * sig * sig);                \
      const double zp2 = 2.0 / (sig * sig) - 8.0 * rr * sscal / (sig * sig * sig)                           \
                         + 6.0 * rr * rr * sscal * sscal / (sig * sig * sig * sig);                           \
      for (int l = 0; l <= l_max; l++) {                                                                     \
        const double f0_ = il[l], f1_ = dilz[l] * zp, f2_ = d2ilz[l] * zp * zp + dilz[l] * zp2;             \
        Fl[l] = amp * f0_;                                                                                   \
        Fl1[l] = ampd * f0_ + amp * f1_;                                                                     \
        Fl2[l] = ampdd * f0_ + 2.0 * ampd * f1_ + amp * f2_;                                                 \
      }                                                                                                      \
      const double sin_t = sin(a->thetas[kk]), cos_t = cos(a->thetas[kk]);                                   \
      const double sin_f = sin(a->phis[kk]), cos_f = cos(a->phis[kk]);                                       \
      nh[0] = sin_t * cos_f; nh[1] = sin_t * sin_f; nh[2] = cos_t;                                           \
      const double tt = nh[2];                                                                               \
      const cplx wc = nh[0] - I * nh[1];                                                                     \
      const cplx ec[3] = {1.0, -I, 0.0};                                                                     \
      for (int q = 0; q < 3; q++) { tvec[q] = -tt * nh[q] * invr; wvec[q] = -wc * nh[q] * invr; }          \
      tvec[2] = tvec[2] + invr;                                                                              \
      for (int q = 0; q < 3; q++) wvec[q] = wvec[q] + ec[q] * invr;                                          \
      if (want2) {                                                                                           \
        for (int bb = 0; bb < 3; bb++)                                                                       \
          for (int aa = 0; aa < 3; aa++) {                                                                   \
            thes[bb * 3 + aa] = (3.0 * tt * nh[aa] * nh[bb]) * invr2;                                        \
            whes[bb * 3 + aa] = (3.0 * wc * nh[aa] * nh[bb] - ec[aa] * nh[bb] - ec[bb] * nh[aa]) * invr2;    \
          }                                                                                                  \
        for (int aa = 0; aa < 3; aa++) {                                                                     \
          thes[aa * 3 + 2] = thes[aa * 3 + 2] - nh[aa] * invr2;                                              \
          thes[2 * 3 + aa] = thes[2 * 3 + aa] - nh[aa] * invr2;                                              \
          thes[aa * 3 + aa] = thes[aa * 3 + aa] - tt * invr2;                                                \
          whes[aa * 3 + aa] = whes[aa * 3 + aa] - wc * invr2;                                                \
        }                                                                                                    \
      }                                                                                                      \
      Qt[0] = 1.0;                                                                                           \
      if (l_max >= 1) { Qt[1] = tt; Qt[2] = 1.0; }                                                          \
      for (int ll = 2; ll <= l_max; ll++) {                                                                  \
        const int kbb = ll * (ll + 1) / 2;                                                                   \
        for (int mm = 0; mm <= ll - 2; mm++) {                                                               \
          const int kq = kbb + mm;                                                                           \
          Qt[kq] = ((double)(2 * ll - 1) * tt * Qt[kq - ll] - (double)(ll + mm - 1) * Qt[kq - 2 * ll + 1])   \
                   / (double)(ll - mm);                                                                      \
        }                                                                                                    \
        Qt[kbb + ll - 1] = (double)(2 * ll - 1) * tt * Qt[kbb + ll - 1 - ll];                                \
        Qt[kbb + ll] = (double)(2 * ll - 1) * Qt[kbb + ll - ll - 1];                                         \
      }                                                                                                      \
      wpow[0] = 0.0; wpow[1] = 0.0; wpow[2] = 1.0;  /* wpow[m + 2] = w^m */                                \
      for (int mm = 1; mm <= l_max; mm++) wpow[mm + 2] = wpow[mm + 1] * wc;                                  \
      for (int kq = 0; kq < k_max; kq++) {                                                                   \
        const int ll = lofk[kq], mm = mofk[kq];                                                              \
        const double q0 = Qt[kq], q1 = (mm + 1 <= ll) ? Qt[kq + 1] : 0.0, q2 = (mm + 2 <= ll) ? Qt[kq + 2] : 0.0; \
        Om[kq] = Ck[kq] * q0 * wpow[mm + 2];                                                                 \
        for (int aa = 0; aa < 3; aa++)                                                                       \
          dOm[kq * 3 + aa] = Ck[kq] * (q1 * tvec[aa] * wpow[mm + 2] + q0 * (double)mm * wpow[mm + 1] * wvec[aa]); \
        if (want2)                                                                                           \
          for (int bb = 0; bb < 3; bb++)                                                                     \
            for (int aa = 0; aa < 3; aa++)                                                                   \
              d2Om[(kq * 3 + bb) * 3 + aa] =                                                                 \
                  Ck[kq] * (q2 * tvec[aa] * tvec[bb] * wpow[mm + 2] + q1 * thes[bb * 3 + aa] * wpow[mm + 2]   \
                            + q1 * (double)mm * wpow[mm + 1] * (tvec[aa] * wvec[bb] + tvec[bb] * wvec[aa])  \
                            + q0 * (double)(mm * (mm - 1)) * wpow[mm] * wvec[aa] * wvec[bb]                  \
                            + q0 * (double)mm * wpow[mm + 1] * whes[bb * 3 + aa]);                           \
      }                                                                                                      \
    } while (0)

    /* the Cartesian, unnormalised derivative of the compressed p for one pair (pair_dp, :1520-1534) */
#define PAIR_DP(kk, i_, d)                                                                                   \
    do {                                                                                                     \
      hs_pair_sph(a, c, i_, kk, trad, tazi, tpol, drad, dazi, dpol, Pb, Pb + n_max * (l_max + 1),           \
                  Pb + 2 * n_max * (l_max + 1), Pb + 3 * n_max * (l_max + 1));                               \
      const double st_ = sin(a->thetas[kk]), ct_ = cos(a->thetas[kk]);                                       \
      const double sf_ = sin(a->phis[kk]), cf_ = cos(a->phis[kk]), ir_ = 1.0 / a->rjs[kk];                   \
      const double cxr = st_ * cf_, cyr = st_ * sf_, czr = ct_;                                              \
      const double pxr = -ct_ * cf_ * ir_, pyr = -ct_ * sf_ * ir_, pzr = st_ * ir_;                          \
      const double axr = -sf_ * ir_, ayr = cf_ * ir_;                                                        \
      for (int kq = 0; kq < n_soap; kq++) {                                                                  \
        (d)[kq * 3 + 0] = cxr * drad[kq] + pxr * dpol[kq] + axr * dazi[kq];                                  \
        (d)[kq * 3 + 1] = cyr * drad[kq] + pyr * dpol[kq] + ayr * dazi[kq];                                  \
        (d)[kq * 3 + 2] = czr * drad[kq] + pzr * dpol[kq];                                                   \
      }                                                                                                      \
    } while (0)

    #pragma omp for schedule(dynamic, 4)
    for (int i = 0; i < n_sites; i++) {
      const int k3 = c->k_first[i];
      const double sv = c->sqrt_dot_p[i], invs = 1.0 / sv, invs3 = invs / (sv * sv), invs5 = invs3 / (sv * sv);
      for (int q = 0; q < n_soap; q++) pvec[q] = soap[(size_t)n_soap * i + q] * sv;
      const double *ci = c->cnk + (size_t)2 * k_max * n_max * i;
      int good;
      /* ---- pass A (:1305-1334) */
      for (int t = 0; t < n_max * k_max * 3; t++) Gacc[t] = 0.0;
      for (int t = 0; t < n_soap * 3; t++) dp1[t] = 0.0;
      for (int j = 1; j < a->n_neigh[i]; j++) {
        const int k2 = k3 + j;
        PAIR_GEOMETRY(k2, good, 0);
        if (!good) continue;
        PAIR_DP(k2, i, dp2);
        for (int t = 0; t < n_soap * 3; t++) dp1[t] = dp1[t] - dp2[t];
        for (int k = 0; k < k_max; k++) {
          const int l = lofk[k];
          const double f0 = Fl[l], f1 = Fl1[l];
          for (int n = 0; n < n_max; n++) {
            const double r0 = fourpi * c->rad[(size_t)k2 * n_max + n], r1 = fourpi * c->rad_der[(size_t)k2 * n_max + n];
            const double g0 = r0 * f0, g1 = r1 * f0 + r0 * f1;
            for (int q = 0; q < 3; q++)
              Gacc[(n * k_max + k) * 3 + q] = Gacc[(n * k_max + k) * 3 + q] + g1 * nh[q] * Om[k] + g0 * dOm[k * 3 + q];
          }
        }
      }
      /* ---- the weight vectors, uncompressed, and their S matrices (:1336-1376) */
      for (int v = 0; v < nv; v++) {
        const double *vin = v < n_vec ? vecs + ((size_t)i * n_vec + v) * n_soap : pvec;
        for (int t = 0; t < n_soap_unc; t++) vunc[t] = 0.0;
        if (c->compress) {
          for (int t = 0; t < a->P_nonzero; t++)
            vunc[a->P_j[t] - 1] = vunc[a->P_j[t] - 1] + a->P_el[t] * vin[a->P_i[t] - 1];
        } else {
          for (int t = 0; t < n_soap; t++) vunc[t] = vin[t];
        }
        for (int t = 0; t < n_soap_unc; t++) if (c->skip[t]) vunc[t] = 0.0;
        for (int t = 0; t < n_max * n_max * (l_max + 1); t++) Smat[t] = 0.0;
        int counter = 0;
        for (int n = 0; n < n_max; n++)
          for (int np = n; np < n_max; np++)
            for (int l = 0; l <= l_max; l++) {
              const double vu = vunc[counter++];
              if (n == np) Smat[(l * n_max + n) * n_max + n] = 2.0 * vu;
              else {
                Smat[(l * n_max + np) * n_max + n] = sqrt2 * vu;
                Smat[(l * n_max + n) * n_max + np] = Smat[(l * n_max + np) * n_max + n];
              }
            }
        for (int k = 0; k < k_max; k++) {
          const int l = lofk[k];
          for (int n = 0; n < n_max; n++) {
            cplx zc = 0.0, b0[3] = {0.0, 0.0, 0.0};
            for (int np = 0; np < n_max; np++) {
              const double smv = Smat[(l * n_max + np) * n_max + n];
              zc = zc + smv * (ci[(size_t)2 * (k_max * np + k)] + I * ci[(size_t)2 * (k_max * np + k) + 1]);
              for (int q = 0; q < 3; q++) b0[q] = b0[q] + smv * Gacc[(np * k_max + k) * 3 + q];
            }
            Zv[(v * n_max + n) * k_max + k] = zc;
            for (int q = 0; q < 3; q++) ZGv[((v * n_max + n) * k_max + k) * 3 + q] = b0[q];
          }
        }
      }
      /* ---- pass B (:1378-1486) */
      for (int t = 0; t < 9 * n_vec; t++) hsum[t] = 0.0;
      for (int j = 1; j < a->n_neigh[i]; j++) {
        const int k2 = k3 + j;
        PAIR_GEOMETRY(k2, good, 1);
        if (!good) continue;
        PAIR_DP(k2, i, dp2);
        for (int t = 0; t < 9 * nv; t++) hv[t] = 0.0;
        for (int t = 0; t < 3 * nv; t++) u2rec[t] = 0.0;
        for (int k = 0; k < k_max; k++) {
          const int l = lofk[k];
          const double f0 = Fl[l], f1 = Fl1[l], f2 = Fl2[l], wmk = wm[k];
          for (int v = 0; v < nv; v++) {
            cplx a0 = 0.0, a1 = 0.0, a2 = 0.0, b0[3] = {0.0, 0.0, 0.0}, b1[3] = {0.0, 0.0, 0.0};
            for (int n = 0; n < n_max; n++) {
              const double r0 = c->rad[(size_t)k2 * n_max + n], r1 = c->rad_der[(size_t)k2 * n_max + n];
              const double r2 = c->rad_der2[(size_t)k2 * n_max + n];
              const cplx zc = conj(Zv[(v * n_max + n) * k_max + k]);
              a0 = a0 + r0 * zc;
              a1 = a1 + r1 * zc;
              a2 = a2 + r2 * zc;
              for (int q = 0; q < 3; q++) {
                const cplx gc = conj(ZGv[((v * n_max + n) * k_max + k) * 3 + q]);
                b0[q] = b0[q] + r0 * gc;
                b1[q] = b1[q] + r1 * gc;
              }
            }
            const cplx z0 = fourpi * f0 * a0, z1 = fourpi * (f0 * a1 + f1 * a0);
            const cplx z2 = fourpi * (f0 * a2 + 2.0 * f1 * a1 + f2 * a0);
            cplx gg0[3], gg1[3];
            for (int q = 0; q < 3; q++) {
              gg0[q] = fourpi * f0 * b0[q];
              gg1[q] = fourpi * (f0 * b1[q] + f1 * b0[q]);
            }
            for (int bb = 0; bb < 3; bb++) u2rec[v * 3 + bb] += wmk * creal(z1 * nh[bb] * Om[k] + z0 * dOm[k * 3 + bb]);
            for (int bb = 0; bb < 3; bb++)
              for (int aa = 0; aa < 3; aa++) {
                cplx tE = (z2 - z1 * invr) * nh[aa] * nh[bb] * Om[k] + z1 * (nh[aa] * dOm[k * 3 + bb] + nh[bb] * dOm[k * 3 + aa])
                          + z0 * d2Om[(k * 3 + bb) * 3 + aa];
                if (aa == bb) tE = tE + z1 * invr * Om[k];
                const cplx tD = gg1[aa] * nh[bb] * Om[k] + gg0[aa] * dOm[k * 3 + bb];
                hv[(v * 3 + bb) * 3 + aa] = hv[(v * 3 + bb) * 3 + aa] - wmk * (creal(tE) + creal(tD));
              }
          }
        }
        for (int v = 0; v < nv; v++) {
          const double *wv = v < n_vec ? vecs + ((size_t)i * n_vec + v) * n_soap : pvec;
          for (int bb = 0; bb < 3; bb++) {
            double refd = 0.0;
            for (int q = 0; q < n_soap; q++) refd += wv[q] * dp2[q * 3 + bb];
            const double e = fabs(u2rec[v * 3 + bb] - refd);
            if (e > chk_err) chk_err = e;
            if (fabs(refd) > chk_ref) chk_ref = fabs(refd);
          }
        }
        /* ---- normalisation (:1414-1484) */
        double t1[3], t2[3], c12[9];
        for (int q = 0; q < 3; q++) {
          t1[q] = 0.0; t2[q] = 0.0;
          for (int s2 = 0; s2 < n_soap; s2++) { t1[q] += pvec[s2] * dp1[s2 * 3 + q]; t2[q] += pvec[s2] * dp2[s2 * 3 + q]; }
        }
        for (int bb = 0; bb < 3; bb++)
          for (int aa = 0; aa < 3; aa++) {
            double acc = 0.0;
            for (int s2 = 0; s2 < n_soap; s2++) acc += dp1[s2 * 3 + aa] * dp2[s2 * 3 + bb];
            c12[bb * 3 + aa] = acc;
          }
        for (int v = 0; v < n_vec; v++) {
          const double *wv = vecs + ((size_t)i * n_vec + v) * n_soap;
          double wp = 0.0, u1[3] = {0, 0, 0}, u2[3] = {0, 0, 0};
          for (int s2 = 0; s2 < n_soap; s2++) {
            wp += wv[s2] * pvec[s2];
            for (int q = 0; q < 3; q++) { u1[q] += wv[s2] * dp1[s2 * 3 + q]; u2[q] += wv[s2] * dp2[s2 * 3 + q]; }
          }
          for (int bb = 0; bb < 3; bb++)
            for (int aa = 0; aa < 3; aa++) {
              const double h = hv[(v * 3 + bb) * 3 + aa] * invs - (u1[aa] * t2[bb] + u2[bb] * t1[aa]) * invs3
                               - wp * (c12[bb * 3 + aa] + hv[(n_vec * 3 + bb) * 3 + aa]) * invs3
                               + 3.0 * wp * t1[aa] * t2[bb] * invs5;
              hess[(((size_t)k2 * n_vec + v) * 3 + bb) * 3 + aa] = h;
              hsum[(v * 3 + bb) * 3 + aa] += h;
            }
        }
      }
      for (int v = 0; v < n_vec; v++)
        for (int t = 0; t < 9; t++) hess[((size_t)k3 * n_vec + v) * 9 + t] = -hsum[v * 9 + t];
    }
#undef PAIR_GEOMETRY
#undef PAIR_DP
    free(Gacc); free(Zv); free(ZGv); free(Smat); free(vunc); free(pvec); free(dp1); free(dp2);
    free(trad); free(tazi); free(tpol); free(drad); free(dazi); free(dpol); free(Pb);
    free(il); free(dilz); free(d2ilz); free(Fl); free(Fl1); free(Fl2); free(Qt);
    free(Om); free(dOm); free(d2Om); free(wpow); free(hv); free(hsum); free(u2rec);
  }
  if (selftest_err) *selftest_err = chk_err / (chk_ref > 1e-300 ? chk_ref : 1e-300);
  free(lofk); free(mofk); free(wm); free(preflm); free(Ck);
  return 0;
}

/* The radial expansion of one species at a list of distances (the columns a
 * masked, in-cutoff pair would get; src/soap_turbo_radial.f90:394-1004,
 * global_scaling not applied).  W is the species' alpha x alpha block. */
int or_radial_eval(int basis, int alpha, double rcut_soft, double rcut_hard, double sigma,
                   double sigma_scaling, double amp_scaling, double nf, const double *W,
                   int scaling_poly, int radial_enhancement, double central_weight, int is_central,
                   int legacy_seed, int n, const double *r, double *out, double *der, double *der2) {
  or_radial_setup st;
  int with_gauss = basis == 1;
  int do_central = with_gauss ? 0 : (central_weight != 0.0);
  if (basis == 2) {
    if (der2) return -1;
    for (int t = 0; t < n; t++)
      or_radial_op_pair(alpha, rcut_soft, rcut_hard, sigma, sigma_scaling, amp_scaling, scaling_poly,
                        radial_enhancement, central_weight, is_central, W, alpha, r[t], out + (size_t)t * alpha,
                        der + (size_t)t * alpha);
    return 0;
  }
  or_radial_init(&st, alpha, rcut_soft, rcut_hard, sigma, sigma_scaling, amp_scaling, nf, W, alpha,
                 scaling_poly, radial_enhancement, 1, do_central, central_weight, with_gauss, legacy_seed);
  if (der2 && or_radial_enable_der2(&st)) return -1;  /* second derivatives need the unified seed */
  for (int t = 0; t < n; t++) {
    double o[32], d[32], d2[32];
    or_radial_pair(&st, r[t], is_central, o, d, der2 ? d2 : NULL);
    for (int q = 0; q < alpha; q++) {
      out[(size_t)t * alpha + q] = o[q];
      der[(size_t)t * alpha + q] = d[q];
      if (der2) der2[(size_t)t * alpha + q] = d2[q];
    }
  }
  return 0;
}

/* Accessors for intermediate arrays (tests compare them stage by stage). */
const double *or_ctx_cnk(const or_ctx *c) { return c->cnk; }
const double *or_ctx_rad(const or_ctx *c) { return c->rad; }
const double *or_ctx_rad_der(const or_ctx *c) { return c->rad_der; }
const double *or_ctx_ang(const or_ctx *c, int which) {
  return which == 0 ? c->ang : which == 1 ? c->ang_r : which == 2 ? c->ang_a : c->ang_p;
}
const double *or_ctx_norm(const or_ctx *c) { return c->sqrt_dot_p; }
int or_ctx_n_max(const or_ctx *c) { return c->n_max; }

/* get_compress_indices, trivial branch, src/soap_turbo_compress.f90:86-119.
 * With P_i == NULL only the dimension is returned ("get_dim"). */
int or_compress_trivial(int n_species, const int *alpha_max, int l_max, int *P_i, int *P_j, double *P_el) {
  int pivot[64], n_max = 0;
  if (n_species > 64) return -1;
  pivot[0] = 1;
  for (int i = 0; i < n_species - 1; i++) pivot[i + 1] = pivot[i] + alpha_max[i];
  for (int i = 0; i < n_species; i++) n_max += alpha_max[i];
  int counter = 0, k = 1;
  for (int n = 1; n <= n_max; n++)
    for (int m = n; m <= n_max; m++)
      for (int l = 0; l <= l_max; l++) {
        int hit = 0;
        for (int s = 0; s < n_species; s++) if (n == pivot[s] || m == pivot[s]) hit = 1;
        if (hit) {
          counter++;
          if (P_i) { P_i[counter - 1] = counter; P_j[counter - 1] = k; P_el[counter - 1] = 1.0; }
        }
        k++;
      }
  return counter;
}

/* get_compress_indices, the Darby branch (compress_mode "nu_R_nu_S", nu_R, nu_S
 * in 0..2), src/soap_turbo_compress.f90:120-303, followed step by step: the
 * combined (species, radial) index ns, the limits N1, N2, S1, S2, the
 * symmetric (nu_R, nu_S both even) and the general recipe, and the
 * dense_to_sparse lookup that numbers the non-zero entries in the order they
 * are met.  Every species must have the same alpha (:134-141; returns -2).
 * With P_i == NULL only P_nonzero is returned; *dim gets the compressed size. */
int or_compress_darby(int n_species, const int *alpha_max, int l_max, int nu_R, int nu_S, int *dim,
                      int *P_i, int *P_j, double *P_el) {
  for (int i = 0; i < n_species; i++)
    if (alpha_max[i] != alpha_max[0]) return -2;
  const int A = alpha_max[0], NS = n_species * A, L1 = l_max + 1;
  int *ns_s = (int *)malloc(sizeof(int) * NS), *ns_n = (int *)malloc(sizeof(int) * NS);
  for (int i = 0, k = 0; i < n_species; i++)
    for (int n = 0; n < A; n++, k++) { ns_s[k] = i; ns_n[k] = n; }
  const int sym = (nu_R % 2 == 0) && (nu_S % 2 == 0);
  const int N1 = nu_R > 0 ? A : 1, N2 = nu_R == 2 ? A : 1;
  const int S1 = nu_S > 0 ? n_species : 1, S2 = nu_S == 2 ? n_species : 1;
  const long n_unc = (long)NS * (NS + 1) / 2 * L1;
  const long n_comp = sym ? (long)N1 * S1 * (N1 * S1 + 1) / 2 * L1 : (long)N1 * S1 * N2 * S2 * L1;
  int *d2s = (int *)calloc((size_t)n_comp * n_unc, sizeof(int)); /* dense_to_sparse(comp, ind) */
  if (!d2s) { free(ns_s); free(ns_n); return -3; }
  int counter = 0;
  long ind = 0;
#define D2S(c, u) d2s[(size_t)(c) * n_unc + (u)]
  for (int i = 0; i < NS; i++) {
    const int z1 = ns_s[i] % S1, a1 = ns_n[i] % N1;
    for (int j = 0; j < NS; j++) {
      const int z2 = ns_s[j] % S2, a2 = ns_n[j] % N2;
      if (j < i) continue; /* the original power spectrum is symmetric */
      for (int l = 0; l <= l_max; l++) {
        if (sym) {
          int ic = z1 * N1 + a1, jc = z2 * N2 + a2;
          if (jc < ic) { const int t = ic; ic = jc; jc = t; }
          const long comp = ((long)ic * (2 * N1 * S1 + 1 - ic) * L1) / 2 + (long)(jc - ic) * L1 + l;
          if (D2S(comp, ind) == 0) D2S(comp, ind) = ++counter;
          const int k = D2S(comp, ind);
          if (P_i) {
            P_el[k - 1] += (i != j && ic == jc) ? sqrt(2.0) : 1.0;
            P_i[k - 1] = (int)comp + 1;
            P_j[k - 1] = (int)ind + 1;
          }
        } else {
          const int ic = z1 * N1 + a1, jc = z2 * N2 + a2;
          /* the compressed indices of the symmetric term that is skipped */
          const int ic2 = (ns_s[j] % S1) * N1 + ns_n[j] % N1, jc2 = (ns_s[i] % S2) * N2 + ns_n[i] % N2;
          const long comp = ((long)ic * S2 * N2 + jc) * L1 + l;
          const long comp2 = ((long)ic2 * S2 * N2 + jc2) * L1 + l;
          if (D2S(comp, ind) == 0) D2S(comp, ind) = ++counter;
          const int k = D2S(comp, ind);
          if (D2S(comp2, ind) == 0 && i != j && comp != comp2) D2S(comp2, ind) = ++counter;
          const int k2 = D2S(comp2, ind);
          if (P_i) {
            if (i == j) {
              P_el[k - 1] += 1.0;
              P_i[k - 1] = (int)comp + 1;
              P_j[k - 1] = (int)ind + 1;
            } else if (comp == comp2) {
              P_el[k - 1] += sqrt(2.0);
              P_i[k - 1] = (int)comp + 1;
              P_j[k - 1] = (int)ind + 1;
            } else {
              P_el[k - 1] += 1.0 / sqrt(2.0);
              P_i[k - 1] = (int)comp + 1;
              P_j[k - 1] = (int)ind + 1;
              P_el[k2 - 1] += 1.0 / sqrt(2.0);
              P_i[k2 - 1] = (int)comp2 + 1;
              P_j[k2 - 1] = (int)ind + 1;
            }
          }
        }
        ind++;
      }
    }
  }
#undef D2S
  free(d2s); free(ns_s); free(ns_n);
  *dim = (int)n_comp;
  return counter;
}

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
