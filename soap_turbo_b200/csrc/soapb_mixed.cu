// soapb_mixed.cu -- the mixed-precision descriptor and force-VJP kernels.
//
// One CTA per central site ("environment").  A site's CSR row of neighbour
// pairs is walked in chunks of NT pairs; each chunk is turned into "entries",
// one per (pair, species) the radial expansion applies to (mask set, inside
// that species' rcut_hard, the self pair only when its central weight is
// used), sorted by species with ballot ranks so every species' entries are a
// contiguous run.
//
// descriptor (get_soap, src/soap_turbo.f90:491-909):
//   A. one thread per entry: FP64 radial expansion (R_n, alpha values), the
//      FP64 angular scalars, FP32 P_l^m; stages 4pi*R_n, e^{-i m phi} and
//      u_k = amp * preflm_k * P_k * ilexp_l in shared memory.
//   B. c_nlm: one thread per (species, k) sums its species' entries in CSR
//      order -- a fixed-order segmented reduction, no atomics.
//   C. power spectrum of the kept components, compression, norm, normalise.
// contract (soap_contract, src/soap_turbo.f90:1723-1884):
//   G -> Gp -> Gu -> H(n,k) in shared memory, then one thread per entry
//   recomputes R_n, dR_n/dr and the four angular factors in registers and
//   contracts them against H; per-pair forces are rotated to Cartesian and the
//   self pair gets minus their sum, all in fixed order.
//
// Everything is deterministic: no atomics touch results, and every reduction
// runs in an order fixed by the launch shape.
#include <cstdio>

#include "soapb_device.cuh"

namespace soapb {

constexpr double kFourPi = 12.566370614359172954;

// ------------------------------------------------------------------ prep
// Block 0 scans n_neigh into CSR offsets; the other blocks pack the mask into
// per-pair species bits and check the pair inputs.
__global__ void k_prep(DevBatch B, int n_species) {
  if (blockIdx.x == 0) {
    __shared__ int warp_tot[32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < B.n_sites; base += blockDim.x) {
      const int i = base + threadIdx.x;
      int v = (i < B.n_sites) ? B.n_neigh[i] : 0;
      if (v < 0) {
        atomicMin(B.err, (unsigned long long)(1ull << 62));
        v = 0;
      }
      int x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) warp_tot[warp] = x;
      __syncthreads();
      if (warp == 0) {
        int t = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, t, o);
          if (lane >= o) t += y;
        }
        warp_tot[lane] = t;  // inclusive over warps
      }
      __syncthreads();
      const int excl = carry + (warp > 0 ? warp_tot[warp - 1] : 0) + x - v;
      if (i < B.n_sites) B.off[i] = excl;
      __syncthreads();
      if (threadIdx.x == blockDim.x - 1) carry = excl + v;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      B.off[B.n_sites] = carry;
      if (carry != B.n_pairs) atomicMin(B.err, (unsigned long long)(1ull << 62));
    }
    return;
  }
  const int k = (blockIdx.x - 1) * blockDim.x + threadIdx.x;
  if (k >= B.n_pairs) return;
  unsigned bits = 0;
  for (int s = 0; s < n_species; ++s)
    if (B.mask[(size_t)s * B.n_pairs + k]) bits |= 1u << s;
  B.bits[k] = (uint8_t)bits;
  const double r = B.rjs[k], t = B.thetas[k], f = B.phis[k];
  if (!(r >= 0.0) || !isfinite(r) || !isfinite(t) || !isfinite(f))
    atomicMin(B.err, (unsigned long long)k);
}

// ------------------------------------------------------------- utilities
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *red) {
  // fixed-order tree: xor shuffles within warps, then warp 0 over partials
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = (lane < NT / 32) ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

struct Chunk {
  int n_ent;
};

// Builds the entry list of one chunk of NT pairs.  Returns, per thread, the
// radial-valid species bits of its own pair and (in slot[]) the entry slot of
// each of them.  Shared: ent[] = chunk-local pair | species << 24, and
// sbase/scnt per species.
template <int NT>
__device__ __forceinline__ int build_entries(const DevParams &P, const DevBatch &B, int p_begin,
                                             int chunk, int p_end, bool vjp, int *ent, int *wcnt,
                                             int *sbase, int *scnt, int *n_ent_out,
                                             int (&slot)[SOAPB_MAX_SPECIES], unsigned &my_bits) {
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = chunk + tid;
  unsigned rb = 0;
  if (k < p_end) {
    const double r = B.rjs[k];
    const unsigned bits = B.bits[k];
    const int j = k - p_begin;
#pragma unroll
    for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) {
      if (s >= P.n_species) break;
      const bool ok = ((bits >> s) & 1u) && r < P.rad[s].rcut_hard &&
                      (vjp ? (j > 0) : (j > 0 || P.rad[s].do_central));
      if (ok) rb |= 1u << s;
    }
  }
  my_bits = rb;
  const unsigned lt = (1u << lane) - 1u;
  int rank[SOAPB_MAX_SPECIES];
#pragma unroll
  for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) {
    rank[s] = 0;
    if (s >= P.n_species) break;
    const unsigned bal = __ballot_sync(0xffffffffu, (rb >> s) & 1u);
    rank[s] = __popc(bal & lt);
    if (lane == 0) wcnt[s * NW + warp] = __popc(bal);
  }
  __syncthreads();
  if (tid < P.n_species) {
    int acc = 0;
    for (int w = 0; w < NW; ++w) {
      const int t = wcnt[tid * NW + w];
      wcnt[tid * NW + w] = acc;
      acc += t;
    }
    scnt[tid] = acc;
  }
  __syncthreads();
  if (tid == 0) {
    int b = 0;
    for (int s = 0; s < P.n_species; ++s) {
      sbase[s] = b;
      b += scnt[s];
    }
    *n_ent_out = b;
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) slot[s] = -1;
#pragma unroll
  for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) {
    if (s >= P.n_species) break;
    if ((rb >> s) & 1u) {
      const int e = sbase[s] + wcnt[s * NW + warp] + rank[s];
      ent[e] = tid | (s << 24);
      slot[s] = e;
    }
  }
  __syncthreads();
  return *n_ent_out;
}

__device__ __forceinline__ int first_species(unsigned bits) { return __ffs(bits) - 1; }

// Shared-memory layout of the kernels (bytes).  Host and device agree on it.
struct Layout {
  size_t W, C, H, R, E, U, P, S, red, ent, wcnt, misc, F, total;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline Layout make_layout(const DevParams &P, int NT, int AMAX, int LC, int mode) {
  // mode 0: descriptor, 1: contract
  Layout L{};
  const size_t KS = (size_t)(P.k_max | 1);
  const size_t nsp = (size_t)P.n_species;
  size_t o = 0;
  L.W = o;   o += nsp * AMAX * AMAX * sizeof(double);
  L.red = o; o += 40 * sizeof(double);
  L.C = o;   o += 2 * (size_t)P.n_max * KS * sizeof(float);
  if (mode == 1) { L.H = o; o += 2 * (size_t)P.n_max * KS * sizeof(float); }
  if (mode == 0) {
    L.R = o; o += (size_t)NT * AMAX * sizeof(float);
    o = align_up(o, 8);
    L.E = o; o += (size_t)NT * (LC + 1) * sizeof(float2);
    L.U = o; o += (size_t)NT * KS * sizeof(float);
  }
  L.P = o;   o += (size_t)P.n_kept * sizeof(float);
  L.S = o;   o += (size_t)P.n_soap * sizeof(float);
  o = align_up(o, 16);
  L.ent = o; o += (size_t)NT * nsp * sizeof(int);
  L.wcnt = o; o += (size_t)SOAPB_MAX_SPECIES * (NT / 32) * sizeof(int);
  L.misc = o; o += 64 * sizeof(int);
  if (mode == 1) { L.F = o; o += (size_t)NT * nsp * 3 * sizeof(float); }
  L.total = align_up(o, 16);
  return L;
}

// Loads the species' W blocks (FP64) into shared memory, AMAX*AMAX apart.
template <int NT, int AMAX>
__device__ __forceinline__ void load_W(const DevParams &P, double *sW) {
  const int n = P.n_species * AMAX * AMAX;
  for (int t = threadIdx.x; t < n; t += NT) {
    const int s = t / (AMAX * AMAX), r = t % (AMAX * AMAX);
    const int a = P.rad[s].alpha;
    sW[t] = (r < a * a) ? P.Wblk[(size_t)s * P.wstride + r] : 0.0;
  }
}

// ------------------------------------------------------------ descriptor
template <int NT, int AMAX, int LC>
__global__ void __launch_bounds__(NT) k_descriptor(const DevParams P, const DevBatch B,
                                                   double *__restrict__ soap_out,
                                                   float *__restrict__ keep_c,
                                                   double *__restrict__ keep_norm, int keep) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int NPLM = (LC + 1) * (LC + 2) / 2;
  const Layout Ly = make_layout(P, NT, AMAX, LC, 0);
  double *sW = (double *)(smem + Ly.W);
  double *sRed = (double *)(smem + Ly.red);
  float *sC = (float *)(smem + Ly.C);
  float *sR = (float *)(smem + Ly.R);
  float2 *sE = (float2 *)(smem + Ly.E);
  float *sU = (float *)(smem + Ly.U);
  float *sP = (float *)(smem + Ly.P);
  float *sS = (float *)(smem + Ly.S);
  int *sEnt = (int *)(smem + Ly.ent);
  int *sW_cnt = (int *)(smem + Ly.wcnt);
  int *sMisc = (int *)(smem + Ly.misc);
  int *sBase = sMisc, *sCnt = sMisc + SOAPB_MAX_SPECIES, *sNent = sMisc + 2 * SOAPB_MAX_SPECIES;

  const int tid = threadIdx.x;
  const int site = blockIdx.x;
  const int KS = P.k_max | 1;
  const int n_max = P.n_max, k_max = P.k_max, L = P.l_max;

  load_W<NT, AMAX>(P, sW);
  for (int t = tid; t < 2 * n_max * KS; t += NT) sC[t] = 0.f;

  const int p_begin = B.off[site];
  const int p_end = min(B.off[site + 1], B.n_pairs);
  __syncthreads();

  for (int chunk = p_begin; chunk < p_end; chunk += NT) {
    int slot[SOAPB_MAX_SPECIES];
    unsigned my_bits;
    const int n_ent = build_entries<NT>(P, B, p_begin, chunk, p_end, false, sEnt, sW_cnt, sBase,
                                        sCnt, sNent, slot, my_bits);
    for (int ebase = 0; ebase < n_ent; ebase += NT) {
      // ---- A. per-entry expansions
      const int e = ebase + tid;
      if (e < n_ent) {
        const int pl = sEnt[e] & 0xffffff, s = sEnt[e] >> 24;
        const int k = chunk + pl;
        const double r = B.rjs[k];
        double val[AMAX], der[AMAX];
        radial_entry<AMAX>(P, P.rad[s], sW + s * AMAX * AMAX, r, k == p_begin, false, val, der);
        const float g4 = (float)(kFourPi * P.rad[s].gscale);
        float *Re = sR + (size_t)(e - ebase) * AMAX;
#pragma unroll
        for (int n = 0; n < AMAX; ++n) Re[n] = g4 * (float)val[n];
        AngScalars<LC> A;
        angular_scalars<LC>(P, first_species(B.bits[k]), r, B.thetas[k], B.phis[k], false, A);
        float plm[NPLM];
        plm_array<LC, float>(L, (float)A.x, (float)A.sq, plm);
        float2 *Ee = sE + (size_t)(e - ebase) * (LC + 1);
#pragma unroll
        for (int m = 0; m <= LC; ++m) Ee[m] = make_float2((float)A.er[m], (float)A.ei[m]);
        float *Ue = sU + (size_t)(e - ebase) * KS;
        const float ampf = (float)A.amp;
#pragma unroll
        for (int l = 0; l <= LC; ++l) {
          if (l > L) break;
          const float il = (float)A.il[l];
#pragma unroll
          for (int m = 0; m <= l; ++m) {
            const int kk = l * (l + 1) / 2 + m;
            Ue[kk] = ampf * P.preflm[kk] * plm[kk] * il;
          }
        }
      }
      __syncthreads();
      // ---- B. c_nlm, fixed-order sum over each species' entries
      const int e_hi = min(ebase + NT, n_ent);
      for (int it = tid; it < P.n_species * k_max; it += NT) {
        const int s = it / k_max, kk = it - s * k_max;
        int l = 0;
        while ((l + 1) * (l + 2) / 2 <= kk) ++l;
        const int m = kk - l * (l + 1) / 2;
        const int lo = max(sBase[s], ebase), hi = min(sBase[s] + sCnt[s], e_hi);
        if (lo >= hi) continue;
        float accr[AMAX], acci[AMAX];
#pragma unroll
        for (int n = 0; n < AMAX; ++n) accr[n] = acci[n] = 0.f;
        for (int e2 = lo; e2 < hi; ++e2) {
          const int el = e2 - ebase;
          const float u = sU[(size_t)el * KS + kk];
          const float2 E = sE[(size_t)el * (LC + 1) + m];
          const float ar = u * E.x, ai = u * E.y;
          const float *Re = sR + (size_t)el * AMAX;
#pragma unroll
          for (int n = 0; n < AMAX; ++n) {
            accr[n] = fmaf(Re[n], ar, accr[n]);
            acci[n] = fmaf(Re[n], ai, acci[n]);
          }
        }
        const int nb = P.rad[s].nbeg, a = P.rad[s].alpha;
#pragma unroll
        for (int n = 0; n < AMAX; ++n) {
          if (n < a) {
            sC[(size_t)(nb + n) * KS + kk] += accr[n];
            sC[(size_t)(n_max + nb + n) * KS + kk] += acci[n];
          }
        }
      }
      __syncthreads();
    }
  }

  // ---- poly3gauss central-atom term (src/soap_turbo.f90:646-662)
  if (P.basis == 1 && tid == 0) {
    const int mult = B.species_mult[site];
    for (int mm = 0; mm < mult; ++mm) {
      const int s = B.species[(size_t)site * B.max_mult + mm] - 1;
      if (s < 0 || s >= P.n_species) continue;
      const int nb = P.rad[s].nbeg, a = P.rad[s].alpha;
      for (int n = 0; n < a; ++n) sC[(size_t)(nb + n) * KS] += (float)P.central[nb + n];
    }
  }
  __syncthreads();

  // ---- C. power spectrum of the kept components (src/soap_turbo.f90:750-795)
  for (int q = tid; q < P.n_kept; q += NT) {
    const int code = P.kept_nnl[q];
    const int n = code & 0xff, np = (code >> 8) & 0xff, l = code >> 16;
    const int kb = l * (l + 1) / 2;
    const float *cn_r = sC + (size_t)n * KS + kb, *cn_i = sC + (size_t)(n_max + n) * KS + kb;
    const float *cp_r = sC + (size_t)np * KS + kb, *cp_i = sC + (size_t)(n_max + np) * KS + kb;
    float acc0 = cn_r[0] * cp_r[0] + cn_i[0] * cp_i[0];
    float acc = 0.f;
    for (int m = 1; m <= l; ++m) acc += cn_r[m] * cp_r[m] + cn_i[m] * cp_i[m];
    const float base = (n == np) ? 1.f : 1.41421356237309504880f;
    sP[q] = base * (acc0 + 2.f * acc);
  }
  __syncthreads();
  // compression and norm (:798-809)
  double nrm2 = 0.0;
  for (int o = tid; o < P.n_soap; o += NT) {
    float v = 0.f;
    for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) v += P.pi_el[t] * sP[P.pi_q[t]];
    sS[o] = v;
    nrm2 += (double)v * (double)v;
  }
  nrm2 = block_sum<NT>(nrm2, sRed);
  double norm = sqrt(nrm2);
  if (norm < 1.0e-5) norm = 1.0;
  const double inv = 1.0 / norm;
  double *out = soap_out + (size_t)site * P.n_soap;
  for (int o = tid; o < P.n_soap; o += NT) out[o] = (double)sS[o] * inv;
  if (keep) {
    float *kc = keep_c + (size_t)site * 2 * n_max * k_max;
    for (int t = tid; t < 2 * n_max * k_max; t += NT) {
      const int row = t / k_max, kk = t - row * k_max;
      kc[t] = sC[(size_t)row * KS + kk];
    }
    if (tid == 0) keep_norm[site] = norm;
  }
}

// ------------------------------------------------------------ contract
template <int NT, int AMAX, int LC>
__global__ void __launch_bounds__(NT) k_contract(const DevParams P, const DevBatch B,
                                                 const double *__restrict__ soap_in,
                                                 const double *__restrict__ G, int g_layout,
                                                 double sgn, const float *__restrict__ keep_c,
                                                 const double *__restrict__ keep_norm,
                                                 double *__restrict__ pair_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int NPLM = (LC + 2) * (LC + 3) / 2;
  const Layout Ly = make_layout(P, NT, AMAX, LC, 1);
  double *sW = (double *)(smem + Ly.W);
  double *sRed = (double *)(smem + Ly.red);
  float *sC = (float *)(smem + Ly.C);
  float *sH = (float *)(smem + Ly.H);
  float *sGu = (float *)(smem + Ly.P);
  float *sGp = (float *)(smem + Ly.S);
  int *sEnt = (int *)(smem + Ly.ent);
  int *sW_cnt = (int *)(smem + Ly.wcnt);
  int *sMisc = (int *)(smem + Ly.misc);
  float *sF = (float *)(smem + Ly.F);
  int *sBase = sMisc, *sCnt = sMisc + SOAPB_MAX_SPECIES, *sNent = sMisc + 2 * SOAPB_MAX_SPECIES;

  const int tid = threadIdx.x;
  const int site = blockIdx.x;
  const int KS = P.k_max | 1;
  const int n_max = P.n_max, k_max = P.k_max, L = P.l_max, n_soap = P.n_soap;
  const int n_sites = B.n_sites;

  load_W<NT, AMAX>(P, sW);
  {
    const float *kc = keep_c + (size_t)site * 2 * n_max * k_max;
    for (int t = tid; t < 2 * n_max * k_max; t += NT) {
      const int row = t / k_max, kk = t - row * k_max;
      sC[(size_t)row * KS + kk] = kc[t];
    }
  }
  // ---- back through the normalisation (src/soap_turbo.f90:1783-1790)
  const double *q = soap_in + (size_t)site * n_soap;
  auto g_at = [&](int o) -> double {
    return g_layout == 0 ? G[(size_t)o * n_sites + site] : G[(size_t)site * n_soap + o];
  };
  double qg = 0.0;
  for (int o = tid; o < n_soap; o += NT) qg += q[o] * g_at(o);
  qg = block_sum<NT>(qg, sRed);
  const double inv = 1.0 / keep_norm[site];
  for (int o = tid; o < n_soap; o += NT) sGp[o] = (float)((g_at(o) - q[o] * qg) * inv);
  __syncthreads();
  // ---- back through the compression (:1791-1798), on the kept components
  for (int t = tid; t < P.n_kept; t += NT) {
    float v = 0.f;
    for (int e = P.pj_off[t]; e < P.pj_off[t + 1]; ++e) v += P.pj_el[e] * sGp[P.pj_o[e]];
    sGu[t] = v;
  }
  __syncthreads();
  // ---- H(k,n) = w(m) sum_np Y(n,np,l) c(k,np) over the non-zero Y (:1800-1835)
  for (int it = tid; it < n_max * k_max; it += NT) {
    const int n = it / k_max, kk = it - n * k_max;
    int l = 0;
    while ((l + 1) * (l + 2) / 2 <= kk) ++l;
    const int m = kk - l * (l + 1) / 2;
    float hr = 0.f, hi = 0.f;
    const int li = l * n_max + n;
    for (int t = P.hl_off[li]; t < P.hl_off[li + 1]; ++t) {
      const float y = P.hl_fac[t] * sGu[P.hl_q[t]];
      const int np = P.hl_np[t];
      hr = fmaf(y, sC[(size_t)np * KS + kk], hr);
      hi = fmaf(y, sC[(size_t)(n_max + np) * KS + kk], hi);
    }
    const float w = (m == 0) ? 1.f : 2.f;
    sH[(size_t)n * KS + kk] = w * hr;
    sH[(size_t)(n_max + n) * KS + kk] = w * hi;
  }
  __syncthreads();

  const int p_begin = B.off[site];
  const int p_end = min(B.off[site + 1], B.n_pairs);
  double self_x = 0.0, self_y = 0.0, self_z = 0.0;

  for (int chunk = p_begin; chunk < p_end; chunk += NT) {
    int slot[SOAPB_MAX_SPECIES];
    unsigned my_bits;
    const int n_ent = build_entries<NT>(P, B, p_begin, chunk, p_end, true, sEnt, sW_cnt, sBase,
                                        sCnt, sNent, slot, my_bits);
    // ---- per entry: expansions and their derivatives, contracted against H
    for (int e = tid; e < n_ent; e += NT) {
      const int pl = sEnt[e] & 0xffffff, s = sEnt[e] >> 24;
      const int k = chunk + pl;
      const double r = B.rjs[k];
      double val[AMAX], der[AMAX];
      radial_entry<AMAX>(P, P.rad[s], sW + s * AMAX * AMAX, r, false, true, val, der);
      const double g4 = kFourPi * P.rad[s].gscale;
      float R[AMAX], Rd[AMAX];
#pragma unroll
      for (int n = 0; n < AMAX; ++n) {
        R[n] = (float)(g4 * val[n]);
        Rd[n] = (float)(g4 * der[n]);
      }
      AngScalars<LC> A;
      angular_scalars<LC>(P, first_species(B.bits[k]), r, B.thetas[k], B.phis[k], true, A);
      float plm[NPLM];
      plm_array<LC + 1, float>(L + 1, (float)A.x, (float)A.sq, plm);
      const float ampf = (float)A.amp, sfac = (float)A.sig_fac;
      const int nb = P.rad[s].nbeg, a = P.rad[s].alpha;
      const float *Hr = sH + (size_t)nb * KS, *Hi = sH + (size_t)(n_max + nb) * KS;
      float f_rad = 0.f, f_azi = 0.f, f_pol = 0.f;
#pragma unroll
      for (int l = 0; l <= LC; ++l) {
        if (l > L) break;
        const float il = (float)A.il[l], ild = (float)A.ild[l];
#pragma unroll
        for (int m = 0; m <= l; ++m) {
          const int kk = l * (l + 1) / 2 + m;
          const float ap = ampf * P.preflm[kk];
          // sin(t) dP/dx and -m P/sin(t), pole-safe forms (src/soap_turbo_angular.f90:194-246)
          float dms, dvs;
          if (m == 0) {
            dms = (l == 0) ? 0.f : -0.5f * plm[l * (l + 1) / 2 + 1];
            dvs = 0.f;
          } else {
            dms = 0.5f * (float)((l + m) * (l - m + 1)) * plm[kk - 1];
            dvs = 0.5f * (float)((l - m + 1) * (l - m + 2)) * plm[(l + 1) * (l + 2) / 2 + m - 1] +
                  0.5f * plm[(l + 1) * (l + 2) / 2 + m + 1];
          }
          if (m != l) dms += -0.5f * plm[kk + 1];
          const float u = ap * plm[kk] * il;
          const float ur = ap * plm[kk] * ild - sfac * u;
          const float ua = ap * dvs * il;
          const float up = ap * dms * il;
          float Ur = 0.f, Ui = 0.f, Vr = 0.f, Vi = 0.f;
#pragma unroll
          for (int n = 0; n < AMAX; ++n) {
            if (n < a) {
              const float hr = Hr[(size_t)n * KS + kk], hi = Hi[(size_t)n * KS + kk];
              Ur = fmaf(Rd[n], hr, Ur);
              Ui = fmaf(Rd[n], hi, Ui);
              Vr = fmaf(R[n], hr, Vr);
              Vi = fmaf(R[n], hi, Vi);
            }
          }
          const float er = (float)A.er[m], ei = (float)A.ei[m];
          const float reU = er * Ur + ei * Ui;
          const float reV = er * Vr + ei * Vi;
          const float imV = ei * Vr - er * Vi;
          f_rad = fmaf(u, reU, fmaf(ur, reV, f_rad));
          f_azi = fmaf(-ua, imV, f_azi);
          f_pol = fmaf(up, reV, f_pol);
        }
      }
      sF[3 * e + 0] = f_rad;
      sF[3 * e + 1] = f_azi;
      sF[3 * e + 2] = f_pol;
    }
    __syncthreads();
    // ---- per pair: sum its entries, rotate to Cartesian (:1864-1875)
    const int k = chunk + tid;
    double px = 0.0, py = 0.0, pz = 0.0;
    if (k < p_end && k > p_begin) {
      double fr = 0.0, fa = 0.0, fp = 0.0;
#pragma unroll
      for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) {
        if (s < P.n_species && slot[s] >= 0) {
          fr += sF[3 * slot[s] + 0];
          fa += sF[3 * slot[s] + 1];
          fp += sF[3 * slot[s] + 2];
        }
      }
      double st, ct, sf, cf;
      sincos(B.thetas[k], &st, &ct);
      sincos(B.phis[k], &sf, &cf);
      const double ir = 1.0 / B.rjs[k];
      px = sgn * (st * cf * fr - ct * cf * ir * fp - sf * ir * fa);
      py = sgn * (st * sf * fr - ct * sf * ir * fp + cf * ir * fa);
      pz = sgn * (ct * fr + st * ir * fp);
      double *po = pair_out + (size_t)3 * k;
      po[0] = px;
      po[1] = py;
      po[2] = pz;
    }
    self_x -= block_sum<NT>(px, sRed);
    self_y -= block_sum<NT>(py, sRed);
    self_z -= block_sum<NT>(pz, sRed);
  }
  if (tid == 0 && p_end > p_begin) {
    double *po = pair_out + (size_t)3 * p_begin;
    po[0] = self_x;
    po[1] = self_y;
    po[2] = self_z;
  }
}

// ------------------------------------------------------------ launchers
template <int NT, int AMAX, int LC>
static cudaError_t run_descriptor(const DevParams &P, const DevBatch &B, cudaStream_t s,
                                  double *soap, float *keep_c, double *keep_norm, int keep) {
  const size_t sm = make_layout(P, NT, AMAX, LC, 0).total;
  cudaError_t e = cudaFuncSetAttribute(k_descriptor<NT, AMAX, LC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  if (P.n_sites > 0)
    k_descriptor<NT, AMAX, LC><<<P.n_sites, NT, sm, s>>>(P, B, soap, keep_c, keep_norm, keep);
  return cudaGetLastError();
}

template <int NT, int AMAX, int LC>
static cudaError_t run_contract(const DevParams &P, const DevBatch &B, cudaStream_t s,
                                const double *soap, const double *G, int g_layout, double sgn,
                                const float *keep_c, const double *keep_norm, double *pair) {
  const size_t sm = make_layout(P, NT, AMAX, LC, 1).total;
  cudaError_t e = cudaFuncSetAttribute(k_contract<NT, AMAX, LC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  if (P.n_sites > 0)
    k_contract<NT, AMAX, LC><<<P.n_sites, NT, sm, s>>>(P, B, soap, G, g_layout, sgn, keep_c,
                                                       keep_norm, pair);
  return cudaGetLastError();
}

static int max_alpha(const DevParams &P) {
  int a = 0;
  for (int s = 0; s < P.n_species; ++s) a = a > P.rad[s].alpha ? a : P.rad[s].alpha;
  return a;
}

cudaError_t launch_prep(const DevParams &P, const DevBatch &B, cudaStream_t s) {
  const int blocks = 1 + (B.n_pairs + 255) / 256;
  k_prep<<<blocks, 256, 0, s>>>(B, P.n_species);
  return cudaGetLastError();
}

#define SOAPB_DISPATCH(FN, ...)                                                    \
  do {                                                                             \
    const int am = max_alpha(P);                                                   \
    const int nt = cfg.threads;                                                    \
    if (am <= 8 && P.l_max <= 8) {                                                 \
      if (nt == 64) return FN<64, 8, 8>(__VA_ARGS__);                              \
      return FN<128, 8, 8>(__VA_ARGS__);                                           \
    }                                                                              \
    return FN<128, 16, 12>(__VA_ARGS__);                                           \
  } while (0)

cudaError_t launch_descriptor(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                              double *soap, float *keep_c, double *keep_norm, int keep) {
  SOAPB_DISPATCH(run_descriptor, P, B, cfg.stream, soap, keep_c, keep_norm, keep);
}

cudaError_t launch_contract(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                            const double *soap, const double *G, int g_layout, double sgn,
                            const float *keep_c, const double *keep_norm, double *pair) {
  SOAPB_DISPATCH(run_contract, P, B, cfg.stream, soap, G, g_layout, sgn, keep_c, keep_norm, pair);
}

size_t descriptor_smem(const DevParams &P, int threads) {
  const bool small = max_alpha(P) <= 8 && P.l_max <= 8;
  return make_layout(P, small ? threads : 128, small ? 8 : 16, small ? 8 : 12, 0).total;
}
size_t contract_smem(const DevParams &P, int threads) {
  const bool small = max_alpha(P) <= 8 && P.l_max <= 8;
  return make_layout(P, small ? threads : 128, small ? 8 : 16, small ? 8 : 12, 1).total;
}

}  // namespace soapb
