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
//   C. power spectrum of the kept components (a dot product per component),
//      compression, norm, normalise.
// contract (soap_contract, src/soap_turbo.f90:1723-1884):
//   G -> Gp -> Gu -> H(n,k) in shared memory, then one thread per entry
//   recomputes R_n, dR_n/dr and the four angular factors in registers and
//   contracts them against H; per-pair forces are rotated to Cartesian and the
//   self pair gets minus their sum, all in fixed order.
//
// Everything is deterministic: no atomics touch results, and every reduction
// runs in an order fixed by the launch shape.
#include <cstdio>
#include <mutex>
#include <vector>

#include "soapb_device.cuh"
#include "soapb_scan.cuh"
#include "soapb_tc.cuh"

namespace soapb {

constexpr double kFourPi = 12.566370614359172954;



// ------------------------------------------------------------------ prep
// The species bits of pair k from the reference's mask(n_pairs, n_species),
// written to B.bits, with the pair's inputs checked.
__device__ __forceinline__ unsigned prep_pair(const DevBatch &B, int k, int n_species) {
  unsigned bits = 0;
  for (int s = 0; s < n_species; ++s)
    if (B.mask[(size_t)s * B.n_pairs + k]) bits |= 1u << s;
  B.bits[k] = (uint8_t)bits;
  const double r = B.rjs[k], t = B.thetas[k], f = B.phis[k];
  if (!(r >= 0.0) || !isfinite(r) || !isfinite(t) || !isfinite(f)) prep_error(B, (unsigned long long)k);
  return bits;
}

// The prep kernel of the plain FP64 path: scan tiles first, then one thread per pair.
constexpr int kPrepThreads = 256;
__global__ void __launch_bounds__(kPrepThreads) k_prep(DevBatch B, int n_species, int scan_tiles) {
  if ((int)blockIdx.x < scan_tiles) {
    __shared__ int sv[kScanTile];
    prep_scan_tile<kPrepThreads>(B, scan_tiles, sv);
    return;
  }
  const int k = ((int)blockIdx.x - scan_tiles) * kPrepThreads + threadIdx.x;
  if (k < B.n_pairs) prep_pair(B, k, n_species);
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

// Three sums at once, same fixed order as block_sum.
template <int NT>
__device__ __forceinline__ void block_sum3(double &a, double &b, double &c, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    red[warp] = a;
    red[8 + warp] = b;
    red[16 + warp] = c;
  }
  __syncthreads();
  if (warp == 0) {
    double x = (lane < NT / 32) ? red[lane] : 0.0;
    double y = (lane < NT / 32) ? red[8 + lane] : 0.0;
    double z = (lane < NT / 32) ? red[16 + lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
      z += __shfl_xor_sync(0xffffffffu, z, o);
    }
    if (lane == 0) {
      red[32] = x;
      red[33] = y;
      red[34] = z;
    }
  }
  __syncthreads();
  a = red[32];
  b = red[33];
  c = red[34];
}

// Builds the entry list of one chunk of NT pairs.  Returns, per thread, the
// radial-valid species bits of its own pair, its distance (my_r) and (in
// slot[]) the entry slot of each of them.  Shared: ent[] = chunk-local pair |
// species << 24, and sbase/scnt per species.
template <int NT>
__device__ __forceinline__ int build_entries(const DevParams &P, const DevBatch &B, int p_begin,
                                             int chunk, int p_end, bool vjp, int *ent, int *wcnt,
                                             int *sbase, int *scnt, int *n_ent_out,
                                             int (&slot)[SOAPB_MAX_SPECIES], unsigned &my_bits,
                                             double &my_r) {
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = chunk + tid;
  unsigned rb = 0;
  my_r = 1.0;
  if (k < p_end) {
    const double r = B.rjs[k];
    my_r = r;
    const unsigned bits = B.bits[k];
    const int j = k - p_begin;
#pragma unroll
    // a pair at or beyond rcut_max has no angular row (the reference zeroes
    // its angular coefficients, src/soap_turbo_angular.f90:549-574); it only
    // matters for poly3operator, whose radial part has no rcut_hard cut
    for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) {
      if (s >= P.n_species) break;
      const bool ok = ((bits >> s) & 1u) && r < P.rad[s].rcut_hard && r < P.rcut_max &&
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

// ------------------------------------------------------------ pair rows
// The angular row of a pair (floats), written by k_pair and read by the site
// kernels: amp i_l, amp di_l/dr, cos(m phi), -sin(m phi) for l, m <= LC, the
// amplitude amp = rcut_max^2 / sigma_t^2, 2 sigma_t_scaling / sigma_t,
// cos(theta), sqrt(1 - cos^2(theta)), then preflm_k P_l^m for l <= l_max (+1
// with derivatives), k = l(l+1)/2 + m.  So u_k = amp preflm_k P_k i_l of
// src/soap_turbo_angular.f90:590-594 is one product of two row values.
__host__ __device__ constexpr int row_il(int) { return 0; }
__host__ __device__ constexpr int row_ild(int LC) { return LC + 1; }
__host__ __device__ constexpr int row_er(int LC) { return 2 * (LC + 1); }
__host__ __device__ constexpr int row_ei(int LC) { return 3 * (LC + 1); }
__host__ __device__ constexpr int row_amp(int LC) { return 4 * (LC + 1); }
__host__ __device__ constexpr int row_sf(int LC) { return 4 * (LC + 1) + 1; }
__host__ __device__ constexpr int row_x(int LC) { return 4 * (LC + 1) + 2; }
__host__ __device__ constexpr int row_sq(int LC) { return 4 * (LC + 1) + 3; }
__host__ __device__ constexpr int row_p(int LC) { return 4 * (LC + 1) + 4; }
__host__ __device__ constexpr int row_len(int LC) { return (row_p(LC) + (LC + 2) * (LC + 3) / 2 + 3) / 4 * 4; }

int ang_row_floats(const DevParams &P) { return row_len(P.amax_t == 8 ? 8 : 12); }
// the pair kernel's staging stride in floats (odd): the whole row, or with TAB
// the larger of its two halves
__host__ __device__ constexpr int pair_stage_stride(int LC, bool TAB) {
  return TAB ? (row_p(LC) > row_len(LC) - row_p(LC) ? row_p(LC) : row_len(LC) - row_p(LC)) + 1 : row_len(LC) + 1;
}

// ------------------------------------------------------------ pair kernel
// One thread per pair, all FP64 work of the path:
//  * the radial expansion of every (pair, species) entry
//    (src/soap_turbo_radial.f90:281-1004), rounded to FP32 with 4 pi and
//    global_scaling folded in, into the radial buffer;
//  * the angular row (src/soap_turbo_angular.f90:267-463, 549-607), staged in
//    shared memory and copied out with coalesced stores.
// The site kernels only read these rows; soap_contract reads the rows of the
// descriptor call that kept its state, as the reference keeps the radial and
// angular expansions between get_soap and soap_contract.
// TAB: R_n and dR_n/dr come from the context's piecewise-polynomial tables
// (FP32 evaluation of the FP64 expansion fitted per species; see RadTab)
// instead of the FP64 expansion itself.
constexpr int kPairThreads = 128;
// CTAs of the pair kernel before its pair CTAs: the scan tiles, and one that
// orders the sites when the batch is one tile and has an order to fill
__host__ __device__ inline int pair_cta_offset(const DevBatch &B, int scan_tiles) {
  return scan_tiles + ((B.order != nullptr && scan_tiles == 1) ? 1 : 0);
}
template <int AMAX, int LC, bool OP, bool TAB>
__global__ void __launch_bounds__(kPairThreads)
    k_pair(const DevParams P, const DevBatch B, int do_der, int scan_tiles, int pair_lo, int pair_hi) {
  constexpr int NT = kPairThreads;
  extern __shared__ __align__(16) unsigned char smem[];
  // the first CTAs scan n_neigh; with a site order to build, one more orders
  // the sites (pair_cta_offset gives the host the same count)
  const int lead = pair_cta_offset(B, scan_tiles);
  if ((int)blockIdx.x < scan_tiles) {
    prep_scan_tile<NT>(B, scan_tiles, (int *)smem);
    return;
  }
  if ((int)blockIdx.x < lead) {
    order_sites<NT>(B, (int *)smem, (int *)smem + kScanTile);
    return;
  }
  constexpr int AW = row_len(LC);
  // odd stride in shared memory: each thread fills its own row, so lanes must
  // not all map to one bank.  TAB stages the row in two halves (the scalars,
  // then the P_l^m values) through half the buffer, for more CTAs per SM.
  constexpr int AWS = pair_stage_stride(LC, TAB);
  const int head = (P.off_rad + P.n_species * SOAPB_RADSP_BYTES) / 16;
  for (int t = threadIdx.x; t < head; t += NT) ((uint4 *)smem)[t] = ((const uint4 *)P.blob)[t];
  float *rows = (float *)(smem + (size_t)head * 16);
  __syncthreads();
  const int k0 = pair_lo + ((int)blockIdx.x - lead) * NT;
  const int k = k0 + threadIdx.x;
  bool active = false;
  double x = 0.0, sq = 0.0;
  unsigned tab_todo = 0u;  // TAB: the species whose tables this pair is evaluated against
  double tab_r = 0.0;
  float *row = rows + threadIdx.x * AWS;
  if (k < pair_hi) {
    const unsigned bits = prep_pair(B, k, P.n_species);
    const double r = B.rjs[k];
    if (bits != 0u && r < P.rcut_max) {
      active = true;
      const int isp = __ffs(bits) - 1;
      if (do_der)
        angular_stage<LC, true>(P, isp, r, B.thetas[k], B.phis[k], row, row_il(LC), row_ild(LC),
                                row_er(LC), row_ei(LC), row_amp(LC), row_sf(LC), x, sq);
      else
        angular_stage<LC, false>(P, isp, r, B.thetas[k], B.phis[k], row, row_il(LC), row_ild(LC),
                                 row_er(LC), row_ei(LC), row_amp(LC), row_sf(LC), x, sq);
      row[row_x(LC)] = (float)x;
      row[row_sq(LC)] = (float)sq;
      if constexpr (!TAB) {
        float *Pr = row + row_p(LC);
        const float *kpx = (const float *)(smem + P.off_kpx);
        plm_rows<LC + 1>(P.l_max + (do_der ? 1 : 0), (float)x, (float)sq,
                         [&](int kk, float v) { Pr[kk] = v * kpx[kk]; });
      }
      // the radial expansion of each species in range, as for a neighbour: the
      // central pair's expansion (:342-355) differs only by the factor
      // central_weight (:638-646), which the descriptor applies to that entry
      const double *sW = (const double *)(smem + P.off_W);
      unsigned todo = 0u;
      for (int s = 0; s < P.n_species; ++s) {
        const RadSp &RS = *(const RadSp *)(smem + P.off_rad + (size_t)s * SOAPB_RADSP_BYTES);
        if (((bits >> s) & 1u) && r < RS.rcut_hard) todo |= 1u << s;
      }
      if constexpr (TAB) {
        tab_todo = todo;
        tab_r = r;
        todo = 0u;
      }
      // species are data, not control flow: lanes of different species share
      // one expansion call
      while (todo) {
        const int s = __ffs(todo) - 1;
        todo &= todo - 1u;
        const RadSp &RS = *(const RadSp *)(smem + P.off_rad + (size_t)s * SOAPB_RADSP_BYTES);
        float4 *o = (float4 *)(B.rad + ((size_t)k * P.n_species + s) * 2 * AMAX);
        double val[AMAX], der[AMAX];
        radial_entry<AMAX, OP>(P, RS, sW + s * AMAX * AMAX, r, false, do_der != 0, val, der);
        const double g4 = kFourPi * RS.gscale;
#pragma unroll
        for (int n4 = 0; n4 < AMAX / 4; ++n4)
          o[n4] = make_float4((float)(g4 * val[4 * n4]), (float)(g4 * val[4 * n4 + 1]),
                              (float)(g4 * val[4 * n4 + 2]), (float)(g4 * val[4 * n4 + 3]));
        if (do_der)
#pragma unroll
          for (int n4 = 0; n4 < AMAX / 4; ++n4)
            o[AMAX / 4 + n4] = make_float4((float)(g4 * der[4 * n4]), (float)(g4 * der[4 * n4 + 1]),
                                           (float)(g4 * der[4 * n4 + 2]), (float)(g4 * der[4 * n4 + 3]));
      }
    }
  }
  if constexpr (TAB) {
    // R_n and dR_n/dr from the tables, a warp's entries of one species at a
    // time: 2 AMAX lanes per entry, lane f evaluating function f, so that the
    // segment's coefficients (stored [degree][function]) are read and the
    // entry's radial row is written as contiguous 64-byte runs
    constexpr int G = 2 * AMAX, EPW = 32 / G;
    static_assert(32 % G == 0, "lanes per entry");
    const int lane = threadIdx.x & 31, f = lane % G, sub = lane / G;
    const int nf = do_der ? G : AMAX;
    for (int s = 0; s < P.n_species; ++s) {
      const bool mine = (tab_todo >> s) & 1u;
      unsigned m = __ballot_sync(0xffffffffu, mine);
      if (!m) continue;
      float t = 0.f;
      int cb = -1;
      if (mine) {
        const RadSp &RS = *(const RadSp *)(smem + P.off_rad + (size_t)s * SOAPB_RADSP_BYTES);
        cb = radial_table_locate<AMAX>(P, RS, P.rtab_sp[s], tab_r, t);
      }
      while (m) {
        unsigned mm = m;
#pragma unroll
        for (int i = 0; i < EPW - 1; ++i)
          if (i < sub) mm &= mm - 1u;
#pragma unroll
        for (int i = 0; i < EPW; ++i) m &= m - 1u;
        const int src = mm ? __ffs(mm) - 1 : 0;
        const int cbe = __shfl_sync(0xffffffffu, cb, src);
        const float te = __shfl_sync(0xffffffffu, t, src);
        if (mm && f < nf) {
          float a = 0.f;
          if (cbe >= 0) {
            const float *c = P.rtab_coef + cbe + f;
            a = c[kRadTabDeg * G];
#pragma unroll
            for (int d = kRadTabDeg - 1; d >= 0; --d) a = fmaf(a, te, c[d * G]);
          }
          const int ke = k0 + (threadIdx.x & ~31) + src;
          B.rad[((size_t)ke * P.n_species + s) * G + f] = a;
        }
      }
    }
  }
  __syncthreads();
  const int nrow = min(NT, pair_hi - k0);
  if constexpr (TAB) {
    // coalesced 16-byte stores of the rows' first parts, then the P_l^m values
    // through the same buffer
    constexpr int P1 = row_p(LC) / 4, P2 = (AW - row_p(LC)) / 4;
    for (int t = threadIdx.x; t < nrow * P1; t += NT) {
      const int i = t / P1, j = t - i * P1;
      const float *src = rows + i * AWS + 4 * j;
      *(float4 *)(B.ang + (size_t)(k0 + i) * AW + 4 * j) = make_float4(src[0], src[1], src[2], src[3]);
    }
    __syncthreads();
    if (active) {
      const float *kpx = (const float *)(smem + P.off_kpx);
      plm_rows<LC + 1>(P.l_max + (do_der ? 1 : 0), (float)x, (float)sq,
                       [&](int kk, float v) { row[kk] = v * kpx[kk]; });
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nrow * P2; t += NT) {
      const int i = t / P2, j = t - i * P2;
      const float *src = rows + i * AWS + 4 * j;
      *(float4 *)(B.ang + (size_t)(k0 + i) * AW + row_p(LC) + 4 * j) =
          make_float4(src[0], src[1], src[2], src[3]);
    }
    return;
  }
  // coalesced 16-byte stores of the CTA's rows (AW is a multiple of 4 floats)
  constexpr int AW4 = AW / 4;
  const int n4 = nrow * AW4;
  float4 *dst = (float4 *)(B.ang + (size_t)k0 * AW);
  for (int t = threadIdx.x; t < n4; t += NT) {
    const int i = t / AW4;
    const float *src = rows + i * AWS + 4 * (t - i * AW4);
    dst[t] = make_float4(src[0], src[1], src[2], src[3]);
  }
}

// ------------------------------------------------------------ layouts
// Shared memory of the site kernels (bytes); host and device agree on it.
// The site part of the constants blob (species constants, per-k tables, item
// maps, kept components, Y lists) comes first.  Region X holds the per-round
// entry staging; outside the chunk loop the same bytes hold per-site arrays.
struct Layout {
  size_t red, ent, wcnt, misc;
  size_t C64, H, Rot, F;
  size_t X;
  size_t R, Rd, A;       // staging inside X
  size_t C, P, S;        // per-site arrays inside X
  size_t total;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
// entries whose rows are staged in shared memory at a time: half the CTA, at
// most 64 for the descriptor (mode 0) and 32 for the contract (mode 1), whose
// longer staged rows would otherwise cost it a CTA per SM
__host__ __device__ constexpr int stage_entries_per_round(int NT, int mode) {
  return NT / 2 < (mode ? 32 : 64) ? NT / 2 : (mode ? 32 : 64);
}
// Staged rows are longer than the global ones and stay 16-byte aligned for the
// asynchronous copies.  The contract (mode 1) pads by 16 floats so that its two
// half-warps, which read neighbouring rows at the same offsets, use disjoint
// bank halves; the descriptor reads one row per thread group and pads by 4.
__host__ __device__ inline int stage_stride(int LC, int mode) { return row_len(LC) + (mode ? 16 : 4); }
// row stride of H: the species blocks padded to AMAX, plus 4 so that 128-bit
// loads of consecutive k rows fall in distinct banks
__host__ __device__ inline int h_stride(int n_species, int AMAX) { return n_species * AMAX + 4; }
// floats per site of the kept c_nlm, padded to a multiple of 4 so that every
// site's block starts 16-byte aligned
__host__ __device__ inline size_t keep_stride(const DevParams &P) {
  return ((size_t)2 * P.n_max * (size_t)(P.k_max | 1) + 3) / 4 * 4;
}
// bytes of constants a site kernel keeps in shared memory (mode 0 descriptor, 1 contract)
__host__ __device__ inline size_t site_blob_bytes(const DevParams &P, int mode) {
  return mode ? (size_t)P.blob_c_bytes : (size_t)(P.blob_bytes - P.off_rad);
}

__host__ __device__ inline Layout make_layout(const DevParams &P, int NT, int AMAX, int LC, int mode) {
  Layout L{};
  const size_t KS = (size_t)(P.k_max | 1);
  const size_t nsp = (size_t)P.n_species, CH = (size_t)stage_entries_per_round(NT, mode);
  const size_t nC = 2 * (size_t)P.n_max * KS;
  size_t o = site_blob_bytes(P, mode);
  L.red = o;  o += 40 * sizeof(double);
  L.ent = o;  o += (size_t)NT * nsp * sizeof(int);
  L.wcnt = o; o += (size_t)SOAPB_MAX_SPECIES * (NT / 32) * sizeof(int);
  L.misc = o; o += 64 * sizeof(int);
  o = align_up(o, 16);
  if (mode == 0) {
    L.C64 = o; o += nC * sizeof(double);
  } else {
    L.H = o;   o += 2 * KS * (size_t)h_stride(P.n_species, AMAX) * sizeof(float);
    L.Rot = o; o += (size_t)NT * 4 * sizeof(float);
    L.F = o;   o += (size_t)NT * nsp * 3 * sizeof(float);
  }
  o = align_up(o, 16);
  L.X = o;
  size_t x = o;
  L.R = x; x += CH * AMAX * sizeof(float);
  if (mode == 1) { L.Rd = x; x += CH * AMAX * sizeof(float); }
  L.A = x; x += CH * (size_t)stage_stride(LC, mode) * sizeof(float);
  const size_t end_stage = x;
  x = o;
  L.C = x; x += nC * sizeof(float);
  L.P = x; x += (size_t)P.n_kept * sizeof(float);
  L.S = x; x += (size_t)P.n_soap * sizeof(float);
  const size_t end_site = x;
  o = end_stage > end_site ? end_stage : end_site;
  L.total = align_up(o, 16);
  return L;
}

template <int NT>
__device__ __forceinline__ void copy_site_blob(const DevParams &P, unsigned char *smem, int mode) {
  const uint4 *src = (const uint4 *)(mode ? P.blob_c : P.blob + P.off_rad);
  uint4 *dst = (uint4 *)smem;
  for (int t = threadIdx.x; t < (int)(site_blob_bytes(P, mode) / 16); t += NT) dst[t] = src[t];
}

// Offset of a blob section inside the site kernels' shared copy.
#define SBLOB(off) (smem + (P.off) - P.off_rad)
#define SBLOBC(off) (smem + (P.off))

__device__ __forceinline__ const RadSp &rad_of(const unsigned char *smem, const DevParams &P, int s) {
  return *(const RadSp *)(smem + (size_t)s * SOAPB_RADSP_BYTES);
}

// Persistent scheduling: every CTA takes sites from a counter until none are
// left; which CTA computes a site does not change its result.  The next site
// is fetched ahead, so that neither the ticket nor the CSR bounds are a round
// trip between two sites: thread 0 takes the next ticket when a site starts,
// loads that site's bounds part-way through (ahead_bounds) and hands the three
// values to the CTA in cur[] when the site ends (ahead_publish, which also
// synchronises).  The first site is fetched by first_site.
// A launch processes the sites [site_lo, site_hi) of the batch.  Each CTA takes
// tickets until one is past the last site, so a launch hands out exactly
// (site_hi - site_lo) + gridDim.x of them; the CTA holding the last one puts
// the counter back to 0 for the next launch.  Returns the site (>= site_hi: none left).
__device__ __forceinline__ int take_ticket(const DevBatch &B, int *ticket) {
  const int n = B.site_hi - B.site_lo;
  const int t = atomicAdd(ticket, 1);
  if (t == n + (int)gridDim.x - 1) atomicExch(ticket, 0);
  return (B.order != nullptr && t < n) ? B.order[t] : B.site_lo + min(t, n);
}
__device__ __forceinline__ void first_site(const DevBatch &B, int *ticket, int *cur) {
  if (threadIdx.x == 0) {
    const int s0 = take_ticket(B, ticket);
    cur[0] = s0;
    cur[1] = s0 < B.site_hi ? B.off[s0] : 0;
    cur[2] = s0 < B.site_hi ? B.off[s0 + 1] : 0;
  }
  __syncthreads();
}
__device__ __forceinline__ void ahead_bounds(const DevBatch &B, int nx, int &nx0, int &nx1) {
  if (threadIdx.x == 0 && nx < B.site_hi) {
    nx0 = B.off[nx];
    nx1 = B.off[nx + 1];
  }
}
// Callers guarantee a __syncthreads between their reads of cur[] at the top of
// the site and this call.
__device__ __forceinline__ void ahead_publish(int *cur, int nx, int nx0, int nx1) {
  if (threadIdx.x == 0) {
    cur[0] = nx;
    cur[1] = nx0;
    cur[2] = nx1;
  }
  __syncthreads();
}

// 16-byte asynchronous global -> shared copy (no register staging).
__device__ __forceinline__ void cp_async16(void *dst_smem, const void *src_gmem) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src_gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Copies the rows of entries [ebase, ebase + n_round) of a chunk into the
// staging area (the angular rows and the radial rows), every 16-byte piece an
// independent asynchronous copy.  The caller synchronises afterwards.
template <int NT, int AMAX, int LC, bool DER>
__device__ __forceinline__ void stage_entries(const DevParams &P, const DevBatch &B, const int *sEnt,
                                              int chunk, int ebase, int n_round, float *sA,
                                              float *sR, float *sRd) {
  constexpr int AW4 = row_len(LC) / 4;
  const int AS = stage_stride(LC, DER ? 1 : 0);
  for (int t = threadIdx.x; t < n_round * AW4; t += NT) {
    const int el = t / AW4, j4 = t - el * AW4;
    const int k = chunk + (sEnt[ebase + el] & 0xffffff);
    cp_async16(sA + (size_t)el * AS + 4 * j4, B.ang + (size_t)k * (4 * AW4) + 4 * j4);
  }
  constexpr int R4 = AMAX / 4, RW4 = DER ? 2 * R4 : R4;
  for (int t = threadIdx.x; t < n_round * RW4; t += NT) {
    const int el = t / RW4, j4 = t - el * RW4;
    const int code = sEnt[ebase + el];
    const int k = chunk + (code & 0xffffff), s = code >> 24;
    const float *src = B.rad + ((size_t)k * P.n_species + s) * 2 * AMAX + 4 * j4;
    float *dst = (j4 < R4) ? sR + (size_t)el * AMAX + 4 * j4 : sRd + (size_t)el * AMAX + 4 * (j4 - R4);
    cp_async16(dst, src);
  }
  cp_async_wait_all();
}

// ------------------------------------------------------------ tensor cores
// 3xTF32 on mma.sync m16n8k8: each FP32 operand is split into a TF32 head and
// a TF32 tail, x = hi + lo to ~22 bits, and a*b is taken as
// lo_a*hi_b + hi_a*lo_b + hi_a*hi_b (small terms first) with FP32 accumulation.
__device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void split_tf32(float x, unsigned &hi, unsigned &lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void mma_3xtf32(float (&d)[4], const float (&a)[4], const float (&b)[2]) {
  unsigned ah[4], al[4], bh[2], bl[2];
#pragma unroll
  for (int i = 0; i < 4; ++i) split_tf32(a[i], ah[i], al[i]);
#pragma unroll
  for (int i = 0; i < 2; ++i) split_tf32(b[i], bh[i], bl[i]);
  mma_tf32(d, al, bh);
  mma_tf32(d, ah, bl);
  mma_tf32(d, ah, bh);
}

// Power spectrum tiles P_l[n][j] = sum_c X_l[n][c] X_l[J_j][c] with
// X_l[n] = (Re c_nl0, r2 Re c_nl1 .. r2 Re c_nll, Im c_nl0, r2 Im c_nl1 ..), r2 = sqrt 2,
// i.e. P_l[n][j] = sum_m w_m Re(c_nlm conj c_{J_j}lm), w_0 = 1, w_m = 2
// (src/soap_turbo.f90:750-795).  A warp per (l, 16-row tile, 8-column tile);
// fragment layouts of m16n8k8: lane = 4 g + t, A rows g / g+8 and columns
// t / t+4, B row t / t+4 and column g, D rows g / g+8 and columns 2t, 2t+1.
template <int NT>
__device__ __forceinline__ void ps_tensor(const DevParams &P, const float *sC, float *sPl, const int *J) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int MT = P.ps_mt, NTJ = P.ps_nt, MR = 16 * MT, JP = 8 * NTJ;
  const int n_max = P.n_max, KS = P.k_max | 1;
  const int per_l = MT * NTJ, n_units = (P.l_max + 1) * per_l;
  for (int u = warp; u < n_units; u += NT / 32) {
    const int l = u / per_l, r = u - l * per_l, mt = r / NTJ, nt = r - mt * NTJ;
    const int kb = l * (l + 1) / 2, KL = 2 * (l + 1);
    const int n0 = 16 * mt + g, n1 = n0 + 8, jn = J[8 * nt + g];
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c0 = 0; c0 < KL; c0 += 8) {
      float a[4], b[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = c0 + t + 4 * h;
        float x0 = 0.f, x1 = 0.f, xj = 0.f;
        if (col < KL) {
          const int im = col > l, m = im ? col - l - 1 : col;
          const float w = m ? 1.41421356237309504880f : 1.f;
          const int off = (im ? n_max * KS : 0) + kb + m;
          if (n0 < n_max) x0 = w * sC[n0 * KS + off];
          if (n1 < n_max) x1 = w * sC[n1 * KS + off];
          if (jn >= 0) xj = w * sC[jn * KS + off];
        }
        a[2 * h] = x0;
        a[2 * h + 1] = x1;
        b[h] = xj;
      }
      mma_3xtf32(d, a, b);
    }
    float *o = sPl + (size_t)(l * MR + n0) * JP + 8 * nt + 2 * t;
    o[0] = d[0];
    o[1] = d[1];
    o[8 * JP] = d[2];
    o[8 * JP + 1] = d[3];
  }
}

// ---- C. of a site, from its c_nlm in sC (FP32, (re/im, n, KS)): the power
// spectrum of the kept components (src/soap_turbo.f90:750-795), the
// compression, the norm and the normalised FP64 output (:798-809, 904-909),
// and with keep the c_nlm and norm the contract reads.  keep: bit 0 keeps, bit
// 1 accumulates into soap_out.  tiles: the power spectrum from tensor-core
// tiles in sPl (the tcgen05 kernel: formed there when ps_ready, else here with
// mma.sync 3xTF32 tiles); else one dot product per kept component on the CUDA
// cores (k_descriptor: measured faster than the mma.sync tiles).
template <int NT>
__device__ __forceinline__ void site_output(const DevParams &P, unsigned char *smem, const float *sC, float *sP,
                                            float *sS, float *sPl, const int *kept, double *sRed, int site,
                                            double *__restrict__ soap_out, float *__restrict__ keep_c,
                                            double *__restrict__ keep_norm, int keep, bool tiles,
                                            bool ps_ready = false) {
  const int tid = threadIdx.x;
  const int KS = P.k_max | 1;
  const int n_max = P.n_max;
    // ---- C. power spectrum of the kept components (src/soap_turbo.f90:750-795)
    float *pout = P.cmap_identity ? sS : sP;
    double nrm2 = 0.0;
    if (tiles) {
      // on the tensor cores, then gathered into the kept components with the
      // sqrt 2 of n != n'
      if (!ps_ready) {
        ps_tensor<NT>(P, sC, sPl, (const int *)SBLOB(off_psj));
        __syncthreads();
      }
      const int *kpos = (const int *)SBLOB(off_kpos);
      for (int q = tid; q < P.n_kept; q += NT) {
        const int code = kpos[q];
        const float v = (code < 0 ? 1.41421356237309504880f : 1.f) * sPl[code & 0x7fffffff];
        pout[q] = v;
        nrm2 += (double)v * (double)v;
      }
    } else
    for (int q = tid; q < P.n_kept; q += NT) {
      const int code = kept[q];
      const int n = code & 0xff, np = (code >> 8) & 0xff, l = code >> 16;
      const int kb = l * (l + 1) / 2;
      const float *cn_r = sC + (size_t)n * KS + kb, *cn_i = sC + (size_t)(n_max + n) * KS + kb;
      const float *cp_r = sC + (size_t)np * KS + kb, *cp_i = sC + (size_t)(n_max + np) * KS + kb;
      const float acc0 = cn_r[0] * cp_r[0] + cn_i[0] * cp_i[0];
      float acc = 0.f;
      for (int m = 1; m <= l; ++m) acc += cn_r[m] * cp_r[m] + cn_i[m] * cp_i[m];
      const float base = (n == np) ? 1.f : 1.41421356237309504880f;
      const float v = base * (acc0 + 2.f * acc);
      pout[q] = v;
      nrm2 += (double)v * (double)v;
    }
    if (!P.cmap_identity) {
      // compression through the map (:798-802)
      __syncthreads();
      nrm2 = 0.0;
      for (int o = tid; o < P.n_soap; o += NT) {
        float v = 0.f;
        for (int t = P.pi_off[o]; t < P.pi_off[o + 1]; ++t) v += P.pi_el[t] * sP[P.pi_q[t]];
        sS[o] = v;
        nrm2 += (double)v * (double)v;
      }
    }
    double *out = soap_out + (size_t)site * P.n_soap;
    // accumulate: the caller's soap row is added before the norm is taken, as
    // the reference adds the compressed descriptor into soap (:798-802).  Each
    // thread reads and writes the same components of the row.
    const bool acc = (keep & 2) != 0;
    if (acc) {
      nrm2 = 0.0;
      for (int o = tid; o < P.n_soap; o += NT) {
        const double v = (double)sS[o] + out[o];
        nrm2 += v * v;
      }
    }
    nrm2 = block_sum<NT>(nrm2, sRed);  // (:805-809)
    double norm = sqrt(nrm2);
    if (norm < 1.0e-5) norm = 1.0;
    const double inv = 1.0 / norm;
    if (acc)
      for (int o = tid; o < P.n_soap; o += NT) out[o] = ((double)sS[o] + out[o]) * inv;
    else
      for (int o = tid; o < P.n_soap; o += NT) out[o] = (double)sS[o] * inv;
    if (keep & 1) {
      float *kc = keep_c + (size_t)site * keep_stride(P);
      const int n4 = (2 * n_max * KS) / 4;
      for (int t = tid; t < n4; t += NT) ((float4 *)kc)[t] = ((const float4 *)sC)[t];
      for (int t = 4 * n4 + tid; t < 2 * n_max * KS; t += NT) kc[t] = sC[t];
      if (tid == 0) keep_norm[site] = norm;
    }
}

// ------------------------------------------------------------ descriptor
template <int NT, int AMAX, int LC>
__global__ void __launch_bounds__(NT, 640 / NT) k_descriptor(const DevParams P, const DevBatch B,
                                                      double *__restrict__ soap_out,
                                                      float *__restrict__ keep_c,
                                                      double *__restrict__ keep_norm, int keep) {
  // keep: bit 0 keeps c_nlm and the norm for the contract, bit 1 accumulates
  // into soap_out
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int CH = stage_entries_per_round(NT, 0);
  constexpr int NH = AMAX / 2;  // radial indices per c_nlm item
  const int AS = stage_stride(LC, 0);
  const Layout Ly = make_layout(P, NT, AMAX, LC, 0);
  const int *klm = (const int *)SBLOB(off_klm);
  const int *citem = (const int *)SBLOB(off_citem);
  const int *kept = (const int *)SBLOB(off_kept);
  const double *central = (const double *)SBLOB(off_central);
  double *sRed = (double *)(smem + Ly.red);
  double *sC64 = (double *)(smem + Ly.C64);
  float *sR = (float *)(smem + Ly.R);
  float *sA = (float *)(smem + Ly.A);
  float *sC = (float *)(smem + Ly.C);
  float *sP = (float *)(smem + Ly.P);
  float *sS = (float *)(smem + Ly.S);
  int *sEnt = (int *)(smem + Ly.ent);
  int *sW_cnt = (int *)(smem + Ly.wcnt);
  int *sMisc = (int *)(smem + Ly.misc);
  int *sBase = sMisc, *sCnt = sMisc + SOAPB_MAX_SPECIES, *sNent = sMisc + 2 * SOAPB_MAX_SPECIES;
  int *sSite = sMisc + 3 * SOAPB_MAX_SPECIES;

  const int tid = threadIdx.x;
  const int KS = P.k_max | 1;
  const int n_max = P.n_max, nsp = P.n_species;

  copy_site_blob<NT>(P, smem, 0);
  first_site(B, B.ticket, sSite);
  for (;;) {
    const int site = sSite[0];
    if (site >= B.site_hi) break;
    const int p_begin = sSite[1];
    const int p_end = min(sSite[2], B.n_pairs);
    int nx = 0, nx0 = 0, nx1 = 0;
    if (tid == 0) nx = take_ticket(B, B.ticket);  // the next site, fetched ahead
    for (int t = tid; t < 2 * n_max * KS; t += NT) sC64[t] = 0.0;
    __syncthreads();

    for (int chunk = p_begin; chunk < p_end; chunk += NT) {
      int slot[SOAPB_MAX_SPECIES];
      unsigned my_bits;
      double my_r;
      const int n_ent = build_entries<NT>(P, B, p_begin, chunk, p_end, false, sEnt, sW_cnt, sBase,
                                          sCnt, sNent, slot, my_bits, my_r);
      for (int ebase = 0; ebase < n_ent; ebase += CH) {
        const int n_round = min(CH, n_ent - ebase);
        // ---- A. the entries' rows
        stage_entries<NT, AMAX, LC, false>(P, B, sEnt, chunk, ebase, n_round, sA, sR, nullptr);
        __syncthreads();
        // the central pair's entries carry central_weight (:638-646); the pair
        // kernel expanded every pair as a neighbour
        if (chunk == p_begin) {
          for (int el = tid; el < n_round; el += NT) {
            const int code = sEnt[ebase + el];
            const double cw = rad_of(smem, P, code >> 24).cw;
            if ((code & 0xffffff) == 0 && cw != 1.0)
#pragma unroll
              for (int n = 0; n < AMAX; ++n) sR[(size_t)el * AMAX + n] *= (float)cw;
          }
          __syncthreads();
        }
        // ---- B. c_nlm: item = (species, k, half of the species' radial block);
        // FP32 partial sums over groups of 4 entries, flushed into FP64
        const int e_hi = ebase + n_round;
        for (int it = tid; it < P.n_citem; it += NT) {
          const int code = citem[it];
          const int s = code & 15, kk = (code >> 4) & 0xff, half = code >> 12;
          const int lo = max(sBase[s], ebase), hi = min(sBase[s] + sCnt[s], e_hi);
          if (lo >= hi) continue;
          const RadSp &RS = rad_of(smem, P, s);
          const int nb = RS.nbeg, a = RS.alpha, n0 = half * NH;
          const int l = klm[kk] & 0xff, m = klm[kk] >> 8;
          double dr[NH], di[NH];
          float pr[NH], pi[NH];
#pragma unroll
          for (int n = 0; n < NH; ++n) {
            dr[n] = di[n] = 0.0;
            pr[n] = pi[n] = 0.f;
          }
          int cnt = 0;
          for (int e2 = lo; e2 < hi; ++e2) {
            const int el = e2 - ebase;
            const float *Ae = sA + (size_t)el * AS;
            // u_k = (preflm_k P_k) (amp i_l) (src/soap_turbo_angular.f90:590-594)
            const float u = Ae[row_p(LC) + kk] * Ae[row_il(LC) + l];
            const float ar = u * Ae[row_er(LC) + m], ai = u * Ae[row_ei(LC) + m];
            const float *Re = sR + (size_t)el * AMAX + n0;
#pragma unroll
            for (int n = 0; n < NH; ++n) {
              pr[n] = fmaf(Re[n], ar, pr[n]);
              pi[n] = fmaf(Re[n], ai, pi[n]);
            }
            if (++cnt == 4) {
              cnt = 0;
#pragma unroll
              for (int n = 0; n < NH; ++n) {
                dr[n] += (double)pr[n];
                di[n] += (double)pi[n];
                pr[n] = pi[n] = 0.f;
              }
            }
          }
#pragma unroll
          for (int n = 0; n < NH; ++n) {
            if (n0 + n < a) {
              sC64[(size_t)(nb + n0 + n) * KS + kk] += dr[n] + (double)pr[n];
              sC64[(size_t)(n_max + nb + n0 + n) * KS + kk] += di[n] + (double)pi[n];
            }
          }
        }
        __syncthreads();
      }
    }

    ahead_bounds(B, nx, nx0, nx1);
    // ---- poly3gauss central-atom term (src/soap_turbo.f90:646-662)
    if (P.basis == 1) {
      const int mult = B.species_mult[site];
      for (int mm = 0; mm < mult; ++mm) {
        const int s = B.species[(size_t)site * B.max_mult + mm] - 1;
        if (s < 0 || s >= nsp) continue;
        const RadSp &RS = rad_of(smem, P, s);
        for (int n = tid; n < RS.alpha; n += NT) sC64[(size_t)(RS.nbeg + n) * KS] += central[RS.nbeg + n];
        __syncthreads();
      }
    }
    __syncthreads();
    for (int t = tid; t < 2 * n_max * KS; t += NT) sC[t] = (float)sC64[t];
    __syncthreads();

    site_output<NT>(P, smem, sC, sP, sS, nullptr, kept, sRed, site, soap_out, keep_c, keep_norm, keep, false);
    ahead_publish(sSite, nx, nx0, nx1);
  }
}

// ------------------------------------------------------------ descriptor on tensor cores
// get_soap's c_nlm (src/soap_turbo.f90:619-664) as a tcgen05 product per site:
// D[2 k + re/im][n] = sum_e A_e(k, re/im) R_e(n), with A_e(k) = u_k e^{-i m phi}
// of entry e (u_k = (preflm_k P_k)(amp i_l), the same FP32 products as the
// CUDA-core kernel) and R_e its species' 4 pi R_n (zero in the other species'
// columns).  M = 128 rows (2 k_max <= 128), N = 32 columns (n_max <= 32), K =
// the entries, 16 at a time (two K-steps of 3xTF32 MMAs); each group's FP32
// partial sums are read from TMEM by the thread that owns the row and added to
// its FP64 accumulators (fixed order, no atomics) -- the accuracy of the
// CUDA-core kernel's FP32 groups flushed into FP64.  Then the poly3gauss
// central term, and k_descriptor's power spectrum, norm and output.
constexpr int kTdGroup = 16;   // entries per group (two K-steps)
constexpr int kTdCols = 32;    // D columns (n)
constexpr int kTdTmemCols = 128;  // c_nlm's 32 columns, then the power spectrum's up to 128

struct TdLayout {
  size_t red, ent, wcnt, misc, mbar, tmem, Ahi, Alo, Bhi, Blo, Phi, Plo, X, R, A, C, P, S, Pl, total;
};
constexpr int kPsTcK = 32;  // K columns of a power-spectrum tile (the host's groups agree)
__host__ __device__ inline TdLayout make_td_layout(const DevParams &P, int NT, int AMAX, int LC) {
  TdLayout L{};
  const size_t KS = (size_t)(P.k_max | 1), nsp = (size_t)P.n_species;
  size_t o = site_blob_bytes(P, 0);
  L.red = o;  o += 40 * sizeof(double);
  L.ent = o;  o += (size_t)NT * nsp * sizeof(int);
  L.wcnt = o; o += (size_t)SOAPB_MAX_SPECIES * (NT / 32) * sizeof(int);
  L.misc = o; o += 64 * sizeof(int);
  L.mbar = align_up(o, 8); o = L.mbar + 8;
  L.tmem = o; o += 8;
  o = align_up(o, 1024);
  // the c_nlm tiles, and afterwards the power-spectrum tiles, in one region
  const size_t tcb = o;
  L.Ahi = o; o += 128 * kTdGroup * 4;
  L.Alo = o; o += 128 * kTdGroup * 4;
  L.Bhi = o; o += kTdCols * kTdGroup * 4;
  L.Blo = o; o += kTdCols * kTdGroup * 4;
  if (P.ps_ng > 0) {
    L.Phi = tcb;
    L.Plo = tcb + 128 * kPsTcK * 4;
    const size_t pe = tcb + 2 * 128 * kPsTcK * 4;
    o = o > pe ? o : pe;
  }
  o = align_up(o, 16);
  L.X = o;
  size_t x = o;
  L.R = x; x += kTdGroup * AMAX * sizeof(float);
  L.A = x; x += kTdGroup * (size_t)stage_stride(LC, 0) * sizeof(float);
  const size_t end_stage = x;
  x = o;
  L.C = x; x += 2 * (size_t)P.n_max * KS * sizeof(float);
  L.P = x; x += (size_t)P.n_kept * sizeof(float);
  L.S = x; x += (size_t)P.n_soap * sizeof(float);
  if (P.ps_mt > 0) {
    x = align_up(x, 16);
    L.Pl = x; x += (size_t)(P.l_max + 1) * 16 * P.ps_mt * 8 * P.ps_nt * sizeof(float);
  }
  L.total = align_up(end_stage > x ? end_stage : x, 16);
  return L;
}

template <int NT, int AMAX, int LC>
__global__ void __launch_bounds__(NT) k_descriptor_tc(const DevParams P, const DevBatch B,
                                                      double *__restrict__ soap_out, float *__restrict__ keep_c,
                                                      double *__restrict__ keep_norm, int keep) {
  static_assert(NT == 128, "one thread per TMEM lane");
  extern __shared__ __align__(16) unsigned char smem[];  // no-swizzle operand tiles need 16-byte alignment
  const int AS = stage_stride(LC, 0);
  const TdLayout Ly = make_td_layout(P, NT, AMAX, LC);
  const int *klm = (const int *)SBLOB(off_klm);
  const int *kept = (const int *)SBLOB(off_kept);
  const double *central = (const double *)SBLOB(off_central);
  double *sRed = (double *)(smem + Ly.red);
  float *sR = (float *)(smem + Ly.R);
  float *sA = (float *)(smem + Ly.A);
  float *sC = (float *)(smem + Ly.C);
  float *sP = (float *)(smem + Ly.P);
  float *sS = (float *)(smem + Ly.S);
  unsigned char *sAhi = smem + Ly.Ahi, *sAlo = smem + Ly.Alo, *sBhi = smem + Ly.Bhi, *sBlo = smem + Ly.Blo;
  uint64_t *mbar = (uint64_t *)(smem + Ly.mbar);
  uint32_t *tmem_slot = (uint32_t *)(smem + Ly.tmem);
  int *sEnt = (int *)(smem + Ly.ent);
  int *sW_cnt = (int *)(smem + Ly.wcnt);
  int *sMisc = (int *)(smem + Ly.misc);
  int *sBase = sMisc, *sCnt = sMisc + SOAPB_MAX_SPECIES, *sNent = sMisc + 2 * SOAPB_MAX_SPECIES;
  int *sSite = sMisc + 3 * SOAPB_MAX_SPECIES;

  const int tid = threadIdx.x, warp = tid >> 5;
  const int KS = P.k_max | 1;
  const int n_max = P.n_max, nsp = P.n_species, k_max = P.k_max;
  const uint32_t idesc = tc::idesc_tf32(128, kTdCols);
  copy_site_blob<NT>(P, smem, 0);
  if (warp == 0) tc::tmem_alloc(tmem_slot, kTdTmemCols);
  if (tid == 0) tc::mbar_init(mbar);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  // this thread's row of D: (k, re/im)
  const int my_k = tid >> 1, my_ri = tid & 1;
  const int my_l = my_k < k_max ? (klm[my_k] & 0xff) : 0, my_m = my_k < k_max ? (klm[my_k] >> 8) : 0;
  const uint32_t tmem = *tmem_slot;
  uint32_t phase = 0;
  bool failed = false;
  int col_s = -1, col_n = 0;  // (tid < 32) the species and local index of D column tid
  if (tid < kTdCols)
    for (int s = 0; s < nsp; ++s) {
      const RadSp &RS = rad_of(smem, P, s);
      if (tid >= RS.nbeg && tid < RS.nbeg + RS.alpha) {
        col_s = s;
        col_n = tid - RS.nbeg;
      }
    }

  first_site(B, B.ticket, sSite);
  for (;;) {
    const int site = sSite[0];
    if (site >= B.site_hi || failed) break;
    const int p_begin = sSite[1];
    const int p_end = min(sSite[2], B.n_pairs);
    int nx = 0, nx0 = 0, nx1 = 0;
    if (tid == 0) nx = take_ticket(B, B.ticket);
    double acc[kTdCols];
#pragma unroll
    for (int n = 0; n < kTdCols; ++n) acc[n] = 0.0;

    for (int chunk = p_begin; chunk < p_end && !failed; chunk += NT) {
      int slot[SOAPB_MAX_SPECIES];
      unsigned my_bits;
      double my_r;
      const int n_ent = build_entries<NT>(P, B, p_begin, chunk, p_end, false, sEnt, sW_cnt, sBase, sCnt, sNent,
                                          slot, my_bits, my_r);
      for (int ebase = 0; ebase < n_ent; ebase += kTdGroup) {
        const int n_g = min(kTdGroup, n_ent - ebase);
        // ---- the group's rows (angular and radial) into shared memory
        stage_entries<NT, AMAX, LC, false>(P, B, sEnt, chunk, ebase, n_g, sA, sR, nullptr);
        __syncthreads();
        // the central pair's entries carry central_weight (:638-646)
        if (chunk == p_begin) {
          for (int el = tid; el < n_g; el += NT) {
            const int code = sEnt[ebase + el];
            const double cw = rad_of(smem, P, code >> 24).cw;
            if ((code & 0xffffff) == 0 && cw != 1.0)
#pragma unroll
              for (int n = 0; n < AMAX; ++n) sR[(size_t)el * AMAX + n] *= (float)cw;
          }
          __syncthreads();
        }
        // ---- A operand: row (k, re/im) of this thread, 16 entries
        {
          float v[kTdGroup];
#pragma unroll
          for (int e = 0; e < kTdGroup; ++e) {
            v[e] = 0.f;
            if (e < n_g && my_k < k_max) {
              const float *Ae = sA + (size_t)e * AS;
              // u_k = (preflm_k P_k)(amp i_l) (src/soap_turbo_angular.f90:590-594)
              const float u = Ae[row_p(LC) + my_k] * Ae[row_il(LC) + my_l];
              v[e] = u * Ae[(my_ri ? row_ei(LC) : row_er(LC)) + my_m];
            }
          }
#pragma unroll
          for (int e4 = 0; e4 < kTdGroup / 4; ++e4) {
            uint4 h, lo;
            tc::split(v[4 * e4], h.x, lo.x);
            tc::split(v[4 * e4 + 1], h.y, lo.y);
            tc::split(v[4 * e4 + 2], h.z, lo.z);
            tc::split(v[4 * e4 + 3], h.w, lo.w);
            const uint32_t off = tc::kmajor_off(tid, 4 * e4, kTdGroup);
            *(uint4 *)(sAhi + off) = h;
            *(uint4 *)(sAlo + off) = lo;
          }
        }
        // ---- B operand: row n, the entries' R_n of their species (else 0)
        if (tid < kTdCols) {
          float v[kTdGroup];
#pragma unroll
          for (int e = 0; e < kTdGroup; ++e) {
            v[e] = 0.f;
            if (e < n_g && col_s >= 0 && (sEnt[ebase + e] >> 24) == col_s) v[e] = sR[(size_t)e * AMAX + col_n];
          }
#pragma unroll
          for (int e4 = 0; e4 < kTdGroup / 4; ++e4) {
            uint4 h, lo;
            tc::split(v[4 * e4], h.x, lo.x);
            tc::split(v[4 * e4 + 1], h.y, lo.y);
            tc::split(v[4 * e4 + 2], h.z, lo.z);
            tc::split(v[4 * e4 + 3], h.w, lo.w);
            const uint32_t off = tc::kmajor_off(tid, 4 * e4, kTdGroup);
            *(uint4 *)(sBhi + off) = h;
            *(uint4 *)(sBlo + off) = lo;
          }
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
          const uint32_t ahi = tc::smem_addr(sAhi), alo = tc::smem_addr(sAlo);
          const uint32_t bhi = tc::smem_addr(sBhi), blo = tc::smem_addr(sBlo);
          for (int k0 = 0; k0 < kTdGroup; k0 += 8)
            tc::mma3_step(tmem, ahi, alo, kTdGroup, bhi, blo, kTdGroup, k0, idesc, k0 > 0);
          tc::commit(mbar);
        }
        const int ok = tc::mbar_wait(mbar, phase, tc::kMaxTries);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
          if (tid == 0) prep_error(B, kErrTc);
          tc::mbar_wait(mbar, phase ^ 1u, tc::kMaxTries);
          failed = true;
          break;
        }
        tc::fence_after_sync();
        // ---- the group's FP32 partial sums into the FP64 accumulators
#pragma unroll
        for (int j = 0; j < kTdCols / 16; ++j) {
          float v[16];
          tc::ld16(tc::taddr(tmem, 32 * warp, 16 * j), v);
#pragma unroll
          for (int q = 0; q < 16; ++q) acc[16 * j + q] += (double)v[q];
        }
        tc::fence_before_sync();
        __syncthreads();
      }
    }
    if (failed) break;
    ahead_bounds(B, nx, nx0, nx1);
    // ---- poly3gauss central-atom term (src/soap_turbo.f90:646-662), row (k = 0, re)
    if (P.basis == 1 && tid == 0) {
      const int mult = B.species_mult[site];
      for (int mm = 0; mm < mult; ++mm) {
        const int s = B.species[(size_t)site * B.max_mult + mm] - 1;
        if (s < 0 || s >= nsp) continue;
        const RadSp &RS = rad_of(smem, P, s);
#pragma unroll
        for (int n = 0; n < kTdCols; ++n)
          if (n >= RS.nbeg && n < RS.nbeg + RS.alpha) acc[n] += central[n];
      }
    }
    // ---- c_nlm to FP32 in sC (re/im, n, KS); the padding column k_max stays 0
    if (my_k < KS)
#pragma unroll
      for (int n = 0; n < kTdCols; ++n)
        if (n < n_max) sC[(size_t)(my_ri * n_max + n) * KS + my_k] = my_k < k_max ? (float)acc[n] : 0.f;
    __syncthreads();
    // ---- power spectrum on the tensor cores (src/soap_turbo.f90:750-795): per
    // group of l, A = rows (l, n) with X_l[n] = (Re c_nl0, r2 Re c_nl1 .., Im
    // c_nl0, r2 Im c_nl1 ..) in l's block of K (zero elsewhere), the J rows
    // first; B = A's first rows, so D[(l, n)][(l, j)] = P_l[n, J_j] (the other
    // blocks of D are zero and unread).  Written to sPl as ps_tensor writes it.
    const bool ps_tc = P.ps_ng > 0;
    if (ps_tc) {
      float *sPl = (float *)(smem + Ly.Pl);
      const int *psrow = (const int *)SBLOB(off_psrow);
      unsigned char *sPhi = smem + Ly.Phi, *sPlo = smem + Ly.Plo;
      const int MR = 16 * P.ps_mt, JP = 8 * P.ps_nt, nJ = P.ps_nj;
      for (int g = 0; g < P.ps_ng && !failed; ++g) {
        const int K = P.ps_gk[g], NB = P.ps_gnb[g];
        int l = -1, n = 0, cb = 0;
        if (tid < P.ps_grows[g]) {
          const int code = psrow[P.ps_grow[g] + tid];
          n = code & 0xff;
          l = (code >> 8) & 0xff;
          cb = code >> 16;
        }
        const int ko = l >= 0 ? P.ps_ko[l] : 0, kb = l * (l + 1) / 2;
        for (int k4 = 0; k4 < K; k4 += 4) {
          float v[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int c = k4 + q - ko;
            v[q] = 0.f;
            if (l >= 0 && c >= 0 && c < 2 * (l + 1)) {
              const int im = c > l, m = im ? c - l - 1 : c;
              const float x = sC[(size_t)(im ? n_max + n : n) * KS + kb + m];
              v[q] = m ? 1.41421356237309504880f * x : x;
            }
          }
          uint4 h, lo;
          tc::split(v[0], h.x, lo.x);
          tc::split(v[1], h.y, lo.y);
          tc::split(v[2], h.z, lo.z);
          tc::split(v[3], h.w, lo.w);
          const uint32_t off = tc::kmajor_off(tid, k4, K);
          *(uint4 *)(sPhi + off) = h;
          *(uint4 *)(sPlo + off) = lo;
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
          const uint32_t phi = tc::smem_addr(sPhi), plo = tc::smem_addr(sPlo);
          const uint32_t id = tc::idesc_tf32(128, NB);
          for (int k0 = 0; k0 < K; k0 += 8) tc::mma3_step(tmem, phi, plo, K, phi, plo, K, k0, id, k0 > 0);
          tc::commit(mbar);
        }
        const int ok = tc::mbar_wait(mbar, phase, tc::kMaxTries);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
          if (tid == 0) prep_error(B, kErrTc);
          tc::mbar_wait(mbar, phase ^ 1u, tc::kMaxTries);
          failed = true;
          break;
        }
        tc::fence_after_sync();
        for (int j = 0; j < NB / 16; ++j) {
          float v[16];
          tc::ld16(tc::taddr(tmem, 32 * warp, 16 * j), v);
          if (l >= 0)
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              const int jc = 16 * j + q - cb;
              if (jc >= 0 && jc < nJ) sPl[(size_t)(l * MR + n) * JP + jc] = v[q];
            }
        }
        tc::fence_before_sync();
        __syncthreads();
      }
      if (failed) break;
    }
    site_output<NT>(P, smem, sC, sP, sS, (float *)(smem + Ly.Pl), kept, sRed, site, soap_out, keep_c, keep_norm,
                    keep, P.ps_mt > 0, ps_tc);
    ahead_publish(sSite, nx, nx0, nx1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTdTmemCols);
}

// ------------------------------------------------------------ contract
constexpr int kHM = 3;  // m values per H item (the host's items must agree)

template <int NT, int AMAX, int LC>
__global__ void __launch_bounds__(NT, 512 / NT) k_contract(const DevParams P, const DevBatch B,
                                                    const double *__restrict__ soap_in,
                                                    const double *__restrict__ G, int g_layout,
                                                    double sgn, const float *__restrict__ keep_c,
                                                    const double *__restrict__ keep_norm,
                                                    double *__restrict__ pair_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int CH = stage_entries_per_round(NT, 1);
  constexpr int KC = (LC + 1) * (LC + 2) / 2;
  constexpr int KJ = (KC + 15) / 16;
  constexpr int GPT = 8;  // G values a thread holds while the norm dot product is reduced
  static_assert(AMAX % 4 == 0, "vector loads of H need AMAX % 4 == 0");
  const int AS = stage_stride(LC, 1);
  constexpr int O_IL = row_il(LC), O_ILD = row_ild(LC), O_ER = row_er(LC), O_EI = row_ei(LC),
                O_SF = row_sf(LC), O_X = row_x(LC), O_SQ = row_sq(LC),
                O_P = row_p(LC);
  const Layout Ly = make_layout(P, NT, AMAX, LC, 1);
  const int4 *kidx = (const int4 *)SBLOBC(off_kidx);
  const float4 *kcoef = (const float4 *)SBLOBC(off_kcoef);
  const int *klm = (const int *)SBLOBC(off_klm_c);
  const int *nmap = (const int *)SBLOBC(off_nmap);
  const int *hitem = (const int *)SBLOBC(off_hitem);
  const int *hloff = (const int *)SBLOBC(off_hloff);
  const int *hl = P.hl_in_blob ? (const int *)SBLOBC(off_hl) : P.hl_packed;
  double *sRed = (double *)(smem + Ly.red);
  float *sH = (float *)(smem + Ly.H);
  float *sRot = (float *)(smem + Ly.Rot);
  float *sF = (float *)(smem + Ly.F);
  float *sC = (float *)(smem + Ly.C);
  float *sGu = (float *)(smem + Ly.P);
  float *sGp = (float *)(smem + Ly.S);
  float *sR = (float *)(smem + Ly.R);
  float *sRd = (float *)(smem + Ly.Rd);
  float *sA = (float *)(smem + Ly.A);
  int *sEnt = (int *)(smem + Ly.ent);
  int *sW_cnt = (int *)(smem + Ly.wcnt);
  int *sMisc = (int *)(smem + Ly.misc);
  int *sBase = sMisc, *sCnt = sMisc + SOAPB_MAX_SPECIES, *sNent = sMisc + 2 * SOAPB_MAX_SPECIES;
  int *sSite = sMisc + 3 * SOAPB_MAX_SPECIES;

  const int tid = threadIdx.x;
  const int KS = P.k_max | 1;
  const int HS = h_stride(P.n_species, AMAX);
  const size_t HPL = (size_t)KS * HS;  // H plane (re, then im)
  const int n_max = P.n_max, k_max = P.k_max, n_soap = P.n_soap, nsp = P.n_species;
  const int n_sites = B.n_sites;
  const int hw = tid >> 4, hl16 = tid & 15;
  float *sGu_eff = P.cmap_identity ? sGp : sGu;

  copy_site_blob<NT>(P, smem, 1);
  for (int t = tid; t < 2 * (int)HPL; t += NT) sH[t] = 0.f;  // entries no item writes stay 0
  first_site(B, B.ticket + 1, sSite);
  for (;;) {
    const int site = sSite[0];
    if (site >= B.site_hi) break;
    const int p_begin = sSite[1];
    const int p_end = min(sSite[2], B.n_pairs);
    int nx = 0, nx0 = 0, nx1 = 0;
    if (tid == 0) nx = take_ticket(B, B.ticket + 1);  // the next site, fetched ahead
    // ---- every per-site load is issued here, so their latencies overlap
    const double knorm = keep_norm[site];
    const double *q = soap_in + (size_t)site * n_soap;
    double gv[GPT], qv[GPT];
#pragma unroll
    for (int j = 0; j < GPT; ++j) {
      const int o = tid + j * NT;
      gv[j] = qv[j] = 0.0;
      if (o < n_soap) {
        gv[j] = g_layout == 0 ? G[(size_t)o * n_sites + site] : G[(size_t)site * n_soap + o];
        qv[j] = q[o];
      }
    }
    {
      const float *kc = keep_c + (size_t)site * keep_stride(P);
      const int n4 = (2 * n_max * KS) / 4;
      for (int t = tid; t < n4; t += NT) cp_async16(sC + 4 * t, kc + 4 * t);
      for (int t = 4 * n4 + tid; t < 2 * n_max * KS; t += NT) sC[t] = kc[t];
      cp_async_wait_all();
    }
    // ---- back through the normalisation (src/soap_turbo.f90:1783-1790)
    double qg = 0.0;
#pragma unroll
    for (int j = 0; j < GPT; ++j) qg += qv[j] * gv[j];
    for (int o = tid + GPT * NT; o < n_soap; o += NT) {
      const double g = g_layout == 0 ? G[(size_t)o * n_sites + site] : G[(size_t)site * n_soap + o];
      sGp[o] = (float)g;  // staged raw; finished below
      qg += q[o] * g;
    }
    qg = block_sum<NT>(qg, sRed);
    const double inv = 1.0 / knorm;
#pragma unroll
    for (int j = 0; j < GPT; ++j) {
      const int o = tid + j * NT;
      if (o < n_soap) sGp[o] = (float)((gv[j] - qv[j] * qg) * inv);
    }
    for (int o = tid + GPT * NT; o < n_soap; o += NT) sGp[o] = (float)(((double)sGp[o] - q[o] * qg) * inv);
    __syncthreads();
    // ---- back through the compression (:1791-1798), unless it is one-to-one
    if (!P.cmap_identity) {
      for (int t = tid; t < P.n_kept; t += NT) {
        float v = 0.f;
        for (int e = P.pj_off[t]; e < P.pj_off[t + 1]; ++e) v += P.pj_el[e] * sGp[P.pj_o[e]];
        sGu[t] = v;
      }
      __syncthreads();
    }
    // ---- H(k,n) = w(m) sum_np Y(n,np,l) c(k,np) over the non-zero Y (:1800-1835);
    // one item per (n, l, m0) walks its Y list once for m = m0 .. m0 + kHM - 1
    // (up to l); the host orders the items heaviest first.  Every H entry an
    // item writes is rewritten at every site; the others stay 0.
    for (int it = tid; it < P.n_hitem; it += NT) {
      const int code = hitem[it];
      const int n = code & 0xff, l = (code >> 8) & 0xff, m0 = code >> 16;
      const int kb = l * (l + 1) / 2 + m0, mn = min(kHM, l + 1 - m0);
      float hr[kHM], hi[kHM];
#pragma unroll
      for (int j = 0; j < kHM; ++j) hr[j] = hi[j] = 0.f;
      const int li = l * n_max + n;
      for (int t = hloff[li]; t < hloff[li + 1]; ++t) {
        const int e = hl[t];
        const int np = e & 0xff, qq = (e >> 8) & 0xffff;
        const float y = ((e >> 31) ? 2.f : 1.41421356237309504880f) * sGu_eff[qq];
        const float *cr = sC + (size_t)np * KS + kb;
        const float *ci = cr + (size_t)n_max * KS;
#pragma unroll
        for (int j = 0; j < kHM; ++j) {
          if (j < mn) {
            hr[j] = fmaf(y, cr[j], hr[j]);
            hi[j] = fmaf(y, ci[j], hi[j]);
          }
        }
      }
      const int nm = nmap[n];
      const int col = (nm & 0xff) * AMAX + (nm >> 8);
#pragma unroll
      for (int j = 0; j < kHM; ++j) {
        if (j < mn) {
          const float w = (m0 + j == 0) ? 1.f : 2.f;
          sH[(size_t)(kb + j) * HS + col] = w * hr[j];
          sH[HPL + (size_t)(kb + j) * HS + col] = w * hi[j];
        }
      }
    }
    __syncthreads();
    ahead_bounds(B, nx, nx0, nx1);

    double self_x = 0.0, self_y = 0.0, self_z = 0.0;

    for (int chunk = p_begin; chunk < p_end; chunk += NT) {
      int slot[SOAPB_MAX_SPECIES];
      unsigned my_bits;
      double my_r;
      const int n_ent = build_entries<NT>(P, B, p_begin, chunk, p_end, true, sEnt, sW_cnt, sBase,
                                          sCnt, sNent, slot, my_bits, my_r);
      for (int ebase = 0; ebase < n_ent; ebase += CH) {
        const int n_round = min(CH, n_ent - ebase);
        // ---- A. the entries' angular rows and radial rows
        stage_entries<NT, AMAX, LC, true>(P, B, sEnt, chunk, ebase, n_round, sA, sR, sRd);
        __syncthreads();
        // ---- B. contraction against H: a half-warp per entry, lanes over k.
        // Lane hl16 of a half-warp handles k = hl16 + 16 j.
        int4 kix[KJ];
        float4 kcf[KJ];
        int klmr[KJ];
#pragma unroll
        for (int j = 0; j < KJ; ++j) {
          const int kk = hl16 + 16 * j;
          const bool v = kk < k_max;
          kix[j] = v ? kidx[kk] : make_int4(0, 0, 0, 0);
          kcf[j] = v ? kcoef[kk] : make_float4(0.f, 0.f, 0.f, 0.f);
          klmr[j] = v ? klm[kk] : -1;
        }
        // The loop bound is uniform per warp (both halves iterate together) so
        // the full-mask shuffles below always see all 32 lanes.
        for (int eb = 2 * (tid >> 5); eb < n_round; eb += NT / 16) {
          const int el = eb + (hw & 1);
          const bool act = el < n_round;
          float f_rad = 0.f, f_azi = 0.f, f_pol = 0.f;
          if (act) {
            const int code = sEnt[ebase + el];
            const int s = code >> 24;
            const float *Ae = sA + (size_t)el * AS;
            const float *Pe = Ae + O_P;
            if (hl16 == 0) {
              // the rotation to Cartesian uses the same angles (:1867-1871)
              float *rot = sRot + 4 * (code & 0xffffff);
              rot[0] = Ae[O_X];
              rot[1] = Ae[O_SQ];
              rot[2] = Ae[O_ER + 1];
              rot[3] = -Ae[O_EI + 1];
            }
            float R[AMAX], Rd[AMAX];
#pragma unroll
            for (int n4 = 0; n4 < AMAX / 4; ++n4) {
              const float4 a = ((const float4 *)(sR + (size_t)el * AMAX))[n4];
              const float4 d = ((const float4 *)(sRd + (size_t)el * AMAX))[n4];
              R[4 * n4] = a.x; R[4 * n4 + 1] = a.y; R[4 * n4 + 2] = a.z; R[4 * n4 + 3] = a.w;
              Rd[4 * n4] = d.x; Rd[4 * n4 + 1] = d.y; Rd[4 * n4 + 2] = d.z; Rd[4 * n4 + 3] = d.w;
            }
            const float sfac = Ae[O_SF];
            const float *Hs = sH + (size_t)s * AMAX;
#pragma unroll
            for (int j = 0; j < KJ; ++j) {
              if (klmr[j] < 0) continue;
              const int kk = hl16 + 16 * j;
              const int l = klmr[j] & 0xff, m = klmr[j] >> 8;
              const float Pk = Pe[kk];
              const float dms = kcf[j].x * Pe[kix[j].x] + kcf[j].y * Pe[kix[j].y];
              const float dvs = kcf[j].z * Pe[kix[j].z] + kcf[j].w * Pe[kix[j].w];
              // rows hold amp i_l, amp di_l/dr and preflm_k P_k; kcoef carries the
              // preflm ratios of the derivative combinations
              const float il = Ae[O_IL + l], ild = Ae[O_ILD + l];
              const float er = Ae[O_ER + m], ei = Ae[O_EI + m];
              const float u = Pk * il;
              const float ur = Pk * ild - sfac * u;
              const float ua = dvs * il;
              const float up = dms * il;
              const float4 *hr4 = (const float4 *)(Hs + (size_t)kk * HS);
              const float4 *hi4 = (const float4 *)(Hs + HPL + (size_t)kk * HS);
              float Ur = 0.f, Ui = 0.f, Vr = 0.f, Vi = 0.f;
#pragma unroll
              for (int n4 = 0; n4 < AMAX / 4; ++n4) {
                const float4 hr = hr4[n4], hi = hi4[n4];
                Ur = fmaf(Rd[4 * n4], hr.x, Ur); Ur = fmaf(Rd[4 * n4 + 1], hr.y, Ur);
                Ur = fmaf(Rd[4 * n4 + 2], hr.z, Ur); Ur = fmaf(Rd[4 * n4 + 3], hr.w, Ur);
                Ui = fmaf(Rd[4 * n4], hi.x, Ui); Ui = fmaf(Rd[4 * n4 + 1], hi.y, Ui);
                Ui = fmaf(Rd[4 * n4 + 2], hi.z, Ui); Ui = fmaf(Rd[4 * n4 + 3], hi.w, Ui);
                Vr = fmaf(R[4 * n4], hr.x, Vr); Vr = fmaf(R[4 * n4 + 1], hr.y, Vr);
                Vr = fmaf(R[4 * n4 + 2], hr.z, Vr); Vr = fmaf(R[4 * n4 + 3], hr.w, Vr);
                Vi = fmaf(R[4 * n4], hi.x, Vi); Vi = fmaf(R[4 * n4 + 1], hi.y, Vi);
                Vi = fmaf(R[4 * n4 + 2], hi.z, Vi); Vi = fmaf(R[4 * n4 + 3], hi.w, Vi);
              }
              const float reU = er * Ur + ei * Ui;
              const float reV = er * Vr + ei * Vi;
              const float imV = ei * Vr - er * Vi;
              f_rad = fmaf(u, reU, fmaf(ur, reV, f_rad));
              f_azi = fmaf(-ua, imV, f_azi);
              f_pol = fmaf(up, reV, f_pol);
            }
          }
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) {
            f_rad += __shfl_xor_sync(0xffffffffu, f_rad, o);
            f_azi += __shfl_xor_sync(0xffffffffu, f_azi, o);
            f_pol += __shfl_xor_sync(0xffffffffu, f_pol, o);
          }
          if (act && hl16 == 0) {
            float *Fe = sF + (size_t)(ebase + el) * 3;
            Fe[0] = f_rad;
            Fe[1] = f_azi;
            Fe[2] = f_pol;
          }
        }
        __syncthreads();
      }
      // ---- per pair: sum its entries, rotate to Cartesian (:1864-1875)
      const int k = chunk + tid;
      if (k < p_end && k > p_begin) {
        double px = 0.0, py = 0.0, pz = 0.0;
        if (my_bits != 0u) {
          double fr = 0.0, fa = 0.0, fp = 0.0;
#pragma unroll
          for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) {
            if (s < nsp && slot[s] >= 0) {
              fr += sF[3 * slot[s] + 0];
              fa += sF[3 * slot[s] + 1];
              fp += sF[3 * slot[s] + 2];
            }
          }
          const float *rot = sRot + 4 * tid;
          const double ct = rot[0], st = rot[1], cf = rot[2], sf = rot[3];
          const double ir = 1.0 / my_r;
          px = sgn * (st * cf * fr - ct * cf * ir * fp - sf * ir * fa);
          py = sgn * (st * sf * fr - ct * sf * ir * fp + cf * ir * fa);
          pz = sgn * (ct * fr + st * ir * fp);
        }
        double *po = pair_out + (size_t)3 * k;
        po[0] = px;
        po[1] = py;
        po[2] = pz;
        self_x -= px;
        self_y -= py;
        self_z -= pz;
      }
    }
    // the central pair is minus the sum of the others (:1875)
    block_sum3<NT>(self_x, self_y, self_z, sRed);
    if (tid == 0 && p_end > p_begin) {
      double *po = pair_out + (size_t)3 * p_begin;
      po[0] = self_x;
      po[1] = self_y;
      po[2] = self_z;
    }
    ahead_publish(sSite, nx, nx0, nx1);
  }
}

// ------------------------------------------------------------ contract on tensor cores
// soap_contract (src/soap_turbo.f90:1723-1884) with the per-entry contraction
// on the tensor cores.  Per site, as k_contract: Gp, Gu and H(k, n) on the CUDA
// cores.  H becomes the B operand of a tcgen05 MMA, [96 columns c = 2k + re/im
// (k < 48, beyond k_max zero) x KB = n_species * AMAX] (K-major, split into
// TF32 head and tail).  The site's entries go in rounds of 64: the A operand
// is [128 x KB], row e < 64 the entry's dR_n/dr and row 64 + e its R_n, each
// in its species' AMAX columns (zero elsewhere), so that one 3xTF32 product
// D = A B^T (9 MMAs of 128 x 96 x 8) gives every entry's
//   U(k) = sum_n dR_n/dr H(k, n)  (rows < 64),   V(k) = sum_n R_n H(k, n)  (rows >= 64)
// in TMEM (the reference's four dot products per n, src/soap_turbo.f90:
// 1842-1866, reassociated over n).  Thread t < 64 then takes U of entry t and
// forms u Re(e conj U); thread 64 + t takes V of entry t and forms the rest of
// the radial, azimuthal and polar sums, each over k in a fixed order, from the
// entry's angular row (read from global memory, where the descriptor's pair
// kernel left it).  The per-pair rotation and the self pair are k_contract's.
constexpr int kTcEntries = 64;   // entries per round
constexpr int kTcCols = 96;      // U / V columns: 2 k + re/im for k < 48
constexpr int kTcTmemCols = 128; // TMEM columns a CTA holds

__host__ __device__ inline int tc_kb(const DevParams &P, int AMAX) { return (P.n_species * AMAX + 7) / 8 * 8; }

struct TcLayout {
  size_t red, ent, wcnt, misc, H, Rot, F, Fu, Bhi, Blo, X, Ahi, Alo, AT, C, Gu, Gp, mbar, tmem, total;
};
__host__ __device__ inline TcLayout make_tc_layout(const DevParams &P, int NT, int AMAX) {
  TcLayout L{};
  const size_t KS = (size_t)(P.k_max | 1), nsp = (size_t)P.n_species, KB = (size_t)tc_kb(P, AMAX);
  size_t o = site_blob_bytes(P, 1);
  L.red = o;  o += 40 * sizeof(double);
  L.ent = o;  o += (size_t)NT * nsp * sizeof(int);
  L.wcnt = o; o += (size_t)SOAPB_MAX_SPECIES * (NT / 32) * sizeof(int);
  L.misc = o; o += 64 * sizeof(int);
  L.mbar = align_up(o, 8); o = L.mbar + 8;
  L.tmem = o; o += 8;
  o = align_up(o, 16);
  L.H = o;   o += 2 * KS * (size_t)h_stride(P.n_species, AMAX) * sizeof(float);
  L.Rot = o; o += (size_t)NT * 4 * sizeof(float);
  L.F = o;   o += (size_t)NT * nsp * 3 * sizeof(float);
  L.Fu = o;  o += (size_t)NT * nsp * sizeof(float);
  o = align_up(o, 1024);
  L.Bhi = o; o += (size_t)kTcCols * KB * 4;
  L.Blo = o; o += (size_t)kTcCols * KB * 4;
  o = align_up(o, 1024);
  L.X = o;
  // per round: the A tiles; per site (before H is built): c_nlm, Gu, Gp
  size_t x = o;
  L.Ahi = x; x += 128 * KB * 4;
  L.Alo = x; x += 128 * KB * 4;
  L.AT = x;  x += (size_t)row_len(AMAX == 8 ? 8 : 12) * kTcEntries * 4;  // the round's angular rows, transposed
  const size_t end_round = x;
  x = o;
  L.C = x;  x += 2 * (size_t)P.n_max * KS * sizeof(float);
  L.Gu = x; x += (size_t)P.n_kept * sizeof(float);
  L.Gp = x; x += (size_t)P.n_soap * sizeof(float);
  L.total = align_up(end_round > x ? end_round : x, 16);
  return L;
}

__host__ __device__ constexpr int tc_l_of(int kk) {
  int l = 0;
  while ((l + 1) * (l + 2) / 2 <= kk) ++l;
  return l;
}
__host__ __device__ constexpr int tc_m_of(int kk) { return kk - tc_l_of(kk) * (tc_l_of(kk) + 1) / 2; }

template <int NT, int AMAX, int LC>
__global__ void __launch_bounds__(NT) k_contract_tc(const DevParams P, const DevBatch B,
                                                    const double *__restrict__ soap_in,
                                                    const double *__restrict__ G, int g_layout, double sgn,
                                                    const float *__restrict__ keep_c,
                                                    const double *__restrict__ keep_norm,
                                                    double *__restrict__ pair_out) {
  static_assert(NT == 128, "one thread per TMEM lane");
  constexpr int KC = (LC + 1) * (LC + 2) / 2;
  static_assert(KC <= 2 * kTcCols / 4 && 2 * KC <= kTcCols, "U/V columns");
  constexpr int GPT = 8;
  constexpr int AW = row_len(LC);
  constexpr int O_IL = row_il(LC), O_ILD = row_ild(LC), O_ER = row_er(LC), O_EI = row_ei(LC),
                O_SF = row_sf(LC), O_X = row_x(LC), O_SQ = row_sq(LC), O_P = row_p(LC);
  extern __shared__ __align__(16) unsigned char smem[];  // no-swizzle operand tiles need 16-byte alignment
  const TcLayout Ly = make_tc_layout(P, NT, AMAX);
  const float4 *kcoef = (const float4 *)SBLOBC(off_kcoef);
  const int *nmap = (const int *)SBLOBC(off_nmap);
  const int *hitem = (const int *)SBLOBC(off_hitem);
  const int *hloff = (const int *)SBLOBC(off_hloff);
  const int *hl = P.hl_in_blob ? (const int *)SBLOBC(off_hl) : P.hl_packed;
  double *sRed = (double *)(smem + Ly.red);
  float *sH = (float *)(smem + Ly.H);
  float *sRot = (float *)(smem + Ly.Rot);
  float *sF = (float *)(smem + Ly.F);
  float *sFu = (float *)(smem + Ly.Fu);
  float *sC = (float *)(smem + Ly.C);
  float *sGu = (float *)(smem + Ly.Gu);
  float *sGp = (float *)(smem + Ly.Gp);
  unsigned char *sAhi = smem + Ly.Ahi, *sAlo = smem + Ly.Alo, *sBhi = smem + Ly.Bhi, *sBlo = smem + Ly.Blo;
  float *sAT = (float *)(smem + Ly.AT);
  uint64_t *mbar = (uint64_t *)(smem + Ly.mbar);
  uint32_t *tmem_slot = (uint32_t *)(smem + Ly.tmem);
  int *sEnt = (int *)(smem + Ly.ent);
  int *sW_cnt = (int *)(smem + Ly.wcnt);
  int *sMisc = (int *)(smem + Ly.misc);
  int *sBase = sMisc, *sCnt = sMisc + SOAPB_MAX_SPECIES, *sNent = sMisc + 2 * SOAPB_MAX_SPECIES;
  int *sSite = sMisc + 3 * SOAPB_MAX_SPECIES;
  int *sFail = sMisc + 3 * SOAPB_MAX_SPECIES + 4;

  const int tid = threadIdx.x, warp = tid >> 5;
  const int KS = P.k_max | 1;
  const int HS = h_stride(P.n_species, AMAX);
  const size_t HPL = (size_t)KS * HS;
  const int n_max = P.n_max, k_max = P.k_max, n_soap = P.n_soap, nsp = P.n_species;
  const int n_sites = B.n_sites;
  const int KB = tc_kb(P, AMAX);
  const uint32_t idesc = tc::idesc_tf32(128, kTcCols);
  float *sGu_eff = P.cmap_identity ? sGp : sGu;

  copy_site_blob<NT>(P, smem, 1);
  for (int t = tid; t < 2 * (int)HPL; t += NT) sH[t] = 0.f;  // entries no item writes stay 0
  if (warp == 0) tc::tmem_alloc(tmem_slot, kTcTmemCols);
  if (tid == 0) {
    tc::mbar_init(mbar);
    *sFail = 0;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  uint32_t phase = 0;
  bool failed = false;

  first_site(B, B.ticket + 1, sSite);
  for (;;) {
    const int site = sSite[0];
    if (site >= B.site_hi || failed) break;
    const int p_begin = sSite[1];
    const int p_end = min(sSite[2], B.n_pairs);
    int nx = 0, nx0 = 0, nx1 = 0;
    if (tid == 0) nx = take_ticket(B, B.ticket + 1);
    // ---- per-site loads, Gp, Gu and H, as k_contract (:1783-1835)
    const double knorm = keep_norm[site];
    const double *q = soap_in + (size_t)site * n_soap;
    double gv[GPT], qv[GPT];
#pragma unroll
    for (int j = 0; j < GPT; ++j) {
      const int o = tid + j * NT;
      gv[j] = qv[j] = 0.0;
      if (o < n_soap) {
        gv[j] = g_layout == 0 ? G[(size_t)o * n_sites + site] : G[(size_t)site * n_soap + o];
        qv[j] = q[o];
      }
    }
    {
      const float *kc = keep_c + (size_t)site * keep_stride(P);
      const int n4 = (2 * n_max * KS) / 4;
      for (int t = tid; t < n4; t += NT) cp_async16(sC + 4 * t, kc + 4 * t);
      for (int t = 4 * n4 + tid; t < 2 * n_max * KS; t += NT) sC[t] = kc[t];
      cp_async_wait_all();
    }
    double qg = 0.0;
#pragma unroll
    for (int j = 0; j < GPT; ++j) qg += qv[j] * gv[j];
    for (int o = tid + GPT * NT; o < n_soap; o += NT) {
      const double g = g_layout == 0 ? G[(size_t)o * n_sites + site] : G[(size_t)site * n_soap + o];
      sGp[o] = (float)g;
      qg += q[o] * g;
    }
    qg = block_sum<NT>(qg, sRed);
    const double inv = 1.0 / knorm;
#pragma unroll
    for (int j = 0; j < GPT; ++j) {
      const int o = tid + j * NT;
      if (o < n_soap) sGp[o] = (float)((gv[j] - qv[j] * qg) * inv);
    }
    for (int o = tid + GPT * NT; o < n_soap; o += NT) sGp[o] = (float)(((double)sGp[o] - q[o] * qg) * inv);
    __syncthreads();
    if (!P.cmap_identity) {
      for (int t = tid; t < P.n_kept; t += NT) {
        float v = 0.f;
        for (int e = P.pj_off[t]; e < P.pj_off[t + 1]; ++e) v += P.pj_el[e] * sGp[P.pj_o[e]];
        sGu[t] = v;
      }
      __syncthreads();
    }
    for (int it = tid; it < P.n_hitem; it += NT) {
      const int code = hitem[it];
      const int n = code & 0xff, l = (code >> 8) & 0xff, m0 = code >> 16;
      const int kb = l * (l + 1) / 2 + m0, mn = min(kHM, l + 1 - m0);
      float hr[kHM], hi[kHM];
#pragma unroll
      for (int j = 0; j < kHM; ++j) hr[j] = hi[j] = 0.f;
      const int li = l * n_max + n;
      for (int t = hloff[li]; t < hloff[li + 1]; ++t) {
        const int e = hl[t];
        const int np = e & 0xff, qq = (e >> 8) & 0xffff;
        const float y = ((e >> 31) ? 2.f : 1.41421356237309504880f) * sGu_eff[qq];
        const float *cr = sC + (size_t)np * KS + kb;
        const float *ci = cr + (size_t)n_max * KS;
#pragma unroll
        for (int j = 0; j < kHM; ++j) {
          if (j < mn) {
            hr[j] = fmaf(y, cr[j], hr[j]);
            hi[j] = fmaf(y, ci[j], hi[j]);
          }
        }
      }
      const int nm = nmap[n];
      const int col = (nm & 0xff) * AMAX + (nm >> 8);
#pragma unroll
      for (int j = 0; j < kHM; ++j) {
        if (j < mn) {
          const float w = (m0 + j == 0) ? 1.f : 2.f;
          sH[(size_t)(kb + j) * HS + col] = w * hr[j];
          sH[HPL + (size_t)(kb + j) * HS + col] = w * hi[j];
        }
      }
    }
    __syncthreads();
    // ---- the B operand: H as [96 x KB], column c = 2 k + (re, im); one row per
    // thread, 16 bytes at a time (H rows are 16-byte aligned: HS is a multiple of 4)
    if (tid < kTcCols) {
      const int c = tid, k = c >> 1;
      const float *hrow = sH + (c & 1) * HPL + (size_t)k * HS;
      for (int kk4 = 0; kk4 < KB; kk4 += 4) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (k < k_max && kk4 < nsp * AMAX) v = *(const float4 *)(hrow + kk4);
        uint4 h, lo;
        tc::split(v.x, h.x, lo.x);
        tc::split(v.y, h.y, lo.y);
        tc::split(v.z, h.z, lo.z);
        tc::split(v.w, h.w, lo.w);
        const uint32_t off = tc::kmajor_off(c, kk4, KB);
        *(uint4 *)(sBhi + off) = h;
        *(uint4 *)(sBlo + off) = lo;
      }
    }
    ahead_bounds(B, nx, nx0, nx1);
    double self_x = 0.0, self_y = 0.0, self_z = 0.0;

    for (int chunk = p_begin; chunk < p_end; chunk += NT) {
      int slot[SOAPB_MAX_SPECIES];
      unsigned my_bits;
      double my_r;
      // (its barriers also order the B tiles' stores before the first round)
      const int n_ent = build_entries<NT>(P, B, p_begin, chunk, p_end, true, sEnt, sW_cnt, sBase, sCnt, sNent,
                                          slot, my_bits, my_r);
      for (int ebase = 0; ebase < n_ent && !failed; ebase += kTcEntries) {
        const int n_round = min(kTcEntries, n_ent - ebase);
        // ---- A operand: rows e < 64 dR/dr, rows 64 + e R, in the species' columns;
        // row tid per thread: its entry's AMAX values, zero in the other columns
        {
          const int e = tid & (kTcEntries - 1);
          int sp = -1;
          float4 rv[AMAX / 4];
#pragma unroll
          for (int j = 0; j < AMAX / 4; ++j) rv[j] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (e < n_round) {
            const int code = sEnt[ebase + e];
            sp = code >> 24;
            const float4 *src = (const float4 *)(B.rad + ((size_t)(chunk + (code & 0xffffff)) * nsp + sp) * 2 * AMAX +
                                                 (tid < kTcEntries ? AMAX : 0));
#pragma unroll
            for (int j = 0; j < AMAX / 4; ++j) rv[j] = src[j];
          }
          for (int kk4 = 0; kk4 < KB; kk4 += 4) {
            const int blk = kk4 / AMAX, j = (kk4 - blk * AMAX) >> 2;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (blk == sp) {
#pragma unroll
              for (int q = 0; q < AMAX / 4; ++q)
                if (q == j) v = rv[q];
            }
            uint4 h, lo;
            tc::split(v.x, h.x, lo.x);
            tc::split(v.y, h.y, lo.y);
            tc::split(v.z, h.z, lo.z);
            tc::split(v.w, h.w, lo.w);
            const uint32_t off = tc::kmajor_off(tid, kk4, KB);
            *(uint4 *)(sAhi + off) = h;
            *(uint4 *)(sAlo + off) = lo;
          }
        }
        // the round's angular rows, transposed to [field][entry] for the epilogue
        // (thread-per-entry reads then fall in distinct banks); pieces of 16 bytes
        for (int t = tid; t < (AW / 4) * kTcEntries; t += NT) {
          const int j4 = t / kTcEntries, e = t - j4 * kTcEntries;
          if (e < n_round) {
            const float4 v = __ldg((const float4 *)(B.ang + (size_t)(chunk + (sEnt[ebase + e] & 0xffffff)) * AW) + j4);
            sAT[(4 * j4) * kTcEntries + e] = v.x;
            sAT[(4 * j4 + 1) * kTcEntries + e] = v.y;
            sAT[(4 * j4 + 2) * kTcEntries + e] = v.z;
            sAT[(4 * j4 + 3) * kTcEntries + e] = v.w;
          }
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
          const uint32_t ahi = tc::smem_addr(sAhi), alo = tc::smem_addr(sAlo);
          const uint32_t bhi = tc::smem_addr(sBhi), blo = tc::smem_addr(sBlo);
          for (int k0 = 0; k0 < KB; k0 += 8) tc::mma3_step(tmem, ahi, alo, KB, bhi, blo, KB, k0, idesc, k0 > 0);
          tc::commit(mbar);
        }
        const int ok = tc::mbar_wait(mbar, phase, tc::kMaxTries);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
          // give up: report, and make sure the MMAs are no longer running
          // before the TMEM is freed
          if (tid == 0) {
            prep_error(B, kErrTc);
            *sFail = 1;
          }
          tc::mbar_wait(mbar, phase ^ 1u, tc::kMaxTries);
          failed = true;
          break;
        }
        tc::fence_after_sync();
        // ---- epilogue: thread tid reads TMEM lane tid
        const bool vrole = tid >= kTcEntries;
        const int e = tid & (kTcEntries - 1);
        const bool act = e < n_round;
        const int code = act ? sEnt[ebase + e] : 0;
        // field f of this entry's row: Ae[f * kTcEntries]
        const float *Ae = sAT + e;
        float il[LC + 1], ild[LC + 1], er[LC + 1], ei[LC + 1], sfac = 0.f;
#pragma unroll
        for (int l = 0; l <= LC; ++l) {
          il[l] = act ? Ae[(O_IL + l) * kTcEntries] : 0.f;
          er[l] = act ? Ae[(O_ER + l) * kTcEntries] : 0.f;
          ei[l] = act ? Ae[(O_EI + l) * kTcEntries] : 0.f;
          ild[l] = (act && vrole) ? Ae[(O_ILD + l) * kTcEntries] : 0.f;
        }
        if (act && vrole) sfac = Ae[O_SF * kTcEntries];
        float f_rad = 0.f, f_azi = 0.f, f_pol = 0.f;
        const float *Pe = Ae + O_P * kTcEntries;
#pragma unroll
        for (int j = 0; j < (2 * KC + 15) / 16; ++j) {
          float v[16];
          tc::ld16(tc::taddr(tmem, 32 * warp, 16 * j), v);
#pragma unroll
          for (int qq = 0; qq < 8; ++qq) {
            const int kk = 8 * j + qq;
            if (kk >= KC) break;
            const int l = tc_l_of(kk), m = tc_m_of(kk);
            if (!act || l > P.l_max) continue;
            const float xr = v[2 * qq], xi = v[2 * qq + 1];
            const float Pk = Pe[kk * kTcEntries];
            const float u = Pk * il[l];
            if (!vrole) {
              f_rad = fmaf(u, er[m] * xr + ei[m] * xi, f_rad);
            } else {
              const float4 cf = kcoef[kk];
              // the derivative forms' P_l^m indices (src/soap_turbo_angular.f90:194-246)
              const int ixx = (m == 0) ? (l > 0 ? l * (l + 1) / 2 + 1 : kk) : kk - 1;
              const int ixy = (m == 0) ? (l > 0 ? l * (l + 1) / 2 + 1 : kk) : (m != l ? kk + 1 : kk);
              const int ixz = (m == 0) ? kk : (l + 1) * (l + 2) / 2 + m - 1;
              const int ixw = (m == 0) ? kk : (l + 1) * (l + 2) / 2 + m + 1;
              const float dms = cf.x * Pe[ixx * kTcEntries] + cf.y * Pe[ixy * kTcEntries];
              const float dvs = cf.z * Pe[ixz * kTcEntries] + cf.w * Pe[ixw * kTcEntries];
              const float ur = Pk * ild[l] - sfac * u;
              const float ua = dvs * il[l];
              const float up = dms * il[l];
              const float reV = er[m] * xr + ei[m] * xi;
              const float imV = ei[m] * xr - er[m] * xi;
              f_rad = fmaf(ur, reV, f_rad);
              f_azi = fmaf(-ua, imV, f_azi);
              f_pol = fmaf(up, reV, f_pol);
            }
          }
        }
        if (act) {
          if (vrole) {
            float *Fe = sF + (size_t)(ebase + e) * 3;
            Fe[0] = f_rad;
            Fe[1] = f_azi;
            Fe[2] = f_pol;
            // the rotation to Cartesian uses the same angles (:1867-1871)
            float *rot = sRot + 4 * (code & 0xffffff);
            rot[0] = Ae[O_X * kTcEntries];
            rot[1] = Ae[O_SQ * kTcEntries];
            rot[2] = er[1];
            rot[3] = -ei[1];
          } else {
            sFu[ebase + e] = f_rad;
          }
        }
        tc::fence_before_sync();
        __syncthreads();
      }
      if (failed) break;
      // ---- per pair: sum its entries, rotate to Cartesian (:1864-1875)
      const int k = chunk + tid;
      if (k < p_end && k > p_begin) {
        double px = 0.0, py = 0.0, pz = 0.0;
        if (my_bits != 0u) {
          double fr = 0.0, fa = 0.0, fp = 0.0;
#pragma unroll
          for (int s = 0; s < SOAPB_MAX_SPECIES; ++s) {
            if (s < nsp && slot[s] >= 0) {
              fr += (double)(sF[3 * slot[s] + 0] + sFu[slot[s]]);
              fa += sF[3 * slot[s] + 1];
              fp += sF[3 * slot[s] + 2];
            }
          }
          const float *rot = sRot + 4 * tid;
          const double ct = rot[0], st = rot[1], cf = rot[2], sf = rot[3];
          const double ir = 1.0 / my_r;
          px = sgn * (st * cf * fr - ct * cf * ir * fp - sf * ir * fa);
          py = sgn * (st * sf * fr - ct * sf * ir * fp + cf * ir * fa);
          pz = sgn * (ct * fr + st * ir * fp);
        }
        double *po = pair_out + (size_t)3 * k;
        po[0] = px;
        po[1] = py;
        po[2] = pz;
        self_x -= px;
        self_y -= py;
        self_z -= pz;
      }
    }
    if (failed) break;
    block_sum3<NT>(self_x, self_y, self_z, sRed);
    if (tid == 0 && p_end > p_begin) {
      double *po = pair_out + (size_t)3 * p_begin;
      po[0] = self_x;
      po[1] = self_y;
      po[2] = self_z;
    }
    ahead_publish(sSite, nx, nx0, nx1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTcTmemCols);
}

// ------------------------------------------------------------ launchers
// What a launch needs from the runtime besides the launch itself -- the
// kernel's dynamic shared memory limit raised, its resident CTAs per SM for a
// persistent grid -- asked once per (kernel, device, CTA size, shared memory)
// and remembered: the drop-in layer launches the same kernels once per site
// chunk, and these queries would otherwise cost it host time on every call.
struct LaunchMemo {
  const void *fn;
  int dev, threads;
  size_t smem;
  int sms, per_sm;
};
struct SmemLimit {
  const void *fn;
  int dev;
  size_t smem;
};
static std::mutex g_launch_mu;
static std::vector<LaunchMemo> g_launch_memo;
static std::vector<SmemLimit> g_smem_limit;

// Raises fn's dynamic shared memory limit on the current device to at least
// smem (never lowers it, so that launches of other sizes stay valid).
template <typename K>
static cudaError_t ensure_smem_limit(K kernel, size_t smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const void *fn = (const void *)kernel;
  std::lock_guard<std::mutex> g(g_launch_mu);
  for (auto &x : g_smem_limit)
    if (x.fn == fn && x.dev == dev) {
      if (x.smem >= smem) return cudaSuccess;
      e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) x.smem = smem;
      return e;
    }
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) g_smem_limit.push_back({fn, dev, smem});
  return e;
}

template <typename K>
static int persistent_grid_query(K kernel, int threads, size_t smem, int dev, int &sms);

template <typename K>
static int persistent_grid(K kernel, int threads, size_t smem, int n_sites, int max_ctas) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  const void *fn = (const void *)kernel;
  bool found = false;
  {
    std::lock_guard<std::mutex> g(g_launch_mu);
    for (const auto &x : g_launch_memo)
      if (x.fn == fn && x.dev == dev && x.threads == threads && x.smem == smem) {
        sms = x.sms;
        per_sm = x.per_sm;
        found = true;
        break;
      }
  }
  if (!found) {
    per_sm = persistent_grid_query(kernel, threads, smem, dev, sms);
    std::lock_guard<std::mutex> g(g_launch_mu);
    g_launch_memo.push_back({fn, dev, threads, smem, sms, per_sm});
  }
  int g = sms * (per_sm > 0 ? per_sm : 1);
  if (max_ctas > 0 && g > max_ctas) g = max_ctas;
  return g < n_sites ? g : n_sites;
}

template <typename K>
static int persistent_grid_query(K kernel, int threads, size_t smem, int dev, int &sms) {
  int per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  // the count from the kernel's registers and shared memory as well: the
  // occupancy query has been seen to answer 1 for CTAs of 66-74 KB that fit
  // three times.  Too many CTAs is harmless here -- a persistent CTA that
  // starts late finds the remaining sites, none waits on another.
  cudaFuncAttributes fa{};
  int sm_per_sm = 0, regs_per_sm = 0;
  if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess &&
      cudaDeviceGetAttribute(&sm_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
      cudaDeviceGetAttribute(&regs_per_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) == cudaSuccess) {
    const int by_smem = (int)((size_t)sm_per_sm / (smem + fa.sharedSizeBytes + 1024));
    const int by_regs = fa.numRegs > 0 ? regs_per_sm / (fa.numRegs * threads) : by_smem;
    const int by_threads = 2048 / threads;
    const int est = by_smem < by_regs ? (by_smem < by_threads ? by_smem : by_threads)
                                      : (by_regs < by_threads ? by_regs : by_threads);
    if (est > per_sm) per_sm = est;
  } else {
    cudaGetLastError();
  }
  return per_sm;
}

// The tensor-core descriptor: definitions with alpha <= 8, l_max <= 8 and n_max
// <= 32 (the D tile's 32 columns).
bool descriptor_tc_fits(const DevParams &P) { return P.tc_descriptor && P.amax_t == 8 && P.n_max <= kTdCols; }
size_t descriptor_tc_smem(const DevParams &P) { return make_td_layout(P, 128, 8, 8).total; }

static cudaError_t run_descriptor_tc(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg, double *soap,
                                     float *keep_c, double *keep_norm, int keep) {
  const size_t sm = descriptor_tc_smem(P);
  auto kern = k_descriptor_tc<128, 8, 8>;
  cudaError_t e = ensure_smem_limit(kern, sm);
  if (e != cudaSuccess) return e;
  if (B.site_hi > B.site_lo) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int cap = sms * (512 / kTdTmemCols);
    const int grid = persistent_grid(kern, 128, sm, B.site_hi - B.site_lo,
                                     cfg.max_ctas > 0 ? (cfg.max_ctas < cap ? cfg.max_ctas : cap) : cap);
    kern<<<grid, 128, sm, cfg.stream>>>(P, B, soap, keep_c, keep_norm, keep);
  }
  return cudaGetLastError();
}

template <int NT, int AMAX, int LC>
static cudaError_t run_descriptor(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                                  double *soap, float *keep_c, double *keep_norm, int keep) {
  if (AMAX == 8 && LC == 8 && descriptor_tc_fits(P))
    return run_descriptor_tc(P, B, cfg, soap, keep_c, keep_norm, keep);
  const size_t sm = make_layout(P, NT, AMAX, LC, 0).total;
  auto kern = k_descriptor<NT, AMAX, LC>;
  cudaError_t e = ensure_smem_limit(kern, sm);
  if (e != cudaSuccess) return e;
  if (B.site_hi > B.site_lo) {
    const int grid = persistent_grid(kern, NT, sm, B.site_hi - B.site_lo, cfg.max_ctas);
    kern<<<grid, NT, sm, cfg.stream>>>(P, B, soap, keep_c, keep_norm, keep);
  }
  return cudaGetLastError();
}

// The tensor-core contract for the alpha <= 8, l_max <= 8 instantiation: a
// persistent grid of at most 4 CTAs per SM, so that the CTAs resident on an SM
// never ask for more than its 512 TMEM columns.
size_t contract_tc_smem(const DevParams &P) { return make_tc_layout(P, 128, 8).total; }

static cudaError_t run_contract_tc(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                                   const double *soap, const double *G, int g_layout, double sgn,
                                   const float *keep_c, const double *keep_norm, double *pair) {
  const size_t sm = contract_tc_smem(P);
  auto kern = k_contract_tc<128, 8, 8>;
  cudaError_t e = ensure_smem_limit(kern, sm);
  if (e != cudaSuccess) return e;
  if (B.site_hi > B.site_lo) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int cap = sms * (512 / kTcTmemCols);
    const int grid = persistent_grid(kern, 128, sm, B.site_hi - B.site_lo,
                                     cfg.max_ctas > 0 ? (cfg.max_ctas < cap ? cfg.max_ctas : cap) : cap);
    kern<<<grid, 128, sm, cfg.stream>>>(P, B, soap, G, g_layout, sgn, keep_c, keep_norm, pair);
  }
  return cudaGetLastError();
}

template <int NT, int AMAX, int LC>
static cudaError_t run_contract(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                                const double *soap, const double *G, int g_layout, double sgn,
                                const float *keep_c, const double *keep_norm, double *pair) {
  if (AMAX == 8 && LC == 8 && P.tc_contract)
    return run_contract_tc(P, B, cfg, soap, G, g_layout, sgn, keep_c, keep_norm, pair);
  const size_t sm = make_layout(P, NT, AMAX, LC, 1).total;
  auto kern = k_contract<NT, AMAX, LC>;
  cudaError_t e = ensure_smem_limit(kern, sm);
  if (e != cudaSuccess) return e;
  if (B.site_hi > B.site_lo) {
    const int grid = persistent_grid(kern, NT, sm, B.site_hi - B.site_lo, cfg.max_ctas);
    kern<<<grid, NT, sm, cfg.stream>>>(P, B, soap, G, g_layout, sgn, keep_c, keep_norm, pair);
  }
  return cudaGetLastError();
}

int prep_err_words(int n_sites) { return 3 + prep_scan_tiles(n_sites); }

unsigned long long prep_error_code(unsigned long long word) {
  return word == 0 ? ~0ull : kErrTop - word;
}

cudaError_t launch_prep(const DevParams &P, const DevBatch &B, cudaStream_t s) {
  const int tiles = prep_scan_tiles(B.n_sites);
  const int blocks = tiles + (B.n_pairs + kPrepThreads - 1) / kPrepThreads;
  if (blocks > 0) k_prep<<<blocks, kPrepThreads, 0, s>>>(B, P.n_species, tiles);
  return cudaGetLastError();
}

template <int AMAX, int LC, bool OP, bool TAB = false>
static cudaError_t run_pair(const DevParams &P, const DevBatch &B, cudaStream_t s, int do_der, int pair_lo,
                            int pair_hi, bool scan) {
  size_t sm = (size_t)P.off_rad + (size_t)P.n_species * SOAPB_RADSP_BYTES +
              (size_t)kPairThreads * pair_stage_stride(LC, TAB) * sizeof(float);
  // scan tiles reuse it: the tile's counts, then the site order's buckets
  if (sm < (kScanTile + kScanOrderBuckets) * sizeof(int)) sm = (kScanTile + kScanOrderBuckets) * sizeof(int);
  auto kern = k_pair<AMAX, LC, OP, TAB>;
  cudaError_t e = ensure_smem_limit(kern, sm);
  if (e != cudaSuccess) return e;
  const int tiles = scan ? prep_scan_tiles(B.n_sites) : 0;
  const int blocks = pair_cta_offset(B, tiles) + (pair_hi - pair_lo + kPairThreads - 1) / kPairThreads;
  if (blocks > 0) kern<<<blocks, kPairThreads, sm, s>>>(P, B, do_der, tiles, pair_lo, pair_hi);
  return cudaGetLastError();
}

cudaError_t launch_pair(const DevParams &P, const DevBatch &B, cudaStream_t s, int do_der, int pair_lo,
                        int pair_hi, bool scan) {
  if (pair_hi < 0) pair_hi = B.n_pairs;
  if (pair_lo < 0 || pair_lo > pair_hi || pair_hi > B.n_pairs) return cudaErrorInvalidValue;
  if (P.basis == kBasisOperator) {
    if (P.amax_t == 8) return run_pair<8, 8, true>(P, B, s, do_der, pair_lo, pair_hi, scan);
    return run_pair<16, 12, true>(P, B, s, do_der, pair_lo, pair_hi, scan);
  }
  if (P.rtab) {
    if (P.amax_t == 8) return run_pair<8, 8, false, true>(P, B, s, do_der, pair_lo, pair_hi, scan);
    return run_pair<16, 12, false, true>(P, B, s, do_der, pair_lo, pair_hi, scan);
  }
  if (P.amax_t == 8) return run_pair<8, 8, false>(P, B, s, do_der, pair_lo, pair_hi, scan);
  return run_pair<16, 12, false>(P, B, s, do_der, pair_lo, pair_hi, scan);
}

// The radial block is fixed by the definition: the host lays the constants
// blob out for amax_t (8 when every alpha <= 8 and l_max <= 8, else 16).  The
// CTA size (threads per site) is a launch choice: 64, 128 or 256.
#define SOAPB_DISPATCH_NT(FN, NT, ...)                    \
  do {                                                    \
    if (P.amax_t == 8) return FN<NT, 8, 8>(__VA_ARGS__);  \
    return FN<NT, 16, 12>(__VA_ARGS__);                   \
  } while (0)
#define SOAPB_DISPATCH(FN, ...)                                             \
  do {                                                                      \
    if (cfg.threads == 64) SOAPB_DISPATCH_NT(FN, 64, __VA_ARGS__);          \
    if (cfg.threads == 256) SOAPB_DISPATCH_NT(FN, 256, __VA_ARGS__);        \
    SOAPB_DISPATCH_NT(FN, 128, __VA_ARGS__);                                \
  } while (0)

cudaError_t launch_descriptor(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                              double *soap, float *keep_c, double *keep_norm, int keep) {
  SOAPB_DISPATCH(run_descriptor, P, B, cfg, soap, keep_c, keep_norm, keep);
}

cudaError_t launch_contract(const DevParams &P, const DevBatch &B, const LaunchCfg &cfg,
                            const double *soap, const double *G, int g_layout, double sgn,
                            const float *keep_c, const double *keep_norm, double *pair) {
  SOAPB_DISPATCH(run_contract, P, B, cfg, soap, G, g_layout, sgn, keep_c, keep_norm, pair);
}

size_t keep_floats_per_site(const DevParams &P) { return keep_stride(P); }

size_t descriptor_smem(const DevParams &P, int threads) {
  return make_layout(P, threads, P.amax_t, P.amax_t == 8 ? 8 : 12, 0).total;
}
size_t contract_smem(const DevParams &P, int threads) {
  return make_layout(P, threads, P.amax_t, P.amax_t == 8 ? 8 : 12, 1).total;
}

}  // namespace soapb
