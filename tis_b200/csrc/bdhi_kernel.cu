// bdhi_kernel.cu -- Brownian dynamics with hydrodynamic interactions
// (Ermak-McCammon, i_simulate_type = BROWNIAN_HI), batched over lanes of
// different sizes, FP64 (precision 1: Cholesky trailing updates on the
// tensor cores in split TF32).
//
// One step of time_integral.F90:429-457 for every lane:
//   [every n_step_hydro steps] D = RPY tensor at x (simu_hydro_tensors.F90:
//       139-182, HI_TENSOR%RPY), L = Cholesky factor of D (:304-324):
//       rpy_kernel, chol_diag_kernel (L_00), then per 64-wide panel k:
//       chol_panel_kernel (L_ik = A_ik L_kk^-T below the diagonal tile),
//       chol_update_kernel or chol_update_tc_kernel (A_ij -= L_ik L_jk^T for
//       the trailing tiles, FP64 or tensor cores; the CTA that finishes tile
//       (k + 1, k + 1) factors it for the next panel)
//   bd_noise_kernel     xi (counter-based or injected r_boxmuller)
//   bd_update_kernel    dx_k = tstep/kT (D F)_k + sqrt(2 tstep) (L xi)_k,
//                       x += dx (one warp per row, HBM-bound matrix-vector)
//   bd_force_kernel     F = FENE + WCA at the new x (force_fene.F90,
//                       force_wca.F90): one warp per bead gathers its records
//
// Matrices are row-major (3N x 3N) per lane at lane.bd0.  Sums run in a fixed
// order (warp butterflies, per-thread loops), so results do not depend on
// scheduling.  A pivot <= 0 sets the lane's not_spd flag (the reference stops
// with util_error); the factorisation continues with a unit pivot so that no
// NaN spreads, and the host reports TIS_E_NOT_SPD.
#include "device_common.cuh"

#include <algorithm>
#include <vector>

namespace tis {

constexpr int CT = 64;          // Cholesky tile
constexpr int CTP = CT + 1;     // padded shared-memory row

// ------------------------------------------------------------ RPY tensor
// The 3x3 block pre1 I + pre2 r r^T of the bead pair (i < j, r = x_j - x_i)
// in simu_hydro_tensors.F90:50-300, each variant's expressions in the
// reference's evaluation order with explicitly rounded operations (the FP64
// D is bit-identical to the reference's arithmetic).  diag_only: the block
// is val I (Zuk-RPY, one bead inside the other).
struct HiBlock { double pre1, pre2; bool diag_only; };

__device__ __forceinline__ HiBlock hi_pair(int type, double rad, double rad_i, double rad_j, double r_sq, double c6,
                                           double c8) {
  const double r_abs = sqrt(r_sq);
  HiBlock b{0.0, 0.0, false};
  auto rpy = [&](double rs) {   // rad_sq-sum form shared by RPY and Zuk-RPY apart
    b.pre1 = __dmul_rn(__ddiv_rn(c8, r_abs), __dadd_rn(1.0, __ddiv_rn(rs, __dmul_rn(3.0, r_sq))));
    b.pre2 = __ddiv_rn(__dmul_rn(__ddiv_rn(c8, r_abs), __dsub_rn(1.0, __ddiv_rn(rs, r_sq))), r_sq);
  };
  if (type == TIS_HI_ZUK_RPY_DEV) {
    if (__dadd_rn(rad_i, rad_j) < r_abs) {
      rpy(__dadd_rn(__dmul_rn(rad_i, rad_i), __dmul_rn(rad_j, rad_j)));
    } else {
      const double rad_s = rad_i < rad_j ? rad_i : rad_j, rad_l = rad_i < rad_j ? rad_j : rad_i;
      if (__dsub_rn(rad_l, rad_s) < r_abs) {
        const double r_cb = __dmul_rn(r_sq, r_abs);
        const double dr = __dsub_rn(rad_i, rad_j), dr2 = __dmul_rn(dr, dr);
        const double y1 = __dadd_rn(dr2, __dmul_rn(3.0, r_sq));
        const double x1 = __dsub_rn(__dmul_rn(__dmul_rn(16.0, r_cb), __dadd_rn(rad_i, rad_j)), __dmul_rn(y1, y1));
        const double cij = __ddiv_rn(__ddiv_rn(c6, rad_i), rad_j);
        b.pre1 = __ddiv_rn(__ddiv_rn(__dmul_rn(cij, x1), 32.0), r_cb);
        const double y2 = __dsub_rn(dr2, r_sq);
        b.pre2 = __ddiv_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(__dmul_rn(cij, 3.0), __dmul_rn(y2, y2)), 32.0), r_cb), r_sq);
      } else {
        b.pre1 = __ddiv_rn(c6, rad_l);
        b.diag_only = true;
      }
    }
    return b;
  }
  const double rad_sq = __dmul_rn(rad, rad);
  if (type == TIS_HI_RPY_DEV || __dmul_rn(2.0, rad) < r_abs) {
    rpy(__dmul_rn(2.0, rad_sq));
  } else if (type == TIS_HI_RPY_OVER_DEV) {
    b.pre1 = __dmul_rn(__ddiv_rn(c6, rad), __dsub_rn(1.0, __ddiv_rn(__dmul_rn(0.28125, r_abs), rad)));
    b.pre2 = __ddiv_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(__ddiv_rn(c6, rad), 3.0), 32.0), rad), r_abs);
  } else {   // ERMAK_OVER
    b.pre1 = __ddiv_rn(__dmul_rn(__ddiv_rn(__ddiv_rn(c8, 2.0), rad), 7.0), 6.0);
    b.pre2 = __ddiv_rn(__ddiv_rn(__ddiv_rn(c8, 2.0), 2.0), r_sq);
  }
  return b;
}

// grid (ceil(N*N / 256), nlane): thread per ordered bead pair (i, j); writes
// the 3x3 block of D and the lower part of L (L = tril(D) before factoring)
__global__ void __launch_bounds__(256) rpy_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc Tp = a.tops[L.top];
  const int N = Tp.nmp, n = 3 * N;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)N * N) return;
  const int i = (int)(e / N), j = (int)(e - (long long)i * N);
  const double T = a.lab_T[a.lstate[lane].label];
  const double c6 = a.boltz * T / (6.0 * a.pi * a.viscosity);
  const double c8 = a.boltz * T / (8.0 * a.pi * a.viscosity);
  const double *hr = a.b_hrad + Tp.bead0;
  const double rad = hr[0];   // radius(1) of RPY, RPY_OVER and ERMAK_OVER
  const int type = a.i_hydro_tensor;
  double blk[3][3];
  if (i == j) {
    const double dv = c6 / (type == TIS_HI_ZUK_RPY_DEV ? hr[i] : rad);
    for (int p = 0; p < 3; ++p)
      for (int q = 0; q < 3; ++q) blk[p][q] = (p == q) ? dv : 0.0;
  } else {
    // the reference fills i < j with r = x_j - x_i and mirrors the block;
    // the block is even in r, so both orders give the same numbers
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const double *x = a.xyz + 3 * (size_t)L.state0;
    double r[3];
    for (int d = 0; d < 3; ++d) r[d] = __dsub_rn(x[3 * hi + d], x[3 * lo + d]);
    const double r_sq = __dadd_rn(__dadd_rn(__dmul_rn(r[0], r[0]), __dmul_rn(r[1], r[1])), __dmul_rn(r[2], r[2]));
    const HiBlock hb = hi_pair(type, rad, hr[lo], hr[hi], r_sq, c6, c8);
    for (int p = 0; p < 3; ++p)
      for (int q = 0; q < 3; ++q) {
        if (hb.diag_only) blk[p][q] = (p == q) ? hb.pre1 : 0.0;
        else if (p == q) blk[p][q] = __dadd_rn(hb.pre1, __dmul_rn(__dmul_rn(hb.pre2, r[p]), r[q]));
        else blk[p][q] = __dmul_rn(__dmul_rn(hb.pre2, r[p]), r[q]);
      }
  }
  // D in FP64 (or FP32, rows padded to 4, for the mixed-precision step),
  // the lower part of L (its upper part is never read)
  double *Lm = a.bd_L + L.bd0;
  for (int p = 0; p < 3; ++p) {
    const size_t row = (size_t)(3 * i + p) * n + 3 * j;
    for (int q = 0; q < 3; ++q) {
      if (a.bd_tc) a.bd_D32[L.bd32 + (size_t)(3 * i + p) * ((n + 3) & ~3) + 3 * j + q] = (float)blk[p][q];
      else a.bd_D[L.bd0 + row + q] = blk[p][q];
      if (a.bd_refine) a.bd_D64[L.bd0 + row + q] = blk[p][q];
      if (3 * j + q <= 3 * i + p) Lm[row + q] = blk[p][q];
    }
  }
}

// ------------------------------------------------------------ Cholesky
__device__ __forceinline__ int lane_tiles(const KArgs &a, const LaneDesc &L, int &n) {
  n = 3 * a.tops[L.top].nmp;
  return (n + CT - 1) / CT;
}

// TF32 split of an FP64 value: hi keeps the top 10 mantissa bits of the
// FP32 rounding (round half up in magnitude), lo = the FP32 rest
__device__ __forceinline__ void tf32_split(double x, float &hi, float &lo) {
  const float xf = (float)x;
  hi = __uint_as_float((__float_as_uint(xf) + 0x1000u) & 0xFFFFE000u);
  lo = xf - hi;
}

// Panel operand planes for the tensor cores: per lane and panel parity
// (two slots: the wide update reads panels k and k + 1), (T + 1) tiles of
// 64 rows x 64 panel columns of TF32 hi parts, then as many of lo parts
// (tile T stays zero: the partner of an odd last row tile).  Inside a tile
// the layout is the K-major, no-swizzle canonical UMMA layout with 8-row
// groups outermost: float offset of (r, c) = (r / 8) 512 + (c / 4) 32 +
// (r % 8) 4 + c % 4, so consecutive row tiles form one operand of 128 rows.
constexpr int PT = CT * CT;   // floats per plane tile
// shared memory of the FP64 tile kernels: a padded tile and an unpadded one
constexpr int U64_SMEM = (CT * CTP + CT * CT) * (int)sizeof(double);

// Factor diagonal tile td of a lane and invert its factor with the 256
// threads of the calling group (tid 0..255, 8 warps; sync() is the group's
// barrier).  The tile A (identity beyond the matrix) sits in shared memory S
// (row stride CTP).  Blocked right-looking Cholesky in the unscaled form
// A_ic -= A_ij A_cj / p_j (p_j the pivot, L_ij = A_ij / sqrt(p_j)), 16
// columns per block:
//   warp 0 factors the block's columns for all rows below in registers (lane
//     l holds rows 16 b + l and 16 b + l + 32), column values passed by warp
//     shuffles, one pivot after the other;
//   all warps apply the block's rank-16 update to the trailing lower part.
// Then W = L^-1 by forward substitution L W = I, four threads per column of
// W (rows t, t + 4, ...), the solved element passed by shuffles.
// A pivot <= 0 is replaced by 1 (no NaN spreads) and flags the lane.  Stores
// L_tt (zero above the diagonal; FP32 copy for mixed precision) and, when a
// panel follows, U_tt = L_tt^-T into the lane's inverse slot.  vec holds
// 4 CT doubles.
template <typename Sync>
__device__ void factor_diag_tile(const KArgs &a, int lane, double *Lm, int n, int td, double *S, double *vec,
                                 int tid, Sync sync) {
  const long long L32 = a.lanes[lane].bd32;
  const int r0 = td * CT, nb = min(CT, n - r0);
  const int warp = tid >> 5, ln = tid & 31;
  double *A = S, *piv = vec, *ipv = vec + CT, *rinv = vec + 2 * CT;
  sync();   // the group's stores to the tile are visible; earlier users of S and vec are done
  {
    double v[CT * CT / 256];   // all loads in flight before the shared-memory stores
#pragma unroll
    for (int q = 0; q < CT * CT / 256; ++q) {
      const int e = tid + 256 * q, i = e >> 6, c = e & 63;
      v[q] = (i < nb && c < nb) ? Lm[(size_t)(r0 + i) * n + r0 + c] : (i == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int q = 0; q < CT * CT / 256; ++q) {
      const int e = tid + 256 * q;
      A[(e >> 6) * CTP + (e & 63)] = v[q];
    }
  }
  int bad = 0;   // warp 0
  for (int b = 0; b < CT / 16; ++b) {
    const int c0 = 16 * b;
    sync();
    if (warp == 0) {
      const int ra = c0 + ln, rb = c0 + ln + 32;
      double pa[16], pb[16];
#pragma unroll
      for (int cc = 0; cc < 16; ++cc) {
        pa[cc] = (ra < CT) ? A[ra * CTP + c0 + cc] : 0.0;
        pb[cc] = (rb < CT) ? A[rb * CTP + c0 + cc] : 0.0;
      }
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        double p = __shfl_sync(0xffffffffu, pa[jj], jj);   // A_jj: row c0 + jj is lane jj's first row
        if (!(p > 0.0)) {
          p = 1.0;
          bad = 1;
        }
        const double ip = 1.0 / p;
        if (ln == 0) {
          piv[c0 + jj] = p;
          ipv[c0 + jj] = ip;
        }
        double cv[16];   // A_{c0 + cc, j}, cc > jj
#pragma unroll
        for (int cc = jj + 1; cc < 16; ++cc) cv[cc] = __shfl_sync(0xffffffffu, pa[jj], cc);
        if (ln > jj && ra < CT) {
          const double m = pa[jj] * ip;
#pragma unroll
          for (int cc = jj + 1; cc < 16; ++cc)
            if (cc <= ln) pa[cc] -= m * cv[cc];
        }
        if (rb < CT) {
          const double m = pb[jj] * ip;
#pragma unroll
          for (int cc = jj + 1; cc < 16; ++cc) pb[cc] -= m * cv[cc];
        }
      }
#pragma unroll
      for (int cc = 0; cc < 16; ++cc) {
        if (ra < CT) A[ra * CTP + c0 + cc] = pa[cc];
        if (rb < CT) A[rb * CTP + c0 + cc] = pb[cc];
      }
    }
    sync();
    // rank-16 update of the trailing lower part: rows and columns >= c0 + 16;
    // thread (ty, tx) owns rows t0 + ty + 16 u and columns t0 + tx + 16 v
    // (u, v < 3), all of them accumulated side by side
    const int t0 = c0 + 16;
    if (t0 < CT) {
      const int tx = tid & 15, ty = tid >> 4;
      double acc[3][3];
#pragma unroll
      for (int u = 0; u < 3; ++u)
#pragma unroll
        for (int v = 0; v < 3; ++v) acc[u][v] = 0.0;
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        double ai[3], ac[3];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          const int i = min(t0 + ty + 16 * u, CT - 1), c = min(t0 + tx + 16 * u, CT - 1);
          ai[u] = A[i * CTP + c0 + jj];
          ac[u] = A[c * CTP + c0 + jj] * ipv[c0 + jj];
        }
#pragma unroll
        for (int u = 0; u < 3; ++u)
#pragma unroll
          for (int v = 0; v < 3; ++v) acc[u][v] += ai[u] * ac[v];
      }
#pragma unroll
      for (int u = 0; u < 3; ++u)
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          const int i = t0 + ty + 16 * u, c = t0 + tx + 16 * v;
          if (i < CT && c <= i) A[i * CTP + c] -= acc[u][v];
        }
    }
  }
  sync();
  if (tid < CT) {
    const double d = sqrt(piv[tid]);
    piv[tid] = d;
    rinv[tid] = 1.0 / d;
  }
  sync();
#pragma unroll
  for (int q = 0; q < CT * CT / 256; ++q) {
    const int e = tid + 256 * q, i = e >> 6, c = e & 63;
    const double l = (c < i) ? A[i * CTP + c] * rinv[c] : (c == i ? piv[c] : 0.0);
    A[i * CTP + c] = l;
    if (i < nb && c < nb) {
      Lm[(size_t)(r0 + i) * n + r0 + c] = l;
      if (a.bd_tc) a.bd_L32[L32 + (size_t)(r0 + i) * ((n + 3) & ~3) + r0 + c] = (float)l;
    }
  }
  if (tid == 0 && bad) atomicOr(&a.not_spd[lane], 1);
  if (r0 + CT < n) {   // a panel of rows below follows (then nb = CT)
    sync();
    // column c of W: thread t of the group of four owns rows t + 4 s
    const int c = tid >> 2, t = tid & 3, lead = ln & ~3;
    double w[16];
#pragma unroll
    for (int s2 = 0; s2 < 16; ++s2) w[s2] = (t + 4 * s2 == c) ? 1.0 : 0.0;
#pragma unroll
    for (int j = 0; j < CT; ++j) {
      double lj[16];   // column j of L for the rows of this thread, loaded off the chain
#pragma unroll
      for (int s2 = (j >> 2); s2 < 16; ++s2) lj[s2] = A[(t + 4 * s2) * CTP + j];
      double wj = 0.0;
      if (t == (j & 3)) {
        w[j >> 2] *= rinv[j];
        wj = w[j >> 2];
      }
      wj = __shfl_sync(0xffffffffu, wj, lead | (j & 3));   // zero while j < c
#pragma unroll
      for (int s2 = (j >> 2); s2 < 16; ++s2)
        if (t + 4 * s2 > j) w[s2] -= lj[s2] * wj;
    }
    double *wout = a.bd_W + (size_t)lane * CT * CT + (size_t)c * CT;   // U[c][i] = W[i][c]
#pragma unroll
    for (int s2 = 0; s2 < 16; ++s2) wout[t + 4 * s2] = w[s2];
  }
}

struct BlockSync {
  __device__ void operator()() const { __syncthreads(); }
};

// grid nlane, 256 threads: the diagonal tile of panel k of every lane.  On
// the tensor-core path the diagonal tile of a later panel is factored by the
// update launch that finishes it (the CTA that owns it), so only panel 0
// needs this launch; the FP64 path launches it for every panel.
__global__ void __launch_bounds__(256) chol_diag_kernel(KArgs a) {
  const int lane = blockIdx.x;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  int n;
  lane_tiles(a, L, n);
  __shared__ double S[CT * CTP], vec[5 * CT];
  if (a.bd_kpanel < lane_tiles(a, L, n)) factor_diag_tile(a, lane, a.bd_L + L.bd0, n, a.bd_kpanel, S, vec, threadIdx.x, BlockSync{});
}

// grid (T - k - 1, nlane), 256 threads: row tile ti = k + 1 + blockIdx.x of
// the panel below the factored diagonal tile: X = A_ik L_kk^-T as a 64 x 64
// x 64 FP64 product with the stored transposed inverse U_kk (thread (ty, tx)
// owns rows ty + 16 u, columns tx + 16 v; sums over m in increasing order),
// stored in FP64 and, for the tensor-core update, split into TF32 hi / lo
// in the panel planes.  Loads and stores are row-contiguous.
__global__ void __launch_bounds__(256) chol_panel_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  int n;
  const int T = lane_tiles(a, L, n), k = a.bd_kpanel;
  const int ti = k + 1 + blockIdx.x;
  if (ti >= T) return;   // rows below the diagonal tile: the panel is full (64 columns)
  const int r0 = k * CT, i0 = ti * CT, mi = min(CT, n - i0);
  double *Lm = a.bd_L + L.bd0;
  extern __shared__ double dsm[];   // U64_SMEM
  double *As = dsm, *Us = As + CT * CTP;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const double *w = a.bd_W + (size_t)lane * CT * CT;
#pragma unroll 4
  for (int e = tid; e < CT * CT; e += 256) {
    const int r = e >> 6, c = e & 63;
    As[r * CTP + c] = (r < mi) ? Lm[(size_t)(i0 + r) * n + r0 + c] : 0.0;
    Us[e] = w[e];
  }
  __syncthreads();
  double acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
#pragma unroll 4
  for (int m = 0; m < CT; ++m) {
    double av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) av[u] = As[(ty + 16 * u) * CTP + m];
#pragma unroll
    for (int v = 0; v < 4; ++v) bv[v] = Us[m * CT + tx + 16 * v];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) As[(ty + 16 * u) * CTP + tx + 16 * v] = acc[u][v];
  __syncthreads();
#pragma unroll 4
  for (int e = tid; e < CT * CT; e += 256) {
    const int r = e >> 6, c = e & 63;
    if (r < mi) {
      Lm[(size_t)(i0 + r) * n + r0 + c] = As[r * CTP + c];
      if (a.bd_tc) a.bd_L32[L.bd32 + (size_t)(i0 + r) * ((n + 3) & ~3) + r0 + c] = (float)As[r * CTP + c];
    }
  }
  if (a.bd_tc) {
    float *ph = a.bd_P + L.bdp0 + (size_t)(k & 1) * 2 * (T + 1) * PT + (size_t)ti * PT;
    float *pl = ph + (size_t)(T + 1) * PT;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q, r = e & 63, g = e >> 6;
      const double *x = As + r * CTP + 4 * g;
      float4 h, l;
      tf32_split(x[0], h.x, l.x);
      tf32_split(x[1], h.y, l.y);
      tf32_split(x[2], h.z, l.z);
      tf32_split(x[3], h.w, l.w);
      const int o = (r >> 3) * 512 + g * 32 + (r & 7) * 4;
      *(float4 *)(ph + o) = h;
      *(float4 *)(pl + o) = l;
    }
  }
}

// grid (nlane, pairs), 256 threads: trailing tile (ti, tj), k < tj <= ti:
// A_ij -= L_ik L_jk^T, a 64x64x64 FP64 product (4x4 outputs per thread)
__global__ void __launch_bounds__(256) chol_update_kernel(KArgs a) {
  const int lane = blockIdx.x;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  int n;
  const int T = lane_tiles(a, L, n), k = a.bd_kpanel;
  const int m = T - k - 1;
  const int p = blockIdx.y;
  if (m <= 0 || p >= m * (m + 1) / 2) return;
  int ii = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
  while (ii * (ii + 1) / 2 > p) --ii;
  while ((ii + 1) * (ii + 2) / 2 <= p) ++ii;
  const int jj = p - ii * (ii + 1) / 2;
  const int ti = k + 1 + ii, tj = k + 1 + jj;
  const int r0 = k * CT, nb = min(CT, n - r0);
  const int i0 = ti * CT, mi = min(CT, n - i0);
  const int j0 = tj * CT, mj = min(CT, n - j0);
  double *Lm = a.bd_L + L.bd0;
  extern __shared__ double sh[];
  double *As = sh, *Bs = sh + CT * CT;   // transposed: As[m][r], Bs[m][c]
  const int tid = threadIdx.x;
  for (int e = tid; e < CT * CT; e += blockDim.x) {
    const int r = e / CT, mm = e - r * CT;
    As[mm * CT + r] = (r < mi && mm < nb) ? Lm[(size_t)(i0 + r) * n + r0 + mm] : 0.0;
    Bs[mm * CT + r] = (r < mj && mm < nb) ? Lm[(size_t)(j0 + r) * n + r0 + mm] : 0.0;
  }
  __syncthreads();
  const int tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
  for (int mm = 0; mm < nb; ++mm) {
    const double2 a01 = *(const double2 *)&As[mm * CT + 4 * ty], a23 = *(const double2 *)&As[mm * CT + 4 * ty + 2];
    const double2 b01 = *(const double2 *)&Bs[mm * CT + 4 * tx], b23 = *(const double2 *)&Bs[mm * CT + 4 * tx + 2];
    const double av[4] = {a01.x, a01.y, a23.x, a23.y}, bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int r = 4 * ty + u;
    if (r >= mi) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int c = 4 * tx + v;
      if (c >= mj) continue;
      Lm[(size_t)(i0 + r) * n + j0 + c] -= acc[u][v];
    }
  }
}

// ------------------------------------------------------------ tensor cores
// Trailing updates on the 5th-generation tensor cores (mixed precision),
// two panels at a time.  For the panel pair (k, k + 1):
//   narrow: A_i,k+1 -= L_ik L_k+1,k^T for the column tile k + 1 (K = 64);
//   wide:   A_ij -= L_ik L_jk^T + L_i,k+1 L_j,k+1^T for j >= k + 2 (K = 128),
// so the FP64 trailing matrix is read and written once per two panels.
// L_ik = hi + lo is split into TF32 parts (the panel planes written by
// chol_panel_kernel, one slot per panel parity), the product taken as
// hi.hi + hi.lo + lo.hi (lo.lo is below FP32 rounding) and accumulated in
// FP32 in tensor memory; the FP64 tile subtracts it.  Diagonal tiles and
// panel solves stay in FP64.
//
// A CTA owns a 128-row block (row tiles ti, ti + 1) and up to UG column
// tiles of it, with one 64-column TMEM accumulator per column tile, and
// runs them as a pipeline of warp roles:
//   warp 0, one thread: bulk copies of the A block of each panel (the
//     second after the first panel's products are done) and of each B tile
//     (two shared-memory stages) from the panel planes;
//   warp 1, one thread: 24 tcgen05.mma (M 128, N 64, K 8) per column tile
//     and panel;
//   warps 2..9: epilogue, as soon as a tile's last panel is in: warp w
//     reads TMEM lanes 32 (w % 4) .. + 31 (rows) and column half (w - 2) / 4,
//     transposes the 32 x 32 block through its own shared-memory stage and
//     updates the FP64 rows with coalesced 256-byte accesses.
// The CTA whose first tile is the diagonal tile of the first updated column
// factors it afterwards (look-ahead for the next panel).  Every wait on a
// barrier is bounded; a wait that gives up flags the lane (not_spd bit 2,
// reported as a device-wait timeout) after the copies and products in
// flight are drained.
constexpr int UG = 8;                                 // column tiles per CTA (8 x 64 TMEM columns)
constexpr int U_A = 2 * 2 * CT * CT * 4;              // A hi + lo, 128 rows, one panel
constexpr int U_B = 2 * CT * CT * 4;                  // one B stage, hi + lo
constexpr int U_STG = 32 * 33 * 4;                    // epilogue transpose stage per warp
constexpr int U_SMEM = U_A + 2 * U_B + 8 * U_STG;
constexpr int U_THREADS = 320;
constexpr uint32_t U_WAIT_NS = 100000;                // suspend hint per poll
constexpr uint32_t U_WAIT_MAX = 20000;                // polls: about 2 s at most

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor: start >> 4 [0,14), LBO >> 4 [16,30),
// SBO >> 4 [32,46), version 1 [46,48), no swizzle (layout type 0 [61,64)).
// K-major without swizzle: LBO = byte step between the two K-adjacent core
// matrices of one K = 8 slice, SBO = byte step between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t it = 0; it < U_WAIT_MAX; ++it) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(parity), "r"(U_WAIT_NS)
                 : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// panel planes of panel kp of a lane: hi, then lo (T + 1 tiles each)
__device__ __forceinline__ const float *plane_hi(const KArgs &a, const LaneDesc &L, int T, int kp) {
  return a.bd_P + L.bdp0 + (size_t)(kp & 1) * 2 * (T + 1) * PT;
}

// One CTA per work item (lane << 16 | R << 8 | g) of the launch (bd_update_items):
// narrow (nph = 1): column tile k + 1 only, panel k; wide (nph = 2): column
// tiles >= k + 2, panels k and k + 1.  U_THREADS threads, one CTA per SM.
__global__ void __launch_bounds__(U_THREADS, 1) chol_update_tc_kernel(KArgs a, const int *items, int nph) {
  const int item = items[blockIdx.x];
  const int lane = item >> 16, R = (item >> 8) & 255, g = item & 255;
  const LaneDesc L = a.lanes[lane];
  int n;
  const int T = lane_tiles(a, L, n), k = a.bd_kpanel;
  const int cf = k + nph;   // first updated row and column tile
  const int m = T - cf;
  if (m <= 0 || 2 * R >= m) return;   // not produced by the item tables; uniform over the CTA
  const int ncol = nph == 1 ? 1 : min(2 * R + 2, m), c0 = g * UG;
  if (c0 >= ncol) return;
  const int nt = min(UG, ncol - c0);
  const int ti0 = cf + 2 * R, tj0 = cf + c0;
  double *Lm = a.bd_L + L.bd0;

  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)tsm + 1023) & ~(uintptr_t)1023);
  const uint32_t s_ahi = smem_u32(base), s_alo = s_ahi + U_A / 2;
  const uint32_t s_b0 = s_ahi + U_A;   // stage s: hi at s_b0 + s U_B, lo 16 KB later
  // fullA, fullB0/1, emptyB0/1, afree, mdone, tfull0..7
  __shared__ __align__(8) uint64_t bars[7 + UG];
  __shared__ uint32_t tmem_slot;
  __shared__ int gaveup;
  const uint32_t b_fullA = smem_u32(&bars[0]), b_fullB = smem_u32(&bars[1]), b_emptyB = smem_u32(&bars[3]);
  const uint32_t b_afree = smem_u32(&bars[5]), b_mdone = smem_u32(&bars[6]), b_tfull = smem_u32(&bars[7]);
  const int tid = threadIdx.x, warp = tid >> 5, lid = tid & 31;
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(UG * CT));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int q = 0; q < 7 + UG; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[q])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    gaveup = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = tmem_slot;

  if (warp == 0) {
    if (lid == 0) {
      bool ok = true;
      int last[2] = {-1, -1};
      for (int p = 0; p < nph && ok; ++p) {
        const float *ph = plane_hi(a, L, T, k + p), *pl = ph + (size_t)(T + 1) * PT;
        // the second panel's A block replaces the first once its products are done
        if (p == 1 && !mbar_wait(b_afree, 0)) { ok = false; break; }
        mbar_expect(b_fullA, U_A);
        bulk_load(s_ahi, ph + (size_t)ti0 * PT, U_A / 2, b_fullA);
        bulk_load(s_alo, pl + (size_t)ti0 * PT, U_A / 2, b_fullA);
        for (int t = 0; t < nt; ++t) {
          const int u = p * nt + t, s = u & 1;
          if (u >= 2 && !mbar_wait(b_emptyB + 8 * s, ((u >> 1) - 1) & 1)) { ok = false; break; }
          const uint32_t dst = s_b0 + (uint32_t)s * U_B;
          mbar_expect(b_fullB + 8 * s, U_B);
          bulk_load(dst, ph + (size_t)(tj0 + t) * PT, U_B / 2, b_fullB + 8 * s);
          bulk_load(dst + U_B / 2, pl + (size_t)(tj0 + t) * PT, U_B / 2, b_fullB + 8 * s);
          last[s] = u;
        }
      }
      // drain: no copy may still be writing shared memory when the CTA ends
      // (the last A load has phase parity nph - 1; the MMA thread waited
      // for the earlier one)
      ok = mbar_wait(b_fullA, (nph - 1) & 1) && ok;
      for (int s = 0; s < 2; ++s)
        if (last[s] >= 0) ok = mbar_wait(b_fullB + 8 * s, (last[s] >> 1) & 1) && ok;
      if (!ok) gaveup = 1;
    }
  } else if (warp == 1) {
    if (lid == 0) {
      // kind::tf32, D F32 [4,6) = 1, A TF32 [7,10) = 2, B TF32 [10,13) = 2,
      // both K-major, N >> 3 at [17,23), M >> 4 at [24,29)
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(CT >> 3) << 17) |
                             ((uint32_t)(2 * CT >> 4) << 24);
      bool ok = true;
      for (int p = 0; p < nph && ok; ++p) {
        if (!mbar_wait(b_fullA, p & 1)) { ok = false; break; }
        for (int t = 0; t < nt; ++t) {
          const int u = p * nt + t, s = u & 1;
          if (!mbar_wait(b_fullB + 8 * s, (u >> 1) & 1)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t bhi = s_b0 + (uint32_t)s * U_B, blo = bhi + U_B / 2;
          const uint32_t dacc = taddr + (uint32_t)(t * CT);
          for (int ks = 0; ks < CT / 8; ++ks) {
            for (int pp = 0; pp < 3; ++pp) {
              const uint32_t sa = (pp == 2 ? s_alo : s_ahi) + (uint32_t)ks * 256u;
              const uint32_t sb = (pp == 1 ? blo : bhi) + (uint32_t)ks * 256u;
              const uint64_t da = umma_desc(sa, 128, 2048), db = umma_desc(sb, 128, 2048);
              const uint32_t acc = (p | ks | pp) ? 1u : 0u;
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
                  :: "r"(dacc), "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
          }
          umma_commit(b_emptyB + 8 * s);
          if (p == nph - 1) umma_commit(b_tfull + 8 * t);
        }
        if (ok && p == 0 && nph > 1) umma_commit(b_afree);
      }
      // every product issued by this thread has landed before TMEM is freed
      umma_commit(b_mdone);
      ok = mbar_wait(b_mdone, 0) && ok;
      if (!ok) gaveup = 1;
    }
  } else {
    const int e = warp - 2, q = warp & 3, h = e >> 2;
    float *stg = (float *)(base + U_A + 2 * U_B + e * U_STG);
    uint32_t eok = 1;
    for (int t = 0; t < nt; ++t) {
      const bool ok = __all_sync(0xffffffffu, mbar_wait(b_tfull + 8 * t, 0));
      if (!ok) {
        if (lid == 0) gaveup = 1;
        eok = 0;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
            "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr + ((uint32_t)(q * 32) << 16) + (uint32_t)(t * CT + h * 32)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // lane = row of the TMEM block: transpose so that a lane owns a column
#pragma unroll
      for (int c = 0; c < 32; ++c) stg[lid * 33 + c] = __uint_as_float(v[c]);
      __syncwarp();
      const int tj = tj0 + t, col = tj * CT + h * 32 + lid;
      double old[32];
#pragma unroll
      for (int rr = 0; rr < 32; ++rr) {
        const int rw = q * 32 + rr, trow = ti0 + (rw >> 6), grow = trow * CT + (rw & 63);
        old[rr] = (grow < n && col < n && trow >= tj) ? Lm[(size_t)grow * n + col] : 0.0;
      }
#pragma unroll
      for (int rr = 0; rr < 32; ++rr) {
        const int rw = q * 32 + rr, trow = ti0 + (rw >> 6), grow = trow * CT + (rw & 63);
        if (grow < n && col < n && trow >= tj) Lm[(size_t)grow * n + col] = old[rr] - (double)stg[rr * 33 + lid];
      }
      __syncwarp();
    }
    if (R == 0 && g == 0) {
      // tile (cf, cf), updated above by this CTA, is final: the eight
      // epilogue warps factor it for the next panel (the operand area is
      // free: every product has been read out of TMEM)
      const auto esync = [] { asm volatile("bar.sync 1, 256;" ::: "memory"); };
      uint32_t all_ok;   // the same on all eight warps
      asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.and.pred p, 1, 256, q;\n\t"
                   "selp.u32 %0, 1, 0, p;\n\t}\n"
                   : "=r"(all_ok)
                   : "r"(eok)
                   : "memory");
      if (all_ok) {
        double *fs = (double *)base, *fv = fs + CT * CTP;
        factor_diag_tile(a, lane, Lm, n, cf, fs, fv, tid - 64, esync);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(UG * CT));
  }
  if (tid == 0 && gaveup) atomicOr(&a.not_spd[lane], 2);   // a tensor-core pipeline wait gave up
}

// ------------------------------------------------------------ step
// grid (ceil(maxN / 128), nlane): xi of every bead
__global__ void __launch_bounds__(128) bd_noise_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const int N = a.tops[L.top].nmp;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double n0, n1, n2;
  noise3(a, lane, L, i, a.bd_istep, a.noise_base, n0, n1, n2);
  double *xi = a.bd_xi + 3 * (size_t)(L.state0 + i);
  xi[0] = n0; xi[1] = n1; xi[2] = n2;
}

// grid (ceil(maxN * 3 / 8), nlane), 256 threads: one warp per row k of the
// lane: dx_k = rlan1 sum_c D_kc F_c + rlan2 sum_{c <= k} L_kc xi_c, x += dx.
// HBM-bound: the mixed-precision path streams FP32 copies of D and L
// (products and sums in FP64), the FP64 path the FP64 matrices.
__device__ __forceinline__ void row_dots64(const double *Drow, const double *Lrow, const double *F,
                                           const double *xi, int n, int k, int lid, double &df, double &dr) {
  df = 0.0;
  dr = 0.0;
  int c = lid;
  for (; c + 96 < n; c += 128)
    df += Drow[c] * F[c] + Drow[c + 32] * F[c + 32] + Drow[c + 64] * F[c + 64] + Drow[c + 96] * F[c + 96];
  for (; c < n; c += 32) df += Drow[c] * F[c];
  c = lid;
  for (; c + 96 <= k; c += 128)
    dr += Lrow[c] * xi[c] + Lrow[c + 32] * xi[c + 32] + Lrow[c + 64] * xi[c + 64] + Lrow[c + 96] * xi[c + 96];
  for (; c <= k; c += 32) dr += Lrow[c] * xi[c];
}

// FP32 rows padded to a multiple of 4 (16-byte aligned): float4 loads for
// the whole 4-column groups inside the matrix, then the < 4 last columns
__device__ __forceinline__ void row_dots32(const float *Drow, const float *Lrow, const double *F, const double *xi,
                                           int n, int k, int lid, double &df, double &dr) {
  df = 0.0;
  dr = 0.0;
  const float4 *D4 = (const float4 *)Drow, *L4 = (const float4 *)Lrow;
  const int n4 = n >> 2;
  // L is zero above the diagonal: whole groups up to column k
  const int k4 = min((k >> 2) + 1, n4);
  auto dot4 = [](const float4 &m, const double *v) {
    return (double)m.x * v[0] + (double)m.y * v[1] + (double)m.z * v[2] + (double)m.w * v[3];
  };
  int g = lid;
  for (; g + 96 < n4; g += 128) {   // four loads in flight per lane
    const float4 d0 = D4[g], d1 = D4[g + 32], d2 = D4[g + 64], d3 = D4[g + 96];
    df += dot4(d0, F + 4 * g) + dot4(d1, F + 4 * g + 128) + dot4(d2, F + 4 * g + 256) + dot4(d3, F + 4 * g + 384);
  }
  for (; g < n4; g += 32) df += dot4(D4[g], F + 4 * g);
  if (lid < n - 4 * n4) df += (double)Drow[4 * n4 + lid] * F[4 * n4 + lid];
  g = lid;
  for (; g + 96 < k4; g += 128) {
    const float4 l0 = L4[g], l1 = L4[g + 32], l2 = L4[g + 64], l3 = L4[g + 96];
    dr += dot4(l0, xi + 4 * g) + dot4(l1, xi + 4 * g + 128) + dot4(l2, xi + 4 * g + 256) + dot4(l3, xi + 4 * g + 384);
  }
  for (; g < k4; g += 32) dr += dot4(L4[g], xi + 4 * g);
  if (4 * k4 + lid <= k) dr += (double)Lrow[4 * k4 + lid] * xi[4 * k4 + lid];
}

__global__ void __launch_bounds__(256) bd_update_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const int n = 3 * a.tops[L.top].nmp;
  const int warp = threadIdx.x >> 5, lid = threadIdx.x & 31;
  const int k = blockIdx.x * 8 + warp;
  if (blockIdx.x == 0 && threadIdx.x == 0) a.lstate[lane].istep = a.bd_istep;
  if (k >= n) return;
  const double *F = a.bd_F + 3 * (size_t)L.state0, *xi = a.bd_xi + 3 * (size_t)L.state0;
  double df, dr;
  if (a.bd_tc) {
    const size_t row = L.bd32 + (size_t)k * ((n + 3) & ~3);
    row_dots32(a.bd_D32 + row, a.bd_L32 + row, F, xi, n, k, lid, df, dr);
    if (a.bd_refine) {   // - (E z)_k / 2
      const float4 *E4 = (const float4 *)(a.bd_E32 + row);
      const double *z = a.bd_z + 3 * (size_t)L.state0;
      const int n4 = n >> 2;
      double ez = 0.0;
      for (int g = lid; g < n4; g += 32) {
        const float4 e = E4[g];
        ez += (double)e.x * z[4 * g] + (double)e.y * z[4 * g + 1] + (double)e.z * z[4 * g + 2] + (double)e.w * z[4 * g + 3];
      }
      if (lid < n - 4 * n4) ez += (double)a.bd_E32[row + 4 * n4 + lid] * z[4 * n4 + lid];
      dr -= 0.5 * ez;
    }
  } else {
    const size_t row = L.bd0 + (size_t)k * n;
    row_dots64(a.bd_D + row, a.bd_L + row, F, xi, n, k, lid, df, dr);
  }
  for (int o = 16; o > 0; o >>= 1) {
    df += __shfl_xor_sync(0xffffffffu, df, o);
    dr += __shfl_xor_sync(0xffffffffu, dr, o);
  }
  if (lid == 0) {
    const double T = a.lab_T[a.lstate[lane].label];
    const double rl1 = a.tstep / (a.boltz * T), rl2 = sqrt(2.0 * a.tstep);
    const double dx = rl1 * df + rl2 * dr;
    const size_t o = 3 * (size_t)L.state0 + k;
    a.xyz[o] += dx;
    a.pxyz[o] += dx;
    a.dxyz[o] += dx;
  }
}

// ------------------------------------------------------------ refinement
// The mixed-precision step samples L xi with the FP32 factor L, whose
// L L^T = D + E differs from D by the rounding of the split-TF32 updates and
// of the FP32 copy (|E| ~ 1e-7 |D|).  M = L - E L^-T / 2 has
// M M^T = D + E L^-T L^-1 E / 4, so the step samples M xi = L xi - E z / 2
// with z = L^-T xi.  E is formed at each refresh with FP64 sums; z and E z
// are FP32 data with FP64 sums (errors of order 1e-7 of a 1e-7 correction).
constexpr int RT = 64;
constexpr int RT_SMEM = 2 * RT * (RT + 1) * (int)sizeof(double);

// grid (Tmax (Tmax + 1) / 2, nlane), 256 threads: tile (I, J), I >= J, of
// E = L L^T - D in FP64, written to both halves of the FP32 E
__global__ void __launch_bounds__(256) refine_residual_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const int n = 3 * a.tops[L.top].nmp, T = (n + RT - 1) / RT, ld = (n + 3) & ~3;
  const int p = blockIdx.x;
  if (p >= T * (T + 1) / 2) return;
  int I = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= p) ++I;
  while (I * (I + 1) / 2 > p) --I;
  const int J = p - I * (I + 1) / 2;
  extern __shared__ double rsm[];
  double *As = rsm, *Bs = rsm + RT * (RT + 1);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int w = 0; w < 4; ++w) acc[q][w] = 0.0;
  const float *Lm = a.bd_L32 + L.bd32;
  for (int K = 0; K <= J; ++K) {   // L_IK L_JK^T; L is zero above its diagonal
    for (int e = threadIdx.x; e < RT * RT; e += 256) {
      const int r = e / RT, c = e - r * RT, gc = K * RT + c, ra = I * RT + r, rb = J * RT + r;
      As[r * (RT + 1) + c] = (ra < n && gc < n) ? (double)Lm[(size_t)ra * ld + gc] : 0.0;
      Bs[r * (RT + 1) + c] = (rb < n && gc < n) ? (double)Lm[(size_t)rb * ld + gc] : 0.0;
    }
    __syncthreads();
    // thread (ty, tx): rows ty * 4 + q, columns tx + 16 w (consecutive tx
    // read rows 65 doubles apart: no shared-memory bank conflicts)
    for (int k = 0; k < RT; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) { av[q] = As[(ty * 4 + q) * (RT + 1) + k]; bv[q] = Bs[(tx + 16 * q) * (RT + 1) + k]; }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int w = 0; w < 4; ++w) acc[q][w] = fma(av[q], bv[w], acc[q][w]);
    }
    __syncthreads();
  }
  const double *D = a.bd_D64 + L.bd0;
  float *E = a.bd_E32 + L.bd32;
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const int row = I * RT + ty * 4 + q, col = J * RT + tx + 16 * w;
      if (row < n && col < n) {
        const float e = (float)(acc[q][w] - D[(size_t)row * n + col]);
        E[(size_t)row * ld + col] = e;
        if (I != J) E[(size_t)col * ld + row] = e;
      }
    }
}

// grid (Tmax, nlane), 64 threads: W_b = inverse of the diagonal tile L_bb of
// the FP32 factor (FP64 forward substitution, one column per thread; rows
// past n act as the identity)
__global__ void __launch_bounds__(64) refine_inverse_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const int n = 3 * a.tops[L.top].nmp, T = (n + RT - 1) / RT, ld = (n + 3) & ~3;
  const int b = blockIdx.x;
  if (b >= T) return;
  extern __shared__ double inv_buf[];   // L_bb, then its inverse (RT_SMEM bytes)
  double *Lt = inv_buf, *X = inv_buf + RT * (RT + 1);
  const float *Lm = a.bd_L32 + L.bd32;
  const int c = threadIdx.x;
  for (int r = 0; r < RT; ++r) {
    const int gr = b * RT + r, gc = b * RT + c;
    Lt[r * (RT + 1) + c] = (gr < n && gc < n) ? (double)Lm[(size_t)gr * ld + gc] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
  for (int i = 0; i < RT; ++i) {
    double x = 0.0;
    if (i >= c) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) s -= Lt[i * (RT + 1) + k] * X[k * (RT + 1) + c];
      x = s / Lt[i * (RT + 1) + i];
    }
    X[i * (RT + 1) + c] = x;
  }
  float *W = a.bd_W32 + L.bdw0 + (size_t)b * RT * RT;
  for (int i = 0; i < RT; ++i) W[i * RT + c] = (float)X[i * (RT + 1) + c];
}

// grid nlane, 1024 threads: z = L^-T xi by blocked back substitution from
// the last tile: rhs_b = xi_b - sum over the rows below of L^T z, then
// z_b = W_b^T rhs_b
constexpr int TRSV_THREADS = 1024;
__global__ void __launch_bounds__(TRSV_THREADS) refine_trsv_kernel(KArgs a) {
  const int lane = blockIdx.x;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const int n = 3 * a.tops[L.top].nmp, T = (n + RT - 1) / RT, ld = (n + 3) & ~3;
  extern __shared__ double trsm_buf[];
  double *zs = trsm_buf;                         // n
  double *part = trsm_buf + ((n + 1) & ~1);      // 16 x 64
  double *rhs = part + 16 * RT;             // 64
  const float *Lm = a.bd_L32 + L.bd32;
  const double *xi = a.bd_xi + 3 * (size_t)L.state0;
  const int c = threadIdx.x & (RT - 1), g = threadIdx.x >> 6;
  for (int b = T - 1; b >= 0; --b) {
    const int j = b * RT + c;
    double sacc = 0.0;
    if (j < n)
      for (int r = (b + 1) * RT + g; r < n; r += 16) sacc += (double)Lm[(size_t)r * ld + j] * zs[r];
    part[g * RT + c] = sacc;
    __syncthreads();
    if (threadIdx.x < RT) {
      double t = 0.0;
      for (int q = 0; q < 16; ++q) t += part[q * RT + c];
      rhs[c] = (j < n) ? xi[j] - t : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < RT) {
      const float *W = a.bd_W32 + L.bdw0 + (size_t)b * RT * RT;
      double z = 0.0;
      for (int i = c; i < RT; ++i) z += (double)W[i * RT + c] * rhs[i];
      if (j < n) zs[j] = z;
    }
    __syncthreads();
  }
  double *zo = a.bd_z + 3 * (size_t)L.state0;
  for (int k = threadIdx.x; k < n; k += TRSV_THREADS) zo[k] = zs[k];
}

// grid (ceil(maxN / 8), nlane), 256 threads: one warp per bead sums its FENE
// and WCA records (force_fene.F90, force_wca.F90) in record order
__global__ void __launch_bounds__(256) bd_force_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int warp = threadIdx.x >> 5, lid = threadIdx.x & 31;
  const int i = blockIdx.x * 8 + warp;
  if (i >= T.nmp) return;
  const double *x = a.xyz + 3 * (size_t)L.state0;
  const int p0 = a.bd_ptr[T.bp0 + i], p1 = a.bd_ptr[T.bp0 + i + 1];
  const double xi0 = x[3 * i], xi1 = x[3 * i + 1], xi2 = x[3 * i + 2];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  int nclamp = 0;
  // entry (j, class * 2 + kind): the record's force on i is f (x_i - x_j),
  // the same numbers as -/+ f (x_i2 - x_i1) in the record's own orientation
  for (int p = p0 + lid; p < p1; p += 32) {
    const int2 ent = a.bd_ent[T.be0 + p];
    const int j = ent.x, cl = ent.y >> 1;
    const double v0 = xi0 - x[3 * j], v1 = xi1 - x[3 * j + 1], v2 = xi2 - x[3 * j + 2];
    double f;
    if (!(ent.y & 1)) {
      const double *pc = a.fene_cls + 3 * (size_t)cl;   // nat, coef, dist2
      const double dist = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
      const double dd = dist - pc[0];
      f = -pc[1] * dd / (1.0 - dd * dd / pc[2]) / dist;
    } else {
      const double *pc = a.wca_cls + 3 * (size_t)cl;    // nat, coef rep, coef att
      const double dist2 = v0 * v0 + v1 * v1 + v2 * v2;
      const double nat2 = pc[0] * pc[0];
      const double ro2 = nat2 / dist2;
      if (ro2 < a.wca_rcut2) continue;
      const double ro4 = ro2 * ro2, ro8 = ro4 * ro4, ro14 = ro8 * ro4 * ro2;
      const double coef = (ro2 > 1.0) ? pc[1] : pc[2];
      f = 12.0 * coef / nat2 * (ro14 - ro8);
      if (f > 50.0) { f = 50.0; nclamp += j > i; }   // DE_MAX; the record is counted once, from its lower bead
    }
    fx += f * v0; fy += f * v1; fz += f * v2;
  }
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
    nclamp += __shfl_xor_sync(0xffffffffu, nclamp, o);
  }
  if (lid == 0) {
    double *F = a.bd_F + 3 * (size_t)(L.state0 + i);
    F[0] = fx; F[1] = fy; F[2] = fz;
    if (nclamp) atomicAdd((unsigned long long *)&a.lstate[lane].nclamp, (unsigned long long)nclamp);
  }
}

// ------------------------------------------------------------ launches
// Work items of the tensor-core updates (lane << 16 | R << 8 | g): for the
// panel pair starting at k (k even) the narrow launch's items are
// items[koff[k] .. koff[k + 1]) and the wide launch's items[koff[k + 1] ..
// koff[k + 2]).  Items that factor the next diagonal tile come first, the
// rest by decreasing tile count.  lane_T = tiles per lane.
void bd_update_items(const std::vector<int> &lane_T, std::vector<int> &items, std::vector<int> &koff) {
  int tmax = 0;
  for (int t : lane_T) tmax = std::max(tmax, t);
  items.clear();
  koff.assign(1, 0);
  for (int k = 0; k < tmax + 1; ++k) {
    const int nph = (k & 1) ? 2 : 1;   // odd entries: the wide launch of the pair starting at k - 1
    const int kp = k & ~1;
    std::vector<std::pair<int, int>> ks;   // (order key, item)
    for (size_t l = 0; l < lane_T.size(); ++l) {
      const int m = lane_T[l] - kp - nph;
      for (int R = 0; 2 * R < m; ++R) {
        const int ncol = nph == 1 ? 1 : std::min(2 * R + 2, m);
        for (int g = 0; g * UG < ncol; ++g) {
          const int nt = std::min(UG, ncol - g * UG);
          const int first = (R == 0 && g == 0) ? 1 << 20 : 0;   // factors the next diagonal tile
          ks.push_back({first + nt, (int)(l << 16) | (R << 8) | g});
        }
      }
    }
    std::stable_sort(ks.begin(), ks.end(), [](const std::pair<int, int> &x, const std::pair<int, int> &y) {
      return x.first > y.first;
    });
    for (auto &e : ks) items.push_back(e.second);
    koff.push_back((int)items.size());
  }
}

cudaError_t bd_refactor_launch(cudaStream_t st, KArgs a, int max_nmp, const int *items, const int *koff) {
  cudaError_t e = cudaFuncSetAttribute(chol_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       U64_SMEM);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(chol_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, U64_SMEM);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(chol_update_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, U_SMEM + 1024);
  if (e != cudaSuccess) return e;
  if (a.bd_tc && (!a.bd_P || !items || !koff)) return cudaErrorInvalidValue;
  const long long nn = (long long)max_nmp * max_nmp;
  rpy_kernel<<<dim3((unsigned)((nn + 255) / 256), a.nlane), 256, 0, st>>>(a);
  a.bd_kpanel = 0;
  chol_diag_kernel<<<a.nlane, 256, 0, st>>>(a);
  const int T = (3 * max_nmp + CT - 1) / CT;
  if (a.bd_tc) {
    // panel pairs: panel k, narrow update (column k + 1), panel k + 1, wide update
    for (int k = 0; k + 1 < T; k += 2) {
      a.bd_kpanel = k;
      chol_panel_kernel<<<dim3(T - k - 1, a.nlane), 256, U64_SMEM, st>>>(a);
      int nit = koff[k + 1] - koff[k];
      if (nit > 0) chol_update_tc_kernel<<<nit, U_THREADS, U_SMEM + 1024, st>>>(a, items + koff[k], 1);
      if (k + 2 < T) {
        KArgs b = a;
        b.bd_kpanel = k + 1;
        chol_panel_kernel<<<dim3(T - k - 2, a.nlane), 256, U64_SMEM, st>>>(b);
        nit = koff[k + 2] - koff[k + 1];
        if (nit > 0) chol_update_tc_kernel<<<nit, U_THREADS, U_SMEM + 1024, st>>>(a, items + koff[k + 1], 2);
      }
    }
  } else {
    for (int k = 0; k + 1 < T; ++k) {
      a.bd_kpanel = k;
      const int m = T - k - 1;
      if (k > 0) chol_diag_kernel<<<a.nlane, 256, 0, st>>>(a);
      chol_panel_kernel<<<dim3(m, a.nlane), 256, U64_SMEM, st>>>(a);
      chol_update_kernel<<<dim3(a.nlane, m * (m + 1) / 2), 256, U64_SMEM, st>>>(a);
    }
    // the last diagonal tile
    a.bd_kpanel = T - 1;
    if (T > 1) chol_diag_kernel<<<a.nlane, 256, 0, st>>>(a);
  }
  if (a.bd_refine) {
    e = cudaFuncSetAttribute(refine_residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, RT_SMEM);
    if (e != cudaSuccess) return e;
    const int TR = (3 * max_nmp + RT - 1) / RT;
    refine_residual_kernel<<<dim3(TR * (TR + 1) / 2, a.nlane), 256, RT_SMEM, st>>>(a);
    e = cudaFuncSetAttribute(refine_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, RT_SMEM);
    if (e != cudaSuccess) return e;
    refine_inverse_kernel<<<dim3(TR, a.nlane), RT, RT_SMEM, st>>>(a);
  }
  return cudaGetLastError();
}

int bd_refactor_launches(int max_nmp, bool tc) {
  const int T = (3 * max_nmp + CT - 1) / CT;
  if (!tc) return 2 + 3 * (T - 1);
  int nl = 2;
  for (int k = 0; k + 1 < T; k += 2) nl += (k + 2 < T) ? 4 : 2;
  return nl;
}

// floats of the panel planes of a lane with N beads (tensor-core update)
long long bd_plane_floats(int nmp) {
  const int T = (3 * nmp + CT - 1) / CT;
  return 2LL * 2 * (T + 1) * PT;   // two panel slots of hi + lo planes
}

cudaError_t bd_step_launch(cudaStream_t st, const KArgs &a, int max_nmp) {
  bd_noise_kernel<<<dim3((max_nmp + 127) / 128, a.nlane), 128, 0, st>>>(a);
  if (a.bd_refine) {
    const size_t sm = (size_t)((3 * max_nmp + 1) & ~1) * sizeof(double) + (16 * RT + RT) * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(refine_trsv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    refine_trsv_kernel<<<a.nlane, TRSV_THREADS, sm, st>>>(a);
  }
  bd_update_kernel<<<dim3((3 * max_nmp + 7) / 8, a.nlane), 256, 0, st>>>(a);
  bd_force_kernel<<<dim3((max_nmp + 7) / 8, a.nlane), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t bd_force_launch(cudaStream_t st, const KArgs &a, int max_nmp) {
  bd_force_kernel<<<dim3((max_nmp + 7) / 8, a.nlane), 256, 0, st>>>(a);
  return cudaGetLastError();
}

} // namespace tis
