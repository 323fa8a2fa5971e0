// bdhi_kernel.cu -- Brownian dynamics with hydrodynamic interactions
// (Ermak-McCammon, i_simulate_type = BROWNIAN_HI), batched over lanes of
// different sizes, FP64.
//
// One step of time_integral.F90:429-457 for every lane:
//   [every n_step_hydro steps] D = RPY tensor at x (simu_hydro_tensors.F90:
//       139-182, HI_TENSOR%RPY), L = Cholesky factor of D (:304-324):
//       rpy_kernel, then per 64-wide panel k: chol_diag_kernel (factor the
//       diagonal tile), chol_panel_kernel (L_ik = A_ik L_kk^-T below it),
//       chol_update_kernel (A_ij -= L_ik L_jk^T for the trailing tiles)
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

namespace tis {

constexpr int CT = 64;          // Cholesky tile
constexpr int CTP = CT + 1;     // padded shared-memory row

// ------------------------------------------------------------ RPY tensor
// grid (ceil(N*N / 256), nlane): thread per ordered bead pair (i, j); writes
// the 3x3 block of D and the lower part of L (L = tril(D) before factoring)
__global__ void __launch_bounds__(256) rpy_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const int N = a.tops[L.top].nmp, n = 3 * N;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)N * N) return;
  const int i = (int)(e / N), j = (int)(e - (long long)i * N);
  const double T = a.lab_T[a.lstate[lane].label];
  const double c6 = a.boltz * T / (6.0 * a.pi * a.viscosity);
  const double c8 = a.boltz * T / (8.0 * a.pi * a.viscosity);
  const double rad = a.hi_radius;
  double blk[3][3];
  if (i == j) {
    for (int p = 0; p < 3; ++p)
      for (int q = 0; q < 3; ++q) blk[p][q] = (p == q) ? c6 / rad : 0.0;
  } else {
    // the reference fills i < j with r = x_j - x_i and mirrors the block;
    // the block is even in r, so both orders give the same numbers
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const double *x = a.xyz + 3 * (size_t)L.state0;
    double r[3];
    for (int d = 0; d < 3; ++d) r[d] = x[3 * hi + d] - x[3 * lo + d];
    const double r_sq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double r_abs = sqrt(r_sq);
    const double rad_sq = rad * rad;
    const double pre1 = c8 / r_abs * (1.0 + 2.0 * rad_sq / (3.0 * r_sq));
    const double pre2 = c8 / r_abs * (1.0 - 2.0 * rad_sq / r_sq) / r_sq;
    for (int p = 0; p < 3; ++p)
      for (int q = 0; q < 3; ++q) blk[p][q] = (p == q ? pre1 : 0.0) + pre2 * r[p] * r[q];
  }
  double *D = a.bd_D + L.bd0, *Lm = a.bd_L + L.bd0;
  for (int p = 0; p < 3; ++p) {
    const size_t row = (size_t)(3 * i + p) * n + 3 * j;
    for (int q = 0; q < 3; ++q) {
      D[row + q] = blk[p][q];
      Lm[row + q] = (3 * j + q <= 3 * i + p) ? blk[p][q] : 0.0;
    }
  }
}

// ------------------------------------------------------------ Cholesky
__device__ __forceinline__ int lane_tiles(const KArgs &a, const LaneDesc &L, int &n) {
  n = 3 * a.tops[L.top].nmp;
  return (n + CT - 1) / CT;
}

// grid nlane, 256 threads (16 x 16): factor the diagonal tile of panel k in
// place; thread (ty, tx) owns rows ty + 16 a and columns tx + 16 b of the tile
__global__ void __launch_bounds__(256) chol_diag_kernel(KArgs a) {
  const int lane = blockIdx.x;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  int n;
  const int T = lane_tiles(a, L, n), k = a.bd_kpanel;
  if (k >= T) return;
  const int r0 = k * CT, nb = min(CT, n - r0);
  double *Lm = a.bd_L + L.bd0;
  __shared__ double A[CT * CTP];
  __shared__ int bad;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  if (tid == 0) bad = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = ty + 16 * u, c = tx + 16 * v;
      A[i * CTP + c] = (i < nb && c < nb) ? Lm[(size_t)(r0 + i) * n + r0 + c] : (i == c ? 1.0 : 0.0);
    }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    if (tid == 0) {
      double d = A[j * CTP + j];
      if (!(d > 0.0)) { bad = 1; d = 1.0; }
      A[j * CTP + j] = sqrt(d);
    }
    __syncthreads();
    if (tid < CT && tid > j) A[tid * CTP + j] /= A[j * CTP + j];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = ty + 16 * u;
      if (i <= j) continue;
      const double lij = A[i * CTP + j];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int c = tx + 16 * v;
        if (c > j && c <= i) A[i * CTP + c] -= lij * A[c * CTP + j];
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = ty + 16 * u, c = tx + 16 * v;
      if (i < nb && c < nb) Lm[(size_t)(r0 + i) * n + r0 + c] = (c <= i) ? A[i * CTP + c] : 0.0;
    }
  if (tid == 0 && bad) atomicOr(&a.not_spd[lane], 1);
}

// grid (tiles - 1, nlane), 256 threads: tile row i = k + 1 + blockIdx.x of
// panel k: solve X L_kk^T = A_ik by forward substitution; four threads per
// row split each dot product (fixed order: strided partials, butterfly)
__global__ void __launch_bounds__(256) chol_panel_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  int n;
  const int T = lane_tiles(a, L, n), k = a.bd_kpanel;
  const int ti = k + 1 + blockIdx.x;
  if (ti >= T) return;
  const int r0 = k * CT, nb = min(CT, n - r0);
  const int i0 = ti * CT, mb = min(CT, n - i0);
  double *Lm = a.bd_L + L.bd0;
  extern __shared__ double shp[];
  double *Lk = shp, *X = shp + CT * CTP;
  const int tid = threadIdx.x, tx = tid & 63, ty = tid >> 6;   // 4 rows of 64 per pass
#pragma unroll 4
  for (int i = ty; i < CT; i += 4) {
    Lk[i * CTP + tx] = (i < nb && tx < nb) ? Lm[(size_t)(r0 + i) * n + r0 + tx] : (i == tx ? 1.0 : 0.0);
    X[i * CTP + tx] = (i < mb && tx < nb) ? Lm[(size_t)(i0 + i) * n + r0 + tx] : 0.0;
  }
  __syncthreads();
  const int row = tid >> 2, part = tid & 3;
  double *x = X + row * CTP;
  for (int c = 0; c < CT; ++c) {
    double p = 0.0;
    for (int m = part; m < c; m += 4) p += x[m] * Lk[c * CTP + m];
    p += __shfl_xor_sync(0xffffffffu, p, 1);
    p += __shfl_xor_sync(0xffffffffu, p, 2);
    if (part == 0) x[c] = (x[c] - p) / Lk[c * CTP + c];
    __syncwarp();
  }
  __syncthreads();
#pragma unroll 4
  for (int i = ty; i < mb; i += 4)
    if (tx < nb) Lm[(size_t)(i0 + i) * n + r0 + tx] = X[i * CTP + tx];
}

// grid (pairs, nlane), 256 threads: trailing tile (ti, tj), k < tj <= ti:
// A_ij -= L_ik L_jk^T, a 64x64x64 FP64 product (4x4 outputs per thread)
__global__ void __launch_bounds__(256) chol_update_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  int n;
  const int T = lane_tiles(a, L, n), k = a.bd_kpanel;
  const int m = T - k - 1;
  const int p = blockIdx.x;
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
// Trailing update on the 5th-generation tensor cores (mixed precision):
// A_ij -= L_ik L_jk^T for a 128 x 64 output block (row tiles ti, ti + 1 of
// panel k, column tile tj) per CTA.  Each FP64 operand x is split into TF32
// parts x = hi + lo (hi keeps the top 10 mantissa bits), and the product is
// hi.hi + hi.lo + lo.hi (the lo.lo term is below FP32 rounding), accumulated
// in FP32 in tensor memory by 24 tcgen05.mma (M = 128, N = 64, K = 8) issued
// by one thread.  Diagonal tiles and panel solves stay in FP64.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, rows 16 B apart, 8-row groups SBO = 128 B
// apart, 4-element K chunks LBO apart (A: 16 groups -> 2048 B; B: 8 -> 1024 B).
constexpr int TC_M = 128, TC_N = 64, TC_K = 64;
constexpr int TC_SMEM = 2 * TC_M * TC_K * 4 + 2 * TC_N * TC_K * 4;   // A hi/lo, B hi/lo (FP32)
constexpr uint32_t TC_WAIT_MAX = 1u << 24;                           // polls of the completion barrier

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor: start >> 4 [0,14), LBO >> 4 [16,30),
// SBO >> 4 [32,46), version 1 [46,48), no swizzle (layout type 0 [61,64))
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// byte offset of element (r, k) in a K-major, no-swizzle tile of `rows` rows
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int rows) {
  return (uint32_t)(((k >> 2) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ void tf32_split(double x, float &hi, float &lo) {
  const float xf = (float)x;
  hi = __uint_as_float((__float_as_uint(xf) + 0x1000u) & 0xFFFFE000u);
  lo = xf - hi;
}

// grid (ceil(m_max / 2) * m_max, nlane), 128 threads (4 warps; warp w owns
// TMEM lanes / output rows 32 w .. 32 w + 31)
__global__ void __launch_bounds__(128) chol_update_tc_kernel(KArgs a, int m_max) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  int n;
  const int T = lane_tiles(a, L, n), k = a.bd_kpanel;
  const int m = T - k - 1;
  const int R = blockIdx.x / m_max, tjr = blockIdx.x - R * m_max;
  if (m <= 0 || 2 * R >= m || tjr >= m || tjr > 2 * R + 1) return;   // uniform over the CTA
  const int ti0 = k + 1 + 2 * R, tj = k + 1 + tjr;
  const int r0 = k * CT, nb = min(CT, n - r0);
  const int j0 = tj * CT, mj = min(CT, n - j0);
  double *Lm = a.bd_L + L.bd0;
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)tsm + 1023) & ~(uintptr_t)1023);
  unsigned char *Ahi = base, *Alo = base + TC_M * TC_K * 4;
  unsigned char *Bhi = Alo + TC_M * TC_K * 4, *Blo = Bhi + TC_N * TC_K * 4;
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(8) uint64_t mbar;
  const int tid = threadIdx.x, warp = tid >> 5, lid = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TC_N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  // operands: rows of tile ti0 then ti0 + 1 (zero past the matrix), columns
  // of panel k; each pass of the block reads 4 rows x 64 columns (coalesced),
  // all loads of a thread in flight before the conversions
  {
    const int kk = tid & 63, rq = tid >> 6;   // 0..1 with 128 threads
    double va[TC_M / 2], vb[TC_N / 2];
#pragma unroll
    for (int u = 0; u < TC_M / 2; ++u) {
      const int r = rq + 2 * u;
      const int grow = (ti0 + (r >> 6)) * CT + (r & 63);
      va[u] = (grow < n && kk < nb) ? Lm[(size_t)grow * n + r0 + kk] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < TC_N / 2; ++u) {
      const int r = rq + 2 * u;
      vb[u] = (r < mj && kk < nb) ? Lm[(size_t)(j0 + r) * n + r0 + kk] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < TC_M / 2; ++u) {
      float hi, lo;
      tf32_split(va[u], hi, lo);
      const uint32_t o = kmajor_off(rq + 2 * u, kk, TC_M);
      *(float *)(Ahi + o) = hi;
      *(float *)(Alo + o) = lo;
    }
#pragma unroll
    for (int u = 0; u < TC_N / 2; ++u) {
      float hi, lo;
      tf32_split(vb[u], hi, lo);
      const uint32_t o = kmajor_off(rq + 2 * u, kk, TC_N);
      *(float *)(Bhi + o) = hi;
      *(float *)(Blo + o) = lo;
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = tmem_slot;
  if (tid == 0) {
    // kind::tf32, D F32 [4,6) = 1, A TF32 [7,10) = 2, B TF32 [10,13) = 2,
    // both K-major, N >> 3 at [17,23), M >> 4 at [24,29)
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                           ((uint32_t)(TC_M >> 4) << 24);
    const uint32_t a_hi = smem_u32(Ahi), a_lo = smem_u32(Alo), b_hi = smem_u32(Bhi), b_lo = smem_u32(Blo);
    for (int s = 0; s < TC_K / 8; ++s) {
      for (int p = 0; p < 3; ++p) {
        const uint32_t sa = (p == 2 ? a_lo : a_hi) + (uint32_t)s * 2u * (TC_M / 8) * 128u;
        const uint32_t sb = (p == 1 ? b_lo : b_hi) + (uint32_t)s * 2u * (TC_N / 8) * 128u;
        const uint64_t da = umma_desc(sa, (TC_M / 8) * 128, 128);
        const uint64_t db = umma_desc(sb, (TC_N / 8) * 128, 128);
        const uint32_t acc = (s | p) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
            :: "r"(taddr), "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(&mbar))
                 : "memory");
  }
  // bounded wait for the products
  uint32_t done = 0;
  for (uint32_t it = 0; it < TC_WAIT_MAX && !done; ++it) {
    asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}\n"
                 : "=r"(done)
                 : "r"(smem_u32(&mbar)), "r"(0u)
                 : "memory");
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // TMEM lane = output row (32 per warp), column = output column: stage the
  // FP32 products in shared memory (the operands are no longer read), then
  // subtract them from the FP64 tiles with coalesced row accesses
  float *stage = (float *)Ahi;   // (TC_M, TC_N + 1), within A hi + A lo
  const int row = warp * 32 + lid;
  for (int c = 0; c < TC_N / 8; ++c) {
    uint32_t v[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 8)));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 8; ++q) stage[row * (TC_N + 1) + c * 8 + q] = __uint_as_float(v[q]);
  }
  __syncthreads();
  if (done) {
    const int col = tid & 63, rq = tid >> 6;
    for (int u = 0; u < TC_M / 2; ++u) {
      const int r = rq + 2 * u;
      const int trow = ti0 + (r >> 6);
      const int grow = trow * CT + (r & 63);
      if (grow < n && col < mj && trow >= tj)
        Lm[(size_t)grow * n + j0 + col] -= (double)stage[r * (TC_N + 1) + col];
    }
  }
  if (tid == 0 && !done) atomicOr(&a.not_spd[lane], 2);   // the tensor-core wait gave up
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(TC_N));
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
  noise3(a, lane, L.state0 + i, a.bd_istep, a.noise_base, n0, n1, n2);
  double *xi = a.bd_xi + 3 * (size_t)(L.state0 + i);
  xi[0] = n0; xi[1] = n1; xi[2] = n2;
}

// grid (ceil(maxN * 3 / 8), nlane), 256 threads: one warp per row k of the
// lane: dx_k = rlan1 sum_c D_kc F_c + rlan2 sum_{c <= k} L_kc xi_c, x += dx
__global__ void __launch_bounds__(256) bd_update_kernel(KArgs a) {
  const int lane = blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const int n = 3 * a.tops[L.top].nmp;
  const int warp = threadIdx.x >> 5, lid = threadIdx.x & 31;
  const int k = blockIdx.x * 8 + warp;
  if (blockIdx.x == 0 && threadIdx.x == 0) a.lstate[lane].istep = a.bd_istep;
  if (k >= n) return;
  const double *Drow = a.bd_D + L.bd0 + (size_t)k * n;
  const double *Lrow = a.bd_L + L.bd0 + (size_t)k * n;
  const double *F = a.bd_F + 3 * (size_t)L.state0, *xi = a.bd_xi + 3 * (size_t)L.state0;
  double df = 0.0, dr = 0.0;
  for (int c = lid; c < n; c += 32) df += Drow[c] * F[c];
  for (int c = lid; c <= k; c += 32) dr += Lrow[c] * xi[c];
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
  double fx = 0.0, fy = 0.0, fz = 0.0;
  int nclamp = 0;
  for (int p = p0 + lid; p < p1; p += 32) {
    const int ent = a.bd_ent[T.be0 + p];
    const int rec = ent >> 1;
    const int *idx = (ent & 1) ? a.wca_idx + 2 * (size_t)rec : a.fene_idx + 2 * (size_t)rec;
    const int i1 = idx[0], i2 = idx[1];
    const double v0 = x[3 * i2] - x[3 * i1], v1 = x[3 * i2 + 1] - x[3 * i1 + 1], v2 = x[3 * i2 + 2] - x[3 * i1 + 2];
    double f;   // force on i2 is f * v21, on i1 -f * v21
    if (!(ent & 1)) {
      const double dist = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
      const double dd = dist - a.fene_nat[rec];
      f = -a.fene_coef[rec] * dd / (1.0 - dd * dd / a.fene_d2[rec]) / dist;
    } else {
      const double dist2 = v0 * v0 + v1 * v1 + v2 * v2;
      const double nat2 = a.wca_nat[rec] * a.wca_nat[rec];
      const double ro2 = nat2 / dist2;
      if (ro2 < a.wca_rcut2) continue;
      const double ro4 = ro2 * ro2, ro8 = ro4 * ro4, ro14 = ro8 * ro4 * ro2;
      const double coef = (ro2 > 1.0) ? a.wca_coef[2 * (size_t)rec] : a.wca_coef[2 * (size_t)rec + 1];
      f = 12.0 * coef / nat2 * (ro14 - ro8);
      if (f > 50.0) { f = 50.0; ++nclamp; }   // DE_MAX
    }
    const double s = (i == i2) ? f : -f;
    fx += s * v0; fy += s * v1; fz += s * v2;
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
cudaError_t bd_refactor_launch(cudaStream_t st, KArgs a, int max_nmp) {
  cudaError_t e = cudaFuncSetAttribute(chol_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       2 * CT * CT * (int)sizeof(double));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(chol_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           2 * CT * CTP * (int)sizeof(double));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(chol_update_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM + 1024);
  if (e != cudaSuccess) return e;
  const long long nn = (long long)max_nmp * max_nmp;
  rpy_kernel<<<dim3((unsigned)((nn + 255) / 256), a.nlane), 256, 0, st>>>(a);
  const int T = (3 * max_nmp + CT - 1) / CT;
  for (int k = 0; k < T; ++k) {
    a.bd_kpanel = k;
    chol_diag_kernel<<<a.nlane, 256, 0, st>>>(a);
    if (k + 1 < T) {
      chol_panel_kernel<<<dim3(T - k - 1, a.nlane), 256, 2 * CT * CTP * sizeof(double), st>>>(a);
      const int m = T - k - 1;
      if (a.bd_tc)
        chol_update_tc_kernel<<<dim3(((m + 1) / 2) * m, a.nlane), 128, TC_SMEM + 1024, st>>>(a, m);
      else
        chol_update_kernel<<<dim3(m * (m + 1) / 2, a.nlane), 256, 2 * CT * CT * sizeof(double), st>>>(a);
    }
  }
  return cudaGetLastError();
}

int bd_refactor_launches(int max_nmp) {
  const int T = (3 * max_nmp + CT - 1) / CT;
  return 1 + T + 2 * (T - 1);
}

cudaError_t bd_step_launch(cudaStream_t st, const KArgs &a, int max_nmp) {
  bd_noise_kernel<<<dim3((max_nmp + 127) / 128, a.nlane), 128, 0, st>>>(a);
  bd_update_kernel<<<dim3((3 * max_nmp + 7) / 8, a.nlane), 256, 0, st>>>(a);
  bd_force_kernel<<<dim3((max_nmp + 7) / 8, a.nlane), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t bd_force_launch(cudaStream_t st, const KArgs &a, int max_nmp) {
  bd_force_kernel<<<dim3((max_nmp + 7) / 8, a.nlane), 256, 0, st>>>(a);
  return cudaGetLastError();
}

} // namespace tis
