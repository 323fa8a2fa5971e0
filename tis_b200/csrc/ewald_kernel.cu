// ewald_kernel.cu -- reciprocal-space Ewald sums on the device, FP64
// (force_ele_coulomb_ewld.F90:62-84 forces, energy_ele_coulomb_ewld.F90:75-89
// energy, k table of mloop_ewld.F90:56-156).
//
// For a charge at x, e^{i k.x} with k = 2 pi (hx, hy, hz) / L factorises
// into e^{i 2 pi hx x / L} e^{i 2 pi hy y / L} e^{i 2 pi hz z / L}.  A first
// kernel tabulates (cos, sin)(2 pi h x_d / L) for h = 0..hmax per charge and
// dimension (negative h by conjugation), so every (k, charge) term costs two
// complex products instead of a sincos:
//
//   ewald_tab_kernel    per charge: 3 (hmax + 1) sincos
//   ewald_sk_kernel     per k and charge block: partial S_c(k) = sum q cos,
//                       S_s(k) = sum q sin (charges in ascending order)
//   ewald_sk_sum_kernel S(k) = the charge-block partials summed in block order
//   ewald_force_kernel  per charge (one warp) and k range (EW_F_SPLIT of
//                       them): partial F = sum_k coef 2 C(k) q (sin S_c -
//                       cos S_s) k, added by the lane kernel in range order
//   ewald_energy_kernel per lane: coef (sum_k C(k) (S_c^2 + S_s^2) + self)
//
// All sums run in a fixed order, so the results do not depend on scheduling.
#include "device_common.cuh"

namespace tis {

constexpr int EW_SK_THREADS = 256;   // k vectors per structure-factor block
constexpr int EW_SK_QCHUNK = 64;     // charges staged in shared memory at a time

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// table entry for integer h (negative h: complex conjugate)
__device__ __forceinline__ double2 tab_get(const double2 *t, int h) {
  const double2 v = t[h < 0 ? -h : h];
  return make_double2(v.x, h < 0 ? -v.y : v.y);
}

// grid (ceil(nq / 128), nlane): tab[(ew0 + kq) * 3 + d][h] = (cos, sin)(2 pi h x_d / L)
__global__ void __launch_bounds__(128) ewald_tab_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.y;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int kq = blockIdx.x * blockDim.x + threadIdx.x;
  if (kq >= T.nq) return;
  const int bead = a.q_bead[T.q0 + kq];
  const double *p = a.pxyz + 3 * (size_t)(L.state0 + bead);
  const int H = a.hmax + 1;
  double2 *t = (double2 *)a.ew_tab + (size_t)(L.ew0 + kq) * 3 * H;
  for (int d = 0; d < 3; ++d) {
    const double th = a.two_pi_L[d] * p[d];
    for (int h = 0; h < H; ++h) {
      double sn, cs;
      sincos((double)h * th, &sn, &cs);
      t[d * H + h] = make_double2(cs, sn);
    }
  }
}

// grid (ceil(nk / 256), nqblk, nlane)
__global__ void __launch_bounds__(EW_SK_THREADS) ewald_sk_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.z;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int H = a.hmax + 1;
  const int k = blockIdx.x * EW_SK_THREADS + threadIdx.x;
  const bool kv = k < a.nk;
  int hx = 0, hy = 0, hz = 0;
  if (kv) { hx = a.ew_h[3 * k]; hy = a.ew_h[3 * k + 1]; hz = a.ew_h[3 * k + 2]; }
  // charges of this block: [q_lo, q_hi)
  const int per = (T.nq + a.nqblk - 1) / a.nqblk;
  const int q_lo = blockIdx.y * per, q_hi = min(T.nq, q_lo + per);
  __shared__ double2 tab[EW_SK_QCHUNK * 3 * 12];
  __shared__ double qv[EW_SK_QCHUNK];
  double sc = 0.0, ss = 0.0;
  const double2 *gt = (const double2 *)a.ew_tab + (size_t)L.ew0 * 3 * H;
  for (int q0 = q_lo; q0 < q_hi; q0 += EW_SK_QCHUNK) {
    const int nqc = min(EW_SK_QCHUNK, q_hi - q0);
    __syncthreads();
    for (int e = threadIdx.x; e < nqc * 3 * H; e += EW_SK_THREADS) tab[e] = gt[(size_t)q0 * 3 * H + e];
    for (int e = threadIdx.x; e < nqc; e += EW_SK_THREADS)
      qv[e] = a.b_charge[T.bead0 + a.q_bead[T.q0 + q0 + e]];
    __syncthreads();
    if (kv) {
      for (int c = 0; c < nqc; ++c) {
        const double2 *t = tab + c * 3 * H;
        const double2 e = cmul(cmul(tab_get(t, hx), tab_get(t + H, hy)), tab_get(t + 2 * H, hz));
        sc += qv[c] * e.x;
        ss += qv[c] * e.y;
      }
    }
  }
  if (kv) {
    double *S = a.ew_S + (((size_t)lane * a.nqblk + blockIdx.y) * a.nk + k) * 2;
    S[0] = sc;
    S[1] = ss;
  }
}

// grid (ceil(nk / 256), nlane): S(k) = sum of the charge-block partials in
// block order, stored in block 0's slot
__global__ void __launch_bounds__(256) ewald_sk_sum_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.y;
  if (lane >= a.nlane) return;
  const int k = blockIdx.x * 256 + threadIdx.x;
  if (k >= a.nk) return;
  double *S = a.ew_S + (size_t)lane * a.nqblk * a.nk * 2;
  double sc = S[2 * (size_t)k], ss = S[2 * (size_t)k + 1];
  for (int b = 1; b < a.nqblk; ++b) {
    sc += S[((size_t)b * a.nk + k) * 2];
    ss += S[((size_t)b * a.nk + k) * 2 + 1];
  }
  S[2 * (size_t)k] = sc;
  S[2 * (size_t)k + 1] = ss;
}

constexpr int EW_F_KCHUNK = 512;     // k vectors staged in shared memory at a time

// grid (ceil(nq / 8), EW_F_SPLIT, nlane), 256 threads: one warp per charge
// over k range blockIdx.y; the CTA stages its 8 charges' tables and
// (S_c, S_s, C(k), h) of EW_F_KCHUNK vectors at a time
constexpr int EW_TAB_MAX = 3 * 16;   // 3 (hmax + 1) table entries per charge staged (hmax <= 15)
__global__ void __launch_bounds__(256) ewald_force_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.z;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int H = a.hmax + 1;
  const int warp = threadIdx.x >> 5, lid = threadIdx.x & 31;
  const int kq = blockIdx.x * 8 + warp;
  const bool qv = kq < T.nq;
  const int bead = qv ? a.q_bead[T.q0 + kq] : 0;
  const double q = qv ? a.b_charge[T.bead0 + bead] : 0.0;
  const double coefT = a.lab_coef[a.lstate[lane].label];
  const double *S = a.ew_S + (size_t)lane * a.nqblk * a.nk * 2;
  __shared__ double2 sT[8 * EW_TAB_MAX];
  __shared__ double2 sS[EW_F_KCHUNK];
  __shared__ double sC[EW_F_KCHUNK];
  __shared__ char4 sH[EW_F_KCHUNK];
  const bool staged = 3 * H <= EW_TAB_MAX;
  const double2 *t = staged ? sT + warp * EW_TAB_MAX
                            : (const double2 *)a.ew_tab + (size_t)(L.ew0 + (qv ? kq : 0)) * 3 * H;
  if (staged && qv) {
    const double2 *g = (const double2 *)a.ew_tab + (size_t)(L.ew0 + kq) * 3 * H;
    for (int e = lid; e < 3 * H; e += 32) sT[warp * EW_TAB_MAX + e] = g[e];
  }
  const int ka = (int)((long long)a.nk * blockIdx.y / EW_F_SPLIT);
  const int kb = (int)((long long)a.nk * (blockIdx.y + 1) / EW_F_SPLIT);
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int k0 = ka; k0 < kb; k0 += EW_F_KCHUNK) {
    const int nkc = min(EW_F_KCHUNK, kb - k0);
    __syncthreads();
    for (int e = threadIdx.x; e < nkc; e += blockDim.x) {
      const int k = k0 + e;
      sS[e] = make_double2(S[2 * (size_t)k], S[2 * (size_t)k + 1]);
      sC[e] = a.ew_coef[k];
      sH[e] = make_char4(a.ew_h[3 * k], a.ew_h[3 * k + 1], a.ew_h[3 * k + 2], 0);
    }
    __syncthreads();
    if (qv) {
      for (int e = lid; e < nkc; e += 32) {
        const char4 h = sH[e];
        const double2 ex = cmul(cmul(tab_get(t, h.x), tab_get(t + H, h.y)), tab_get(t + 2 * H, h.z));
        const double2 sk = sS[e];
        // qs * scos - qc * ssin (force_ele_coulomb_ewld.F90:74-80)
        const double dv = coefT * 2.0 * sC[e] * (q * ex.y * sk.x - q * ex.x * sk.y);
        fx += dv * (a.two_pi_L[0] * h.x);
        fy += dv * (a.two_pi_L[1] * h.y);
        fz += dv * (a.two_pi_L[2] * h.z);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (qv && lid == 0) {
    double *f = a.f_ext + 3 * ((size_t)blockIdx.y * a.nbead_total + L.state0 + bead);
    f[0] = fx; f[1] = fy; f[2] = fz;
  }
}

// grid nlane, 256 threads: adds coef (E_f + E_s) to E_ELE and E_TOTAL of each
// lane's energy (energy_ele_coulomb_ewld.F90:75-89 and the self term :212)
__global__ void __launch_bounds__(256) ewald_energy_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.x;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int label = (a.elabel && a.elabel[lane] >= 0) ? a.elabel[lane] : a.lstate[lane].label;
  const double *S = a.ew_S + (size_t)lane * a.nqblk * a.nk * 2;
  double ef = 0.0, qq = 0.0;
  for (int k = threadIdx.x; k < a.nk; k += blockDim.x) {
    const double sc = S[2 * (size_t)k], ss = S[2 * (size_t)k + 1];
    ef += a.ew_coef[k] * (sc * sc + ss * ss);
  }
  for (int kq = threadIdx.x; kq < T.nq; kq += blockDim.x) {
    const double q = a.b_charge[T.bead0 + a.q_bead[T.q0 + kq]];
    qq += q * q;
  }
  __shared__ double red[2][8];
  for (int o = 16; o > 0; o >>= 1) {
    ef += __shfl_xor_sync(0xffffffffu, ef, o);
    qq += __shfl_xor_sync(0xffffffffu, qq, o);
  }
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = ef; red[1][threadIdx.x >> 5] = qq; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0, s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { e += red[0][w]; s += red[1][w]; }
    const double add = a.lab_coef[label] * (e + a.ewld_self * s);
    double *E = a.out_energy + (size_t)lane * N_ETYPE;
    E[7] += add;
    E[0] += add;
  }
}

// Launches tab, structure factors and forces (into f_ext) for one lane
// (only_lane >= 0) or every lane.  nq_max: largest charge count of a lane.
cudaError_t ewald_recip_launch(cudaStream_t st, const KArgs &a, int nq_max, bool forces) {
  if (forces && !a.f_ext) return cudaErrorInvalidValue;
  const int nl = a.only_lane >= 0 ? 1 : a.nlane;
  ewald_tab_kernel<<<dim3((nq_max + 127) / 128, nl), 128, 0, st>>>(a);
  ewald_sk_kernel<<<dim3((a.nk + EW_SK_THREADS - 1) / EW_SK_THREADS, a.nqblk, nl), EW_SK_THREADS, 0, st>>>(a);
  if (a.nqblk > 1) ewald_sk_sum_kernel<<<dim3((a.nk + 255) / 256, nl), 256, 0, st>>>(a);
  if (forces) ewald_force_kernel<<<dim3((nq_max + 7) / 8, EW_F_SPLIT, nl), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t ewald_energy_launch(cudaStream_t st, const KArgs &a) {
  ewald_energy_kernel<<<a.only_lane >= 0 ? 1 : a.nlane, 256, 0, st>>>(a);
  return cudaGetLastError();
}

} // namespace tis
