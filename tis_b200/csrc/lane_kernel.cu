// lane_kernel.cu -- persistent force-and-integrate kernel, one CTA per lane.
//
// Each CTA keeps its lane's coordinates, velocities and accelerations in
// shared memory for the whole launch and runs the reference step
// (src/time_integral.F90:57-190) nsteps times without leaving the SM:
//
//   neighbour trigger -> [rebuild lists] -> x update -> bonded terms into
//   per-interaction slots -> [valence pruning] -> per-bead gather of
//   non-bonded pairs + bonded slots (FP64 accumulation) -> v / a update
//
// Real = double is the plain FP64 path; Real = float computes pair and
// bonded forces in FP32 and accumulates each bead's force in FP64 (state,
// integration and neighbour decisions are FP64 in both).
//
// Determinism: every bead sums its contributions in a fixed order (its
// neighbour row in ascending j, then its incidence list in slot order) and
// the G threads of a bead group combine their partial sums with a fixed
// xor-butterfly, so results do not depend on scheduling.  Neighbour pair
// sets are bit-exact with the reference: the FP64 distance test is evaluated
// with explicitly rounded operations in the Fortran order.
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"

namespace tis {

__device__ __forceinline__ double sqr_rn(double x) { return __dmul_rn(x, x); }

// util_pbneighbor.F90:198-212 on one component; returns imi (0, 1, 2)
__device__ __forceinline__ int pb1(double &v, double L, double h) {
  if (v > h) { v = __dsub_rn(v, L); return 0; }
  if (v < -h) { v = __dadd_rn(v, L); return 1; }
  return 2;
}

// util_periodic.F90:163-173 on one coordinate, exact FP64 operation order
__device__ __forceinline__ double wrap1(double tx, double pw) {
  double pmax = __dmul_rn(0.5, pw), pmin = __dmul_rn(-0.5, pw);
  if (tx > pmax) {
    long long k = (long long)__ddiv_rn(__dsub_rn(tx, pmax), pw);
    tx = __dsub_rn(tx, __dmul_rn(pw, (double)(k + 1)));
  } else if (tx < pmin) {
    long long k = (long long)__ddiv_rn(__dsub_rn(pmin, tx), pw);
    tx = __dadd_rn(tx, __dmul_rn(pw, (double)(k + 1)));
  }
  return tx;
}

template <typename Real> struct R3 { Real x, y, z; };

template <typename Real> __device__ __forceinline__ Real rsqrt_(Real x);
template <> __device__ __forceinline__ double rsqrt_<double>(double x) { return 1.0 / sqrt(x); }
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return 1.0f / sqrtf(x); }

// ------------------------------------------------------------ shared state
template <typename Real>
struct Smem {
  double *X, *Y, *Z;        // xyz_mp_rep (unwrapped)
  double *PX, *PY, *PZ;     // pxyz_mp_rep (alias of X,Y,Z when not periodic)
  double *VX, *VY, *VZ;
  double *AX, *AY, *AZ;
  double *DX, *DY, *DZ;     // dxyz_mp (skin rule only)
  Real *rad, *eps, *q;      // pair parameters per bead
  int8_t *typ, *cls;
  int *misc;                // see MISC_*
  double *red;              // 64 doubles of reduction scratch
};
enum { MISC_EXCESS = 0, MISC_REBUILD = 1, MISC_CLAMP = 2, MISC_NEXV = 3, MISC_NELE = 4, MISC_NAN = 5,
       MISC_UNITS = 8 /* neigh_unit bytes start here (as ints) */ };

__host__ __device__ inline size_t smem_bytes(int N, bool periodic, bool skin, int real_size, int nunit) {
  size_t nd = 9 * (size_t)N;                 // X, V, A
  if (periodic) nd += 3 * (size_t)N;
  if (skin) nd += 3 * (size_t)N;
  nd += 64;                                  // red
  size_t b = nd * 8;
  b += 3 * (size_t)N * real_size;
  b += 2 * (size_t)N;
  b = (b + 15) & ~(size_t)15;
  b += (MISC_UNITS + (size_t)nunit * nunit + 8) * 4;
  return b;
}

template <typename Real>
__device__ Smem<Real> carve(void *base, int N, bool periodic, bool skin, int nunit) {
  Smem<Real> s;
  double *d = (double *)base;
  s.X = d; s.Y = d + N; s.Z = d + 2 * N; d += 3 * N;
  s.VX = d; s.VY = d + N; s.VZ = d + 2 * N; d += 3 * N;
  s.AX = d; s.AY = d + N; s.AZ = d + 2 * N; d += 3 * N;
  if (periodic) { s.PX = d; s.PY = d + N; s.PZ = d + 2 * N; d += 3 * N; }
  else { s.PX = s.X; s.PY = s.Y; s.PZ = s.Z; }
  if (skin) { s.DX = d; s.DY = d + N; s.DZ = d + 2 * N; d += 3 * N; }
  else { s.DX = s.DY = s.DZ = nullptr; }
  s.red = d; d += 64;
  Real *r = (Real *)d;
  s.rad = r; s.eps = r + N; s.q = r + 2 * N; r += 3 * N;
  int8_t *b = (int8_t *)r;
  s.typ = b; s.cls = b + N; b += 2 * N;
  uintptr_t p = ((uintptr_t)b + 15) & ~(uintptr_t)15;
  s.misc = (int *)p;
  return s;
}

// --------------------------------------------------------------- noise
// Gaussian triple for (lane, step, bead): counter-based Philox + Box-Muller,
// or the injected r_boxmuller array when one is set.
__device__ __forceinline__ void noise3(const KArgs &a, int lane, int gbead, long long istep, int noise_step,
                                       double &n0, double &n1, double &n2) {
  if (a.noise) {
    if (noise_step < a.noise_nsteps) {
      const double *r = a.noise + ((size_t)noise_step * a.nbead_total + gbead) * 3;
      n0 = r[0]; n1 = r[1]; n2 = r[2];
    } else {
      n0 = n1 = n2 = 0.0;
      atomicOr(&a.lstate[lane].flags, LF_NOISE_EXHAUSTED);
    }
    return;
  }
  U4 c = {(uint32_t)istep, (uint32_t)((unsigned long long)istep >> 32), (uint32_t)gbead, 0x4E4F4953u};
  U4 o = philox4x32(c, (uint32_t)a.seed ^ (0x9E3779B9u * (uint32_t)(lane + 1)), (uint32_t)(a.seed >> 32));
  float u1 = u01f_open0(o.x), u2 = u01f_open0(o.y), u3 = u01f_open0(o.z), u4 = u01f_open0(o.w);
  float r1 = sqrtf(-2.0f * logf(u1)), r2 = sqrtf(-2.0f * logf(u3));
  float s1, c1, s2, c2;
  sincospif(2.0f * u2, &s1, &c1);
  sincospif(2.0f * u4, &s2, &c2);
  n0 = (double)(r1 * c1); n1 = (double)(r1 * s1); n2 = (double)(r2 * c2);
}

__device__ __forceinline__ double lane_uniform(const KArgs &a, int lane, const LaneDesc &L, long long istep,
                                               int &draw) {
  LaneState &st = a.lstate[lane];
  if (a.unif) {
    if (st.unif_pos < a.n_unif) return a.unif[(size_t)L.unif0 + st.unif_pos++];
    st.flags |= LF_UNIF_EXHAUSTED;
    return 0.5;
  }
  U4 c = {(uint32_t)istep, (uint32_t)((unsigned long long)istep >> 32), (uint32_t)draw++, 0x50524E45u};
  U4 o = philox4x32(c, (uint32_t)a.seed ^ (0x85EBCA6Bu * (uint32_t)(lane + 1)), (uint32_t)(a.seed >> 32) ^ 0x5bd1e995u);
  return u01_open0(o.x);
}

// ------------------------------------------------------------ list build
// neighbor_list.F90:49-90 + neighbor_assign.F90:481-559 (+ sort) and
// neighbor_list_ele.F90:123-210, evaluated once per unordered pair into two
// symmetric bit matrices, then expanded into per-bead rows in ascending j.
template <typename Real>
__device__ void build_lists(const KArgs &a, int lane, const LaneDesc &L, const TopDesc &T, Smem<Real> &s) {
  const int N = T.nmp;
  const int W = (N + 31) >> 5;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int warp = tid >> 5, lid = tid & 31, nwarp = nth >> 5;
  LaneState &st = a.lstate[lane];
  uint32_t *mexv = a.mask + L.mask0;
  uint32_t *mele = mexv + (size_t)N * W;
  // wrap pxyz (util_periodic.F90)
  if (a.periodic) {
    for (int i = tid; i < N; i += nth) {
      s.PX[i] = wrap1(s.PX[i], a.psize[0]);
      s.PY[i] = wrap1(s.PY[i], a.psize[1]);
      s.PZ[i] = wrap1(s.PZ[i], a.psize[2]);
    }
  }
  for (int k = tid; k < 2 * N * W; k += nth) mexv[k] = 0u;
  if (tid == 0) { s.misc[MISC_NEXV] = 0; s.misc[MISC_NELE] = 0; }
  // unit prescreen (neighbor_pre.F90:174-252), thread 0
  const int nu = T.nunit;
  int *nunit_ok = s.misc + MISC_UNITS;
  if (tid == 0) {
    double cm[3 * 32], md[32];
    for (int u = 0; u < nu && u < 32; ++u) {
      int is = a.u_lunit[2 * (T.unit0 + u)], ie = a.u_lunit[2 * (T.unit0 + u) + 1];
      if (a.u_class[T.unit0 + u] == 4 /* ION */) { md[u] = 0; cm[3*u] = cm[3*u+1] = cm[3*u+2] = 0; continue; }
      double sx = 0, sy = 0, sz = 0;
      for (int i = is; i <= ie; ++i) { sx += s.X[i]; sy += s.Y[i]; sz += s.Z[i]; }
      double n = (double)(ie - is + 1);
      cm[3 * u] = sx / n; cm[3 * u + 1] = sy / n; cm[3 * u + 2] = sz / n;
      double m = 0;
      for (int i = is; i <= ie; ++i) {
        double dx = s.X[i] - cm[3 * u], dy = s.Y[i] - cm[3 * u + 1], dz = s.Z[i] - cm[3 * u + 2];
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 > m) m = d2;
      }
      md[u] = sqrt(m);
      if (a.periodic) for (int d = 0; d < 3; ++d) cm[3 * u + d] = wrap1(cm[3 * u + d], a.psize[d]);
    }
    for (int u = 0; u < nu; ++u)
      for (int v = u; v < nu; ++v) {
        int ok;
        if (a.u_class[T.unit0 + u] == 4 || a.u_class[T.unit0 + v] == 4 || u == v || u >= 32 || v >= 32) ok = 1;
        else {
          double w[3] = {cm[3 * v] - cm[3 * u], cm[3 * v + 1] - cm[3 * u + 1], cm[3 * v + 2] - cm[3 * u + 2]};
          if (a.periodic) for (int d = 0; d < 3; ++d) pb1(w[d], a.psize[d], a.psizeh[d]);
          ok = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) <
               md[u] + md[v] + sqrt(a.rneigh2[T.rn0 + u * nu + v]);
        }
        nunit_ok[u * nu + v] = ok;
        nunit_ok[v * nu + u] = ok;
      }
  }
  __syncthreads();
  const double rele2 = (a.i_ele != 0) ? a.lab_rele2[st.label] : -1.0;
  uint8_t *mir = a.periodic ? (a.mirror + L.mirror0) : nullptr;
  // pair tests: warp w takes rows i = w, w + nwarp, ...; lanes take j > i
  for (int i = warp; i < N - 1; i += nwarp) {
    const int ui = a.b_unit[T.bead0 + i];
    const int ci = s.cls[i];
    const int nsep = (s.typ[i] == 2) ? a.nsep[0] : (s.typ[i] == 4 ? a.nsep[1] : (s.typ[i] == 3 ? a.nsep[2] : -1));
    const double xi = s.PX[i], yi = s.PY[i], zi = s.PZ[i];
    const bool qi = fabs((double)a.b_charge[T.bead0 + i]) >= 1.0e-6;
    for (int j = i + 1 + lid; j < N; j += 32) {
      const int uj = a.b_unit[T.bead0 + j];
      if (!nunit_ok[ui * nu + uj]) continue;
      double v0 = __dsub_rn(s.PX[j], xi), v1 = __dsub_rn(s.PY[j], yi), v2 = __dsub_rn(s.PZ[j], zi);
      int im = 27;
      if (a.periodic) {
        int m0 = pb1(v0, a.psize[0], a.psizeh[0]);
        int m1 = pb1(v1, a.psize[1], a.psizeh[1]);
        int m2 = pb1(v2, a.psize[2], a.psizeh[2]);
        im = 9 * m0 + 3 * m1 + m2 + 1;
      }
      const double d2 = __dadd_rn(__dadd_rn(sqr_rn(v0), sqr_rn(v1)), sqr_rn(v2));
      bool ex = d2 < a.rneigh2[T.rn0 + ui * nu + uj];
      if (ex) {
        const int cj = s.cls[j];
        if (ui == uj) {
          if (ci == 2 /* RNA */ && j < i + nsep) ex = false;
        } else if (!((ci == 2 && cj == 2) || (ci == 2 && cj == 4) || (ci == 4 && cj == 2) ||
                     (ci == 4 && cj == 3) || (ci == 3 && cj == 4))) {
          ex = false;
        }
      }
      bool el = false;
      if (a.i_ele != 0 && qi && fabs((double)a.b_charge[T.bead0 + j]) >= 1.0e-6) el = d2 < rele2;
      if (ex || el) {
        const uint32_t bj = 1u << (j & 31), bi = 1u << (i & 31);
        if (ex) {
          atomicOr(&mexv[(size_t)i * W + (j >> 5)], bj);
          atomicOr(&mexv[(size_t)j * W + (i >> 5)], bi);
          atomicAdd(&s.misc[MISC_NEXV], 1);
        }
        if (el) {
          atomicOr(&mele[(size_t)i * W + (j >> 5)], bj);
          atomicOr(&mele[(size_t)j * W + (i >> 5)], bi);
          atomicAdd(&s.misc[MISC_NELE], 1);
        }
        if (mir) mir[(size_t)i * N + j] = (uint8_t)im;
      }
    }
  }
  __syncthreads();
  // rows: warp per bead, ascending j
  uint32_t *nbr = a.nbr + L.nbr0;
  int *rowcnt = a.rowcnt + L.rowcnt0;
  for (int r = warp; r < N; r += nwarp) {
    uint32_t *row = nbr + (size_t)r * (N > 1 ? N - 1 : 1);
    int base = 0;
    for (int w0 = 0; w0 < W; w0 += 32) {
      const int w = w0 + lid;
      uint32_t e = 0, l = 0;
      if (w < W) { e = mexv[(size_t)r * W + w]; l = mele[(size_t)r * W + w]; }
      uint32_t u = e | l;
      int c = __popc(u);
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lid >= o) incl += t;
      }
      int pos = base + incl - c;
      while (u) {
        int b = __ffs(u) - 1;
        u &= u - 1;
        int j = (w << 5) + b;
        uint32_t ent = (uint32_t)j;
        if (e & (1u << b)) ent |= (1u << 16);
        if (l & (1u << b)) ent |= (1u << 17);
        if (mir) {
          uint32_t im = (r < j) ? mir[(size_t)r * N + j] : mir[(size_t)j * N + r];
          ent |= (im << 18);
        }
        row[pos++] = ent;
      }
      base += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lid == 0) rowcnt[r] = base;
  }
  // hbond neighbour flags (neighbor_list_hb.F90:335-354)
  uint8_t *hbf = a.hb_flag + L.hb0;
  for (int h = tid; h < T.nhb; h += nth) {
    const int *m = a.hb_idx + 6 * (size_t)(T.hb0 + h);
    double v0, v1, v2;
    v0 = __dsub_rn(s.PX[m[0]], s.PX[m[1]]);
    v1 = __dsub_rn(s.PY[m[0]], s.PY[m[1]]);
    v2 = __dsub_rn(s.PZ[m[0]], s.PZ[m[1]]);
    if (a.periodic) { pb1(v0, a.psize[0], a.psizeh[0]); pb1(v1, a.psize[1], a.psizeh[1]); pb1(v2, a.psize[2], a.psizeh[2]); }
    double d2 = __dadd_rn(__dadd_rn(sqr_rn(v0), sqr_rn(v1)), sqr_rn(v2));
    hbf[h] = (d2 < a.hb_nd2[T.hb0 + h]) ? 1 : 0;
  }
  __syncthreads();
  if (tid == 0) {
    st.nrebuild++;
    st.nexv = s.misc[MISC_NEXV];
    st.nele = s.misc[MISC_NELE];
  }
}

// ------------------------------------------------------------ bonded terms
template <typename Real>
__device__ __forceinline__ void put_slot(void *slots, size_t k, Real fx, Real fy, Real fz) {
  Real *p = (Real *)slots + 3 * k;
  p[0] = fx; p[1] = fy; p[2] = fz;
}

template <typename Real>
__device__ __forceinline__ R3<Real> dvec(const Smem<Real> &s, int i, int j) {   // x_j - x_i (unwrapped)
  return R3<Real>{(Real)(s.X[j] - s.X[i]), (Real)(s.Y[j] - s.Y[i]), (Real)(s.Z[j] - s.Z[i])};
}

template <typename Real> __device__ __forceinline__ Real dot(R3<Real> a, R3<Real> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename Real> __device__ __forceinline__ R3<Real> crs(R3<Real> a, R3<Real> b) {
  return R3<Real>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename Real> __device__ __forceinline__ Real wrap_pi(Real d) {
  const Real PI = (Real)3.14159265358979323846, TPI = (Real)(2.0 * 3.14159265358979323846);
  if (d > PI) d -= TPI; else if (d < -PI) d += TPI;
  return d;
}

// force_bond.F90:41-56
template <typename Real>
__device__ void term_bond(const KArgs &a, const TopDesc &T, const Smem<Real> &s, void *slots, int k) {
  const int *m = a.bd_idx + 2 * (size_t)(T.bd0 + k);
  R3<Real> v = dvec(s, m[0], m[1]);
  Real dist = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
  Real dd = dist - (Real)a.bd_nat[T.bd0 + k];
  Real f = (Real)a.bd_coef[T.bd0 + k] * ((Real)-2.0 * dd / dist);
  put_slot<Real>(slots, 2 * k, -f * v.x, -f * v.y, -f * v.z);
  put_slot<Real>(slots, 2 * k + 1, f * v.x, f * v.y, f * v.z);
}

// force_bangle.F90:103-147
template <typename Real>
__device__ void term_angle(const KArgs &a, const TopDesc &T, const Smem<Real> &s, void *slots, int k) {
  const size_t sb = T.slot_ba + 3 * (size_t)k;
  const Real cf = (Real)a.ba_coef[T.ba0 + k];
  if (cf < (Real)1.0e-6) {
    put_slot<Real>(slots, sb, 0, 0, 0); put_slot<Real>(slots, sb + 1, 0, 0, 0); put_slot<Real>(slots, sb + 2, 0, 0, 0);
    return;
  }
  const int *m = a.ba_idx + 3 * (size_t)(T.ba0 + k);
  R3<Real> v21 = dvec(s, m[0], m[1]), v32 = dvec(s, m[1], m[2]);
  Real c11 = dot(v21, v21), c22 = dot(v32, v32), c21 = dot(v32, v21);
  Real co = -c21 / sqrt(c11 * c22);
  if (co > (Real)1) co = 1; else if (co < (Real)-1) co = -1;
  Real dba = acos(co) - (Real)a.ba_nat[T.ba0 + k];
  Real t3 = c11 * c22 - c21 * c21;
  if (t3 <= (Real)1) t3 = 1;
  Real f = (Real)2 * cf * dba / sqrt(t3);
  Real a1 = c21 / c11, a2 = c21 / c22;
  R3<Real> f21{f * (v21.x * a1 - v32.x), f * (v21.y * a1 - v32.y), f * (v21.z * a1 - v32.z)};
  R3<Real> f32{f * (v32.x * a2 - v21.x), f * (v32.y * a2 - v21.y), f * (v32.z * a2 - v21.z)};
  put_slot<Real>(slots, sb, -f21.x, -f21.y, -f21.z);
  put_slot<Real>(slots, sb + 1, f21.x - f32.x, f21.y - f32.y, f21.z - f32.z);
  put_slot<Real>(slots, sb + 2, f32.x, f32.y, f32.z);
}

// force_dtrna_stack.F90:54-165
template <typename Real>
__device__ void term_stack(const KArgs &a, const TopDesc &T, const Smem<Real> &s, void *slots, int k, double u0) {
  const int *m = a.st_idx + 7 * (size_t)(T.st0 + k);
  const double *nat = a.st_nat + 3 * (size_t)(T.st0 + k);
  const double *cf = a.st_coef + 3 * (size_t)(T.st0 + k);
  R3<Real> v21 = dvec(s, m[0], m[1]);
  R3<Real> v34 = dvec(s, m[3], m[2]);
  R3<Real> v54 = dvec(s, m[3], m[4]);
  R3<Real> v56 = dvec(s, m[5], m[4]);
  R3<Real> v76 = dvec(s, m[5], m[6]);
  const Real k1 = (Real)cf[0], k2 = (Real)cf[1], k3 = (Real)cf[2];
  Real fr[7][3];
  Real ediv = 1;
  Real dist = sqrt(dot(v21, v21));
  Real dd = dist - (Real)nat[0];
  ediv += k1 * dd * dd;
  Real g = (Real)2 * k1 * dd / dist;
  fr[0][0] = -g * v21.x; fr[0][1] = -g * v21.y; fr[0][2] = -g * v21.z;
  fr[1][0] = g * v21.x; fr[1][1] = g * v21.y; fr[1][2] = g * v21.z;
  R3<Real> mm = crs(v34, v54), nn = crs(v54, v56);
  Real dmm = dot(mm, mm), dnn = dot(nn, nn);
  Real d5454 = dot(v54, v54), abs54 = sqrt(d5454);
  Real d5654 = dot(v56, v54);
  Real d3454o = dot(v34, v54) / d5454, d5654o = d5654 / d5454;
  Real dih = atan2(dot(v34, nn) * abs54, dot(mm, nn));
  Real d = wrap_pi(dih - (Real)nat[1]);
  ediv += k2 * d * d;
  Real gi = (Real)2 * k2 * d * abs54 / dmm, gl = -(Real)2 * k2 * d * abs54 / dnn;
  R3<Real> fi{gi * mm.x, gi * mm.y, gi * mm.z}, fl{gl * nn.x, gl * nn.y, gl * nn.z};
  const Real fiv[3] = {fi.x, fi.y, fi.z}, flv[3] = {fl.x, fl.y, fl.z};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    fr[2][q] = fiv[q];
    fr[3][q] = ((Real)-1 + d3454o) * fiv[q] - d5654o * flv[q];
    fr[4][q] = ((Real)-1 + d5654o) * flv[q] - d3454o * fiv[q];
    fr[5][q] = flv[q];
    fr[6][q] = 0;
  }
  mm = crs(v76, v56);
  nn.x = -nn.x; nn.y = -nn.y; nn.z = -nn.z;
  dmm = dot(mm, mm);
  Real d5656 = dot(v56, v56), abs56 = sqrt(d5656);
  Real d7656o = dot(v76, v56) / d5656, d5456o = d5654 / d5656;
  dih = atan2(dot(v76, nn) * abs56, dot(mm, nn));
  d = wrap_pi(dih - (Real)nat[2]);
  ediv += k3 * d * d;
  gi = (Real)2 * k3 * d * abs56 / dmm; gl = -(Real)2 * k3 * d * abs56 / dnn;
  const Real f2i[3] = {gi * mm.x, gi * mm.y, gi * mm.z}, f2l[3] = {gl * nn.x, gl * nn.y, gl * nn.z};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    fr[6][q] += f2i[q];
    fr[5][q] += ((Real)-1 + d7656o) * f2i[q] - d5456o * f2l[q];
    fr[4][q] += -d7656o * f2i[q] + ((Real)-1 + d5456o) * f2l[q];
    fr[3][q] += f2l[q];
  }
  const Real pre = (Real)(u0 / ((double)ediv * (double)ediv));
  const size_t sb = T.slot_st + 7 * (size_t)k;
#pragma unroll
  for (int p = 0; p < 7; ++p) put_slot<Real>(slots, sb + p, pre * fr[p][0], pre * fr[p][1], pre * fr[p][2]);
}

// force_dtrna_hbond15.F90:91-353 (one hbond of the neighbour list).
// Returns the energy; active = |d| <= hb_cutoff_dist.
template <typename Real>
__device__ double term_hbond(const KArgs &a, const TopDesc &T, const Smem<Real> &s, void *slots, int k, bool &active) {
  const int *m = a.hb_idx + 6 * (size_t)(T.hb0 + k);
  const double *nat = a.hb_nat + 6 * (size_t)(T.hb0 + k);
  const double *cf = a.hb_coef + 7 * (size_t)(T.hb0 + k);
  // v12 = x1 - x2 (pxyz + minimum image when periodic)
  double w0 = s.PX[m[0]] - s.PX[m[1]], w1 = s.PY[m[0]] - s.PY[m[1]], w2 = s.PZ[m[0]] - s.PZ[m[1]];
  if (a.periodic) { pb1(w0, a.psize[0], a.psizeh[0]); pb1(w1, a.psize[1], a.psizeh[1]); pb1(w2, a.psize[2], a.psizeh[2]); }
  R3<Real> v12{(Real)w0, (Real)w1, (Real)w2};
  Real d1212 = dot(v12, v12);
  Real a12 = sqrt(d1212);
  Real d = a12 - (Real)nat[0];
  if (fabs((double)d) > a.hb_cutoff_dist) { active = false; return 0.0; }
  active = true;
  auto dv = [&](int p, int q) {   // x_p - x_q with minimum image when periodic
    double u0 = s.X[m[p]] - s.X[m[q]], u1 = s.Y[m[p]] - s.Y[m[q]], u2 = s.Z[m[p]] - s.Z[m[q]];
    if (a.periodic) { pb1(u0, a.psize[0], a.psizeh[0]); pb1(u1, a.psize[1], a.psizeh[1]); pb1(u2, a.psize[2], a.psizeh[2]); }
    return R3<Real>{(Real)u0, (Real)u1, (Real)u2};
  };
  R3<Real> v13 = dv(0, 2), v53 = dv(4, 2), v42 = dv(3, 1), v46 = dv(3, 5);
  Real fo[6][3];
  Real ex = -(Real)cf[1] * d * d;
  Real g = (Real)2 * (Real)cf[1] * d / a12;
  fo[0][0] = g * v12.x; fo[0][1] = g * v12.y; fo[0][2] = g * v12.z;
  fo[1][0] = -fo[0][0]; fo[1][1] = -fo[0][1]; fo[1][2] = -fo[0][2];
#pragma unroll
  for (int p = 2; p < 6; ++p) fo[p][0] = fo[p][1] = fo[p][2] = 0;
  Real d1313 = dot(v13, v13), d4242 = dot(v42, v42);
  Real a13 = sqrt(d1313), a42 = sqrt(d4242);
  Real d1213 = dot(v13, v12), d1242 = dot(v12, v42), d4246 = dot(v42, v46), d1353 = dot(v13, v53);
  Real d1213o1212 = d1213 / d1212, d1213o1313 = d1213 / d1313, d1242o1212 = d1242 / d1212;
  Real d4246o4242 = d4246 / d4242, d1242o4242 = d1242 / d4242, d1353o1313 = d1353 / d1313;
  const Real MAXC = (Real)a.max_abscos;
  const Real v12a[3] = {v12.x, v12.y, v12.z}, v13a[3] = {v13.x, v13.y, v13.z}, v42a[3] = {v42.x, v42.y, v42.z};
  // angle 3-1=2
  Real cos312 = d1213 / (a13 * a12);
  if (fabs(cos312) > MAXC) d1213 = copysign(a12 * a13 * MAXC, cos312);
  d = acos(cos312) - (Real)nat[1];
  Real pre = (Real)2 * (Real)cf[2] * d / sqrt(d1313 * d1212 - d1213 * d1213);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    Real fi = pre * (v12a[q] - d1213o1313 * v13a[q]);
    Real fk = pre * (v13a[q] - d1213o1212 * v12a[q]);
    fo[2][q] += fi; fo[1][q] += fk; fo[0][q] = fo[0][q] - fi - fk;
  }
  ex -= (Real)cf[2] * d * d;
  // angle 1=2-4
  Real cos124 = d1242 / (a12 * a42);
  if (fabs(cos124) > MAXC) d1242 = copysign(a12 * a42 * MAXC, cos124);
  d = acos(cos124) - (Real)nat[2];
  pre = (Real)2 * (Real)cf[3] * d / sqrt(d1212 * d4242 - d1242 * d1242);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    Real fi = -pre * (v42a[q] - d1242o1212 * v12a[q]);
    Real fk = -pre * (v12a[q] - d1242o4242 * v42a[q]);
    fo[0][q] += fi; fo[3][q] += fk; fo[1][q] = fo[1][q] - fi - fk;
  }
  ex -= (Real)cf[3] * d * d;
  // dihedral 4-2=1=3
  R3<Real> c4212 = crs(v42, v12), c1213 = crs(v12, v13);
  Real c4212_2 = dot(c4212, c4212), c1213_2 = dot(c1213, c1213);
  const Real sin2 = (Real)1 - MAXC * MAXC;
  if (fabs(cos124) > MAXC) c4212_2 = d4242 * d1212 * sin2;
  if (fabs(cos312) > MAXC) c1213_2 = d1212 * d1313 * sin2;
  Real dih = atan2(dot(v42, c1213) * a12, dot(c4212, c1213));
  d = wrap_pi(dih - (Real)nat[3]);
  ex -= (Real)cf[4] * d * d;
  pre = (Real)2 * (Real)cf[4] * d * a12;
  {
    const Real ca[3] = {c4212.x, c4212.y, c4212.z}, cb[3] = {c1213.x, c1213.y, c1213.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Real fi = pre / c4212_2 * ca[q], fl = -pre / c1213_2 * cb[q];
      fo[3][q] += fi;
      fo[1][q] += ((Real)-1 + d1242o1212) * fi - d1213o1212 * fl;
      fo[0][q] += ((Real)-1 + d1213o1212) * fl - d1242o1212 * fi;
      fo[2][q] += fl;
    }
  }
  // dihedral 5-3-1=2
  R3<Real> c5313 = crs(v53, v13);
  R3<Real> n{-c1213.x, -c1213.y, -c1213.z};
  Real c5313_2 = dot(c5313, c5313);
  Real cos531 = d1353 / (a13 * sqrt(dot(v53, v53)));
  if (fabs(cos531) > MAXC) c5313_2 = dot(v53, v53) * d1313 * sin2;
  dih = atan2(dot(v53, n) * a13, dot(c5313, n));
  d = wrap_pi(dih - (Real)nat[4]);
  ex -= (Real)cf[5] * d * d;
  pre = (Real)2 * (Real)cf[5] * d * a13;
  {
    const Real ca[3] = {c5313.x, c5313.y, c5313.z}, cb[3] = {n.x, n.y, n.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Real fi = pre / c5313_2 * ca[q], fl = -pre / c1213_2 * cb[q];
      fo[4][q] += fi;
      fo[2][q] += ((Real)-1 + d1353o1313) * fi - d1213o1313 * fl;
      fo[0][q] += ((Real)-1 + d1213o1313) * fl - d1353o1313 * fi;
      fo[1][q] += fl;
    }
  }
  // dihedral 1=2-4-6
  n = R3<Real>{-c4212.x, -c4212.y, -c4212.z};
  R3<Real> c4246 = crs(v42, v46);
  Real c4246_2 = dot(c4246, c4246);
  Real cos246 = d4246 / (a42 * sqrt(dot(v46, v46)));
  if (fabs(cos246) > MAXC) c4246_2 = dot(v46, v46) * d4242 * sin2;
  dih = atan2(dot(v12, c4246) * a42, dot(n, c4246));
  d = wrap_pi(dih - (Real)nat[5]);
  ex -= (Real)cf[6] * d * d;
  pre = (Real)2 * (Real)cf[6] * d * a42;
  {
    const Real ca[3] = {n.x, n.y, n.z}, cb[3] = {c4246.x, c4246.y, c4246.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Real fi = pre / c4212_2 * ca[q], fl = -pre / c4246_2 * cb[q];
      fo[0][q] += fi;
      fo[1][q] += ((Real)-1 + d1242o4242) * fi - d4246o4242 * fl;
      fo[3][q] += ((Real)-1 + d4246o4242) * fl - d1242o4242 * fi;
      fo[5][q] += fl;
    }
  }
  const double ene = cf[0] * exp((double)ex);
  const Real e = (Real)ene;
  const size_t sb = T.slot_hb + 6 * (size_t)k;
#pragma unroll
  for (int p = 0; p < 6; ++p) put_slot<Real>(slots, sb + p, e * fo[p][0], e * fo[p][1], e * fo[p][2]);
  return ene;
}

// force_dtrna_hbond15.F90:373-509, run by one thread of the lane
template <typename Real>
__device__ void prune_hbonds(const KArgs &a, int lane, const LaneDesc &L, const TopDesc &T, long long istep,
                             double beta, bool zero_energy) {
  uint8_t *hbf = a.hb_flag + L.hb0;
  double *ene = a.hb_ene + L.hb0;
  int *exc = a.site_exc + L.site0;
  const int ns = T.nsite;
  for (int s = 0; s < ns; ++s) exc[s] -= a.site_val[T.site0 + s];
  int draw = 0;
  for (int guard = 0; guard < 4 * (T.nhb + 1); ++guard) {
    int nex = 0;
    for (int s = 0; s < ns; ++s) nex += (exc[s] > 0);
    if (nex == 0) break;
    double rnd = lane_uniform(a, lane, L, istep, draw);
    int pick = (int)ceil(rnd * nex);
    pick = pick < 1 ? 1 : (pick > nex ? nex : pick);
    int site = -1;
    for (int s = 0, c = 0; s < ns; ++s)
      if (exc[s] > 0 && ++c == pick) { site = s; break; }
    // hb_seq: active hbonds at the site, in list_hb_at_hbsite order
    int seq[128];
    int nseq = 0;
    for (int p = a.site_ptr[T.site0 + site]; p < a.site_ptr[T.site0 + site + 1]; ++p) {
      int h = a.site_hb[T.sitehb0 + p];
      if (hbf[h] & 2) {
        if (nseq < 128) seq[nseq++] = h;
        else a.lstate[lane].flags |= LF_OVERFLOW;
      }
    }
    for (int i = 0; i < nseq; ++i) {
      rnd = lane_uniform(a, lane, L, istep, draw);
      int isw = (int)ceil(rnd * nseq);
      isw = isw < 1 ? 1 : (isw > nseq ? nseq : isw);
      int t = seq[i]; seq[i] = seq[isw - 1]; seq[isw - 1] = t;
    }
    if (nseq == 0) break;
    int idel = seq[0];
    for (int i = 1; i < nseq; ++i) {
      int jhb = seq[i];
      double ratio = exp((ene[jhb] - ene[idel]) * beta);
      rnd = lane_uniform(a, lane, L, istep, draw);
      if (rnd < ratio) idel = jhb;
    }
    hbf[idel] &= ~2;
    if (zero_energy) ene[idel] = 0.0;
    const int *sites = a.hb_site + 6 * (size_t)(T.hb0 + idel);
    for (int i = 0; i < 3; ++i) {
      int s1 = sites[i], s2 = sites[3 + i];
      if (s1 >= 0 && exc[s1] > 0) exc[s1] -= 1;
      if (s2 >= 0 && exc[s2] > 0) exc[s2] -= 1;
    }
  }
}

// ------------------------------------------------------------ force pass
// Bonded terms into slots, pruning, then per-bead gather.  On return the
// owner thread (g == 0) of each bead group has called sink(i, fx, fy, fz).
template <typename Real, typename Sink>
__device__ void force_pass(const KArgs &a, int lane, const LaneDesc &L, const TopDesc &T, Smem<Real> &s,
                           long long istep, Sink sink) {
  const int N = T.nmp;
  const int tid = threadIdx.x, nth = blockDim.x;
  LaneState &st = a.lstate[lane];
  const int label = st.label;
  void *slots = (Real *)a.slots + 3 * (size_t)L.slot0;
  uint8_t *hbf = a.hb_flag + L.hb0;
  double *hbe = a.hb_ene + L.hb0;
  int *exc = a.site_exc + L.site0;
  // (site counters were cleared by the caller before the previous barrier)
  const int nb = T.nbd, na = T.nba, nst = T.nst, nhb = T.nhb;
  const int total = nb + na + nst + nhb;
  const double *u0 = a.lab_u0 + a.lab_u0off[label];
  for (int k = tid; k < total; k += nth) {
    if (k < nb) term_bond<Real>(a, T, s, slots, k);
    else if (k < nb + na) term_angle<Real>(a, T, s, slots, k - nb);
    else if (k < nb + na + nst) term_stack<Real>(a, T, s, slots, k - nb - na, u0[k - nb - na]);
    else {
      const int h = k - nb - na - nst;
      uint8_t f = hbf[h] & 1;
      if (f) {
        bool act;
        double e = term_hbond<Real>(a, T, s, slots, h, act);
        hbe[h] = act ? e : 0.0;
        if (act) {
          f |= 2;
          const int *sites = a.hb_site + 6 * (size_t)(T.hb0 + h);
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            int sid = sites[q];
            if (sid >= 0) {
              int old = atomicAdd(&exc[sid], 1);
              if (old + 1 > a.site_val[T.site0 + sid]) s.misc[MISC_EXCESS] = 1;
            }
          }
        }
      } else {
        hbe[h] = 0.0;
      }
      hbf[h] = f;
    }
  }
  __syncthreads();
  if (s.misc[MISC_EXCESS]) {
    if (tid == 0) {
      const double beta = a.hb_beta_global ? a.beta_hbond15 : a.lab_beta[label];
      prune_hbonds<Real>(a, lane, L, T, istep, beta, true);
    }
    __syncthreads();
  }
  // gather
  const int G = a.group;
  const int g = tid & (G - 1);
  const int grp = tid / G, ngrp = nth / G;
  const uint32_t *nbr = a.nbr + L.nbr0;
  const int *rowcnt = a.rowcnt + L.rowcnt0;
  const double a_exv = a.exv_adjust;
  const Real ra = (Real)a_exv, ra2 = ra * ra;
  const double cdist = a.lab_cdist[label];
  const Real rcd = (Real)(1.0 / cdist);
  const double cut2d = (a.cutoff_ele * cdist) * (a.cutoff_ele * cdist);
  const Real cut2 = (Real)cut2d;
  const double coefT = a.lab_coef[label];
  const Real dist_ps = (Real)a.exv_dist_PS, dist_rr = (Real)a.exv_dist;
  const int rowlen = N > 1 ? N - 1 : 1;
  int nclamp = 0;
  const int iters = (N + ngrp - 1) / ngrp;
  for (int it = 0; it < iters; ++it) {
    const int i = grp + it * ngrp;
    const bool valid = i < N;
    double fx = 0, fy = 0, fz = 0;
    if (valid) {
      const double xi = s.PX[i], yi = s.PY[i], zi = s.PZ[i];
      const int ti = s.typ[i], ci = s.cls[i];
      const Real radi = s.rad[i], epsi = s.eps[i];
      const double qi = (double)s.q[i];
      const uint32_t *row = nbr + (size_t)i * rowlen;
      const int cnt = rowcnt[i];
      for (int e = g; e < cnt; e += G) {
        const uint32_t ent = row[e];
        const int j = ent & 0xFFFF;
        double w0 = s.PX[j] - xi, w1 = s.PY[j] - yi, w2 = s.PZ[j] - zi;
        if (a.periodic) {
          const int im = (int)(ent >> 18) - 1;   // canonical (min, max) mirror
          const int sgn = (j > i) ? 1 : -1;
          const int m0 = im / 9, m1 = (im / 3) % 3, m2 = im % 3;
          if (m0 != 2) w0 += sgn * (m0 == 0 ? -a.psize[0] : a.psize[0]);
          if (m1 != 2) w1 += sgn * (m1 == 0 ? -a.psize[1] : a.psize[1]);
          if (m2 != 2) w2 += sgn * (m2 == 0 ? -a.psize[2] : a.psize[2]);
        }
        const Real wx = (Real)w0, wy = (Real)w1, wz = (Real)w2;
        const Real r2 = wx * wx + wy * wy + wz * wz;
        Real dv = 0;
        if (ent & (1u << 16)) {       // force_exv_dt15.F90:204-265
          const int tj = s.typ[j], cj = s.cls[j];
          Real dij;
          if ((ti == 2 && tj == 4) || (ti == 4 && tj == 2)) dij = dist_ps;
          else if (ci == 2 && cj == 2) dij = dist_rr;
          else dij = radi + s.rad[j];
          const Real dist = sqrt(r2);
          if (dist <= dij) {
            const Real coef = epsi * s.eps[j];
            const Real dr = dist + ra - dij;
            const Real ro2 = ra2 / (dr * dr);
            const Real ro4 = ro2 * ro2, ro8 = ro4 * ro4, ro14 = ro2 * ro4 * ro8;
            Real f = fabs((Real)12 * coef * (ro14 - ro8) * dr / ra2 / dist);
            if (f > (Real)50) { f = 50; ++nclamp; }
            dv += f;
          }
        }
        if ((ent & (1u << 17)) && r2 <= cut2) {   // force_ele_DH.F90:72-117
          const Real ce = (Real)(qi * (double)s.q[j] * coefT);
          const Real dist1 = sqrt(r2);
          const Real rd = (Real)1 / dist1;
          Real f = ce * rd * rd * (rd + rcd) * exp(-dist1 * rcd);
          if (f > (Real)50) { f = 50; ++nclamp; }
          dv += f;
        }
        if (dv != (Real)0) {
          fx -= (double)(dv * wx); fy -= (double)(dv * wy); fz -= (double)(dv * wz);
        }
      }
      // bonded slots (incidence list, ascending slot id)
      const int p0 = a.inc_ptr[T.inc0 + i], p1 = a.inc_ptr[T.inc0 + i + 1];
      const Real *sl = (const Real *)slots;
      for (int p = p0 + g; p < p1; p += G) {
        const int sid = a.inc_slot[p];
        if (sid >= T.slot_hb) {
          const int h = (sid - T.slot_hb) / 6;
          if (!(hbf[h] & 2)) continue;
        }
        fx += (double)sl[3 * (size_t)sid]; fy += (double)sl[3 * (size_t)sid + 1]; fz += (double)sl[3 * (size_t)sid + 2];
      }
    }
    // fixed-order butterfly over the G threads of the group
    for (int o = G >> 1; o > 0; o >>= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o, G);
      fy += __shfl_xor_sync(0xffffffffu, fy, o, G);
      fz += __shfl_xor_sync(0xffffffffu, fz, o, G);
    }
    if (valid && g == 0) sink(i, fx, fy, fz);
  }
  if (nclamp) atomicAdd(&s.misc[MISC_CLAMP], nclamp);
}

// ------------------------------------------------------------ the kernel
template <typename Real>
__global__ void __launch_bounds__(MAX_THREADS) lane_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.x;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int N = T.nmp;
  const int tid = threadIdx.x, nth = blockDim.x;
  const bool skin = a.n_step_neighbor <= 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<Real> s = carve<Real>(smem_raw, N, a.periodic != 0, skin, T.nunit);
  LaneState &st = a.lstate[lane];
  // load state
  for (int i = tid; i < N; i += nth) {
    const size_t o = 3 * (size_t)(L.state0 + i);
    s.X[i] = a.xyz[o]; s.Y[i] = a.xyz[o + 1]; s.Z[i] = a.xyz[o + 2];
    if (a.periodic) { s.PX[i] = a.pxyz[o]; s.PY[i] = a.pxyz[o + 1]; s.PZ[i] = a.pxyz[o + 2]; }
    s.VX[i] = a.velo[o]; s.VY[i] = a.velo[o + 1]; s.VZ[i] = a.velo[o + 2];
    s.AX[i] = a.accel[o]; s.AY[i] = a.accel[o + 1]; s.AZ[i] = a.accel[o + 2];
    if (skin) { s.DX[i] = a.dxyz[o]; s.DY[i] = a.dxyz[o + 1]; s.DZ[i] = a.dxyz[o + 2]; }
    const int b = T.bead0 + i;
    s.rad[i] = (Real)a.b_radius[b]; s.eps[i] = (Real)a.b_eps[b]; s.q[i] = (Real)a.b_charge[b];
    s.typ[i] = a.b_type[b]; s.cls[i] = a.b_class[b];
  }
  if (tid < MISC_UNITS) s.misc[tid] = 0;
  int *exc = a.site_exc + L.site0;
  for (int k = tid; k < T.nsite; k += nth) exc[k] = 0;
  __syncthreads();

  const int label0 = st.label;
  const double *c1 = a.lab_c1 + a.lab_c1off[label0];
  const int gb0 = L.state0;

  if (a.mode == KM_NEIGHBOR) {
    build_lists<Real>(a, lane, L, T, s);
  } else if (a.mode == KM_FORCE) {
    double *out = a.out_force;
    force_pass<Real>(a, lane, L, T, s, st.istep, [&](int i, double fx, double fy, double fz) {
      const size_t o = 3 * (size_t)(L.state0 + i);
      out[o] = fx; out[o + 1] = fy; out[o + 2] = fz;
    });
  } else if (a.mode == KM_PRE) {
    build_lists<Real>(a, lane, L, T, s);
    // dxyz_mp = 0 (time_integral_pre.F90:79)
    if (skin) for (int i = tid; i < N; i += nth) { s.DX[i] = 0.0; s.DY[i] = 0.0; s.DZ[i] = 0.0; }
    __syncthreads();
    const long long is = st.istep;
    force_pass<Real>(a, lane, L, T, s, is, [&](int i, double fx, double fy, double fz) {
      double n0, n1, n2;
      noise3(a, lane, gb0 + i, is, a.noise_base, n0, n1, n2);
      const double rc = a.b_rcmass[T.bead0 + i], cc = c1[i];
      s.AX[i] = fx * rc + cc * n0; s.AY[i] = fy * rc + cc * n1; s.AZ[i] = fz * rc + cc * n2;
    });
  } else {  // KM_STEP
    for (int step = 0; step < a.nsteps; ++step) {
      const long long istep = st.istep + 1;
      // neighbour trigger (time_integral.F90:57-110)
      bool rebuild;
      if (!skin) {
        rebuild = (istep % a.n_step_neighbor) == 1 || istep == 1;
      } else {
        double m1 = 0, m2 = 0;
        for (int i = tid; i < N; i += nth) {
          double d2 = s.DX[i] * s.DX[i] + s.DY[i] * s.DY[i] + s.DZ[i] * s.DZ[i];
          if (d2 > m1) { m2 = m1; m1 = d2; } else if (d2 > m2) m2 = d2;
        }
        for (int o = 16; o > 0; o >>= 1) {
          double o1 = __shfl_xor_sync(0xffffffffu, m1, o), o2 = __shfl_xor_sync(0xffffffffu, m2, o);
          double n1 = fmax(m1, o1), n2 = fmax(fmin(m1, o1), fmax(m2, o2));
          m1 = n1; m2 = n2;
        }
        if ((tid & 31) == 0) { s.red[2 * (tid >> 5)] = m1; s.red[2 * (tid >> 5) + 1] = m2; }
        __syncthreads();
        if (tid == 0) {
          double b1 = 0, b2 = 0;
          for (int w = 0; w < (nth >> 5); ++w) {
            double o1 = s.red[2 * w], o2 = s.red[2 * w + 1];
            double n1 = fmax(b1, o1), n2 = fmax(fmin(b1, o1), fmax(b2, o2));
            b1 = n1; b2 = n2;
          }
          s.misc[MISC_REBUILD] = (sqrt(b1) + sqrt(b2) > a.neigh_margin) ? 1 : 0;
        }
        __syncthreads();
        rebuild = s.misc[MISC_REBUILD] != 0;
      }
      if (rebuild) {
        build_lists<Real>(a, lane, L, T, s);
        // dxyz_mp(:,:,irep) = 0 after a skin-triggered rebuild (time_integral.F90:89)
        if (skin) for (int i = tid; i < N; i += nth) { s.DX[i] = 0.0; s.DY[i] = 0.0; s.DZ[i] = 0.0; }
        __syncthreads();
      }
      // x update (time_integral.F90:152-161); clear hbond-site counters
      for (int i = tid; i < N; i += nth) {
        const int b = T.bead0 + i;
        const double c4 = a.b_c4[b];
        double dx = c4 * s.VX[i] + a.tstep2 * s.AX[i];
        double dy = c4 * s.VY[i] + a.tstep2 * s.AY[i];
        double dz = c4 * s.VZ[i] + a.tstep2 * s.AZ[i];
        s.X[i] += dx; s.Y[i] += dy; s.Z[i] += dz;
        if (a.periodic) { s.PX[i] += dx; s.PY[i] += dy; s.PZ[i] += dz; }
        if (skin) { s.DX[i] += dx; s.DY[i] += dy; s.DZ[i] += dz; }
      }
      for (int k = tid; k < T.nsite; k += nth) exc[k] = 0;
      if (tid == 0) s.misc[MISC_EXCESS] = 0;
      __syncthreads();
      const int nstep_noise = a.noise_base + step;
      force_pass<Real>(a, lane, L, T, s, istep, [&](int i, double fx, double fy, double fz) {
        // time_integral.F90:169-183
        double n0, n1, n2;
        noise3(a, lane, gb0 + i, istep, nstep_noise, n0, n1, n2);
        const int b = T.bead0 + i;
        const double rc = a.b_rcmass[b], cc = c1[i], c2 = a.b_c2[b], c3 = a.b_c3[b];
        const double ax = fx * rc + cc * n0, ay = fy * rc + cc * n1, az = fz * rc + cc * n2;
        s.VX[i] = c2 * s.VX[i] + c3 * (s.AX[i] + ax);
        s.VY[i] = c2 * s.VY[i] + c3 * (s.AY[i] + ay);
        s.VZ[i] = c2 * s.VZ[i] + c3 * (s.AZ[i] + az);
        s.AX[i] = ax; s.AY[i] = ay; s.AZ[i] = az;
        if (!(fx == fx && fy == fy && fz == fz)) s.misc[MISC_NAN] = 1;
      });
      if (tid == 0) st.istep = istep;
      __syncthreads();
    }
  }
  __syncthreads();
  // write back
  for (int i = tid; i < N; i += nth) {
    const size_t o = 3 * (size_t)(L.state0 + i);
    a.xyz[o] = s.X[i]; a.xyz[o + 1] = s.Y[i]; a.xyz[o + 2] = s.Z[i];
    if (a.periodic) { a.pxyz[o] = s.PX[i]; a.pxyz[o + 1] = s.PY[i]; a.pxyz[o + 2] = s.PZ[i]; }
    else { a.pxyz[o] = s.X[i]; a.pxyz[o + 1] = s.Y[i]; a.pxyz[o + 2] = s.Z[i]; }
    a.velo[o] = s.VX[i]; a.velo[o + 1] = s.VY[i]; a.velo[o + 2] = s.VZ[i];
    a.accel[o] = s.AX[i]; a.accel[o + 1] = s.AY[i]; a.accel[o + 2] = s.AZ[i];
    if (skin) { a.dxyz[o] = s.DX[i]; a.dxyz[o + 1] = s.DY[i]; a.dxyz[o + 2] = s.DZ[i]; }
  }
  if (tid == 0) {
    st.nclamp += s.misc[MISC_CLAMP];
    if (s.misc[MISC_NAN]) st.flags |= LF_NAN;
  }
}

template __global__ void lane_kernel<double>(KArgs);
template __global__ void lane_kernel<float>(KArgs);

size_t smem_bytes_host(int N, bool periodic, bool skin, int real_size, int nunit) {
  return smem_bytes(N, periodic, skin, real_size, nunit);
}

cudaError_t lane_kernel_set_smem(bool mixed, int bytes) {
  if (mixed) return cudaFuncSetAttribute(lane_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return cudaFuncSetAttribute(lane_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t lane_kernel_launch(bool mixed, int grid, int block, size_t smem, cudaStream_t st, const KArgs &a) {
  if (mixed) lane_kernel<float><<<grid, block, smem, st>>>(a);
  else lane_kernel<double><<<grid, block, smem, st>>>(a);
  return cudaGetLastError();
}

} // namespace tis

// =====================================================================
// energy_sumup (src/energy_sumup.F90:11-530) for one lane per CTA, FP64.
// Terms follow the energy twins: energy_bond, energy_bangle (via
// util_bondangle), energy_dtrna_stack, energy_dtrna_hbond15, energy_exv_dt15,
// energy_ele_DH and energy_kinetic.  Sums are reduced in a fixed order.
// =====================================================================
namespace tis {

__device__ __forceinline__ double3 gpos(const double *x, int idx) {
  return make_double3(x[3 * (size_t)idx], x[3 * (size_t)idx + 1], x[3 * (size_t)idx + 2]);
}
__device__ __forceinline__ double3 sub3(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double wrapd(double d) {
  const double PI = 3.14159265358979323846;
  if (d > PI) d -= 2.0 * PI; else if (d < -PI) d += 2.0 * PI;
  return d;
}

enum { ES_VELO, ES_BOND, ES_ANGLE, ES_STACK, ES_HB, ES_EXV, ES_ELE, ES_N };

__global__ void __launch_bounds__(256) energy_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.x;
  if (lane >= a.nlane) return;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int N = T.nmp;
  const int tid = threadIdx.x, nth = blockDim.x;
  LaneState &st = a.lstate[lane];
  const int label = (a.elabel && a.elabel[lane] >= 0) ? a.elabel[lane] : st.label;
  const double *X = a.xyz + 3 * (size_t)L.state0;
  const double *P = a.pxyz + 3 * (size_t)L.state0;
  const double *V = a.velo + 3 * (size_t)L.state0;
  __shared__ double red[ES_N][8];
  __shared__ int excess_flag;
  double es[ES_N];
  for (int k = 0; k < ES_N; ++k) es[k] = 0.0;
  if (tid == 0) excess_flag = 0;
  int *exc = a.site_exc + L.site0;
  uint8_t *hbf = a.hb_flag + L.hb0;
  double *hbe = a.hb_ene + L.hb0;
  if (!a.reuse_hb) for (int k = tid; k < T.nsite; k += nth) exc[k] = 0;
  __syncthreads();
  // kinetic
  for (int i = tid; i < N; i += nth) {
    double3 v = gpos(V, i);
    es[ES_VELO] += 0.5 * a.b_cmass[T.bead0 + i] * (v.x * v.x + v.y * v.y + v.z * v.z);
  }
  for (int k = tid; k < T.nbd; k += nth) {
    const int *m = a.bd_idx + 2 * (size_t)(T.bd0 + k);
    double3 v = sub3(gpos(X, m[1]), gpos(X, m[0]));
    double dd = sqrt(v.x * v.x + v.y * v.y + v.z * v.z) - a.bd_nat[T.bd0 + k];
    es[ES_BOND] += a.bd_coef[T.bd0 + k] * (dd * dd);
  }
  for (int k = tid; k < T.nba; k += nth) {
    const int *m = a.ba_idx + 3 * (size_t)(T.ba0 + k);
    double3 v21 = sub3(gpos(X, m[1]), gpos(X, m[0])), v32 = sub3(gpos(X, m[2]), gpos(X, m[1]));
    double c11 = dot3(v21, v21), c22 = dot3(v32, v32), c21 = dot3(v32, v21);
    double co = -c21 / sqrt(c11 * c22);
    if (co > 1.0) co = 1.0; else if (co < -1.0) co = -1.0;
    double dba = acos(co) - a.ba_nat[T.ba0 + k];
    es[ES_ANGLE] += a.ba_coef[T.ba0 + k] * (dba * dba);
  }
  const double *u0 = a.lab_u0 + a.lab_u0off[label];
  for (int k = tid; k < T.nst; k += nth) {
    const int *m = a.st_idx + 7 * (size_t)(T.st0 + k);
    const double *nat = a.st_nat + 3 * (size_t)(T.st0 + k);
    const double *cf = a.st_coef + 3 * (size_t)(T.st0 + k);
    double3 v21 = sub3(gpos(X, m[1]), gpos(X, m[0])), v34 = sub3(gpos(X, m[2]), gpos(X, m[3]));
    double3 v54 = sub3(gpos(X, m[4]), gpos(X, m[3])), v56 = sub3(gpos(X, m[4]), gpos(X, m[5]));
    double3 v76 = sub3(gpos(X, m[6]), gpos(X, m[5]));
    double ediv = 1.0;
    double dd = sqrt(dot3(v21, v21)) - nat[0];
    ediv += cf[0] * dd * dd;
    double3 mm = cross3(v34, v54), nn = cross3(v54, v56);
    double d = wrapd(atan2(dot3(v34, nn) * sqrt(dot3(v54, v54)), dot3(mm, nn)) - nat[1]);
    ediv += cf[1] * d * d;
    mm = cross3(v76, v56);
    nn = make_double3(-nn.x, -nn.y, -nn.z);
    d = wrapd(atan2(dot3(v76, nn) * sqrt(dot3(v56, v56)), dot3(mm, nn)) - nat[2]);
    ediv += cf[2] * d * d;
    es[ES_STACK] += u0[k] / ediv;
  }
  // non-bonded pairs j > i from the neighbour rows
  const uint32_t *nbr = a.nbr + L.nbr0;
  const int *rowcnt = a.rowcnt + L.rowcnt0;
  const int rowlen = N > 1 ? N - 1 : 1;
  const double cdist = a.lab_cdist[label], coefT = a.lab_coef[label];
  const double cut2 = (a.i_DH_cutoff_type == 0) ? (a.cutoff_ele * cdist) * (a.cutoff_ele * cdist)
                                                : a.cutoff_ele * a.cutoff_ele;
  const double rcd = 1.0 / cdist;
  for (int i = tid; i < N; i += nth) {
    const uint32_t *row = nbr + (size_t)i * rowlen;
    const int cnt = rowcnt[i];
    const int ti = a.b_type[T.bead0 + i], ci = a.b_class[T.bead0 + i];
    for (int e = 0; e < cnt; ++e) {
      const uint32_t ent = row[e];
      const int j = ent & 0xFFFF;
      if (j < i) continue;
      double3 w = sub3(gpos(P, j), gpos(P, i));
      if (a.periodic) {
        const int im = (int)(ent >> 18) - 1;
        const int m0 = im / 9, m1 = (im / 3) % 3, m2 = im % 3;
        if (m0 != 2) w.x += (m0 == 0 ? -a.psize[0] : a.psize[0]);
        if (m1 != 2) w.y += (m1 == 0 ? -a.psize[1] : a.psize[1]);
        if (m2 != 2) w.z += (m2 == 0 ? -a.psize[2] : a.psize[2]);
      }
      const double r2 = dot3(w, w);
      if (ent & (1u << 16)) {
        const int tj = a.b_type[T.bead0 + j], cj = a.b_class[T.bead0 + j];
        double dij;
        if ((ti == 2 && tj == 4) || (ti == 4 && tj == 2)) dij = a.exv_dist_PS;
        else if (ci == 2 && cj == 2) dij = a.exv_dist;
        else dij = a.b_radius[T.bead0 + i] + a.b_radius[T.bead0 + j];
        double dist = sqrt(r2);
        if (dist <= dij) {
          dist = dist + a.exv_adjust - dij;
          double ene;
          if (dist > 0.2 /* exv_inf */) {
            double ro = a.exv_adjust / dist, ro2 = ro * ro, ro6 = ro2 * ro2 * ro2;
            ene = a.b_eps[T.bead0 + i] * a.b_eps[T.bead0 + j] * (ro6 * ro6 - 2 * ro6 + 1.0);
          } else {
            ene = 1.0e10;
          }
          es[ES_EXV] += ene;
        }
      }
      if ((ent & (1u << 17)) && a.i_ele == 1 && r2 <= cut2) {
        const double dist1 = sqrt(r2);
        const double ce = a.b_charge[T.bead0 + i] * a.b_charge[T.bead0 + j] * coefT;
        es[ES_ELE] += ce / dist1 * exp(-dist1 * rcd);
      }
    }
  }
  // hydrogen bonds (energy_dtrna_hbond15.F90)
  if (!a.reuse_hb) {
    for (int h = tid; h < T.nhb; h += nth) {
      uint8_t f = hbf[h] & 1;
      hbe[h] = 0.0;
      if (f) {
        const int *m = a.hb_idx + 6 * (size_t)(T.hb0 + h);
        const double *nat = a.hb_nat + 6 * (size_t)(T.hb0 + h);
        const double *cf = a.hb_coef + 7 * (size_t)(T.hb0 + h);
        auto dv = [&](int p, int q) {
          double3 u = sub3(gpos(a.periodic ? P : X, m[p]), gpos(a.periodic ? P : X, m[q]));
          if (a.periodic) { pb1(u.x, a.psize[0], a.psizeh[0]); pb1(u.y, a.psize[1], a.psizeh[1]); pb1(u.z, a.psize[2], a.psizeh[2]); }
          return u;
        };
        double3 v12 = dv(0, 1);
        double a12 = sqrt(dot3(v12, v12));
        double d = a12 - nat[0];
        if (fabs(d) <= a.hb_cutoff_dist) {
          f |= 2;
          const int *sites = a.hb_site + 6 * (size_t)(T.hb0 + h);
          for (int q = 0; q < 6; ++q)
            if (sites[q] >= 0) {
              int old = atomicAdd(&exc[sites[q]], 1);
              if (old + 1 > a.site_val[T.site0 + sites[q]]) excess_flag = 1;
            }
          double ex = -cf[1] * d * d;
          double3 v13 = dv(0, 2), v53 = dv(4, 2), v42 = dv(3, 1), v46 = dv(3, 5);
          double a13 = sqrt(dot3(v13, v13)), a42 = sqrt(dot3(v42, v42));
          double d1213 = dot3(v13, v12), d1242 = dot3(v12, v42);
          d = acos(d1213 / (a13 * a12)) - nat[1];
          ex -= cf[2] * d * d;
          d = acos(d1242 / (a12 * a42)) - nat[2];
          ex -= cf[3] * d * d;
          double3 c4212 = cross3(v42, v12), c1213 = cross3(v12, v13);
          d = wrapd(atan2(dot3(v42, c1213) * a12, dot3(c4212, c1213)) - nat[3]);
          ex -= cf[4] * d * d;
          double3 mm = cross3(v53, v13), n = make_double3(-c1213.x, -c1213.y, -c1213.z);
          d = wrapd(atan2(dot3(v53, n) * a13, dot3(mm, n)) - nat[4]);
          ex -= cf[5] * d * d;
          mm = make_double3(-c4212.x, -c4212.y, -c4212.z);
          n = cross3(v42, v46);
          d = wrapd(atan2(dot3(v12, n) * a42, dot3(mm, n)) - nat[5]);
          ex -= cf[6] * d * d;
          hbe[h] = cf[0] * exp(ex);
        }
      }
      hbf[h] = f;
    }
    __syncthreads();
    if (excess_flag && tid == 0)
      prune_hbonds<double>(a, lane, L, T, st.istep, a.ebeta_lane ? a.ebeta_lane[lane] : a.ebeta, false);
    __syncthreads();
  }
  for (int h = tid; h < T.nhb; h += nth)
    if ((hbf[h] & 3) == 3) es[ES_HB] += hbe[h];
  // deterministic block reduction: warp butterfly, then warps in order
  for (int k = 0; k < ES_N; ++k)
    for (int o = 16; o > 0; o >>= 1) es[k] += __shfl_xor_sync(0xffffffffu, es[k], o);
  if ((tid & 31) == 0)
    for (int k = 0; k < ES_N; ++k) red[k][tid >> 5] = es[k];
  __syncthreads();
  if (tid == 0) {
    double tot[ES_N];
    for (int k = 0; k < ES_N; ++k) {
      tot[k] = 0.0;
      for (int w = 0; w < (nth >> 5); ++w) tot[k] += red[k][w];
    }
    double *E = a.out_energy + (size_t)lane * N_ETYPE;
    for (int k = 0; k < N_ETYPE; ++k) E[k] = 0.0;
    E[1] = tot[ES_VELO];
    E[2] = tot[ES_BOND];
    E[3] = tot[ES_ANGLE];
    E[7] = tot[ES_ELE];
    E[15] = tot[ES_STACK];
    E[16] = tot[ES_HB];
    E[17] = tot[ES_EXV];
    double sum = 0.0;
    for (int k = 2; k < N_ETYPE; ++k) sum += E[k];
    E[0] = sum;
  }
}

// velocity rescale after an accepted temperature swap
// (simu_replica_exchange.F90:272-300): scale > 0 multiplies, scale < 0
// divides by -scale, 0 leaves the lane alone.
__global__ void scale_velo_kernel(double *velo, const LaneDesc *lanes, const TopDesc *tops, const double *scale, int nlane);

cudaError_t energy_kernel_launch(int grid, cudaStream_t st, const KArgs &a) {
  energy_kernel<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t scale_velo_launch(int nlane, cudaStream_t st, double *velo, const LaneDesc *lanes, const TopDesc *tops,
                              const double *scale) {
  scale_velo_kernel<<<nlane, 128, 0, st>>>(velo, lanes, tops, scale, nlane);
  return cudaGetLastError();
}

__global__ void scale_velo_kernel(double *velo, const LaneDesc *lanes, const TopDesc *tops, const double *scale, int nlane) {
  const int lane = blockIdx.x;
  if (lane >= nlane) return;
  const double f = scale[lane];
  if (f == 0.0) return;
  const LaneDesc L = lanes[lane];
  const int N = tops[L.top].nmp;
  double *v = velo + 3 * (size_t)L.state0;
  if (f > 0.0) for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) v[k] = f * v[k];
  else for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) v[k] = v[k] / (-f);
}

} // namespace tis
