// device_common.cuh -- device helpers and the shared-memory layout of the
// lane kernels (one CTA per lane, see lane_kernel.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"

namespace tis {

// Optional per-phase cycle counters (compiled only with -DTIS_PHASE_TIMING,
// read with tis_phase_read): thread 0 of CTA 0 accumulates clock64 spans.
#ifdef TIS_PHASE_TIMING
static __device__ unsigned long long g_phase[128];
#define PHASE_T0(v) long long v = clock64()
#define PHASE_ADD(k, t0) do { if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(&g_phase[k], (unsigned long long)(clock64() - (t0))); } while (0)
#ifdef TIS_PHASE_LIGHT
#define PHASE_ALL(k, t0) do {} while (0)
#else
#define PHASE_ALL(k, t0) do { if (blockIdx.x == 0) { atomicAdd(&g_phase[k], (unsigned long long)(clock64() - (t0))); atomicAdd(&g_phase[(k) + 16], 1ull); } } while (0)
#endif
// per-warp spans of the first two CTAs: slots base + 16 blockIdx.x + warp
#define PHASE_WARP(base, t0) do { if (blockIdx.x < 2 && (threadIdx.x & 31) == 0) atomicAdd(&g_phase[(base) + 16 * blockIdx.x + (threadIdx.x >> 5)], (unsigned long long)(clock64() - (t0))); } while (0)
#else
#define PHASE_WARP(base, t0) do {} while (0)
#define PHASE_ALL(k, t0) do {} while (0)
#define PHASE_T0(v) do {} while (0)
#define PHASE_ADD(k, t0) do {} while (0)
#endif

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

// Divisions and reciprocal square roots of the bonded terms: IEEE in the
// FP64 path, the hardware approximations (<= 2 ulp) in the FP32 path.
template <typename Real> __device__ __forceinline__ Real fdiv(Real a, Real b);
template <> __device__ __forceinline__ double fdiv<double>(double a, double b) { return a / b; }
template <> __device__ __forceinline__ float fdiv<float>(float a, float b) { return __fdividef(a, b); }
template <typename Real> __device__ __forceinline__ Real frsq(Real a);
template <> __device__ __forceinline__ double frsq<double>(double a) { return 1.0 / sqrt(a); }
template <> __device__ __forceinline__ float frsq<float>(float a) { return rsqrtf(a); }

template <typename Real> __device__ __forceinline__ Real rsqrt_(Real x);
template <> __device__ __forceinline__ double rsqrt_<double>(double x) { return 1.0 / sqrt(x); }
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return 1.0f / sqrtf(x); }

template <typename Real> struct V4;
template <> struct V4<float> { typedef float4 T; };
template <> struct V4<double> { typedef double4 T; };

// ------------------------------------------------------------ shared state
// Per-CTA shared memory.  The neighbour lists are two symmetric bit
// matrices (exv, ele): bit j of row i is set when the pair (min, max) is in
// the reference's list.  The matrices, bonded slots and incidence lists live
// in shared memory when they fit; otherwise they are used in global memory.
constexpr size_t MASK_SMEM_MAX = 64 * 1024;    // bit matrices kept in shared memory up to this size

// MISC_EXCESS, MISC_NEAR_DISP and MISC_DMAX have a second copy (+1) for odd
// steps: the two-CTA kernel sets a flag for the next step while the current
// one is read.
enum { MISC_EXCESS = 0, MISC_CLAMP = 2, MISC_NEXV = 3, MISC_NELE = 4, MISC_NAN = 5,
       MISC_REBUILT = 6, MISC_NEAR_BAD = 7, MISC_NEAR_DISP = 8, MISC_PMF = 10, MISC_CHUNK = 11,
       MISC_DMAX = 12 /* and 13 */, MISC_UNITS = 14 /* neigh_unit ints start here */ };

// Excluded-volume near lists: at a recording pass every bead keeps, per
// thread of its group, the exv-list partners within (screen radius +
// NEAR_SKIN); later passes visit only those until the lists are stale (a
// rebuild, or a bead displaced by more than NEAR_DISP_MAX since the
// recording: two beads then close in by less than NEAR_SKIN - 0.05 A).
// Visiting a sub-list in ascending j is the same summation as the full
// screen, so the forces are bitwise the same either way.
constexpr int NEAR_CAP = 32;                   // entries per bead, split over its group
constexpr float NEAR_SKIN = 1.0f;
constexpr float NEAR_DISP_MAX = 0.475f;

template <typename Real>
struct Smem {
  double *X, *Y, *Z;        // xyz_mp_rep (unwrapped)
  double *PX, *PY, *PZ;     // pxyz_mp_rep (alias of X,Y,Z when not periodic)
  double *VX, *VY, *VZ;
  double *AX, *AY, *AZ;
  double *DX, *DY, *DZ;     // dxyz_mp (skin rule only)
  double *QX, *QY, *QZ;     // periodic: pxyz wrapped at the last rebuild
  double *XN, *YN, *ZN;     // two-CTA lanes: next-step positions (double buffer)
  double *DD;               // skin rule: dot_product(dxyz, dxyz) of every bead
  double *red;              // 64 doubles of reduction scratch
  double *ch_part;          // (3 * CHMAX) partial Debye-Hueckel force of each chunk
  double *rn2;              // rneighbordist2_unit (nunit x nunit)
  typename V4<Real>::T *A4; // (px, py, pz, q) rounded to Real
  typename V4<Real>::T *B4; // (exv radius, exv sqrt(eps), exv screen radius, 0)
  typename V4<Real>::T *L4; // (px, py, pz) - A4 rounded to Real: hi + lo carries pxyz to ~2^-48
  typename V4<Real>::T *A4N, *L4N;   // two-CTA lanes: next-step A4, L4
  int *qb;                  // charged bead indices (nq)
  int *qidx;                // charge row of each bead (-1: uncharged)
  int *inc_ptr;             // (N + 1), relative to the lane's incidence entries
  int *misc;                // see MISC_*
  int16_t *unit;            // unit index of each bead
  int8_t *typ, *cls;
  uint32_t *mask;           // exv rows then ele rows, W words each (shared or global)
  uint16_t *near;           // (N, NEAR_CAP) exv near lists (shared only)
  uint8_t *near_cnt;        // (N, 8) entries per group thread, 0xFF = overflow
  float4 *NR4;              // positions at the last near-list recording
  Real *slots;              // shared or global
  const int *inc_slot;      // shared copy or global
  int W;                    // words per bit row
  double *C1, *C2, *C3, *C4, *RC;   // rlan_const(1..4) and 1/m of each bead (cst_on)
  double *NX, *NY, *NZ;              // this step's Gaussian noise, drawn in the bonded sweep (cst_on)
  int *exc;                 // hbond-site occupancy counters (shared when they fit, else the lane's global copy)
  int16_t *sched;           // fixed deal of the bonded sweep: warp w takes chunks sched[33 + sched[w] ..]
  int sched_cap;
  bool mask_smem, slots_smem, inc_smem, near_on, cst_on, exc_smem;
  bool fits;                // the base layout fits the launch's dynamic shared memory
};

// Entries of the bonded sweep's fixed deal: 33 per-warp offsets, then the
// chunk ids (at most sched_cap: every kind's items, at most nslot / 2, the
// electrostatic row chunks, at most CHMAX, and the noise of N beads, in
// chunks of 32, one partial chunk per kind) and as many scratch entries
__host__ __device__ inline int sched_cap(int N, int nslot) {
  return (nslot + CHMAX + N) / 32 + 16;
}

struct SmemPlan { size_t base, mask, slots, inc, near, cst, exc; };

// Byte layout of one lane (host and device use the same arithmetic).
__host__ __device__ inline SmemPlan smem_plan(int N, int nq, int nslot, int ninc, bool periodic, bool skin,
                                              int real_size, int nunit, bool dbuf = false, int nsite = 0) {
  size_t nd = 9 * (size_t)N + 64 + 3 * (size_t)CHMAX + (size_t)nunit * nunit + 2;
  if (periodic) nd += 6 * (size_t)N;
  if (skin) nd += 3 * (size_t)N;
  if (dbuf) nd += 3 * (size_t)N;
  if (skin) nd += (size_t)N;
  size_t b = nd * 8;
  b += 12 * (size_t)N * real_size;                  // A4, B4, L4
  if (dbuf) b += 8 * (size_t)N * real_size;         // A4N, L4N
  b = (b + 15) & ~(size_t)15;
  b += 4 * ((size_t)nq + N + (N + 1) + MISC_UNITS + (size_t)nunit * nunit + 8);
  b += 4 * (size_t)N;                               // unit, typ, cls
  b = (b + 15) & ~(size_t)15;
  b += 2 * (33 + 2 * (size_t)sched_cap(N, nslot));  // sweep deal
  b = (b + 15) & ~(size_t)15;
  SmemPlan p;
  p.base = b;
  p.mask = 8 * (size_t)N * ((N + 31) / 32);
  p.slots = ((3 * (size_t)nslot * real_size) + 15) & ~(size_t)15;
  p.inc = ((4 * (size_t)ninc) + 15) & ~(size_t)15;
  p.near = 16 * (size_t)N + 2 * (size_t)NEAR_CAP * N + 8 * (size_t)N + 16;
  p.cst = 8 * 8 * (size_t)N + 16;
  p.exc = ((4 * (size_t)nsite) + 15) & ~(size_t)15;
  return p;
}

// pxyz of bead i as the unevaluated sum A4 + L4 in Real
template <typename Real, typename S>
__device__ __forceinline__ void set_pos(S &s, int i) {
  const Real hx = (Real)s.PX[i], hy = (Real)s.PY[i], hz = (Real)s.PZ[i];
  s.A4[i].x = hx; s.A4[i].y = hy; s.A4[i].z = hz;
  s.L4[i].x = (Real)(s.PX[i] - (double)hx); s.L4[i].y = (Real)(s.PY[i] - (double)hy);
  s.L4[i].z = (Real)(s.PZ[i] - (double)hz); s.L4[i].w = (Real)0;
}

// error-free sum (Knuth TwoSum): hi + lo carries the running sum exactly
__device__ __forceinline__ void two_sum_add(float &hi, float &lo, float x) {
  const float s = hi + x;
  const float bp = s - hi;
  lo += (hi - (s - bp)) + (x - bp);
  hi = s;
}

template <typename Real>
__device__ Smem<Real> carve(unsigned char *base, int total, const KArgs &a, const LaneDesc &L, const TopDesc &T,
                            bool periodic, bool skin, bool dbuf = false) {
  const int N = T.nmp;
  Smem<Real> s;
  SmemPlan pl = smem_plan(N, T.nq, T.nslot, T.ninc, periodic, skin, (int)sizeof(Real), T.nunit, dbuf, T.nsite);
  double *d = (double *)base;
  s.X = d; s.Y = d + N; s.Z = d + 2 * N; d += 3 * N;
  s.VX = d; s.VY = d + N; s.VZ = d + 2 * N; d += 3 * N;
  s.AX = d; s.AY = d + N; s.AZ = d + 2 * N; d += 3 * N;
  if (periodic) {
    s.PX = d; s.PY = d + N; s.PZ = d + 2 * N; d += 3 * N;
    s.QX = d; s.QY = d + N; s.QZ = d + 2 * N; d += 3 * N;
  } else {
    s.PX = s.X; s.PY = s.Y; s.PZ = s.Z;
    s.QX = s.QY = s.QZ = nullptr;
  }
  if (skin) { s.DX = d; s.DY = d + N; s.DZ = d + 2 * N; d += 3 * N; }
  else { s.DX = s.DY = s.DZ = nullptr; }
  if (dbuf) { s.XN = d; s.YN = d + N; s.ZN = d + 2 * N; d += 3 * N; }
  else { s.XN = s.YN = s.ZN = nullptr; }
  if (skin) { s.DD = d; d += N; }
  else s.DD = nullptr;
  s.red = d; d += 64;
  s.ch_part = d; d += 3 * CHMAX;
  s.rn2 = d; d += T.nunit * T.nunit;
  typedef typename V4<Real>::T V;
  V *v4 = (V *)(((uintptr_t)d + 15) & ~(uintptr_t)15);
  s.A4 = v4; s.B4 = v4 + N; s.L4 = v4 + 2 * N; v4 += 3 * N;
  if (dbuf) { s.A4N = v4; s.L4N = v4 + N; v4 += 2 * N; }
  else { s.A4N = s.L4N = nullptr; }
  int *ip = (int *)(((uintptr_t)v4 + 15) & ~(uintptr_t)15);
  s.qb = ip; ip += T.nq;
  s.qidx = ip; ip += N;
  s.inc_ptr = ip; ip += N + 1;
  s.misc = ip; ip += MISC_UNITS + T.nunit * T.nunit + 8;
  s.unit = (int16_t *)ip;
  int8_t *b = (int8_t *)(s.unit + N);
  s.typ = b; s.cls = b + N; b += 2 * N;
  s.sched = (int16_t *)(((uintptr_t)b + 15) & ~(uintptr_t)15);
  s.sched_cap = sched_cap(N, T.nslot);
  unsigned char *u = (unsigned char *)(s.sched + 33 + 2 * s.sched_cap);
  u = (unsigned char *)(((uintptr_t)u + 15) & ~(uintptr_t)15);
  size_t used = (size_t)(u - base);
  s.fits = used <= (size_t)total;
  size_t left = (size_t)total > used ? (size_t)total - used : 0;
  s.W = (N + 31) >> 5;
  s.mask_smem = pl.mask <= MASK_SMEM_MAX && pl.mask <= left;
  if (s.mask_smem) { s.mask = (uint32_t *)u; u += pl.mask; left -= pl.mask; }
  else s.mask = a.mask + L.mask0;
  s.inc_smem = pl.inc <= left;
  if (s.inc_smem) { s.inc_slot = (const int *)u; u += pl.inc; left -= pl.inc; }
  else s.inc_slot = a.inc_slot + a.inc_ptr[T.inc0];
  s.slots_smem = pl.slots <= left;
  if (s.slots_smem) { s.slots = (Real *)u; u += pl.slots; left -= pl.slots; }
  else s.slots = (Real *)a.slots + 3 * (size_t)L.slot0;
  s.near_on = pl.near <= left;
  if (s.near_on) {
    s.NR4 = (float4 *)(((uintptr_t)u + 15) & ~(uintptr_t)15);
    s.near = (uint16_t *)(s.NR4 + N);
    s.near_cnt = (uint8_t *)(s.near + (size_t)NEAR_CAP * N);
    u = (unsigned char *)(s.near_cnt + 8 * (size_t)N);
    left = (size_t)total > (size_t)(u - base) ? (size_t)total - (size_t)(u - base) : 0;
  } else {
    s.NR4 = nullptr; s.near = nullptr; s.near_cnt = nullptr;
  }
  s.cst_on = pl.cst <= left;
  if (s.cst_on) {
    double *c = (double *)(((uintptr_t)u + 15) & ~(uintptr_t)15);
    s.C1 = c; s.C2 = c + N; s.C3 = c + 2 * N; s.C4 = c + 3 * N; s.RC = c + 4 * N;
    s.NX = c + 5 * N; s.NY = c + 6 * N; s.NZ = c + 7 * N;
    u = (unsigned char *)(c + 8 * (size_t)N);
    left = (size_t)total > (size_t)(u - base) ? (size_t)total - (size_t)(u - base) : 0;
  } else {
    s.C1 = s.C2 = s.C3 = s.C4 = s.RC = s.NX = s.NY = s.NZ = nullptr;
  }
  // hbond-site counters: shared atomics instead of returning L2 atomics
  s.exc_smem = T.nsite > 0 && pl.exc <= left;
  if (s.exc_smem) s.exc = (int *)(((uintptr_t)u + 15) & ~(uintptr_t)15);
  else s.exc = a.site_exc + L.site0;
  return s;
}

// --------------------------------------------------------------- noise
// Gaussian triple for (replica, step, bead i): counter-based Philox +
// Box-Muller keyed by the replica's key_lane / key_bead0, or the injected
// r_boxmuller array (indexed by the bead's place in this context) when one
// is set.
__device__ __forceinline__ void noise3(const KArgs &a, int lane, const LaneDesc &L, int i, long long istep,
                                       int noise_step, double &n0, double &n1, double &n2) {
  if (a.noise) {
    if (noise_step < a.noise_nsteps) {
      const double *r = a.noise + ((size_t)noise_step * a.nbead_total + L.state0 + i) * 3;
      n0 = r[0]; n1 = r[1]; n2 = r[2];
    } else {
      n0 = n1 = n2 = 0.0;
      atomicOr(&a.lstate[lane].flags, LF_NOISE_EXHAUSTED);
    }
    return;
  }
  U4 c = {(uint32_t)istep, (uint32_t)((unsigned long long)istep >> 32), (uint32_t)(L.key_bead0 + i), 0x4E4F4953u};
  U4 o = philox4x32(c, (uint32_t)a.seed ^ (0x9E3779B9u * (uint32_t)(L.key_lane + 1)), (uint32_t)(a.seed >> 32));
  float u1 = u01f_open0(o.x), u2 = u01f_open0(o.y), u3 = u01f_open0(o.z), u4 = u01f_open0(o.w);
  float r1 = sqrtf(-2.0f * logf(u1)), r2 = sqrtf(-2.0f * logf(u3));
  float s1, c1, s2, c2;
  sincospif(2.0f * u2, &s1, &c1);
  sincospif(2.0f * u4, &s2, &c2);
  n0 = (double)(r1 * c1); n1 = (double)(r1 * s1); n2 = (double)(r2 * c2);
}

// component d of noise3 (the same operations for that component)
__device__ __forceinline__ double noise1(const KArgs &a, int lane, const LaneDesc &L, int i, long long istep,
                                         int noise_step, int d) {
  if (a.noise) {
    if (noise_step < a.noise_nsteps) return a.noise[((size_t)noise_step * a.nbead_total + L.state0 + i) * 3 + d];
    atomicOr(&a.lstate[lane].flags, LF_NOISE_EXHAUSTED);
    return 0.0;
  }
  U4 c = {(uint32_t)istep, (uint32_t)((unsigned long long)istep >> 32), (uint32_t)(L.key_bead0 + i), 0x4E4F4953u};
  U4 o = philox4x32(c, (uint32_t)a.seed ^ (0x9E3779B9u * (uint32_t)(L.key_lane + 1)), (uint32_t)(a.seed >> 32));
  float sn, cs;
  if (d < 2) {
    const float u1 = u01f_open0(o.x), u2 = u01f_open0(o.y);
    const float r1 = sqrtf(-2.0f * logf(u1));
    sincospif(2.0f * u2, &sn, &cs);
    return (double)(r1 * (d ? sn : cs));
  }
  const float u3 = u01f_open0(o.z), u4 = u01f_open0(o.w);
  const float r2 = sqrtf(-2.0f * logf(u3));
  sincospif(2.0f * u4, &sn, &cs);
  return (double)(r2 * cs);
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
  U4 o = philox4x32(c, (uint32_t)a.seed ^ (0x85EBCA6Bu * (uint32_t)(L.key_lane + 1)),
                    (uint32_t)(a.seed >> 32) ^ 0x5bd1e995u);
  return u01_open0(o.x);
}

// ------------------------------------------------------------ bonded terms
// Destination of the bonded slots: the slot of a bead goes to `loc`, or to
// `peer` when the bead belongs to the other CTA of a two-CTA lane (beads
// outside [lo, hi)).  peer == nullptr: one CTA per lane, everything local.
struct SlotDst {
  void *loc, *peer;
  int lo, hi;
};

template <typename Real>
__device__ __forceinline__ void put_slot(const SlotDst &d, size_t k, int bead, Real fx, Real fy, Real fz) {
  void *base = (d.peer && (bead < d.lo || bead >= d.hi)) ? d.peer : d.loc;
  Real *p = (Real *)base + 3 * k;
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
// Interaction tables are constant for a launch: read them through the
// read-only data path, which the cluster barriers' acquire does not discard.
template <typename T> __device__ __forceinline__ T ldro(const T *p) { return __ldg(p); }

template <typename Real> __device__ __forceinline__ Real wrap_pi(Real d) {
  const Real PI = (Real)3.14159265358979323846, TPI = (Real)(2.0 * 3.14159265358979323846);
  if (d > PI) d -= TPI; else if (d < -PI) d += TPI;
  return d;
}

// force_bond.F90:41-56
template <typename Real>
__device__ void term_bond(const KArgs &a, const TopDesc &T, const Smem<Real> &s, const SlotDst &slots, int k) {
  const int *mp = a.bd_idx + 2 * (size_t)(T.bd0 + k);
  const int m[2] = {ldro(mp), ldro(mp + 1)};
  R3<Real> v = dvec(s, m[0], m[1]);
  Real dist = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
  Real dd = dist - (Real)ldro(a.bd_nat + T.bd0 + k);
  Real f = (Real)ldro(a.bd_coef + T.bd0 + k) * ((Real)-2.0 * fdiv(dd, dist));
  put_slot<Real>(slots, 2 * k, m[0], -f * v.x, -f * v.y, -f * v.z);
  put_slot<Real>(slots, 2 * k + 1, m[1], f * v.x, f * v.y, f * v.z);
}

// force_bangle.F90:103-147
template <typename Real>
__device__ void term_angle(const KArgs &a, const TopDesc &T, const Smem<Real> &s, const SlotDst &slots, int k) {
  const size_t sb = T.slot_ba + 3 * (size_t)k;
  const Real cf = (Real)ldro(a.ba_coef + T.ba0 + k);
  const int *mp = a.ba_idx + 3 * (size_t)(T.ba0 + k);
  const int m[3] = {ldro(mp), ldro(mp + 1), ldro(mp + 2)};
  if (cf < (Real)1.0e-6) {
    put_slot<Real>(slots, sb, m[0], 0, 0, 0); put_slot<Real>(slots, sb + 1, m[1], 0, 0, 0);
    put_slot<Real>(slots, sb + 2, m[2], 0, 0, 0);
    return;
  }
  R3<Real> v21 = dvec(s, m[0], m[1]), v32 = dvec(s, m[1], m[2]);
  Real c11 = dot(v21, v21), c22 = dot(v32, v32), c21 = dot(v32, v21);
  Real co = -c21 * frsq(c11 * c22);
  if (co > (Real)1) co = 1; else if (co < (Real)-1) co = -1;
  Real th, t3;
  if (sizeof(Real) == 4 && fabs(co) > (Real)0.99) {
    // FP32 near 0 or 180 degrees: the angle as atan2(|v21 x v32|, -v21.v32)
    // and t3 = |v21 x v32|^2 (= c11 c22 - c21^2), the same quantities as the
    // reference's acos of the cosine, without the rounding that acos and the
    // difference amplify there (up to 1e-4 rad at 179.97 degrees)
    const R3<Real> cr = crs(v21, v32);
    t3 = dot(cr, cr);
    th = atan2(sqrt(t3), -c21);
  } else {
    th = acos(co);
    t3 = c11 * c22 - c21 * c21;
  }
  Real dba = th - (Real)ldro(a.ba_nat + T.ba0 + k);
  if (t3 <= (Real)1) t3 = 1;
  Real f = (Real)2 * cf * dba * frsq(t3);
  Real a1 = fdiv(c21, c11), a2 = fdiv(c21, c22);
  R3<Real> f21{f * (v21.x * a1 - v32.x), f * (v21.y * a1 - v32.y), f * (v21.z * a1 - v32.z)};
  R3<Real> f32{f * (v32.x * a2 - v21.x), f * (v32.y * a2 - v21.y), f * (v32.z * a2 - v21.z)};
  put_slot<Real>(slots, sb, m[0], -f21.x, -f21.y, -f21.z);
  put_slot<Real>(slots, sb + 1, m[1], f21.x - f32.x, f21.y - f32.y, f21.z - f32.z);
  put_slot<Real>(slots, sb + 2, m[2], f32.x, f32.y, f32.z);
}

// st_status of secondary stack k (force_dtrna_stack_nlocal.F90:83-92): off
// when an exclusive tertiary stack of it is within 10 A of its native
// distance; FP64 in the reference's operation order, so the decision is the
// reference's
template <typename Real>
__device__ __forceinline__ bool stack_excluded(const KArgs &a, const TopDesc &T, const Smem<Real> &s, int k) {
  if (T.ntst == 0) return false;
  for (int e = a.stx_ptr[T.stx0 + k]; e < a.stx_ptr[T.stx0 + k + 1]; ++e) {
    const int t = a.stx_tst[e];
    const int *m = a.tst_idx + 6 * (size_t)(T.tst0 + t);
    double v0 = s.PX[m[0]] - s.PX[m[1]], v1 = s.PY[m[0]] - s.PY[m[1]], v2 = s.PZ[m[0]] - s.PZ[m[1]];
    if (a.periodic) { pb1(v0, a.psize[0], a.psizeh[0]); pb1(v1, a.psize[1], a.psizeh[1]); pb1(v2, a.psize[2], a.psizeh[2]); }
    const double d = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2))) -
                     a.tst_nat[6 * (size_t)(T.tst0 + t)];
    if (d < 10.0) return true;
  }
  return false;
}

// force_dtrna_stack_nlocal.F90:60-263: tertiary stack k into its six slots,
// FP64 in both paths for the reason given at term_stack
template <typename Real>
__device__ void term_tstack(const KArgs &a, const TopDesc &T, const Smem<Real> &s, const SlotDst &slots, int k) {
  const int *m = a.tst_idx + 6 * (size_t)(T.tst0 + k);
  const double *nat = a.tst_nat + 6 * (size_t)(T.tst0 + k);
  const double *cf = a.tst_coef + 7 * (size_t)(T.tst0 + k);
  typedef double W;   // working precision of this term
  auto dv = [&](int p, int q) {   // x_p - x_q (pxyz + minimum image when periodic)
    double w0 = s.PX[m[p]] - s.PX[m[q]], w1 = s.PY[m[p]] - s.PY[m[q]], w2 = s.PZ[m[p]] - s.PZ[m[q]];
    if (a.periodic) { pb1(w0, a.psize[0], a.psizeh[0]); pb1(w1, a.psize[1], a.psizeh[1]); pb1(w2, a.psize[2], a.psizeh[2]); }
    return R3<W>{w0, w1, w2};
  };
  const R3<W> v12 = dv(0, 1), v13 = dv(0, 2), v53 = dv(4, 2), v42 = dv(3, 1), v46 = dv(3, 5);
  const W d1212 = dot(v12, v12), d1313 = dot(v13, v13), d4242 = dot(v42, v42);
  const W a12 = sqrt(d1212), a13 = sqrt(d1313), a42 = sqrt(d4242);
  const W d1213 = dot(v13, v12), d1242 = dot(v12, v42), d4246 = dot(v42, v46), d1353 = dot(v13, v53);
  const W o1213_1212 = fdiv<W>(d1213, d1212), o1213_1313 = fdiv<W>(d1213, d1313);
  const W o1242_1212 = fdiv<W>(d1242, d1212), o4246_4242 = fdiv<W>(d4246, d4242);
  const W o1242_4242 = fdiv<W>(d1242, d4242), o1353_1313 = fdiv<W>(d1353, d1313);
  W fr[6][3];
  W ediv = 1;
  // distance 1=2
  W d = a12 - (W)nat[0];
  ediv += (W)cf[1] * d * d;
  {
    const W g = fdiv<W>((W)2 * (W)cf[1] * d, a12);
    fr[0][0] = g * v12.x; fr[0][1] = g * v12.y; fr[0][2] = g * v12.z;
    fr[1][0] = -fr[0][0]; fr[1][1] = -fr[0][1]; fr[1][2] = -fr[0][2];
  }
  const W v12a[3] = {v12.x, v12.y, v12.z}, v13a[3] = {v13.x, v13.y, v13.z}, v42a[3] = {v42.x, v42.y, v42.z};
#pragma unroll
  for (int q = 0; q < 3; ++q) { fr[2][q] = 0; fr[3][q] = 0; fr[4][q] = 0; fr[5][q] = 0; }
  // angle 3-1=2
  {
    W co = fdiv<W>(d1213, a13 * a12);
    co = co > (W)1 ? (W)1 : (co < (W)-1 ? (W)-1 : co);
    const W th = acos(co), sn2 = d1313 * d1212 - d1213 * d1213;
    d = th - (W)nat[1];
    const W pre = (W)2 * (W)cf[2] * d * frsq<W>(sn2);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const W fi = pre * (v12a[q] - o1213_1313 * v13a[q]), fk = pre * (v13a[q] - o1213_1212 * v12a[q]);
      fr[2][q] += fi; fr[1][q] += fk; fr[0][q] -= fi + fk;
    }
    ediv += (W)cf[2] * d * d;
  }
  // angle 1=2-4
  {
    W co = fdiv<W>(d1242, a12 * a42);
    co = co > (W)1 ? (W)1 : (co < (W)-1 ? (W)-1 : co);
    const W th = acos(co), sn2 = d1212 * d4242 - d1242 * d1242;
    d = th - (W)nat[2];
    const W pre = (W)2 * (W)cf[3] * d * frsq<W>(sn2);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const W fi = -pre * (v42a[q] - o1242_1212 * v12a[q]), fk = -pre * (v12a[q] - o1242_4242 * v42a[q]);
      fr[0][q] += fi; fr[3][q] += fk; fr[1][q] -= fi + fk;
    }
    ediv += (W)cf[3] * d * d;
  }
  // dihedral 4-2=1=3
  const R3<W> c4212 = crs(v42, v12), c1213 = crs(v12, v13);
  const W c4212_2 = dot(c4212, c4212), c1213_2 = dot(c1213, c1213);
  {
    d = wrap_pi(atan2(dot(v42, c1213) * a12, dot(c4212, c1213)) - (W)nat[3]);
    ediv += (W)cf[4] * d * d;
    const W pre = (W)2 * (W)cf[4] * d * a12;
    const W gi = fdiv<W>(pre, c4212_2), gl = -fdiv<W>(pre, c1213_2);
    const W fi[3] = {gi * c4212.x, gi * c4212.y, gi * c4212.z}, fl[3] = {gl * c1213.x, gl * c1213.y, gl * c1213.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      fr[3][q] += fi[q];
      fr[1][q] += ((W)-1 + o1242_1212) * fi[q] - o1213_1212 * fl[q];
      fr[0][q] += ((W)-1 + o1213_1212) * fl[q] - o1242_1212 * fi[q];
      fr[2][q] += fl[q];
    }
  }
  // dihedral 5-3-1=2
  {
    const R3<W> mm = crs(v53, v13), nn{-c1213.x, -c1213.y, -c1213.z};
    d = wrap_pi(atan2(dot(v53, nn) * a13, dot(mm, nn)) - (W)nat[4]);
    ediv += (W)cf[5] * d * d;
    const W pre = (W)2 * (W)cf[5] * d * a13;
    const W gi = fdiv<W>(pre, dot(mm, mm)), gl = -fdiv<W>(pre, c1213_2);
    const W fi[3] = {gi * mm.x, gi * mm.y, gi * mm.z}, fl[3] = {gl * nn.x, gl * nn.y, gl * nn.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      fr[4][q] += fi[q];
      fr[2][q] += ((W)-1 + o1353_1313) * fi[q] - o1213_1313 * fl[q];
      fr[0][q] += ((W)-1 + o1213_1313) * fl[q] - o1353_1313 * fi[q];
      fr[1][q] += fl[q];
    }
  }
  // dihedral 1=2-4-6
  {
    const R3<W> mm{-c4212.x, -c4212.y, -c4212.z}, nn = crs(v42, v46);
    d = wrap_pi(atan2(dot(v12, nn) * a42, dot(mm, nn)) - (W)nat[5]);
    ediv += (W)cf[6] * d * d;
    const W pre = (W)2 * (W)cf[6] * d * a42;
    const W gi = fdiv<W>(pre, c4212_2), gl = -fdiv<W>(pre, dot(nn, nn));
    const W fi[3] = {gi * mm.x, gi * mm.y, gi * mm.z}, fl[3] = {gl * nn.x, gl * nn.y, gl * nn.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      fr[0][q] += fi[q];
      fr[1][q] += ((W)-1 + o1242_4242) * fi[q] - o4246_4242 * fl[q];
      fr[3][q] += ((W)-1 + o4246_4242) * fl[q] - o1242_4242 * fi[q];
      fr[5][q] += fl[q];
    }
  }
  const W pre = cf[0] / (ediv * ediv);
  const size_t sb = T.slot_tst + 6 * (size_t)k;
#pragma unroll
  for (int p = 0; p < 6; ++p)
    put_slot<Real>(slots, sb + p, m[p], (Real)(pre * fr[p][0]), (Real)(pre * fr[p][1]), (Real)(pre * fr[p][2]));
}

// force_dtrna_stack.F90:54-165 in FP64 whatever Real is, for a stack whose
// dihedrals run through a nearly straight triple: their cross products of
// nearly parallel bond vectors, and force terms that cancel, are resolved by
// FP32 only to ~1e-4 (measured on a C4 chain).
template <typename Real>
__device__ void term_stack64(const KArgs &a, const TopDesc &T, const Smem<Real> &s, const SlotDst &slots, int k, double u0) {
  const int *mp = a.st_idx + 7 * (size_t)(T.st0 + k);
  const int m[7] = {ldro(mp), ldro(mp + 1), ldro(mp + 2), ldro(mp + 3), ldro(mp + 4), ldro(mp + 5), ldro(mp + 6)};
  const double *natp = a.st_nat + 3 * (size_t)(T.st0 + k), *cfp = a.st_coef + 3 * (size_t)(T.st0 + k);
  const double nat[3] = {ldro(natp), ldro(natp + 1), ldro(natp + 2)};
  const double cf[3] = {ldro(cfp), ldro(cfp + 1), ldro(cfp + 2)};
  typedef double W;   // working precision of this term
  auto dv = [&](int i, int j) {   // x_j - x_i (unwrapped), FP64
    return R3<W>{s.X[j] - s.X[i], s.Y[j] - s.Y[i], s.Z[j] - s.Z[i]};
  };
  R3<W> v21 = dv(m[0], m[1]);
  R3<W> v34 = dv(m[3], m[2]);
  R3<W> v54 = dv(m[3], m[4]);
  R3<W> v56 = dv(m[5], m[4]);
  R3<W> v76 = dv(m[5], m[6]);
  const W k1 = cf[0], k2 = cf[1], k3 = cf[2];
  W fr[7][3];
  W ediv = 1;
  W dist = sqrt(dot(v21, v21));
  W dd = dist - (W)nat[0];
  ediv += k1 * dd * dd;
  W g = (W)2 * k1 * fdiv<W>(dd, dist);
  fr[0][0] = -g * v21.x; fr[0][1] = -g * v21.y; fr[0][2] = -g * v21.z;
  fr[1][0] = g * v21.x; fr[1][1] = g * v21.y; fr[1][2] = g * v21.z;
  R3<W> mm = crs(v34, v54), nn = crs(v54, v56);
  W dmm = dot(mm, mm), dnn = dot(nn, nn);
  W d5454 = dot(v54, v54), abs54 = sqrt(d5454);
  W d5654 = dot(v56, v54);
  W d3454o = fdiv<W>(dot(v34, v54), d5454), d5654o = fdiv<W>(d5654, d5454);
  W dih = atan2(dot(v34, nn) * abs54, dot(mm, nn));
  W d = wrap_pi(dih - (W)nat[1]);
  ediv += k2 * d * d;
  W gi = fdiv<W>((W)2 * k2 * d * abs54, dmm), gl = -fdiv<W>((W)2 * k2 * d * abs54, dnn);
  R3<W> fi{gi * mm.x, gi * mm.y, gi * mm.z}, fl{gl * nn.x, gl * nn.y, gl * nn.z};
  const W fiv[3] = {fi.x, fi.y, fi.z}, flv[3] = {fl.x, fl.y, fl.z};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    fr[2][q] = fiv[q];
    fr[3][q] = ((W)-1 + d3454o) * fiv[q] - d5654o * flv[q];
    fr[4][q] = ((W)-1 + d5654o) * flv[q] - d3454o * fiv[q];
    fr[5][q] = flv[q];
    fr[6][q] = 0;
  }
  mm = crs(v76, v56);
  nn.x = -nn.x; nn.y = -nn.y; nn.z = -nn.z;
  dmm = dot(mm, mm);
  W d5656 = dot(v56, v56), abs56 = sqrt(d5656);
  W d7656o = fdiv<W>(dot(v76, v56), d5656), d5456o = fdiv<W>(d5654, d5656);
  dih = atan2(dot(v76, nn) * abs56, dot(mm, nn));
  d = wrap_pi(dih - (W)nat[2]);
  ediv += k3 * d * d;
  gi = fdiv<W>((W)2 * k3 * d * abs56, dmm); gl = -fdiv<W>((W)2 * k3 * d * abs56, dnn);
  const W f2i[3] = {gi * mm.x, gi * mm.y, gi * mm.z}, f2l[3] = {gl * nn.x, gl * nn.y, gl * nn.z};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    fr[6][q] += f2i[q];
    fr[5][q] += ((W)-1 + d7656o) * f2i[q] - d5456o * f2l[q];
    fr[4][q] += -d7656o * f2i[q] + ((W)-1 + d5456o) * f2l[q];
    fr[3][q] += f2l[q];
  }
  const W pre = u0 / (ediv * ediv);
  const size_t sb = T.slot_st + 7 * (size_t)k;
#pragma unroll
  for (int p = 0; p < 7; ++p)
    put_slot<Real>(slots, sb + p, m[p], (Real)(pre * fr[p][0]), (Real)(pre * fr[p][1]), (Real)(pre * fr[p][2]));
}

// force_dtrna_stack.F90:54-165 (skipped when st_status is off).  The FP64
// path evaluates it as written; the mixed path in FP32 unless one of the
// dihedrals' triples is within ~2 degrees of straight (sin^2 < 1e-3), which
// goes to term_stack64
template <typename Real>
__device__ void term_stack(const KArgs &a, const TopDesc &T, const Smem<Real> &s, const SlotDst &slots, int k, double u0) {
  const int *mp = a.st_idx + 7 * (size_t)(T.st0 + k);
  const int m[7] = {ldro(mp), ldro(mp + 1), ldro(mp + 2), ldro(mp + 3), ldro(mp + 4), ldro(mp + 5), ldro(mp + 6)};
  if (stack_excluded<Real>(a, T, s, k)) {
    const size_t sb = T.slot_st + 7 * (size_t)k;
#pragma unroll
    for (int p = 0; p < 7; ++p) put_slot<Real>(slots, sb + p, m[p], 0, 0, 0);
    return;
  }
  const double *natp = a.st_nat + 3 * (size_t)(T.st0 + k), *cfp = a.st_coef + 3 * (size_t)(T.st0 + k);
  const double nat[3] = {ldro(natp), ldro(natp + 1), ldro(natp + 2)};
  const double cf[3] = {ldro(cfp), ldro(cfp + 1), ldro(cfp + 2)};
  R3<Real> v21 = dvec(s, m[0], m[1]);
  R3<Real> v34 = dvec(s, m[3], m[2]);
  R3<Real> v54 = dvec(s, m[3], m[4]);
  R3<Real> v56 = dvec(s, m[5], m[4]);
  R3<Real> v76 = dvec(s, m[5], m[6]);
  if constexpr (sizeof(Real) == 4) {
    const R3<Real> c1 = crs(v34, v54), c2 = crs(v54, v56), c3 = crs(v76, v56);
    const Real l54 = dot(v54, v54), l56 = dot(v56, v56);
    const Real lim = (Real)1e-3;
    if (dot(c1, c1) < lim * dot(v34, v34) * l54 || dot(c2, c2) < lim * l54 * l56 ||
        dot(c3, c3) < lim * dot(v76, v76) * l56) {
      term_stack64<Real>(a, T, s, slots, k, u0);
      return;
    }
  }
  const Real k1 = (Real)cf[0], k2 = (Real)cf[1], k3 = (Real)cf[2];
  Real fr[7][3];
  Real ediv = 1;
  Real dist = sqrt(dot(v21, v21));
  Real dd = dist - (Real)nat[0];
  ediv += k1 * dd * dd;
  Real g = (Real)2 * k1 * fdiv(dd, dist);
  fr[0][0] = -g * v21.x; fr[0][1] = -g * v21.y; fr[0][2] = -g * v21.z;
  fr[1][0] = g * v21.x; fr[1][1] = g * v21.y; fr[1][2] = g * v21.z;
  R3<Real> mm = crs(v34, v54), nn = crs(v54, v56);
  Real dmm = dot(mm, mm), dnn = dot(nn, nn);
  Real d5454 = dot(v54, v54), abs54 = sqrt(d5454);
  Real d5654 = dot(v56, v54);
  Real d3454o = fdiv(dot(v34, v54), d5454), d5654o = fdiv(d5654, d5454);
  Real dih = atan2(dot(v34, nn) * abs54, dot(mm, nn));
  Real d = wrap_pi(dih - (Real)nat[1]);
  ediv += k2 * d * d;
  Real gi = fdiv((Real)2 * k2 * d * abs54, dmm), gl = -fdiv((Real)2 * k2 * d * abs54, dnn);
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
  Real d7656o = fdiv(dot(v76, v56), d5656), d5456o = fdiv(d5654, d5656);
  dih = atan2(dot(v76, nn) * abs56, dot(mm, nn));
  d = wrap_pi(dih - (Real)nat[2]);
  ediv += k3 * d * d;
  gi = fdiv((Real)2 * k3 * d * abs56, dmm); gl = -fdiv((Real)2 * k3 * d * abs56, dnn);
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
  for (int p = 0; p < 7; ++p) put_slot<Real>(slots, sb + p, m[p], pre * fr[p][0], pre * fr[p][1], pre * fr[p][2]);
}

// force_dtrna_hbond15.F90:91-353 (one hbond of the neighbour list).
// Returns the energy; active = |d| <= hb_cutoff_dist.
template <typename Real>
__device__ double term_hbond(const KArgs &a, const TopDesc &T, const Smem<Real> &s, const SlotDst &slots, int k, bool &active) {
  const int *mp = a.hb_idx + 6 * (size_t)(T.hb0 + k);
  const int m[6] = {ldro(mp), ldro(mp + 1), ldro(mp + 2), ldro(mp + 3), ldro(mp + 4), ldro(mp + 5)};
  const double *natp = a.hb_nat + 6 * (size_t)(T.hb0 + k), *cfp = a.hb_coef + 7 * (size_t)(T.hb0 + k);
  double nat[6], cf[7];
#pragma unroll
  for (int q = 0; q < 6; ++q) nat[q] = ldro(natp + q);
#pragma unroll
  for (int q = 0; q < 7; ++q) cf[q] = ldro(cfp + q);
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
  Real g = fdiv((Real)2 * (Real)cf[1] * d, a12);
  fo[0][0] = g * v12.x; fo[0][1] = g * v12.y; fo[0][2] = g * v12.z;
  fo[1][0] = -fo[0][0]; fo[1][1] = -fo[0][1]; fo[1][2] = -fo[0][2];
#pragma unroll
  for (int p = 2; p < 6; ++p) fo[p][0] = fo[p][1] = fo[p][2] = 0;
  Real d1313 = dot(v13, v13), d4242 = dot(v42, v42);
  Real a13 = sqrt(d1313), a42 = sqrt(d4242);
  Real d1213 = dot(v13, v12), d1242 = dot(v12, v42), d4246 = dot(v42, v46), d1353 = dot(v13, v53);
  Real d1213o1212 = fdiv(d1213, d1212), d1213o1313 = fdiv(d1213, d1313), d1242o1212 = fdiv(d1242, d1212);
  Real d4246o4242 = fdiv(d4246, d4242), d1242o4242 = fdiv(d1242, d4242), d1353o1313 = fdiv(d1353, d1313);
  const Real MAXC = (Real)a.max_abscos;
  const Real v12a[3] = {v12.x, v12.y, v12.z}, v13a[3] = {v13.x, v13.y, v13.z}, v42a[3] = {v42.x, v42.y, v42.z};
  // angle 3-1=2 (the |cos| cap keeps acos away from +-1, so FP32 resolves
  // it: the sine is at least that of the cap)
  Real cos312 = fdiv(d1213, a13 * a12);
  if (fabs(cos312) > MAXC) d1213 = copysign(a12 * a13 * MAXC, cos312);
  d = acos(cos312) - (Real)nat[1];
  Real pre = (Real)2 * (Real)cf[2] * d * frsq(d1313 * d1212 - d1213 * d1213);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    Real fi = pre * (v12a[q] - d1213o1313 * v13a[q]);
    Real fk = pre * (v13a[q] - d1213o1212 * v12a[q]);
    fo[2][q] += fi; fo[1][q] += fk; fo[0][q] = fo[0][q] - fi - fk;
  }
  ex -= (Real)cf[2] * d * d;
  // angle 1=2-4
  Real cos124 = fdiv(d1242, a12 * a42);
  if (fabs(cos124) > MAXC) d1242 = copysign(a12 * a42 * MAXC, cos124);
  d = acos(cos124) - (Real)nat[2];
  pre = (Real)2 * (Real)cf[3] * d * frsq(d1212 * d4242 - d1242 * d1242);
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
      Real fi = fdiv(pre, c4212_2) * ca[q], fl = -fdiv(pre, c1213_2) * cb[q];
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
  Real cos531 = fdiv(d1353, a13 * sqrt(dot(v53, v53)));
  if (fabs(cos531) > MAXC) c5313_2 = dot(v53, v53) * d1313 * sin2;
  dih = atan2(dot(v53, n) * a13, dot(c5313, n));
  d = wrap_pi(dih - (Real)nat[4]);
  ex -= (Real)cf[5] * d * d;
  pre = (Real)2 * (Real)cf[5] * d * a13;
  {
    const Real ca[3] = {c5313.x, c5313.y, c5313.z}, cb[3] = {n.x, n.y, n.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Real fi = fdiv(pre, c5313_2) * ca[q], fl = -fdiv(pre, c1213_2) * cb[q];
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
  Real cos246 = fdiv(d4246, a42 * sqrt(dot(v46, v46)));
  if (fabs(cos246) > MAXC) c4246_2 = dot(v46, v46) * d4242 * sin2;
  dih = atan2(dot(v12, c4246) * a42, dot(n, c4246));
  d = wrap_pi(dih - (Real)nat[5]);
  ex -= (Real)cf[6] * d * d;
  pre = (Real)2 * (Real)cf[6] * d * a42;
  {
    const Real ca[3] = {n.x, n.y, n.z}, cb[3] = {c4246.x, c4246.y, c4246.z};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Real fi = fdiv(pre, c4212_2) * ca[q], fl = -fdiv(pre, c4246_2) * cb[q];
      fo[0][q] += fi;
      fo[1][q] += ((Real)-1 + d1242o4242) * fi - d4246o4242 * fl;
      fo[3][q] += ((Real)-1 + d4246o4242) * fl - d1242o4242 * fi;
      fo[5][q] += fl;
    }
  }
  const Real e = (Real)cf[0] * exp(ex);
  const double ene = (double)e;
  const size_t sb = T.slot_hb + 6 * (size_t)k;
#pragma unroll
  for (int p = 0; p < 6; ++p) put_slot<Real>(slots, sb + p, m[p], e * fo[p][0], e * fo[p][1], e * fo[p][2]);
  return ene;
}

// force_dtrna_hbond15.F90:373-509, run by one thread of the lane
template <typename Real>
__device__ void prune_hbonds(const KArgs &a, int lane, const LaneDesc &L, const TopDesc &T, long long istep,
                             double beta, bool zero_energy, int *exc) {
  uint8_t *hbf = a.hb_flag + L.hb0;
  double *ene = a.hb_ene + L.hb0;
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

} // namespace tis
