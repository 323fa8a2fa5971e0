// lane_kernel.cu -- persistent force-and-integrate kernel, one CTA per lane.
//
// Each CTA keeps its lane's coordinates, velocities and accelerations in
// shared memory for the whole launch and runs the reference step
// (src/time_integral.F90:57-190) nsteps times without leaving the SM:
//
//   neighbour trigger -> [rebuild the list bit matrices] -> x update ->
//   phase 1: hbonds, stacks, Debye-Hueckel row chunks, angles, bonds
//            (one balanced sweep, most expensive items first) ->
//   [valence pruning] ->
//   phase 2: per bead, exv pairs + bonded slots + Debye-Hueckel partials,
//            summed in FP64, then the v / a update.
//
// Real = double is the plain FP64 path; Real = float computes pair and
// bonded forces in FP32 and accumulates each bead's force in FP64 (state,
// integration and neighbour decisions are FP64 in both).
//
// Determinism: each bead sums its contributions in a fixed order (bits of its
// rows in ascending j, its incidence list in slot order, its Debye-Hueckel
// chunks in order) and the threads of a bead group combine their partial
// sums with a fixed xor-butterfly, so results do not depend on scheduling.
// Neighbour pair sets are bit-exact with the reference: the FP64 distance
// test uses explicitly rounded operations in the Fortran order.
#include <cooperative_groups.h>

#include "device_common.cuh"

namespace tis {

namespace cg = cooperative_groups;

// Split of one lane over the CTAs of its cluster: this CTA owns beads
// [lo, hi) (their x / v / a updates, list rows, near lists, force sums).
// nrank == 1: one CTA per lane, owns every bead.
struct Clu {
  int rank, nrank;
  int lo, hi;
  int kq_lo, kq_hi;   // charged rows (electrostatic chunks) of the own beads
};

// the same shared-memory object in the other CTA of a two-CTA cluster
template <typename T>
__device__ __forceinline__ T *peer_ptr(T *p, const Clu &cu) {
  return cg::this_cluster().map_shared_rank(p, cu.rank ^ 1);
}

// ------------------------------------------------------------ skin rule
// time_integral.F90:57-93: rebuild when sqrt(d2max) + sqrt(d2max_2nd) >
// neigh_margin, d2 = dot_product(dxyz_mp, dxyz_mp) of each bead.  The pair
// (d2max, d2max_2nd) is the top two of the multiset of d2 values, so partial
// results merge exactly in any order: each warp folds its beads, every warp
// then folds the per-warp pairs (of both CTAs of a cluster) and reaches the
// same decision without another barrier.
__device__ __forceinline__ void top2_add(double &m1, double &m2, double d2) {
  if (d2 > m1) { m2 = m1; m1 = d2; } else if (d2 > m2) m2 = d2;
}
__device__ __forceinline__ void top2_merge(double &m1, double &m2, double o1, double o2) {
  const double n1 = fmax(m1, o1), n2 = fmax(fmin(m1, o1), fmax(m2, o2));
  m1 = n1; m2 = n2;
}
__device__ __forceinline__ void top2_warp(double &m1, double &m2) {
  for (int o = 16; o > 0; o >>= 1) {
    const double o1 = __shfl_xor_sync(0xffffffffu, m1, o), o2 = __shfl_xor_sync(0xffffffffu, m2, o);
    top2_merge(m1, m2, o1, o2);
  }
}
// dot_product(dxyz, dxyz) in the Fortran operation order, no contraction
__device__ __forceinline__ double disp2(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}
// per-warp pair of this thread's (m1, m2) into red[2 w], red[2 w + 1]; every
// thread of the CTA calls it
__device__ __forceinline__ void top2_store(double m1, double m2, double *red) {
  top2_warp(m1, m2);
  if ((threadIdx.x & 31) == 0) { red[2 * (threadIdx.x >> 5)] = m1; red[2 * (threadIdx.x >> 5) + 1] = m2; }
}
// sqrt(d2max) + sqrt(d2max_2nd) > margin from every lane's pair (the
// decision is the same in every lane)
__device__ __forceinline__ bool skin_decide(double m1, double m2, double margin) {
  top2_warp(m1, m2);
  // FP32 screen: the float sum is within ~4e-7 (relative) of the FP64 one,
  // so outside a 1e-4 band around the margin it decides the same way
  const float sf = sqrtf((float)m1) + sqrtf((float)m2), mf = (float)margin;
  if (sf < mf * 0.9999f) return false;
  if (sf > mf * 1.0001f) return true;
  return __dadd_rn(sqrt(m1), sqrt(m2)) > margin;
}
// The trigger from the d2 of every bead (DD) and M, their maximum rounded
// up to float: M rules the skin out while 2 sqrt(M) is 1e-4 below the
// margin (sqrt(d2max) + sqrt(d2max_2nd) <= 2 sqrt(M)); else every warp
// takes the top two d2 of DD.  Every thread reaches the same decision.
__device__ __forceinline__ bool skin_trigger(int Mbits, const double *DD, int N, double margin) {
  const float M = __int_as_float(Mbits);
  if (2.0f * sqrtf(M) < (float)margin * 0.9999f) return false;
  double m1 = 0.0, m2 = 0.0;
  for (int b = (threadIdx.x & 31); b < N; b += 32) top2_add(m1, m2, DD[b]);
  return skin_decide(m1, m2, margin);
}
// the trigger from the per-warp pairs of this CTA (lanes 0 .. nwarp - 1) and,
// with two CTAs, of the other one (lanes 16 .. 16 + nwarp - 1, nwarp <= 16)
__device__ __forceinline__ bool skin_fires(const double *red, const double *peer_red, int nwarp, double margin) {
  const int lid = threadIdx.x & 31;
  double m1 = 0.0, m2 = 0.0;
  if (lid < nwarp) { m1 = red[2 * lid]; m2 = red[2 * lid + 1]; }
  else if (peer_red && lid >= 16 && lid - 16 < nwarp) { m1 = peer_red[2 * (lid - 16)]; m2 = peer_red[2 * (lid - 16) + 1]; }
  return skin_decide(m1, m2, margin);
}

// a b + c d of the integration: in the FP64 path each product rounded as
// the reference evaluates it (no contraction), so the update is the
// reference's to the last bit; the mixed path lets the compiler contract
template <typename Real>
__device__ __forceinline__ double mad2(double a, double b, double c, double d) {
  if constexpr (sizeof(Real) == 8) return __dadd_rn(__dmul_rn(a, b), __dmul_rn(c, d));
  else return a * b + c * d;
}
template <typename Real>
__device__ __forceinline__ double add_rn(double a, double b) {
  if constexpr (sizeof(Real) == 8) return __dadd_rn(a, b);
  else return a + b;
}

// ------------------------------------------------------------ list build
constexpr int CELL_MIN = 384;   // beads of a one-CTA lane from which the build bins them
// neighbor_list.F90:49-90 + neighbor_assign.F90:481-559 (the EXV_DT15 type
// sort keeps the generation order) and neighbor_list_ele.F90:123-210: every
// unordered pair is tested once and sets its bit in both rows of the exv
// and/or ele matrix.  Periodic systems also record the mirror index of the
// canonical (min, max) orientation (neighbor_assign.F90:742-770).
__device__ __forceinline__ void rebuild_counts(LaneState &st, int nexv, int nele, long long istep) {
  st.nrebuild++;
  st.last_rebuild = istep;
  st.nexv = nexv;
  st.nele = nele;
}

template <typename Real, int CL>
__device__ void build_lists(const KArgs &a, int lane, const LaneDesc &L, const TopDesc &T, Smem<Real> &s,
                            const Clu &cu, long long istep) {
  const int N = T.nmp, W = s.W;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int warp = tid >> 5, lid = tid & 31, nwarp = nth >> 5;
  LaneState &st = a.lstate[lane];
  uint32_t *mexv = s.mask;
  uint32_t *mele = mexv + (size_t)N * W;
  // wrap pxyz (util_periodic.F90)
  if (a.periodic) {
    for (int i = tid; i < N; i += nth) {
      s.PX[i] = wrap1(s.PX[i], a.psize[0]);
      s.PY[i] = wrap1(s.PY[i], a.psize[1]);
      s.PZ[i] = wrap1(s.PZ[i], a.psize[2]);
      s.QX[i] = s.PX[i]; s.QY[i] = s.PY[i]; s.QZ[i] = s.PZ[i];
      set_pos<Real>(s, i);
    }
  }
  if (CL == 1) {
    for (int k = tid; k < 2 * N * W; k += nth) mexv[k] = 0u;
  } else {
    // own rows only: the other CTA writes its own rows (and, with a global
    // matrix, nothing else) before the barrier below
    const int nw = (cu.hi - cu.lo) * W;
    for (int k = tid; k < nw; k += nth) {
      mexv[(size_t)cu.lo * W + k] = 0u;
      mele[(size_t)cu.lo * W + k] = 0u;
    }
  }
  if (tid == 0) {
    s.misc[MISC_NEXV] = 0; s.misc[MISC_NELE] = 0; s.misc[MISC_REBUILT] = 1;
    s.misc[MISC_NEAR_BAD] = 1;
  }
  // unit prescreen (neighbor_pre.F90:174-252), thread 0
  const int nu = T.nunit;
  int *nunit_ok = s.misc + MISC_UNITS;
  if (tid == 0 && nu == 1) {
    nunit_ok[0] = 1;
  } else if (tid == 0) {
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
          ok = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) < md[u] + md[v] + sqrt(s.rn2[u * nu + v]);
        }
        nunit_ok[u * nu + v] = ok;
        nunit_ok[v * nu + u] = ok;
      }
  }
  __syncthreads();
  const double rele2 = (a.i_ele != 0) ? a.lab_rele2[st.label] : -1.0;
  uint8_t *mir = a.periodic ? (a.mirror + L.mirror0) : nullptr;
  int nexv_l = 0, nele_l = 0;
  // two CTAs: every row must be cleared before either CTA sets bits in it
  uint32_t *pexv = mexv, *pele = mele;
  if (CL == 2) {
    cg::this_cluster().sync();
    if (s.mask_smem) { pexv = peer_ptr(mexv, cu); pele = peer_ptr(mele, cu); }
  }
  PHASE_T0(t_pairs);
  const bool one_unit = nu == 1;
  const double rn2_00 = s.rn2[0];
  // the pair test of row i, partner j > i
  auto pair = [&](int i, int j, int ui, int ci, int nsep, double xi, double yi, double zi, bool qi) {
    const int uj = one_unit ? 0 : s.unit[j];
    if (!one_unit && !nunit_ok[ui * nu + uj]) return;
    double v0 = __dsub_rn(s.PX[j], xi), v1 = __dsub_rn(s.PY[j], yi), v2 = __dsub_rn(s.PZ[j], zi);
    int im = 27;
    if (a.periodic) {
      int m0 = pb1(v0, a.psize[0], a.psizeh[0]);
      int m1 = pb1(v1, a.psize[1], a.psizeh[1]);
      int m2 = pb1(v2, a.psize[2], a.psizeh[2]);
      im = 9 * m0 + 3 * m1 + m2 + 1;
    }
    const double d2 = __dadd_rn(__dadd_rn(sqr_rn(v0), sqr_rn(v1)), sqr_rn(v2));
    bool ex = d2 < (one_unit ? rn2_00 : s.rn2[ui * nu + uj]);
    const bool el = qi && fabs((double)s.A4[j].w) >= 1.0e-6 && d2 < rele2;
    if (ex) {
      if (ui == uj) {
        if (ci == 2 /* RNA */ && j < i + nsep) ex = false;
      } else {
        const int cj = s.cls[j];
        if (!((ci == 2 && cj == 2) || (ci == 2 && cj == 4) || (ci == 4 && cj == 2) ||
              (ci == 4 && cj == 3) || (ci == 3 && cj == 4)))
          ex = false;
        else if (a.dt19 && ((ci == 2 && cj == 4) || (ci == 4 && cj == 2))) {
          // neighbor_assign.F90:524-537: no exv between a charged phosphate and an ion
          const int pb = (s.typ[i] == 2) ? i : ((s.typ[j] == 2) ? j : -1);
          if (pb >= 0 && fabs((double)s.A4[pb].w) > 1.0e-6) ex = false;
        }
      }
    }
    if (ex || el) {
      const uint32_t bj = 1u << (j & 31), bi = 1u << (i & 31);
      const bool own_i = CL == 1 || (i >= cu.lo && i < cu.hi);
      const bool own_j = CL == 1 || (j >= cu.lo && j < cu.hi);
      if (ex) {
        atomicOr(&(own_i ? mexv : pexv)[(size_t)i * W + (j >> 5)], bj);
        atomicOr(&(own_j ? mexv : pexv)[(size_t)j * W + (i >> 5)], bi);
        ++nexv_l;
      }
      if (el) {
        atomicOr(&(own_i ? mele : pele)[(size_t)i * W + (j >> 5)], bj);
        atomicOr(&(own_j ? mele : pele)[(size_t)j * W + (i >> 5)], bi);
        ++nele_l;
      }
      if (mir) mir[(size_t)i * N + j] = (uint8_t)im;
    }
  };
  auto nsep_of = [&](int i) {
    return (s.typ[i] == 2) ? a.nsep[0] : (s.typ[i] == 4 ? a.nsep[1] : (s.typ[i] == 3 ? a.nsep[2] : -1));
  };
  auto q_of = [&](int i) { return a.i_ele != 0 && fabs((double)s.A4[i].w) >= 1.0e-6; };
  // ---- cell list (one CTA, large lanes): bins at least as wide as the
  // largest list cutoff, so a pair within it lies in the same or a
  // neighbouring bin (across the box when periodic); a row tests only the
  // beads of the 27 bins around its own.  The test is the all-pairs one, so
  // are the lists.  Scratch: the Debye-Hueckel partials, unused while the
  // lists are built.
  int *cl = (int *)s.ch_part;
  int nb[3] = {0, 0, 0};
  double blo[3] = {0, 0, 0}, bw[3] = {1, 1, 1};
  bool cells = false;
  if (CL == 1 && N >= CELL_MIN) {
    double rc2 = rele2;
    for (int k = 0; k < nu * nu; ++k) rc2 = fmax(rc2, s.rn2[k]);
    const double wmin = sqrt(rc2) * (1.0 + 1.0e-9) + 1.0e-9;
    double ext[3];
    if (a.periodic) {
      for (int d = 0; d < 3; ++d) { blo[d] = -a.psizeh[d]; ext[d] = a.psize[d]; }
    } else {
      // bounding box of the lane: per-warp extremes, then every thread
      double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
      for (int i = tid; i < N; i += nth) {
        const double q[3] = {s.PX[i], s.PY[i], s.PZ[i]};
        for (int d = 0; d < 3; ++d) { mn[d] = fmin(mn[d], q[d]); mx[d] = fmax(mx[d], q[d]); }
      }
      for (int o = 16; o > 0; o >>= 1)
        for (int d = 0; d < 3; ++d) {
          mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
          mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
      double *red = (double *)cl;
      if (lid == 0)
        for (int d = 0; d < 3; ++d) { red[d * 32 + warp] = mn[d]; red[(3 + d) * 32 + warp] = mx[d]; }
      __syncthreads();
      for (int d = 0; d < 3; ++d) {
        for (int w = 0; w < nwarp; ++w) { mn[d] = fmin(mn[d], red[d * 32 + w]); mx[d] = fmax(mx[d], red[(3 + d) * 32 + w]); }
        blo[d] = mn[d];
        ext[d] = mx[d] - mn[d];
      }
      __syncthreads();   // red is overwritten below
    }
    // bins of width >= wmin, widened until their tables fit the scratch
    const long long room = 6 * CHMAX - 1 - N - 56 * nwarp;
    double w = wmin;
    for (int tries = 0; tries < 40 && !cells; ++tries, w *= 1.25) {
      long long ncell = 1;
      bool ok = true;
      for (int d = 0; d < 3; ++d) {
        const double nf = floor(ext[d] / w) + (a.periodic ? 0.0 : 1.0);
        nb[d] = nf < 1.0 ? 1 : (nf > 4096.0 ? 4096 : (int)nf);
        bw[d] = a.periodic ? ext[d] / nb[d] : w;
        if (a.periodic && nb[d] < 3) ok = false;   // neighbouring bins must be distinct
        ncell *= nb[d];
      }
      if (!ok || ncell <= 27) break;   // too few bins to gain over the all-pairs scan
      cells = 2 * ncell <= room;
    }
  }
  if (cells) {
    const int ncell = nb[0] * nb[1] * nb[2];
    int *start = cl, *fill = cl + ncell + 1, *cb = fill + ncell, *wsc = cb + N;
    auto bin_of = [&](int i, int &x, int &y, int &z) {
      x = min(max((int)floor((s.PX[i] - blo[0]) / bw[0]), 0), nb[0] - 1);
      y = min(max((int)floor((s.PY[i] - blo[1]) / bw[1]), 0), nb[1] - 1);
      z = min(max((int)floor((s.PZ[i] - blo[2]) / bw[2]), 0), nb[2] - 1);
    };
    for (int k = tid; k <= ncell; k += nth) start[k] = 0;
    __syncthreads();
    for (int i = tid; i < N; i += nth) {
      int x, y, z;
      bin_of(i, x, y, z);
      atomicAdd(&start[(z * nb[1] + y) * nb[0] + x + 1], 1);
    }
    __syncthreads();
    if (warp == 0) {   // inclusive scan: start[c] = first slot of bin c, start[ncell] = N
      const int seg = (ncell + 1 + 31) / 32, k0 = lid * seg, k1 = min(k0 + seg, ncell + 1);
      int sum = 0;
      for (int k = k0; k < k1; ++k) sum += start[k];
      int incl = sum;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lid >= o) incl += t;
      }
      int run = incl - sum;
      for (int k = k0; k < k1; ++k) { run += start[k]; start[k] = run; }
    }
    __syncthreads();
    for (int c = tid; c < ncell; c += nth) fill[c] = start[c];
    __syncthreads();
    for (int i = tid; i < N; i += nth) {
      int x, y, z;
      bin_of(i, x, y, z);
      cb[atomicAdd(&fill[(z * nb[1] + y) * nb[0] + x], 1)] = i;
    }
    __syncthreads();
    int *wp = wsc + 56 * warp;   // per warp: 28 candidate offsets, 27 bin starts
    for (int i = warp; i < N - 1; i += nwarp) {
      int x, y, z;
      bin_of(i, x, y, z);
      int n_l = 0, st_l = 0;
      if (lid < 27) {
        int bx = x + lid % 3 - 1, by = y + (lid / 3) % 3 - 1, bz = z + lid / 9 - 1;
        bool in = true;
        if (a.periodic) {
          bx = (bx + nb[0]) % nb[0]; by = (by + nb[1]) % nb[1]; bz = (bz + nb[2]) % nb[2];
        } else {
          in = bx >= 0 && bx < nb[0] && by >= 0 && by < nb[1] && bz >= 0 && bz < nb[2];
        }
        if (in) {
          const int c = (bz * nb[1] + by) * nb[0] + bx;
          st_l = start[c];
          n_l = start[c + 1] - st_l;
        }
      }
      int incl = n_l;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lid >= o) incl += t;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      if (lid < 28) wp[lid] = incl - n_l;
      if (lid < 27) wp[28 + lid] = st_l;
      __syncwarp();
      const int ui = s.unit[i], ci = s.cls[i], nsep = nsep_of(i);
      const double xi = s.PX[i], yi = s.PY[i], zi = s.PZ[i];
      const bool qi = q_of(i);
      for (int k = lid; k < total; k += 32) {
        int b = 0;   // the last bin whose candidates start at or before k
        for (int st = 16; st > 0; st >>= 1)
          if (b + st < 27 && wp[b + st] <= k) b += st;
        const int j = cb[wp[28 + b] + k - wp[b]];
        if (j > i) pair(i, j, ui, ci, nsep, xi, yi, zi, qi);
      }
      __syncwarp();
    }
  } else {
    // every pair: warp w takes rows i = w, w + nwarp, ...; its lanes take
    // j > i (two CTAs: CTA r takes the rows of parity r and sets each bit
    // in the copy of the row's owner)
    const int rstep = nwarp * CL;
    for (int i = warp * CL + cu.rank; i < N - 1; i += rstep) {
      const int ui = s.unit[i], ci = s.cls[i], nsep = nsep_of(i);
      const double xi = s.PX[i], yi = s.PY[i], zi = s.PZ[i];
      const bool qi = q_of(i);
      for (int j = i + 1 + lid; j < N; j += 32) pair(i, j, ui, ci, nsep, xi, yi, zi, qi);
    }
  }
  if (nexv_l) atomicAdd(&s.misc[MISC_NEXV], nexv_l);
  if (nele_l) atomicAdd(&s.misc[MISC_NELE], nele_l);
  PHASE_ADD(7, t_pairs);
  // hbond neighbour flags (neighbor_list_hb.F90:335-354); two CTAs: the
  // first one, which evaluates every hbond
  uint8_t *hbf = a.hb_flag + L.hb0;
  for (int h = tid; h < (cu.rank == 0 ? T.nhb : 0); h += nth) {
    const int *m = a.hb_idx + 6 * (size_t)(T.hb0 + h);
    double v0, v1, v2;
    v0 = __dsub_rn(s.PX[m[0]], s.PX[m[1]]);
    v1 = __dsub_rn(s.PY[m[0]], s.PY[m[1]]);
    v2 = __dsub_rn(s.PZ[m[0]], s.PZ[m[1]]);
    if (a.periodic) { pb1(v0, a.psize[0], a.psizeh[0]); pb1(v1, a.psize[1], a.psizeh[1]); pb1(v2, a.psize[2], a.psizeh[2]); }
    double d2 = __dadd_rn(__dadd_rn(sqr_rn(v0), sqr_rn(v1)), sqr_rn(v2));
    hbf[h] = (d2 < a.hb_nd2[T.hb0 + h]) ? 1 : 0;
  }
  // one CTA: the lists and counts are complete after this barrier; two CTAs:
  // the rows are read only after the step's next cluster barrier, after
  // which the first CTA adds up both counts (rebuild_counts)
  if (CL == 1) {
    __syncthreads();
    if (tid == 0) rebuild_counts(st, s.misc[MISC_NEXV], s.misc[MISC_NELE], istep);
  }
}

// ------------------------------------------------------------ force pass
// exp for the Debye-Hueckel factor: FP64 in the FP64 path; the fast
// single-precision exponential in the mixed path (relative error about
// |x| 2^-22 for the arguments here, |x| <= 25)
template <typename Real> __device__ __forceinline__ Real fexp(Real x);
template <> __device__ __forceinline__ double fexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float fexp<float>(float x) { return __expf(x); }

template <typename Real>
__device__ __forceinline__ void group_reduce(double &fx, double &fy, double &fz, int G) {
  for (int o = G >> 1; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o, G);
    fy += __shfl_xor_sync(0xffffffffu, fy, o, G);
    fz += __shfl_xor_sync(0xffffffffu, fz, o, G);
  }
}

__device__ __forceinline__ int pow2_floor_clamp(int x, int hi) {
  int g = 1;
  while (g * 2 <= x && g * 2 <= hi) g *= 2;
  return g;
}

// Periodic image of the pair fixed at the last rebuild (d_mirror(:, imirror)
// of the canonical (min, max) orientation, negated for the reverse one),
// recomputed from the positions wrapped at that rebuild with the same
// rounded FP64 operations as the list build: the same image as its mirror
// table, without a global-memory lookup.
template <typename T, typename S>
__device__ __forceinline__ void mirror_shift(const KArgs &a, const S &s, int i, int j, T &w0, T &w1, T &w2) {
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  const T sg = (j > i) ? (T)1 : (T)-1;
  const double v0 = __dsub_rn(s.QX[hi], s.QX[lo]), v1 = __dsub_rn(s.QY[hi], s.QY[lo]),
               v2 = __dsub_rn(s.QZ[hi], s.QZ[lo]);
  if (v0 > a.psizeh[0]) w0 -= sg * (T)a.psize[0]; else if (v0 < -a.psizeh[0]) w0 += sg * (T)a.psize[0];
  if (v1 > a.psizeh[1]) w1 -= sg * (T)a.psize[1]; else if (v1 < -a.psizeh[1]) w1 += sg * (T)a.psize[1];
  if (v2 > a.psizeh[2]) w2 -= sg * (T)a.psize[2]; else if (v2 < -a.psizeh[2]) w2 += sg * (T)a.psize[2];
}

template <typename Real> __device__ __forceinline__ Real rsq(Real x);
template <> __device__ __forceinline__ double rsq<double>(double x) { return 1.0 / sqrt(x); }
template <> __device__ __forceinline__ float rsq<float>(float x) { return rsqrtf(x); }

// Debye-Hueckel chunk geometry: charged row k is cut into cpr chunks of gw
// words of its ele bit row; chunk c covers row c / cpr.
struct ChunkGeo { int cpr, gw, nch; };
__device__ __forceinline__ ChunkGeo chunk_geo(int NQ, int W) {
  ChunkGeo g;
  int cpr = NQ > 0 ? CHMAX / NQ : 1;
  if (cpr < 1) cpr = 1;
  if (cpr > W) cpr = W;
  g.gw = (W + cpr - 1) / cpr;
  g.cpr = (W + g.gw - 1) / g.gw;
  g.nch = NQ * g.cpr;
  return g;
}

// Items of the bonded sweep of this CTA, [x0, x1) per kind (all of them
// for one CTA per lane; with two CTAs every hbond goes to the first one, as
// the valence pruning that may follow is serial, the rows of the own
// charged beads, and halves of the stacks, angles and bonds), cut into
// chunks of 32 items of one kind, and dealt to the warps in one of three
// ways (sweep_mode; two CTAs per lane always take the first):
//  0  chunks numbered hbonds (two CTAs), stacks, tertiary stacks,
//     Debye-Hueckel row chunks, angles, hbonds (one CTA), bonds, noise --
//     kinds in measured cost order, with a formed hbond the longest serial
//     chain -- and round r gives chunk r nwarp + w to warp w (r even) or to
//     warp nwarp - 1 - w (r odd), so the costly first chunks and the cheap
//     last ones even out over the warps and the SM's four schedulers;
//  1  tertiary stacks (FP64), Debye-Hueckel chunks, stacks, hbonds, angles,
//     bonds, noise -- longest first -- each warp taking the next chunk from
//     a shared counter as it finishes one;
//  2  the numbering of 0, dealt once per launch by sweep_deal.
// Measured on B200: 0 for C3 (one or two chunks per warp, where the cost of
// an hbond chunk depends on how many hbonds are formed), 1 and 2 for
// C4's long chains (many chunks per warp).
struct Sweep {
  int hb_0, hb_1, st_0, st_1, ts_0, ts_1, ch_0, ch_1, ba_0, ba_1, bd_0, bd_1, nz_0, nz_1;
  int c_hb, c_st, c_ts, c_ch, c_ba, c_bd, c_nz, c_end;
  int n_hbc, n_stc, n_tsc, n_chc, n_bac, n_bdc, n_nzc;
};

template <int CL>
__device__ __forceinline__ Sweep sweep_plan(const KArgs &a, const TopDesc &T, const Clu &cu, int nch, int cpr,
                                            bool noise, bool dyn) {
  Sweep w;
  const int nhb = T.nhb, nst = T.nst, nba = T.nba, nbd = T.nbd, ntst = T.ntst;
  w.hb_0 = 0; w.hb_1 = nhb; w.st_0 = 0; w.st_1 = nst; w.ts_0 = 0; w.ts_1 = ntst;
  w.ch_0 = 0; w.ch_1 = nch; w.ba_0 = 0; w.ba_1 = nba; w.bd_0 = 0; w.bd_1 = nbd;
  if (CL == 2) {
    if (cu.rank == 1) w.hb_1 = 0;
    w.st_0 = cu.rank ? nst / 2 : 0; w.st_1 = cu.rank ? nst : nst / 2;
    w.ts_0 = cu.rank ? ntst / 2 : 0; w.ts_1 = cu.rank ? ntst : ntst / 2;
    w.ba_0 = cu.rank ? nba / 2 : 0; w.ba_1 = cu.rank ? nba : nba / 2;
    w.bd_0 = cu.rank ? nbd / 2 : 0; w.bd_1 = cu.rank ? nbd : nbd / 2;
    w.ch_0 = nch ? cu.kq_lo * cpr : 0; w.ch_1 = nch ? cu.kq_hi * cpr : 0;
  }
  w.nz_0 = cu.lo; w.nz_1 = noise ? cu.hi : cu.lo;
  w.n_hbc = (w.hb_1 - w.hb_0 + 31) >> 5; w.n_stc = (w.st_1 - w.st_0 + 31) >> 5;
  w.n_tsc = (w.ts_1 - w.ts_0 + 31) >> 5; w.n_chc = (w.ch_1 - w.ch_0 + 31) >> 5;
  w.n_bac = (w.ba_1 - w.ba_0 + 31) >> 5; w.n_bdc = (w.bd_1 - w.bd_0 + 31) >> 5;
  w.n_nzc = (w.nz_1 - w.nz_0 + 31) >> 5;
  if (dyn) {
    w.c_ts = 0; w.c_ch = w.c_ts + w.n_tsc; w.c_st = w.c_ch + w.n_chc; w.c_hb = w.c_st + w.n_stc;
    w.c_ba = w.c_hb + w.n_hbc; w.c_bd = w.c_ba + w.n_bac; w.c_nz = w.c_bd + w.n_bdc;
  } else {
    w.c_st = (CL == 2) ? w.n_hbc : 0; w.c_ts = w.c_st + w.n_stc; w.c_ch = w.c_ts + w.n_tsc;
    w.c_ba = w.c_ch + w.n_chc; w.c_hb = (CL == 2) ? 0 : w.c_ba + w.n_bac;
    w.c_bd = w.c_ba + w.n_bac + ((CL == 2) ? 0 : w.n_hbc); w.c_nz = w.c_bd + w.n_bdc;
  }
  w.c_end = w.c_nz + w.n_nzc;
  return w;
}

// The fixed deal (thread 0, once per launch): chunks in decreasing
// estimated latency -- per kind, relative to a bond chunk (measured on
// B200): tertiary stack 16, stack 9, Debye-Hueckel 1 + 10 per word of a
// row, hbond and angle 5, bond 4, noise 3 -- each to the warp with
// the least estimated load (ties: the least loaded of the SM's four
// schedulers, then the lowest warp); warp w's chunks are
// sched[33 + sched[w] .. 33 + sched[w + 1]).
__device__ void sweep_deal(const Sweep &w, int gw, int nwarp, int16_t *sched, int cap) {
  struct K { int c0, n, wt; } k[7] = {{w.c_ts, w.n_tsc, 16}, {w.c_st, w.n_stc, 9}, {w.c_ch, w.n_chc, 1 + 10 * gw},
                                      {w.c_hb, w.n_hbc, 5},  {w.c_ba, w.n_bac, 5},  {w.c_bd, w.n_bdc, 4},
                                      {w.c_nz, w.n_nzc, 3}};
  for (int x = 1; x < 7; ++x)   // stable insertion sort by weight, descending
    for (int y = x; y > 0 && k[y].wt > k[y - 1].wt; --y) { K t = k[y]; k[y] = k[y - 1]; k[y - 1] = t; }
  int load[32], cnt[33], sm[4] = {0, 0, 0, 0};
  for (int v = 0; v < 32; ++v) { load[v] = 0; cnt[v] = 0; }
  int16_t *asg = sched + 33 + cap;   // warp of each chunk id
  const int nc = w.c_end < cap ? w.c_end : cap;
  for (int x = 0; x < 7; ++x)
    for (int c = k[x].c0; c < k[x].c0 + k[x].n && c < nc; ++c) {
      int best = 0;
      for (int v = 1; v < nwarp; ++v)
        if (load[v] < load[best] || (load[v] == load[best] && sm[v & 3] < sm[best & 3])) best = v;
      load[best] += k[x].wt; sm[best & 3] += k[x].wt; ++cnt[best];
      asg[c] = (int16_t)best;
    }
  int o = 0;
  for (int v = 0; v < nwarp; ++v) { sched[v] = (int16_t)o; o += cnt[v]; cnt[v] = sched[v]; }
  sched[nwarp] = (int16_t)o;
  // each warp's chunks in the order the deal gave them (longest first)
  for (int x = 0; x < 7; ++x)
    for (int c = k[x].c0; c < k[x].c0 + k[x].n && c < nc; ++c) sched[33 + cnt[asg[c]]++] = (int16_t)c;
}

// Phase 1 runs every interaction-level item in one balanced sweep: stacks,
// tertiary stacks, Debye-Hueckel chunks (force_ele_DH.F90:72-117 over a word range of one
// charged bead's ele row, summed by one thread into ch_part), angles,
// hbonds, bonds.  Phase 2 gives each bead a group of GA
// threads that sums its exv pairs, its bonded slots and its Debye-Hueckel
// chunk partials; the group's owner thread hands the FP64 total to `sink`.
struct NoFin {
  __device__ void operator()(int) const {}
};

template <typename Real, int CL, typename Sink, typename Fin = NoFin>
__device__ void force_pass(const KArgs &a, int lane, const LaneDesc &L, const TopDesc &T, Smem<Real> &s,
                           long long istep, const Clu &cu, int noise_step, Sink sink, int par = 0, Fin fin = Fin()) {
  typedef typename V4<Real>::T V;
  const int N = T.nmp, NQ = T.nq, W = s.W;
  const int tid = threadIdx.x, nth = blockDim.x;
  LaneState &st = a.lstate[lane];
  const int label = st.label;
  // slots of beads owned by the other CTA go to its copy (one global array
  // when the slots do not fit shared memory)
  const SlotDst slots{s.slots, (CL == 2 && s.slots_smem) ? (void *)peer_ptr(s.slots, cu) : nullptr, cu.lo, cu.hi};
  const Real *my_slots = s.slots;
  uint8_t *hbf = a.hb_flag + L.hb0;
  double *hbe = a.hb_ene + L.hb0;
  int *exc = s.exc;
  const uint32_t *mexv = s.mask, *mele = s.mask + (size_t)N * W;
  const uint8_t *mir = a.periodic ? (a.mirror + L.mirror0) : nullptr;
  int nclamp = 0;
  // (site counters and this step's MISC_EXCESS copy were cleared by the
  // caller before its barrier; par selects the copies of this step)
  const int f_exc = MISC_EXCESS + par, f_disp = MISC_NEAR_DISP + par;
  const int nhb = T.nhb, nst = T.nst, nba = T.nba, nbd = T.nbd, ntst = T.ntst;
  const ChunkGeo geo = chunk_geo(NQ, W);
  const int nch = (a.i_ele != 0) ? geo.nch : 0;
  const int k_st = nhb, k_ch = k_st + nst, k_ba = k_ch + nch, k_bd = k_ba + nba, total = k_bd + nbd;
  const double *u0 = a.lab_u0 + a.lab_u0off[label];
  const double cdist = a.lab_cdist[label];
  const double coefT = a.lab_coef[label];
  const Real rcd = (Real)(1.0 / cdist);
  // DH: the force cutoff is always scaled by the Debye length
  // (force_ele_DH.F90:44); Ewald: real-space cutoff in A
  const bool ewald = a.i_ele == 2, coul = a.i_ele == 3;
  const Real cut2 = (ewald || coul) ? (Real)(a.cutoff_ele * a.cutoff_ele)
                                    : (Real)((a.cutoff_ele * cdist) * (a.cutoff_ele * cdist));
  const Real ew_a = (Real)a.ewld_alpha, ew_a2 = (Real)(a.ewld_alpha * a.ewld_alpha), ew_b = (Real)a.ewld_beta;
  // near-list state: read here (after the caller's barrier), rewritten by
  // thread 0 only after the end-of-phase-1 barrier
  const bool near_rec = s.near_on && (s.misc[MISC_NEAR_BAD] != 0 ||
                                      __int_as_float(s.misc[f_disp]) > NEAR_DISP_MAX * NEAR_DISP_MAX);
  PHASE_T0(t_p1);
  // warp-uniform schedule: 32-item chunks of one kind (no divergence between
  // kinds), dealt to the warps as below
  const int nwarp = nth >> 5, warp = tid >> 5, lid = tid & 31;
  const int mode = (CL == 1) ? a.sweep_mode : 0;
  const bool dyn = mode == 1;
  // the sink's Gaussian noise of the own beads is drawn in the sweep, where warps have slack
  const Sweep sw = sweep_plan<CL>(a, T, cu, nch, geo.cpr, noise_step >= 0 && s.cst_on && a.noise_in_sweep, dyn);
  const int hb_0 = sw.hb_0, hb_1 = sw.hb_1, st_0 = sw.st_0, st_1 = sw.st_1, ts_0 = sw.ts_0, ts_1 = sw.ts_1;
  const int ch_0 = sw.ch_0, ch_1 = sw.ch_1, ba_0 = sw.ba_0, ba_1 = sw.ba_1, bd_0 = sw.bd_0, bd_1 = sw.bd_1;
  const int c_hb = sw.c_hb, c_st = sw.c_st, c_ts = sw.c_ts, c_ch = sw.c_ch, c_ba = sw.c_ba, c_bd = sw.c_bd;
  const int c_nz = sw.c_nz, c_end = sw.c_end;
  const int n_hbc = sw.n_hbc, n_stc = sw.n_stc, n_tsc = sw.n_tsc, n_chc = sw.n_chc, n_bac = sw.n_bac,
            n_bdc = sw.n_bdc;
  (void)k_st; (void)k_ch; (void)k_ba; (void)k_bd; (void)total;
  // (the counter was cleared after the last pass's bonded sweep; the deal
  // was made at the start of the launch)
  int k = 0, kend = 0, c = warp;
  if (dyn) {
    if (lid == 0) c = atomicAdd(&s.misc[MISC_CHUNK], 1);
    c = __shfl_sync(0xffffffffu, c, 0);
  } else if (mode == 2) {
    k = s.sched[warp]; kend = s.sched[warp + 1];
    c = (k < kend) ? s.sched[33 + k] : c_end;
  }
  while (c < c_end) {
    // the next chunk of this warp, requested before this one is processed
    int cn;
    if (dyn) {
      cn = 0;
      if (lid == 0) cn = atomicAdd(&s.misc[MISC_CHUNK], 1);
    } else if (mode == 2) {
      cn = (++k < kend) ? s.sched[33 + k] : c_end;
    } else {
      ++k;
      cn = k * nwarp + ((k & 1) ? nwarp - 1 - warp : warp);
    }
    PHASE_T0(t_item);
    int kind;
    if (c >= c_hb && c < c_hb + n_hbc) {
      kind = 0;
      const int h = hb_0 + ((c - c_hb) << 5) + lid;
      if (h < hb_1) {
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
              int sid = ldro(sites + q);
              if (sid >= 0) {
                int old = atomicAdd(&exc[sid], 1);
                if (old + 1 > ldro(a.site_val + T.site0 + sid)) {
                  s.misc[f_exc] = 1;
                  if (CL == 2) peer_ptr(s.misc, cu)[f_exc] = 1;
                }
              }
            }
          }
        } else {
          hbe[h] = 0.0;
        }
        hbf[h] = f;
      }
    } else if (c >= c_st && c < c_st + n_stc) {
      kind = 1;
      const int k = st_0 + ((c - c_st) << 5) + lid;
      if (k < st_1) term_stack<Real>(a, T, s, slots, k, ldro(u0 + k));
    } else if (c >= c_ts && c < c_ts + n_tsc) {
      kind = 1;
      const int k = ts_0 + ((c - c_ts) << 5) + lid;
      if (k < ts_1) term_tstack<Real>(a, T, s, slots, k);
    } else if (c >= c_ch && c < c_ch + n_chc) {
      kind = 2;
      const int cc = ch_0 + ((c - c_ch) << 5) + lid;
      if (cc < ch_1) {
        // force_ele_DH.F90:72-117 over a word range of one charged bead's
        // ele row; two pairs in flight per iteration
        const int kq = cc / geo.cpr, part = cc - kq * geo.cpr;
        const int i = s.qb[kq];
        const V pi = s.A4[i];
        const Real qci = (Real)((double)pi.w * coefT);
        const uint32_t *row = mele + (size_t)i * W;
        // DT19: Mg-P pairs within pmf_rmax take the table force (force_ele_DH.F90:87-97)
        const int tq = s.typ[i];
        const double *pmf_row = (a.pmf_f && (tq == 2 || tq == 5)) ? a.pmf_f + (size_t)label * a.pmf_nbin : nullptr;
        const int w1 = min(W, (part + 1) * geo.gw);
        // partial sums over at most a few words of the row, in Real (the
        // chunk totals enter each bead's FP64 sum)
        Real axs = 0, ays = 0, azs = 0;
        for (int w = part * geo.gw; w < w1; ++w) {
          uint32_t m = row[w];
          while (m) {
            const int j0 = (w << 5) + __ffs(m) - 1;
            m &= m - 1;
            const bool two = m != 0;
            const int j1 = two ? (w << 5) + __ffs(m) - 1 : j0;
            if (two) m &= m - 1;
            const V p0 = s.A4[j0], p1 = s.A4[j1];
            Real ax, ay, az, bx, by, bz;
            if (mir) {   // FP64 difference and image shift (see the exv gather)
              double ex = (double)p0.x - (double)pi.x, ey = (double)p0.y - (double)pi.y, ez = (double)p0.z - (double)pi.z;
              double fx_ = (double)p1.x - (double)pi.x, fy_ = (double)p1.y - (double)pi.y, fz_ = (double)p1.z - (double)pi.z;
              mirror_shift<double>(a, s, i, j0, ex, ey, ez);
              mirror_shift<double>(a, s, i, j1, fx_, fy_, fz_);
              ax = (Real)ex; ay = (Real)ey; az = (Real)ez; bx = (Real)fx_; by = (Real)fy_; bz = (Real)fz_;
            } else {
              ax = p0.x - pi.x; ay = p0.y - pi.y; az = p0.z - pi.z;
              bx = p1.x - pi.x; by = p1.y - pi.y; bz = p1.z - pi.z;
            }
            const Real ra2 = ax * ax + ay * ay + az * az, rb2 = bx * bx + by * by + bz * bz;
            const Real ria = rsq<Real>(ra2), rib = rsq<Real>(rb2);
            const Real da = ra2 * ria, db = rb2 * rib;
            Real fa, fb;
            if (coul) {
              // force_ele_coulomb.F90:66-71 (no clamp)
              fa = qci * p0.w * ria * ria * ria;
              fb = qci * p1.w * rib * rib * rib;
            } else if (!ewald) {
              fa = qci * p0.w * ria * ria * (ria + rcd) * fexp<Real>(-da * rcd);
              fb = qci * p1.w * rib * rib * (rib + rcd) * fexp<Real>(-db * rcd);
              if (pmf_row) {
                bool low = false;
                if (mg_p_pair(tq, s.typ[j0]) && (double)da <= a.pmf_rmax)
                  fa = (Real)pmf_row[pmf_bin(a, (double)da, low)] * ria;
                if (two && mg_p_pair(tq, s.typ[j1]) && (double)db <= a.pmf_rmax)
                  fb = (Real)pmf_row[pmf_bin(a, (double)db, low)] * rib;
                if (low) s.misc[MISC_PMF] = 1;
              }
            } else {
              // force_ele_coulomb_ewld.F90:118-137 (real space, no clamp)
              fa = qci * p0.w * (erfc(ew_a * da) * ria + ew_b * exp(-ew_a2 * ra2)) * ria * ria;
              fb = qci * p1.w * (erfc(ew_a * db) * rib + ew_b * exp(-ew_a2 * rb2)) * rib * rib;
            }
            if (!(ra2 <= cut2)) fa = 0;
            if (!(rb2 <= cut2) || !two) fb = 0;
            if (!ewald && !coul) {   // DE_MAX clamp, each pair counted once (from its lower bead)
              if (fa > (Real)50) { fa = 50; nclamp += j0 > i; }
              if (fb > (Real)50) { fb = 50; nclamp += j1 > i; }
            }
            axs -= fa * ax + fb * bx;
            ays -= fa * ay + fb * by;
            azs -= fa * az + fb * bz;
          }
        }
        s.ch_part[3 * cc] = axs; s.ch_part[3 * cc + 1] = ays; s.ch_part[3 * cc + 2] = azs;
      }
    } else if (c >= c_ba && c < c_ba + n_bac) {
      kind = 3;
      const int k = ba_0 + ((c - c_ba) << 5) + lid;
      if (k < ba_1) term_angle<Real>(a, T, s, slots, k);
    } else if (c >= c_bd && c < c_bd + n_bdc) {
      kind = 4;
      const int k = bd_0 + ((c - c_bd) << 5) + lid;
      if (k < bd_1) term_bond<Real>(a, T, s, slots, k);
    } else {
      kind = 4;
      const int i = cu.lo + ((c - c_nz) << 5) + lid;
      if (i < cu.hi) {
        double n0, n1, n2;
        noise3(a, lane, L, i, istep, noise_step, n0, n1, n2);
        s.NX[i] = n0; s.NY[i] = n1; s.NZ[i] = n2;
      }
    }
    PHASE_ALL(32 + kind, t_item);
    c = dyn ? __shfl_sync(0xffffffffu, cn, 0) : cn;
  }
  PHASE_ADD(3, t_p1);
  PHASE_WARP(64, t_p1);
  PHASE_T0(t_b2);
  if (CL == 1) __syncthreads(); else cg::this_cluster().sync();
  PHASE_ADD(9, t_b2);
  // (two CTAs: the caller clears the displacement flag of the step after next)
  if (tid == 0) {
    s.misc[MISC_CHUNK] = 0;   // every warp has taken its last chunk
    if (s.near_on) { s.misc[MISC_NEAR_BAD] = 0; if (CL == 1) s.misc[f_disp] = 0; }
    if (CL == 1) s.misc[MISC_DMAX] = 0;
  }
  // both CTAs hold the same flag (the first one sets it in both), so both
  // take the same barriers
  if (s.misc[f_exc]) {
    if (tid == 0 && cu.rank == 0) {
      const double beta = a.hb_beta_global ? (a.rex ? a.rex->beta_global : a.beta_hbond15) : a.lab_beta[label];
      prune_hbonds<Real>(a, lane, L, T, istep, beta, true, s.exc);
    }
    if (CL == 1) __syncthreads(); else cg::this_cluster().sync();
  }
  PHASE_T0(t_p2);
  // ---- phase 2: exv pairs + bonded slots + Debye-Hueckel chunk partials
  const int nown = cu.hi - cu.lo;
  const int GA = a.group > 0 ? a.group : pow2_floor_clamp(nth / nown, 8);
  const int g = tid & (GA - 1), grp = tid / GA, ngrp = nth / GA;
  const Real ra = (Real)a.exv_adjust, ra2 = ra * ra, inv_ra2 = (Real)(1.0 / (a.exv_adjust * a.exv_adjust));
  const Real dist_ps = (Real)a.exv_dist_PS, dist_rr = (Real)a.exv_dist;
  const int iters = (nown + ngrp - 1) / ngrp;
  for (int it = 0; it < iters; ++it) {
    const int i = cu.lo + grp + it * ngrp;
    const bool valid = i < cu.hi;
    double fx = 0, fy = 0, fz = 0;
    PHASE_T0(t_e0);
    PHASE_T0(t_e2);
    if (valid) {
      const V pi = s.A4[i], bi = s.B4[i], li = s.L4[i];
      const int ti = s.typ[i], ci = s.cls[i];
      const Real scr2 = bi.z * bi.z;   // (screen radius)^2, rounding margin included
      const Real nscr = bi.z + (Real)NEAR_SKIN, nscr2 = nscr * nscr;
      const uint32_t *row = mexv + (size_t)i * W;
      // force_exv_dt15.F90:204-265 for partner j: one 16-byte load screens
      // the pair; pairs inside the screen radius use the hi + lo difference
      // (the FP64 difference to ~1e-12 relative).  rec: record j in lst when
      // it is within the near radius.
      auto visit = [&](int j, bool rec, int &cnt, uint16_t *lst, int ncap) {
        const V pj = s.A4[j];
        Real sx, sy, sz;
        if (mir) {
          // across the box the two coordinates are ~L apart: difference and
          // image shift in FP64, so only the short result is rounded
          double ex = (double)pj.x - (double)pi.x, ey = (double)pj.y - (double)pi.y, ez = (double)pj.z - (double)pi.z;
          mirror_shift<double>(a, s, i, j, ex, ey, ez);
          sx = (Real)ex; sy = (Real)ey; sz = (Real)ez;
        } else {
          sx = pj.x - pi.x; sy = pj.y - pi.y; sz = pj.z - pi.z;
        }
        const Real d2s = sx * sx + sy * sy + sz * sz;
        if (rec && d2s <= nscr2) {
          if (cnt < ncap) lst[cnt] = (uint16_t)j;
          ++cnt;
        }
        if (d2s > scr2) return;
        const V lj = s.L4[j];
        const Real wx = sx + (lj.x - li.x), wy = sy + (lj.y - li.y), wz = sz + (lj.z - li.z);
        const Real r2 = wx * wx + wy * wy + wz * wz;
        const int tj = s.typ[j], cj = s.cls[j];
        const V bj = s.B4[j];
        Real dij;
        if (a.dt19) dij = (ti == 3 && tj == 3) ? dist_rr : bi.x + bj.x;   // force_exv_dt15.F90:60-66
        else if ((ti == 2 && tj == 4) || (ti == 4 && tj == 2)) dij = dist_ps;
        else if (ci == 2 && cj == 2) dij = dist_rr;
        else dij = bi.x + bj.x;
        if (r2 > dij * dij) return;
        Real rinv = rsq<Real>(r2);
        Real dr = r2 * rinv + ra - dij;
        if (sizeof(Real) == 4 && dr < (Real)1.5) {
          // on the steep part of the potential (dr = dist + a - d_ij small)
          // the rounding of the FP32 distance is amplified ~13 / dr: the
          // distance and dr in FP64 from the exact hi + lo difference
          const double ex = (double)sx + ((double)lj.x - (double)li.x);
          const double ey = (double)sy + ((double)lj.y - (double)li.y);
          const double ez = (double)sz + ((double)lj.z - (double)li.z);
          const double d64 = sqrt(ex * ex + ey * ey + ez * ez);
          double dij64;
          if (a.dt19) dij64 = (ti == 3 && tj == 3) ? a.exv_dist : (double)bi.x + (double)bj.x;
          else if ((ti == 2 && tj == 4) || (ti == 4 && tj == 2)) dij64 = a.exv_dist_PS;
          else if (ci == 2 && cj == 2) dij64 = a.exv_dist;
          else dij64 = (double)bi.x + (double)bj.x;
          rinv = (Real)(1.0 / d64);
          dr = (Real)(d64 + a.exv_adjust - dij64);
        }
        const Real coef = bi.y * bj.y;
        const Real ro2 = fdiv(ra2, dr * dr);
        const Real ro4 = ro2 * ro2, ro8 = ro4 * ro4, ro14 = ro2 * ro4 * ro8;
        Real f = fabs((Real)12 * coef * (ro14 - ro8) * dr * inv_ra2 * rinv);
        // DE_MAX clamp; each pair is visited from both beads and counted once
        if (f > (Real)50) { f = 50; nclamp += j > i; }
        fx -= (double)(f * wx); fy -= (double)(f * wy); fz -= (double)(f * wz);
      };
      const int ncap = NEAR_CAP / GA;
      uint16_t *lst = s.near_on ? s.near + (size_t)i * NEAR_CAP + g * ncap : nullptr;
      const int have = s.near_on ? (int)s.near_cnt[i * 8 + g] : 0xFF;
      int cnt = 0;
      if (s.near_on && !near_rec && have != 0xFF) {
        for (int k = 0; k < have; ++k) visit((int)lst[k], false, cnt, lst, ncap);
      } else {
        for (int w = g; w < W; w += GA) {
          uint32_t m = row[w];
          while (m) {
            const int j = (w << 5) + __ffs(m) - 1;
            m &= m - 1;
            visit(j, near_rec, cnt, lst, ncap);
          }
        }
        if (near_rec) {
          s.near_cnt[i * 8 + g] = (uint8_t)(cnt > ncap ? 0xFF : cnt);
          if (g == 0) s.NR4[i] = make_float4((float)pi.x, (float)pi.y, (float)pi.z, 0.f);
        }
      }
      PHASE_ALL(40, t_e0);
#ifdef TIS_PHASE_TIMING
      t_e2 = clock64();
#endif
      // bonded slots (incidence list, ascending slot id)
      const int p0 = s.inc_ptr[i], p1 = s.inc_ptr[i + 1];
      for (int p = p0 + g; p < p1; p += GA) {
        const int sid = s.inc_slot[p];
        if (sid >= T.slot_hb) {
          const int h = (sid - T.slot_hb) / 6;
          if (!(hbf[h] & 2)) continue;
        }
        fx += (double)my_slots[3 * (size_t)sid]; fy += (double)my_slots[3 * (size_t)sid + 1];
        fz += (double)my_slots[3 * (size_t)sid + 2];
      }
      const int kq = s.qidx[i];
      if (nch > 0 && kq >= 0) {
        for (int c = kq * geo.cpr + g; c < (kq + 1) * geo.cpr; c += GA) {
          fx += s.ch_part[3 * c]; fy += s.ch_part[3 * c + 1]; fz += s.ch_part[3 * c + 2];
        }
      }
    }
    if (valid) PHASE_ALL(41, t_e2);
    PHASE_T0(t_e1);
    // every thread of the group holds the same totals: thread d of the group
    // (d < GA) hands component d (and d + GA, ...) to the sink, then its
    // first thread finishes the bead after the components are written
    group_reduce<Real>(fx, fy, fz, GA);
    if (valid) {
      for (int d = g; d < 3; d += GA) {
        double f = d == 0 ? fx : (d == 1 ? fy : fz);
        if (a.f_ext)   // the reciprocal-space partial forces, in k-range order
          for (int p = 0; p < EW_F_SPLIT; ++p) f += a.f_ext[3 * ((size_t)p * a.nbead_total + L.state0 + i) + d];
        sink(i, d, f);
      }
    }
    __syncwarp();
    if (valid && g == 0) fin(i);
    if (valid && g == 0) PHASE_ALL(42, t_e1);
  }
  if (nclamp) atomicAdd(&s.misc[MISC_CLAMP], nclamp);
  PHASE_WARP(96, t_p2);
#ifdef TIS_PHASE_TIMING
  __syncthreads();
  PHASE_ADD(5, t_p2);
#endif
}

// ------------------------------------------------------------ the kernel
// CL = 1: one CTA per lane.  CL = 2 (mixed precision, KM_STEP, no periodic
// box, fixed rebuild cadence): a cluster of two CTAs per lane; CTA r owns
// half of the beads (x / v / a updates, list rows, force sums) and half of
// the bonded items; new positions go to both CTAs' double-buffered copies
// through distributed shared memory.  Per step: one cluster barrier after
// the x update, one after the bonded sweep (two more at a rebuild, one more
// after a valence pruning).  Every branch that decides a cluster barrier is
// uniform over both CTAs.
template <typename Real, int NT, int CL, bool SKIN2 = false>
__global__ void __launch_bounds__(NT) lane_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane
                                      : (a.lane_order ? a.lane_order[blockIdx.x / CL] : (int)(blockIdx.x / CL));
  if (lane >= a.nlane) return;
  if (CL == 2 && a.mode != KM_STEP) return;
  // replicas that have reached their exchange step wait (time_integral.F90:134)
  if (a.lane_nsteps && (a.mode == KM_XSTEP || a.mode == KM_VSTEP || a.mode == KM_VXSTEP) &&
      a.step_k >= a.lane_nsteps[lane])
    return;
  const int lane_steps = (a.lane_nsteps && a.mode == KM_STEP) ? min(a.nsteps, a.lane_nsteps[lane]) : a.nsteps;
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int N = T.nmp, NQ = T.nq;
  const int tid = threadIdx.x, nth = blockDim.x;
  // the two-CTA kernel is compiled once per rebuild rule (its registers are
  // scarce); the one-CTA kernel decides at run time
  const bool skin = (CL == 2) ? SKIN2 : a.n_step_neighbor <= 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<Real> s = carve<Real>(smem_raw, a.smem_total, a, L, T, a.periodic != 0, skin, CL == 2);
  // a layout larger than the launch's shared memory (the host sizes the
  // launch so this cannot happen) touches nothing: the lane is flagged
  if (!s.fits) {
    if (tid == 0) atomicOr(&a.lstate[lane].flags, LF_SMEM);
    return;
  }
  LaneState &st = a.lstate[lane];
  Clu cu;
  cu.nrank = CL;
  cu.rank = (CL == 2) ? (int)cg::this_cluster().block_rank() : 0;
  cu.lo = (CL == 2 && cu.rank == 1) ? (N + 1) / 2 : 0;
  cu.hi = (CL == 2 && cu.rank == 0) ? (N + 1) / 2 : N;
  cu.kq_lo = 0; cu.kq_hi = NQ;
  const long long istep0 = st.istep;   // two CTAs: written only after the final cluster barrier
  // ---- load state, per-bead parameters, incidence lists, list bit matrices
  for (int i = tid; i < N; i += nth) {
    const size_t o = 3 * (size_t)(L.state0 + i);
    s.X[i] = a.xyz[o]; s.Y[i] = a.xyz[o + 1]; s.Z[i] = a.xyz[o + 2];
    if (a.periodic) {
      s.PX[i] = a.pxyz[o]; s.PY[i] = a.pxyz[o + 1]; s.PZ[i] = a.pxyz[o + 2];
      s.QX[i] = a.p0xyz[o]; s.QY[i] = a.p0xyz[o + 1]; s.QZ[i] = a.p0xyz[o + 2];
    }
    s.VX[i] = a.velo[o]; s.VY[i] = a.velo[o + 1]; s.VZ[i] = a.velo[o + 2];
    s.AX[i] = a.accel[o]; s.AY[i] = a.accel[o + 1]; s.AZ[i] = a.accel[o + 2];
    if (skin) { s.DX[i] = a.dxyz[o]; s.DY[i] = a.dxyz[o + 1]; s.DZ[i] = a.dxyz[o + 2]; }
    const int b = T.bead0 + i;
    set_pos<Real>(s, i);
    s.A4[i].w = (Real)bead_charge(a, st.label, b);
    if (s.A4N) { s.A4N[i].w = s.A4[i].w; s.L4N[i].w = (Real)0; }   // the next-step copies keep .w
    s.B4[i].x = (Real)a.b_radius[b]; s.B4[i].y = (Real)a.b_eps[b];
    s.B4[i].z = (Real)(a.b_screen[b] * (1.0 + 1.0e-4) + 1.0e-3); s.B4[i].w = (Real)0;
    s.typ[i] = a.b_type[b]; s.cls[i] = a.b_class[b];
    s.unit[i] = a.b_unit[b];
    s.qidx[i] = -1;
  }
  const int inc_base = a.inc_ptr[T.inc0];
  for (int i = tid; i <= N; i += nth) s.inc_ptr[i] = a.inc_ptr[T.inc0 + i] - inc_base;
  if (s.inc_smem)
    for (int k = tid; k < T.ninc; k += nth) ((int *)s.inc_slot)[k] = a.inc_slot[inc_base + k];
  for (int k = tid; k < NQ; k += nth) s.qb[k] = a.q_bead[T.q0 + k];
  for (int k = tid; k < T.nunit * T.nunit; k += nth) s.rn2[k] = a.rneigh2[T.rn0 + k];
  if (s.mask_smem && a.mode != KM_NEIGHBOR && a.mode != KM_PRE) {
    const uint32_t *gm = a.mask + L.mask0;
    for (int k = tid; k < 2 * N * s.W; k += nth) s.mask[k] = gm[k];
  }
  if (tid < MISC_UNITS) s.misc[tid] = 0;
  int *exc = s.exc;
  for (int k = tid; k < T.nsite; k += nth) exc[k] = 0;
  __syncthreads();
  for (int k = tid; k < NQ; k += nth) s.qidx[s.qb[k]] = k;
  if (tid == 0) s.misc[MISC_NEAR_BAD] = 1;
  __syncthreads();
  if (CL == 2) {
    // charged rows of the own beads (q_bead ascends in bead index)
    int ql = 0, qh = 0;
    for (int k = 0; k < NQ; ++k) { ql += s.qb[k] < cu.lo; qh += s.qb[k] < cu.hi; }
    cu.kq_lo = ql; cu.kq_hi = qh;
  }
  // the fixed deal of the bonded sweep, for the launch (modes with a force pass)
  if (CL == 1 && a.mode != KM_NEIGHBOR && a.sweep_mode == 2) {
    if (tid == 0) {
      const ChunkGeo geo = chunk_geo(NQ, s.W);
      const Sweep sw = sweep_plan<CL>(a, T, cu, a.i_ele != 0 ? geo.nch : 0, geo.cpr,
                                      a.mode != KM_FORCE && s.cst_on && a.noise_in_sweep, false);
      sweep_deal(sw, geo.gw, nth >> 5, s.sched, s.sched_cap);
    }
    __syncthreads();
  }

  const int label0 = st.label;
  const double *c1 = a.lab_c1 + a.lab_c1off[label0];
  if (s.cst_on) {
    for (int i = tid; i < N; i += nth) {
      const int b = T.bead0 + i;
      s.C1[i] = c1[i]; s.C2[i] = a.b_c2[b]; s.C3[i] = a.b_c3[b]; s.C4[i] = a.b_c4[b]; s.RC[i] = a.b_rcmass[b];
    }
    __syncthreads();
  }
  // time_integral.F90:169-183: v / a update of component d of bead i from
  // its force (the components of a bead are three independent updates)
  auto vstep = [&](long long istep, int nstep_noise) {
    return [&, istep, nstep_noise](int i, int d, double f) {
      double n, rc, cc, c2, c3;
      if (s.cst_on) {
        // drawn in the bonded sweep, or here
        n = a.noise_in_sweep ? s.NX[d * N + i] : noise1(a, lane, L, i, istep, nstep_noise, d);
        rc = s.RC[i]; cc = s.C1[i]; c2 = s.C2[i]; c3 = s.C3[i];
      } else {
        n = noise1(a, lane, L, i, istep, nstep_noise, d);
        const int b = T.bead0 + i;
        rc = a.b_rcmass[b]; cc = c1[i]; c2 = a.b_c2[b]; c3 = a.b_c3[b];
      }
      // each product rounded, as the reference evaluates it (no contraction)
      double *V = s.VX + d * N, *A = s.AX + d * N;
      const double acc = mad2<Real>(f, rc, cc, n);
      V[i] = mad2<Real>(c2, V[i], c3, add_rn<Real>(A[i], acc));
      A[i] = acc;
      if (!(f == f)) s.misc[MISC_NAN] = 1;
    };
  };

  // skin rule: the trigger of the first step from the displacements loaded
  // above (two CTAs: in the copy of the step's parity; the other CTA's pairs
  // are read after the cluster barrier below)
  bool skin_fire = false;
  double *red0 = s.red + ((CL == 2) ? 32 * (int)(istep0 & 1) : 0);
  if (skin && (a.mode == KM_STEP || a.mode == KM_XSTEP || a.mode == KM_VXSTEP)) {
    double m1 = 0.0, m2 = 0.0;
    for (int i = cu.lo + tid; i < cu.hi; i += nth) top2_add(m1, m2, disp2(s.DX[i], s.DY[i], s.DZ[i]));
    top2_store(m1, m2, red0);
    if (CL == 1) {
      __syncthreads();
      skin_fire = skin_fires(red0, nullptr, nth >> 5, a.neigh_margin);
    }
  }

  if constexpr (CL == 2) {
    typedef typename V4<Real>::T V;
    cg::this_cluster().sync();   // both CTAs are running before any distributed access
    if (skin) skin_fire = skin_fires(red0, peer_ptr(red0, cu), nth >> 5, a.neigh_margin);
    // x update of step n + 1 of own bead i (time_integral.F90:152-161) from
    // the v / a of step n: positions into the next-step buffers of both CTAs;
    // skin rule: dxyz restarts from zero when step n + 1 rebuilds
    // (time_integral.F90:89), and (m1, m2) collect the top two of the new
    // dxyz for the trigger of step n + 2; the near-list displacement flag of
    // step n + 1 goes to the copy of its parity
    auto xnext = [&](int i, int d, bool fire) {
      const double c4 = s.cst_on ? s.C4[i] : a.b_c4[T.bead0 + i];
      const double dx = mad2<Real>(c4, s.VX[d * N + i], a.tstep2, s.AX[d * N + i]);
      const double nx = s.X[d * N + i] + dx;
      if (skin) {
        double *D = s.DX + d * N;
        D[i] = fire ? dx : D[i] + dx;
      }
      s.XN[d * N + i] = nx;
      peer_ptr(s.XN, cu)[d * N + i] = nx;
      const Real hi = (Real)nx, lo = (Real)(nx - (double)hi);
      (&s.A4N[i].x)[d] = hi; (&s.L4N[i].x)[d] = lo;
      (&peer_ptr(s.A4N, cu)[i].x)[d] = hi; (&peer_ptr(s.L4N, cu)[i].x)[d] = lo;
    };
    // after the three components of bead i: dot_product(dxyz, dxyz) into DD
    // of both CTAs and, rounded up to float, into the running maximum of the
    // step (flag copy f_dmax, both CTAs); the near-list displacement check
    auto xfin = [&](int i, int f_disp, int f_dmax) {
      if (skin) {
        const double d2 = disp2(s.DX[i], s.DY[i], s.DZ[i]);
        s.DD[i] = d2;
        peer_ptr(s.DD, cu)[i] = d2;
        const int bits = __float_as_int(__double2float_ru(d2));   // order-preserving for d2 >= 0
        atomicMax(&s.misc[f_dmax], bits);
        atomicMax(&peer_ptr(s.misc, cu)[f_dmax], bits);
      }
      if (s.near_on) {
        const V av = s.A4N[i];
        const float ex = (float)av.x - s.NR4[i].x, ey = (float)av.y - s.NR4[i].y, ez = (float)av.z - s.NR4[i].z;
        const float e2 = ex * ex + ey * ey + ez * ez;
        if (!(e2 <= NEAR_DISP_MAX * NEAR_DISP_MAX)) atomicMax(&s.misc[f_disp], 0x7f000000);
      }
    };
    // the first step's x update; the later ones run in the v / a update of
    // the step before (the lists of a rebuild come from the positions before
    // the update, which stay in the current buffers until the swap)
    {
      const long long is1 = istep0 + 1;
      for (int i = cu.lo + tid; i < cu.hi; i += nth) {
        for (int d = 0; d < 3; ++d) xnext(i, d, skin_fire);
        xfin(i, MISC_NEAR_DISP + (int)(is1 & 1), MISC_DMAX + (int)(is1 & 1));
      }
      if (cu.rank == 0) for (int k = tid; k < T.nsite; k += nth) exc[k] = 0;
      if (tid == 0) s.misc[MISC_EXCESS + (int)(is1 & 1)] = 0;
    }
    for (int step = 0; step < lane_steps; ++step) {
      const long long istep = istep0 + step + 1;
      const int par = (int)(istep & 1);
      const bool last = step + 1 == lane_steps;
      // neighbour trigger: the skin rule (time_integral.F90:57-93) or the
      // fixed cadence (:94); the decision is the same in both CTAs
      PHASE_T0(t_reb);
      const bool rebuild = skin ? skin_fire : ((istep % a.n_step_neighbor) == 1 || istep == 1);
      if (rebuild) {
        __syncthreads();   // the last force pass has finished with the rows
        build_lists<Real, 2>(a, lane, L, T, s, cu, istep);
      }
      PHASE_ADD(1, t_reb);
      PHASE_T0(t_b1);
      // the next-step buffers (and, after a rebuild, the list rows) of both
      // CTAs are complete
      cg::this_cluster().sync();
      PHASE_ADD(8, t_b1);
      if (rebuild && tid == 0 && cu.rank == 0)
        rebuild_counts(st, s.misc[MISC_NEXV] + peer_ptr(s.misc, cu)[MISC_NEXV],
                       s.misc[MISC_NELE] + peer_ptr(s.misc, cu)[MISC_NELE], istep);
      // trigger of the next step from the dxyz of this one
      if (skin) skin_fire = skin_trigger(s.misc[MISC_DMAX + par], s.DD, N, a.neigh_margin);
      // flags of the next step: their last readers passed this barrier
      if (tid == 0) {
        s.misc[MISC_EXCESS + (par ^ 1)] = 0; s.misc[MISC_NEAR_DISP + (par ^ 1)] = 0; s.misc[MISC_DMAX + (par ^ 1)] = 0;
      }
      { double *t; t = s.X; s.X = s.XN; s.XN = t; t = s.Y; s.Y = s.YN; s.YN = t; t = s.Z; s.Z = s.ZN; s.ZN = t; }
      s.PX = s.X; s.PY = s.Y; s.PZ = s.Z;
      { V *t; t = s.A4; s.A4 = s.A4N; s.A4N = t; t = s.L4; s.L4 = s.L4N; s.L4N = t; }
      PHASE_T0(t_fp);
      const int nstep_noise = a.noise_base + step;
      const bool fire_next = skin_fire;
      force_pass<Real, 2>(
          a, lane, L, T, s, istep, cu, nstep_noise,
          [&](int i, int d, double f) {
            vstep(istep, nstep_noise)(i, d, f);
            if (!last) xnext(i, d, fire_next);
          },
          par,
          [&](int i) {
            if (!last) xfin(i, MISC_NEAR_DISP + (par ^ 1), MISC_DMAX + (par ^ 1));
          });
      if (!last) {
        // hbond-site counters of the next step (read only in the bonded sweep
        // and the valence pruning, both behind this step's cluster barriers)
        if (cu.rank == 0) for (int k = tid; k < T.nsite; k += nth) exc[k] = 0;
      }
      PHASE_ADD(6, t_fp);
    }
    cg::this_cluster().sync();   // no distributed shared-memory access after this
  } else if (a.mode == KM_NEIGHBOR) {
    build_lists<Real, 1>(a, lane, L, T, s, cu, st.istep);
  } else if (a.mode == KM_FORCE) {
    double *out = a.out_force;
    force_pass<Real, 1>(a, lane, L, T, s, st.istep, cu, -1,
                        [&](int i, int d, double f) { out[3 * (size_t)(L.state0 + i) + d] = f; });
  } else if (a.mode == KM_PRE) {
    build_lists<Real, 1>(a, lane, L, T, s, cu, st.istep);
    // dxyz_mp = 0 (time_integral_pre.F90:79)
    if (skin) for (int i = tid; i < N; i += nth) { s.DX[i] = 0.0; s.DY[i] = 0.0; s.DZ[i] = 0.0; }
    __syncthreads();
    const long long is = st.istep;
    force_pass<Real, 1>(a, lane, L, T, s, is, cu, a.noise_base, [&](int i, int d, double f) {
      const double n = (s.cst_on && a.noise_in_sweep) ? s.NX[d * N + i] : noise1(a, lane, L, i, is, a.noise_base, d);
      s.AX[d * N + i] = mad2<Real>(f, a.b_rcmass[T.bead0 + i], c1[i], n);
    });
  } else {
    // KM_STEP (nsteps), KM_XSTEP and KM_VSTEP (the two halves of one step),
    // KM_VXSTEP (the second half of one step and the first of the next)
    auto xpart = [&](long long istep) {
      // time_integral.F90:57-161: neighbour trigger, rebuild, x update
      PHASE_T0(t_trig);
      const bool rebuild = skin ? skin_fire : ((istep % a.n_step_neighbor) == 1 || istep == 1);
      PHASE_ADD(0, t_trig);
      PHASE_T0(t_reb);
      if (rebuild) {
        build_lists<Real, 1>(a, lane, L, T, s, cu, istep);
        // dxyz_mp(:,:,irep) = 0 after a skin-triggered rebuild (time_integral.F90:89)
        if (skin) for (int i = tid; i < N; i += nth) { s.DX[i] = 0.0; s.DY[i] = 0.0; s.DZ[i] = 0.0; }
        __syncthreads();
      }
      PHASE_ADD(1, t_reb);
      PHASE_T0(t_xu);
      // x update (time_integral.F90:152-161), each product rounded as the
      // reference evaluates it; clear hbond-site counters
      for (int i = tid; i < N; i += nth) {
        const double c4 = s.cst_on ? s.C4[i] : a.b_c4[T.bead0 + i];
        const double dx = mad2<Real>(c4, s.VX[i], a.tstep2, s.AX[i]);
        const double dy = mad2<Real>(c4, s.VY[i], a.tstep2, s.AY[i]);
        const double dz = mad2<Real>(c4, s.VZ[i], a.tstep2, s.AZ[i]);
        s.X[i] += dx; s.Y[i] += dy; s.Z[i] += dz;
        if (a.periodic) { s.PX[i] += dx; s.PY[i] += dy; s.PZ[i] += dz; }
        if (skin) {
          s.DX[i] += dx; s.DY[i] += dy; s.DZ[i] += dz;
          const double d2 = disp2(s.DX[i], s.DY[i], s.DZ[i]);
          s.DD[i] = d2;
          atomicMax(&s.misc[MISC_DMAX], __float_as_int(__double2float_ru(d2)));   // order-preserving for d2 >= 0
        }
        set_pos<Real>(s, i);
        if (s.near_on) {
          const float ex = (float)s.A4[i].x - s.NR4[i].x, ey = (float)s.A4[i].y - s.NR4[i].y,
                      ez = (float)s.A4[i].z - s.NR4[i].z;
          const float e2 = ex * ex + ey * ey + ez * ez;
          if (!(e2 <= NEAR_DISP_MAX * NEAR_DISP_MAX)) atomicMax(&s.misc[MISC_NEAR_DISP], 0x7f000000);
        }
      }
      for (int k = tid; k < T.nsite; k += nth) exc[k] = 0;
      if (tid == 0) s.misc[MISC_EXCESS] = 0;
      __syncthreads();
      // the next step's trigger (MISC_DMAX is cleared after the force
      // pass's first barrier, before the next x update)
      if (skin) skin_fire = skin_trigger(s.misc[MISC_DMAX], s.DD, N, a.neigh_margin);
      PHASE_ADD(2, t_xu);
    };
    const int nloop = (a.mode == KM_STEP) ? lane_steps : 1;
    for (int step = 0; step < nloop; ++step) {
      const long long istep = st.istep + 1;
      if (a.mode == KM_STEP || a.mode == KM_XSTEP) xpart(istep);
      if (a.mode != KM_XSTEP) {
        // time_integral.F90:162-183: forces (+ f_ext), v / a update
        const int nstep_noise = a.noise_base + step;
        PHASE_T0(t_fp);
        force_pass<Real, 1>(a, lane, L, T, s, istep, cu, nstep_noise, vstep(istep, nstep_noise));
        if (tid == 0) st.istep = istep;
        __syncthreads();
        PHASE_ADD(6, t_fp);
      }
      // the next step's x update, unless this replica stops at this step
      if (a.mode == KM_VXSTEP && (!a.lane_nsteps || a.step_k + 1 < a.lane_nsteps[lane])) xpart(istep + 1);
    }
  }
  __syncthreads();
  // the global copy of the bit matrices is read by the energy kernel and the list exports
  if (s.misc[MISC_REBUILT] && s.mask_smem) {
    uint32_t *gm = a.mask + L.mask0;
    if (CL == 1) {
      for (int k = tid; k < 2 * N * s.W; k += nth) gm[k] = s.mask[k];
    } else {   // own rows of both matrices
      const int nw = (cu.hi - cu.lo) * s.W;
      for (int k = tid; k < nw; k += nth) {
        const size_t o = (size_t)cu.lo * s.W + k;
        gm[o] = s.mask[o];
        gm[(size_t)N * s.W + o] = s.mask[(size_t)N * s.W + o];
      }
    }
  }
  // write back
  for (int i = cu.lo + tid; i < cu.hi; i += nth) {
    const size_t o = 3 * (size_t)(L.state0 + i);
    a.xyz[o] = s.X[i]; a.xyz[o + 1] = s.Y[i]; a.xyz[o + 2] = s.Z[i];
    if (a.periodic) {
      a.pxyz[o] = s.PX[i]; a.pxyz[o + 1] = s.PY[i]; a.pxyz[o + 2] = s.PZ[i];
      a.p0xyz[o] = s.QX[i]; a.p0xyz[o + 1] = s.QY[i]; a.p0xyz[o + 2] = s.QZ[i];
    } else {
      a.pxyz[o] = s.X[i]; a.pxyz[o + 1] = s.Y[i]; a.pxyz[o + 2] = s.Z[i];
    }
    a.velo[o] = s.VX[i]; a.velo[o + 1] = s.VY[i]; a.velo[o + 2] = s.VZ[i];
    a.accel[o] = s.AX[i]; a.accel[o + 1] = s.AY[i]; a.accel[o + 2] = s.AZ[i];
    if (skin) { a.dxyz[o] = s.DX[i]; a.dxyz[o + 1] = s.DY[i]; a.dxyz[o + 2] = s.DZ[i]; }
  }
  if (tid == 0) {
    if (CL == 1) {
      st.nclamp += s.misc[MISC_CLAMP];
      if (s.misc[MISC_NAN]) st.flags |= LF_NAN;
      if (s.misc[MISC_PMF]) st.flags |= LF_PMF;
    } else {
      if (s.misc[MISC_CLAMP]) atomicAdd((unsigned long long *)&st.nclamp, (unsigned long long)s.misc[MISC_CLAMP]);
      if (s.misc[MISC_NAN]) atomicOr(&st.flags, LF_NAN);
      if (s.misc[MISC_PMF]) atomicOr(&st.flags, LF_PMF);
      if (cu.rank == 0) st.istep = istep0 + lane_steps;
    }
  }
}

// r_boxmuller(3, nmp, nrep) of the counter-based generator for steps
// istep0 .. istep0 + gridDim.y - 1 (the noise the lane kernel draws at
// those steps): block (lane, k) writes out[k][bead][3]
__global__ void noise_kernel(KArgs a, long long istep0, double *out) {
  const int lane = blockIdx.x, k = blockIdx.y;
  const LaneDesc L = a.lanes[lane];
  const int N = a.tops[L.top].nmp;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    double n0, n1, n2;
    noise3(a, lane, L, i, istep0 + k, 0, n0, n1, n2);
    const size_t o = ((size_t)k * a.nbead_total + L.state0 + i) * 3;
    out[o] = n0; out[o + 1] = n1; out[o + 2] = n2;
  }
}

cudaError_t noise_launch(cudaStream_t st, KArgs a, long long istep0, int nstep, double *out) {
  a.noise = nullptr;   // always the counter-based generator
  noise_kernel<<<dim3(a.nlane, nstep), 256, 0, st>>>(a, istep0, out);
  return cudaGetLastError();
}

#ifdef TIS_PHASE_TIMING
extern "C" int tis_phase_read(unsigned long long *out) {
  return (int)cudaMemcpyFromSymbol(out, g_phase, sizeof(unsigned long long) * 128);
}
#endif

template __global__ void lane_kernel<double, 512, 1>(KArgs);
template __global__ void lane_kernel<float, 512, 1>(KArgs);
template __global__ void lane_kernel<float, 1024, 1>(KArgs);
template __global__ void lane_kernel<float, 512, 2, false>(KArgs);
template __global__ void lane_kernel<float, 512, 2, true>(KArgs);

// Dynamic shared memory to request for a topology: base layout + bit
// matrices + incidence lists + slots, capped at the 227 KB a CTA may use.
size_t smem_bytes_host(int N, int nq, int nslot, int ninc, bool periodic, bool skin, int real_size, int nunit,
                       bool dbuf, int nsite) {
  SmemPlan p = smem_plan(N, nq, nslot, ninc, periodic, skin, real_size, nunit, dbuf, nsite);
  size_t want = p.base + (p.mask <= MASK_SMEM_MAX ? p.mask : 0) + p.inc + p.slots + p.near + p.cst + p.exc + 64;
  return want < 227 * 1024 ? want : 227 * 1024;
}

size_t smem_base_host(int N, int nq, int nslot, int ninc, bool periodic, bool skin, int real_size, int nunit,
                      bool dbuf) {
  return smem_plan(N, nq, nslot, ninc, periodic, skin, real_size, nunit, dbuf).base;
}

cudaError_t lane_kernel_set_smem(bool mixed, int bytes, int bytes2) {
  cudaError_t e;
  if (mixed) {
    e = cudaFuncSetAttribute(lane_kernel<float, 512, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(lane_kernel<float, 1024, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    if (bytes2 > 0) {
      e = cudaFuncSetAttribute(lane_kernel<float, 512, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes2);
      if (e != cudaSuccess) return e;
      return cudaFuncSetAttribute(lane_kernel<float, 512, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes2);
    }
    return cudaSuccess;
  }
  return cudaFuncSetAttribute(lane_kernel<double, 512, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// block: threads per CTA (mixed: up to 1024, FP64: up to 512)
cudaError_t lane_kernel_launch(bool mixed, int grid, int block, size_t smem, cudaStream_t st, const KArgs &a) {
  if (mixed && block > 512) lane_kernel<float, 1024, 1><<<grid, block, smem, st>>>(a);
  else if (mixed) lane_kernel<float, 512, 1><<<grid, block, smem, st>>>(a);
  else lane_kernel<double, 512, 1><<<grid, block, smem, st>>>(a);
  return cudaGetLastError();
}

// Two CTAs per lane (clusters of 2): nlane lanes, 512 threads, KM_STEP only.
cudaError_t lane_kernel_launch_pair(int nlane, size_t smem, cudaStream_t st, const KArgs &a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * nlane, 1, 1);
  cfg.blockDim = dim3(512, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (a.n_step_neighbor <= 0) return cudaLaunchKernelEx(&cfg, lane_kernel<float, 512, 2, true>, a);
  return cudaLaunchKernelEx(&cfg, lane_kernel<float, 512, 2, false>, a);
}

} // namespace tis
