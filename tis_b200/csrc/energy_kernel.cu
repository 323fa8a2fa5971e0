// energy_kernel.cu -- energy_sumup on the device and the replica-exchange
// velocity rescale.
#include "device_common.cuh"

// =====================================================================
// energy_sumup (src/energy_sumup.F90:11-530) for one lane per CTA, FP64.
// Terms follow the energy twins: energy_bond, energy_bangle (via
// util_bondangle), energy_dtrna_stack, energy_dtrna_stack_nlocal,
// energy_dtrna_hbond15, energy_exv_dt15,
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

enum { ES_VELO, ES_BOND, ES_ANGLE, ES_STACK, ES_HB, ES_EXV, ES_ELE, ES_WREP, ES_WATT, ES_TST, ES_THB, ES_N };

constexpr int EK_THREADS = 512;
// beads whose (pxyz, charge) the energy kernels stage in shared memory:
// 1472 x 32 bytes and the kernels' static arrays fit the 48 KB a launch gets
// without opting in; larger lanes read pxyz from global memory
constexpr int EK_STAGE_MAX = 1472;

__device__ __forceinline__ void energy_lane(const KArgs &a, int lane) {
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const int N = T.nmp;
  const int tid = threadIdx.x, nth = blockDim.x;
  LaneState &st = a.lstate[lane];
  const int label = (a.elabel && a.elabel[lane] >= 0) ? a.elabel[lane] : st.label;
  const double *X = a.xyz + 3 * (size_t)L.state0;
  const double *P = a.pxyz + 3 * (size_t)L.state0;
  const double *V = a.velo + 3 * (size_t)L.state0;
  __shared__ double red[ES_N][EK_THREADS / 32];
  // the pair loops read pxyz and the charge of every partner: staged in
  // shared memory (the same doubles) when the lane fits
  extern __shared__ double4 ek_pq[];
  const bool staged = N <= EK_STAGE_MAX;
  if (staged)
    for (int i = tid; i < N; i += nth) {
      const double3 p = gpos(P, i);
      ek_pq[i] = make_double4(p.x, p.y, p.z, bead_charge(a, label, T.bead0 + i));
    }
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
  // energy_fene.F90 (added to E_TYPE%BOND) and energy_wca.F90
  for (int k = tid; k < T.nfe; k += nth) {
    const int r = T.fe0 + k;
    double3 v = sub3(gpos(X, a.fene_idx[2 * r + 1]), gpos(X, a.fene_idx[2 * r]));
    const double dd = sqrt(dot3(v, v)) - a.fene_nat[r];
    es[ES_BOND] += -0.5 * a.fene_coef[r] * a.fene_d2[r] * log(1.0 - dd * dd / a.fene_d2[r]);
  }
  for (int k = tid; k < T.nwc; k += nth) {
    const int r = T.wc0 + k;
    double3 v = sub3(gpos(X, a.wca_idx[2 * r + 1]), gpos(X, a.wca_idx[2 * r]));
    const double ro2 = a.wca_nat[r] * a.wca_nat[r] / dot3(v, v);
    if (ro2 < a.wca_rcut2) continue;
    const double ro3 = ro2 * ro2 * ro2, ro6 = ro3 * ro3;
    if (ro2 >= 1.0) {
      es[ES_WREP] += a.wca_coef[2 * (size_t)r] * (ro6 - 2.0 * ro3 + 1.0);
      es[ES_WATT] += -a.wca_coef[2 * (size_t)r + 1];
    } else {
      es[ES_WATT] += a.wca_coef[2 * (size_t)r + 1] * (ro6 - 2.0 * ro3);
    }
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
  // energy_dtrna_stack_nlocal.F90:106-232: U0 / ediv of every tertiary stack
  auto tdv = [&](const int *m, int p, int q) {   // x_p - x_q (pxyz + minimum image when periodic)
    double3 u = sub3(gpos(a.periodic ? P : X, m[p]), gpos(a.periodic ? P : X, m[q]));
    if (a.periodic) { pb1(u.x, a.psize[0], a.psizeh[0]); pb1(u.y, a.psize[1], a.psizeh[1]); pb1(u.z, a.psize[2], a.psizeh[2]); }
    return u;
  };
  for (int k = tid; k < T.ntst; k += nth) {
    const int *m = a.tst_idx + 6 * (size_t)(T.tst0 + k);
    const double *nat = a.tst_nat + 6 * (size_t)(T.tst0 + k);
    const double *cf = a.tst_coef + 7 * (size_t)(T.tst0 + k);
    const double3 v12 = tdv(m, 0, 1), v13 = tdv(m, 0, 2), v53 = tdv(m, 4, 2), v42 = tdv(m, 3, 1), v46 = tdv(m, 3, 5);
    const double d1212 = dot3(v12, v12), d1313 = dot3(v13, v13), d4242 = dot3(v42, v42);
    const double a12 = sqrt(d1212), a13 = sqrt(d1313), a42 = sqrt(d4242);
    double ediv = 1.0;
    double d = a12 - nat[0];
    ediv += cf[1] * d * d;
    d = acos(dot3(v13, v12) / (a13 * a12)) - nat[1];
    ediv += cf[2] * d * d;
    d = acos(dot3(v12, v42) / (a12 * a42)) - nat[2];
    ediv += cf[3] * d * d;
    const double3 c4212 = cross3(v42, v12), c1213 = cross3(v12, v13);
    d = wrapd(atan2(dot3(v42, c1213) * sqrt(d1212), dot3(c4212, c1213)) - nat[3]);
    ediv += cf[4] * d * d;
    const double3 n1 = make_double3(-c1213.x, -c1213.y, -c1213.z);
    d = wrapd(atan2(dot3(v53, n1) * a13, dot3(cross3(v53, v13), n1)) - nat[4]);
    ediv += cf[5] * d * d;
    const double3 m2 = make_double3(-c4212.x, -c4212.y, -c4212.z), n2 = cross3(v42, v46);
    d = wrapd(atan2(dot3(v12, n2) * a42, dot3(m2, n2)) - nat[5]);
    ediv += cf[6] * d * d;
    es[ES_TST] += cf[0] / ediv;
  }
  const double *u0 = a.lab_u0 + a.lab_u0off[label];
  for (int k = tid; k < T.nst; k += nth) {
    const int *m = a.st_idx + 7 * (size_t)(T.st0 + k);
    // st_status (energy_dtrna_stack_nlocal.F90:121-129): an exclusive
    // tertiary stack within 10 A of its native distance turns the stack off
    bool off = false;
    for (int e = (T.ntst ? a.stx_ptr[T.stx0 + k] : 0); e < (T.ntst ? a.stx_ptr[T.stx0 + k + 1] : 0); ++e) {
      const int t = a.stx_tst[e];
      const int *mt = a.tst_idx + 6 * (size_t)(T.tst0 + t);
      const double3 u = tdv(mt, 0, 1);
      const double dd = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(u.x, u.x), __dmul_rn(u.y, u.y)), __dmul_rn(u.z, u.z))) -
                        a.tst_nat[6 * (size_t)(T.tst0 + t)];
      if (dd < 10.0) off = true;
    }
    if (off) continue;
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
  // non-bonded pairs j > i from the global copy of the list bit matrices
  const int W = (N + 31) >> 5;
  const uint32_t *mexv = a.mask + L.mask0, *mele = mexv + (size_t)N * W;
  const uint8_t *mir = a.periodic ? (a.mirror + L.mirror0) : nullptr;
  const double cdist = a.lab_cdist[label], coefT = a.lab_coef[label];
  // DH: energy_ele_DH.F90:33 scales the cutoff only for i_DH_cutoff_type 0;
  // Ewald: real-space cutoff in A (energy_ele_coulomb_ewld.F90:137)
  const double cut2 = (a.i_ele == 1 && a.i_DH_cutoff_type == 0) ? (a.cutoff_ele * cdist) * (a.cutoff_ele * cdist)
                                                                : a.cutoff_ele * a.cutoff_ele;
  const double rcd = 1.0 / cdist;
  auto ppos = [&](int i) {
    if (staged) { const double4 v = ek_pq[i]; return make_double3(v.x, v.y, v.z); }
    return gpos(P, i);
  };
  auto pq = [&](int i) { return staged ? ek_pq[i].w : bead_charge(a, label, T.bead0 + i); };
  auto shifted = [&](int i, int j) {   // j > i: canonical orientation
    double3 w = sub3(ppos(j), ppos(i));
    if (mir) {
      const int im = (int)mir[(size_t)i * N + j] - 1;
      const int m0 = im / 9, m1 = (im / 3) % 3, m2 = im % 3;
      if (m0 != 2) w.x += (m0 == 0 ? -a.psize[0] : a.psize[0]);
      if (m1 != 2) w.y += (m1 == 0 ? -a.psize[1] : a.psize[1]);
      if (m2 != 2) w.z += (m2 == 0 ? -a.psize[2] : a.psize[2]);
    }
    return w;
  };
  // one item per (row i, word w) of the upper triangle, so the rows of
  // charged beads with many partners spread over many threads
  for (int it = tid; it < N * W; it += nth) {
    const int i = it / W, w = it - i * W;
    if (w < ((i + 1) >> 5)) continue;
    const int ti = a.b_type[T.bead0 + i], ci = a.b_class[T.bead0 + i];
    const double q_i = pq(i);
    const bool qi = fabs(q_i) >= 1.0e-6;
    {
      uint32_t me = mexv[(size_t)i * W + w], ml = (a.i_ele != 0 && qi) ? mele[(size_t)i * W + w] : 0u;
      if (w == ((i + 1) >> 5)) {   // keep bits j > i only
        const uint32_t keep = ((i + 1) & 31) ? ~((1u << ((i + 1) & 31)) - 1u) : 0xffffffffu;
        me &= keep; ml &= keep;
      }
      while (me) {
        const int j = (w << 5) + __ffs(me) - 1;
        me &= me - 1;
        const double3 v = shifted(i, j);
        const int tj = a.b_type[T.bead0 + j], cj = a.b_class[T.bead0 + j];
        double dij;
        if (a.dt19)   // energy_exv_dt15.F90:67-73
          dij = (ti == 3 && tj == 3) ? a.exv_dist : a.b_radius[T.bead0 + i] + a.b_radius[T.bead0 + j];
        else if ((ti == 2 && tj == 4) || (ti == 4 && tj == 2)) dij = a.exv_dist_PS;
        else if (ci == 2 && cj == 2) dij = a.exv_dist;
        else dij = a.b_radius[T.bead0 + i] + a.b_radius[T.bead0 + j];
        double dist = sqrt(dot3(v, v));
        if (dist <= dij) {
          dist = dist + a.exv_adjust - dij;
          double ene;
          if (dist > a.exv_inf) {
            double ro = a.exv_adjust / dist, ro2 = ro * ro, ro6 = ro2 * ro2 * ro2;
            ene = a.b_eps[T.bead0 + i] * a.b_eps[T.bead0 + j] * (ro6 * ro6 - 2 * ro6 + 1.0);
          } else {
            ene = 1.0e10;   // HIGH_ENERGY
          }
          es[ES_EXV] += ene;
        }
      }
      while (ml) {
        const int j = (w << 5) + __ffs(ml) - 1;
        ml &= ml - 1;
        const double3 v = shifted(i, j);
        const double r2 = dot3(v, v);
        if (r2 <= cut2) {
          const double dist1 = sqrt(r2);
          if (a.pmf_e && mg_p_pair(ti, a.b_type[T.bead0 + j]) && dist1 <= a.pmf_rmax) {
            // energy_ele_DH.F90:77-95: linear between the table points
            bool low = false;
            const int ib = pmf_bin(a, dist1, low);
            const double *pe = a.pmf_e + (size_t)label * a.pmf_nbin, *pf = a.pmf_f + (size_t)label * a.pmf_nbin;
            es[ES_ELE] += pe[ib] - pf[ib] * (dist1 - (a.pmf_rmin + (double)ib * a.pmf_rbin));
            continue;
          }
          const double ce = q_i * pq(j) * coefT;
          if (a.i_ele == 1) es[ES_ELE] += ce / dist1 * exp(-dist1 * rcd);
          else if (a.i_ele == 3) es[ES_ELE] += ce * (1.0e0 / dist1 - 1.0e0 / a.cutoff_ele);   // energy_ele_coulomb.F90:66
          else es[ES_ELE] += ce * erfc(a.ewld_alpha * dist1) / dist1;
        }
      }
    }
  }
  // hydrogen bonds (energy_dtrna_hbond15.F90)
  if (!a.reuse_hb) {
    for (int h = tid; h < T.nhb; h += nth) {
      uint8_t f = (a.hb_flag_src ? a.hb_flag_src + L.hb0 : hbf)[h] & 1;
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
      prune_hbonds<double>(a, lane, L, T, st.istep,
                           a.ebeta_lane ? a.ebeta_lane[lane] : (a.rex ? a.rex->beta_global : a.ebeta), false, exc);
    __syncthreads();
  }
  // energy_dtrna_hbond15.F90:135-143: tertiary ('T') bonds count separately
  for (int h = tid; h < T.nhb; h += nth)
    if ((hbf[h] & 3) == 3) es[(a.hb_tert && a.hb_tert[T.hb0 + h]) ? ES_THB : ES_HB] += hbe[h];
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
    E[22] = tot[ES_WREP];
    E[23] = tot[ES_WATT];
    E[18] = tot[ES_TST];
    E[19] = tot[ES_THB];
    double sum = 0.0;
    for (int k = 2; k < N_ETYPE; ++k) sum += E[k];
    E[0] = sum;
  }
}

__global__ void __launch_bounds__(EK_THREADS) energy_kernel(KArgs a) {
  const int lane = (a.only_lane >= 0) ? a.only_lane : (int)blockIdx.x;
  if (lane >= a.nlane) return;
  energy_lane(a, lane);
}

// The two energy passes of an exchange in one launch: block l < nlane the
// own label of lane l (args a), block nlane + l the partner label (args b,
// whose hbond recomputation uses its own scratch, so the passes can run
// together)
__global__ void __launch_bounds__(EK_THREADS) energy_pair_kernel(KArgs a, KArgs b) {
  const int l = (int)blockIdx.x;
  if (l < a.nlane) energy_lane(a, l);
  else if (l < 2 * a.nlane) energy_lane(b, l - a.nlane);
}

// dynamic shared memory for the largest lane that stages (every lane with
// N <= EK_STAGE_MAX stages, so the launch must hold min(max_nmp, EK_STAGE_MAX))
inline size_t ek_smem(int max_nmp) { return (size_t)(max_nmp < EK_STAGE_MAX ? max_nmp : EK_STAGE_MAX) * sizeof(double4); }

cudaError_t energy_kernel_launch(int grid, int max_nmp, cudaStream_t st, const KArgs &a) {
  const size_t smem = ek_smem(max_nmp);
  energy_kernel<<<grid, EK_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t energy_pair_launch(int nlane, int max_nmp, cudaStream_t st, const KArgs &a, const KArgs &b) {
  const size_t smem = ek_smem(max_nmp);
  energy_pair_kernel<<<2 * nlane, EK_THREADS, smem, st>>>(a, b);
  return cudaGetLastError();
}

// ----------------------------------------------------------------------
// st_status of every secondary stack of one lane (force_dtrna_stack_nlocal.
// F90:83-92) at the lane's current coordinates, for the restart's DTRNA15
// block; the same FP64 test as the force pass.
__global__ void st_status_kernel(KArgs a, int lane, int *out) {
  const LaneDesc L = a.lanes[lane];
  const TopDesc T = a.tops[L.top];
  const double *X = a.xyz + 3 * (size_t)L.state0;
  const double *P = a.pxyz + 3 * (size_t)L.state0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < T.nst; k += gridDim.x * blockDim.x) {
    int on = 1;
    for (int e = (T.ntst ? a.stx_ptr[T.stx0 + k] : 0); e < (T.ntst ? a.stx_ptr[T.stx0 + k + 1] : 0); ++e) {
      const int t = a.stx_tst[e];
      const int *m = a.tst_idx + 6 * (size_t)(T.tst0 + t);
      double3 u = sub3(gpos(a.periodic ? P : X, m[0]), gpos(a.periodic ? P : X, m[1]));
      if (a.periodic) { pb1(u.x, a.psize[0], a.psizeh[0]); pb1(u.y, a.psize[1], a.psizeh[1]); pb1(u.z, a.psize[2], a.psizeh[2]); }
      const double d = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(u.x, u.x), __dmul_rn(u.y, u.y)), __dmul_rn(u.z, u.z))) -
                       a.tst_nat[6 * (size_t)(T.tst0 + t)];
      if (d < 10.0) on = 0;
    }
    out[k] = on;
  }
}

cudaError_t st_status_launch(cudaStream_t st, const KArgs &a, int lane, int nst, int *out) {
  if (nst <= 0) return cudaSuccess;
  st_status_kernel<<<(nst + 127) / 128, 128, 0, st>>>(a, lane, out);
  return cudaGetLastError();
}

// ----------------------------------------------------------------------
// Replica exchange on the device (simu_replica_exchange.F90:121-300, one
// temperature dimension).  rex_prep_kernel: the partner label of every lane
// for this exchange's odd/even pairing and the partner's beta; the energy
// kernel then evaluates every lane at its partner label.
// rex_exchange_kernel (one CTA): thread 0 runs the Metropolis decisions in
// label order with counter-based uniforms (or injected ones), updates the
// label maps, the pair alternation and beta_hbond15; then the CTA writes the
// lanes' labels.  vscale_kernel then rescales the velocities of the swapped
// lanes, one block per lane.


__global__ void rex_prep_kernel(KArgs a, const int *rep2lab, int *elabel, double *ebeta) {
  const int lane = blockIdx.x * blockDim.x + threadIdx.x;
  if (lane >= a.nlane) return;
  const int lo = rex_pair(rep2lab[lane] + 1, a.nlane, a.rex->idx_pair);
  elabel[lane] = lo ? lo - 1 : -1;
  ebeta[lane] = lo ? 1.0e0 / (a.lab_T[lo - 1] * a.boltz) : a.rex->beta_global;
}

__global__ void __launch_bounds__(256) rex_exchange_kernel(KArgs a, RexState *rex, int *rep2lab, int *lab2rep,
                                                           const double *e_own, const double *e_opp,
                                                           const double *u, double *scale, double *velo) {
  const int n = a.nlane, tid = threadIdx.x;
  const int ip = rex->idx_pair;
  const unsigned long long ctr = rex->counter;
  __shared__ int s_npair, s_nacc;
  for (int r = tid; r < n; r += blockDim.x) scale[r] = 0.0;
  if (tid == 0) { s_npair = 0; s_nacc = 0; }
  __syncthreads();
  // simu_replica_exchange.F90:121-267.  The pairs of one exchange are
  // disjoint, so each is decided by its own thread; the k-th pair in label
  // order takes the k-th uniform, as the reference's serial loop draws them.
  for (int li = 1 + tid; li <= n; li += blockDim.x) {
    const int lj = rex_pair(li, n, ip);
    if (lj < li) continue;
    const int k = (ip == 1) ? (li - 1) / 2 : (li - 2) / 2;
    atomicAdd(&s_npair, 1);
    double uu;
    if (u) {
      uu = u[k];
    } else {
      const unsigned long long c = ctr + (unsigned long long)k;
      const U4 o = philox4x32(U4{(uint32_t)c, (uint32_t)(c >> 32), 0x52454D44u, 0u}, (uint32_t)a.seed,
                              (uint32_t)(a.seed >> 32));
      uu = u01_open0(o.x) - 2.3283064365386963e-10;   // [0, 1)
    }
    const int ri = lab2rep[li - 1], rj = lab2rep[lj - 1];
    const double tm = a.lab_T[li - 1], tn = a.lab_T[lj - 1];
    const double pim = e_own[(size_t)ri * N_ETYPE], pin = e_opp[(size_t)ri * N_ETYPE];
    const double pjn = e_own[(size_t)rj * N_ETYPE], pjm = e_opp[(size_t)rj * N_ETYPE];
    const double delta = ((pjm - pim) / tm - (pjn - pin) / tn) / a.boltz;
    if (delta < 0.0e0 || uu <= exp(-delta)) {
      rep2lab[ri] = lj - 1; rep2lab[rj] = li - 1;
      lab2rep[li - 1] = rj; lab2rep[lj - 1] = ri;
      const double sf = sqrt(tn / tm);
      scale[ri] = sf;
      scale[rj] = -sf;
      atomicAdd(&s_nacc, 1);
    }
  }
  __syncthreads();
  if (tid == 0) {
    rex->counter = u ? ctr : ctr + (unsigned long long)s_npair;
    rex->nacc = s_nacc;
    rex->idx_pair = (ip == 2) ? 1 : ip + 1;
    rex->beta_global = 1.0e0 / (a.lab_T[rep2lab[n - 1]] * a.boltz);
  }
  for (int r = tid; r < n; r += blockDim.x) a.lstate[r].label = rep2lab[r];
  (void)velo;   // the velocities of the swapped replicas are rescaled by vscale_kernel
}

// velocity rescale of the lanes a ladder exchange swapped: lane l's
// velocities times scale[l] (> 0) or divided by -scale[l] (< 0), as the
// device exchange does; one block per lane
__global__ void vscale_kernel(KArgs a, const double *scale, double *velo) {
  const int lane = blockIdx.x;
  const double f = scale[lane];
  if (f == 0.0) return;
  const LaneDesc L = a.lanes[lane];
  const int N = a.tops[L.top].nmp;
  double *v = velo + 3 * (size_t)L.state0;
  if (f > 0.0) for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) v[k] = f * v[k];
  else for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) v[k] = v[k] / (-f);
}

cudaError_t vscale_launch(cudaStream_t st, const KArgs &a, const double *scale, double *velo) {
  vscale_kernel<<<a.nlane, 128, 0, st>>>(a, scale, velo);
  return cudaGetLastError();
}

cudaError_t rex_launch(cudaStream_t st, const KArgs &a, RexState *rex, int *rep2lab, int *lab2rep, int *elabel,
                       double *ebeta) {
  rex_prep_kernel<<<(a.nlane + 127) / 128, 128, 0, st>>>(a, rep2lab, elabel, ebeta);
  (void)lab2rep; (void)rex;
  return cudaGetLastError();
}

cudaError_t rex_exchange_launch(cudaStream_t st, const KArgs &a, RexState *rex, int *rep2lab, int *lab2rep,
                                const double *e_own, const double *e_opp, const double *u, double *scale,
                                double *velo) {
  rex_exchange_kernel<<<1, 256, 0, st>>>(a, rex, rep2lab, lab2rep, e_own, e_opp, u, scale, velo);
  // time_integral.F90 velocity rescale of the swapped replicas, one block each
  vscale_kernel<<<a.nlane, 128, 0, st>>>(a, scale, velo);
  return cudaGetLastError();
}

} // namespace tis
