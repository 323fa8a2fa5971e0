// common.cuh -- device-side data layout shared by the lane kernels and the
// host API of libtis_b200.so.
//
// A *lane* is one system replica (one CTA of the persistent kernel).  Lanes
// point at a *topology* (interaction tables shared by the replicas of one
// chain) and at a *label* (temperature-dependent parameters; labels are
// swapped between lanes by replica exchange).  All per-bead state is FP64,
// Fortran order (xyz fastest): x[3*(state0 + i) + d].
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#endif

namespace tis {

constexpr int MAX_THREADS = 1024;
constexpr int N_ETYPE = 25;   // E_TYPE%MAX
constexpr int CHMAX = 1024;   // electrostatic row chunks per lane (at least one per charged bead)
constexpr int EW_F_SPLIT = 4; // k ranges of the reciprocal-space forces: f_ext holds one (3, nbead_total)
                              // plane of partial forces per range, added in range order
// HI_TENSOR (const_index.F90:39-45)
constexpr int TIS_HI_RPY_DEV = 1, TIS_HI_RPY_OVER_DEV = 2, TIS_HI_ERMAK_OVER_DEV = 3, TIS_HI_ZUK_RPY_DEV = 4;

// per-topology descriptor (offsets into the concatenated topology arrays)
struct TopDesc {
  int nmp, nunit;
  int bead0;        // per-bead topology arrays
  int unit0;        // lunit2mp / iclass_unit (2 ints per unit) and rneigh2 (nunit^2 doubles at rn0)
  int rn0;
  int bd0, nbd;
  int ba0, nba;
  int st0, nst;
  int tst0, ntst;   // tertiary stacks
  int stx0;         // per secondary stack: stx_ptr[stx0 + k] .. (+1) -> tertiary stacks that can disable it
  int hb0, nhb;
  int site0, nsite;
  int sitehb0;      // CSR of hbonds per site: site_ptr[site0 + s] .. (+1), entries at sitehb0
  int inc0;         // incidence CSR: inc_ptr[inc0 + i] (nmp + 1 entries), values index inc_slot
  int ninc;         // incidence entries of this topology
  int q0, nq;       // charged beads (|q| >= ZERO_JUDGE), bead indices at q_bead[q0 ..], ascending
  int fe0, nfe;     // FENE records
  int wc0, nwc;     // WCA records
  int bp0, be0;     // Brownian-HI force incidence: bd_ptr[bp0 .. bp0 + nmp], entries from bd_ent[be0]
  int nslot;        // 2 nbd + 3 nba + 7 nst + 6 ntst + 6 nhb
  int slot_ba, slot_st, slot_tst, slot_hb;   // slot bases inside a lane (bonds start at 0)
  int nlabel;       // labels that belong to this topology
};

// per-lane descriptor
struct LaneDesc {
  int top;
  int state0;       // bead offset of this lane's state
  int mask0;        // list bit matrices: exv then ele, nmp rows of ceil(nmp / 32) words
  long long mirror0;// periodic: nmp x nmp bytes (canonical pair mirror index)
  int slot0;        // slots x 3 values
  int hb0;          // hb flags / status / energies (nhb each)
  int site0;        // per-lane hbond-site excess counters (nsite ints)
  int unif0;        // injected uniform stream (n_uniform per lane)
  int ew0;          // Ewald: first charge of this lane in the per-lane charge tables
  long long bd0;    // Brownian-HI: first element of this lane's (3N)^2 diffusion / Cholesky matrices
  long long bdp0;   // Brownian-HI, tensor cores: first float of this lane's TF32 panel planes
  long long bd32;   // Brownian-HI, mixed precision: first float of this lane's FP32 D and L (rows padded to 4)
  long long bdw0;   // Brownian-HI refinement: first float of this lane's inverses of the diagonal tiles of L
  int key_lane;     // counter-based noise and uniforms: the replica's key (its global replica number - 1)
  int key_bead0;    // and the counter of its first bead (so a replica draws the same numbers in any context)
};

// Mutable per-lane scalar state, kept in global memory between launches.
struct LaneState {
  long long istep;
  long long nrebuild;
  long long nclamp;
  long long last_rebuild;   // istep of the last neighbour rebuild (-1: none)
  int label;          // global label index
  int unif_pos;
  int flags;          // bit 0 list overflow, 1 nan, 2 uniforms exhausted, 3 noise exhausted
  int nexv, nele;     // half-list sizes at the last rebuild
  int need_rebuild;
};

enum LaneFlags { LF_OVERFLOW = 1, LF_NAN = 2, LF_UNIF_EXHAUSTED = 4, LF_NOISE_EXHAUSTED = 8, LF_PMF = 16,
                 LF_SMEM = 32 /* the lane's base layout did not fit the launch's shared memory: nothing ran */ };

enum KMode {
  KM_NEIGHBOR = 1,     // rebuild lists (wrap pxyz if periodic)
  KM_FORCE = 2,        // force_sumup -> out_force
  KM_PRE = 3,          // time_integral_pre: lists, force, a(0)
  KM_STEP = 4,         // nsteps of time_integral
  KM_XSTEP = 5,        // first half of one step: trigger, rebuild, x update
  KM_VSTEP = 6,        // second half of one step: forces (+ f_ext), v / a update
  KM_VXSTEP = 7,       // KM_VSTEP, then the KM_XSTEP of the next step
};

// Kernel arguments (all device pointers).
struct KArgs {
  // sizes
  int nlane;
  int nsteps;
  int mode;
  int only_lane;       // -1: every lane
  int group;           // threads per bead in the gather pass (power of two <= 32)
  // constants
  int periodic;
  double psize[3], psizeh[3];
  double neigh_margin;
  int n_step_neighbor;
  double exv_dist, exv_dist_PS, exv_adjust, exv_inf;
  int nsep[3];         // P, S, B
  int i_ele;           // 0 none, 1 DH, 2 Ewald
  double cutoff_ele;   // DH: in Debye lengths; Ewald: real-space cutoff in A
  // Ewald (force_ele_coulomb_ewld.F90, mloop_ewld.F90)
  double ewld_alpha, ewld_beta;   // alpha, 2 alpha / sqrt(pi)
  double ewld_self;               // -alpha / sqrt(pi)
  int nk;                         // reciprocal vectors, all +-h with |h| <= hmax
  int hmax;                       // ceil(hmax): per-dimension table length - 1
  int nqblk;                      // charge blocks of the structure-factor partial sums
  double two_pi_L[3];             // 2 pi / L
  const int8_t *ew_h;             // (nk, 3) integer h
  const double *ew_coef;          // (nk) 2 pi / L^3 exp(-k^2 / 4 alpha^2) / k^2
  double *ew_tab;                 // (q, 3, hmax + 1) of (cos, sin)(2 pi h x / L), per lane's charges
  double *ew_S;                   // (lane, nqblk, nk, 2) partial sums of q cos, q sin
  double *f_ext;                  // (3, nbead_total) force added to each bead's sum, or null
  // Brownian dynamics with hydrodynamic interactions (time_integral.F90:429-457)
  const int *fene_idx; const double *fene_nat, *fene_coef, *fene_d2;   // force_fene.F90
  const int *wca_idx; const double *wca_nat, *wca_coef;                 // force_wca.F90 (coef: rep, att)
  double wca_rcut2;                // 1 / cutoff_wca^2
  const int *bd_ptr;               // per bead: range of its records in bd_ent
  const int2 *bd_ent;              // (partner bead, parameter class * 2 + kind (0 FENE, 1 WCA))
  const double *fene_cls, *wca_cls;// parameter classes: FENE (nat, coef, dist2), WCA (nat, coef rep, coef att)
  double *bd_D, *bd_L;             // per lane (3N x 3N, row-major): diffusion tensor (FP64 path), Cholesky factor
  float *bd_D32, *bd_L32;          // mixed precision: FP32 D and lower factor read by the step's matrix-vector products
  double *bd_F, *bd_xi;            // per lane (3N): force, Gaussian noise of the step
  float *bd_P;                     // per lane: TF32 hi / lo planes of the current Cholesky panel
  double *bd_W;                    // per lane: 64 x 64 transposed inverse of the current diagonal tile
  int *not_spd;                    // per lane: a Cholesky pivot was <= 0
  double hi_radius, viscosity;
  int i_hydro_tensor;              // HI_TENSOR: 1 RPY, 2 RPY_OVER, 3 ERMAK_OVER, 4 ZUK_RPY
  // refinement of the mixed-precision noise: E = L L^T - D (FP32 L of the step, FP64 sums), W = inverses
  // of the diagonal 64 x 64 tiles of L, z = L^-T xi; the step adds -E z / 2 to L xi
  int bd_refine;
  double *bd_D64;                  // per lane (3N x 3N, row-major): D in FP64 (refinement)
  float *bd_E32;                   // per lane: E, rows padded like bd_D32
  float *bd_W32;                   // per lane: (T, 64, 64) inverses of the diagonal tiles
  double *bd_z;                    // per lane (3N): z
  const double *b_hrad;            // per bead: hydrodynamic radius (ZUK_RPY; the others take bead 1's)
  double boltz, pi;                // BOLTZ_KCAL_MOL and F_PI of const_physical.F90
  long long bd_istep;              // step being taken (1-based)
  int bd_kpanel;                   // Cholesky panel of this launch
  int bd_tc;                       // 1: trailing updates on the tensor cores (3xTF32 split, FP32 accumulation)
  double hb_cutoff_dist;
  double max_abscos;   // MAX_ANG_ABSCOS_HBOND15 == MAX_DIH_ABSCOS_HBOND15
  double tstep, tstep2, tsteph;
  double beta_hbond15; // global quirk value (used when hb_beta_global and rex is null)
  const struct RexState *rex;   // device replica-exchange state (its beta_global overrides beta_hbond15)
  int hb_beta_global;
  unsigned long long seed;
  // descriptors
  const TopDesc *tops;
  const LaneDesc *lanes;
  LaneState *lstate;
  // topology arrays
  const int8_t *b_type;    // MPTYPE
  const int8_t *b_class;   // CLASS of the bead's unit
  const int16_t *b_unit;   // unit index (local)
  const double *b_rcmass, *b_fric, *b_radius, *b_eps, *b_charge;
  const double *b_screen;  // largest exv contact distance of the bead with any bead of its topology
  const int *u_lunit;      // (first, last) 0-based per unit
  const int *u_class;
  const double *rneigh2;   // per topology nunit x nunit
  const int *bd_idx; const double *bd_nat, *bd_coef;
  const int *ba_idx; const double *ba_nat, *ba_coef;
  const int *st_idx; const double *st_nat, *st_coef;
  const int *tst_idx; const double *tst_nat, *tst_coef;   // tertiary stacks: 6 beads, 6 natives, U0 + 6 coefs
  const int *stx_ptr, *stx_tst;    // secondary stack -> exclusive tertiary stacks (topology-local index)
  const int *hb_idx; const double *hb_nat, *hb_coef; const int *hb_site; const double *hb_nd2;
  const uint8_t *hb_tert;            // (hb) 1: tertiary hydrogen bond; null when there are none
  const int *site_val; const int *site_ptr; const int *site_hb;
  const int *inc_ptr; const int *inc_slot;
  const int *q_bead;
  // DT19 semi-explicit ions and Manning charges (simu_ele_set.F90:107-253)
  int dt19;                // i_dtrna_model == 2019
  const uint8_t *b_qkind;  // per bead 1: the charge is -Zp of the lane's label; null: no such bead
  const double *lab_zp;    // per label
  const double *pmf_e, *pmf_f;   // per label, pmf_nbin each: Mg-P energy and force tables; null: none
  int pmf_nbin;
  double pmf_rmin, pmf_rbin, pmf_rbininv, pmf_rmax;
  // labels (temperature-dependent parameters)
  const double *lab_T, *lab_coef, *lab_cdist, *lab_beta, *lab_rele2;
  const int *lab_u0off; const double *lab_u0;   // stack U0(T) per label
  const int *lab_c1off; const double *lab_c1;   // rlan_const(1) per label and bead
  const double *b_c2, *b_c3, *b_c4;             // rlan_const(2..4) per bead
  // state
  double *xyz, *pxyz, *velo, *accel, *dxyz;
  double *p0xyz;           // periodic: pxyz as wrapped at the last rebuild (fixes each pair's image)
  // lists and scratch
  uint32_t *mask; uint8_t *mirror;
  int smem_total;          // dynamic shared memory bytes of the launch
  void *slots;             // float or double triplets
  uint8_t *hb_flag;        // bit0 in neighbour list, bit1 status
  double *hb_ene;
  int *site_exc;
  // energy evaluation (energy_kernel)
  const int *elabel;       // per lane label override (-1: own label)
  int reuse_hb;            // 1: sum the hbond energies of the last force pass (flg_hb_energy)
  const uint8_t *hb_flag_src; // energy pass with its own hbond scratch (hb_flag, hb_ene, site_exc):
                              // the list bits of the lanes' hb_flag are read from here; null: hb_flag
  double ebeta;            // beta_hbond15 for a recomputed hbond pruning
  const double *ebeta_lane;// per lane beta (overrides ebeta when set)
  double *out_energy;      // (N_ETYPE) per lane
  const double *b_cmass;
  int i_DH_cutoff_type;
  // io
  double *out_force;       // (3, nmp) per lane at state0
  const double *noise;     // injected: (3, nbead_total, noise_nsteps)
  int noise_nsteps;
  int noise_base;          // noise step consumed by the first step of this launch
  const double *unif;      // injected uniforms per lane
  int n_unif;
  int nbead_total;
  int noise_in_sweep;      // 1: the sink's noise is drawn in the bonded sweep (kept in shared memory)
  int sweep_mode;          // bonded sweep of one CTA per lane: 0 snake deal, 1 shared counter, 2 longest-first deal
  const int *lane_nsteps;  // per lane: steps of this launch (KM_STEP) or 1 + the last step index that
                           // moves the lane (KM_XSTEP / KM_VSTEP); null: every lane takes nsteps
  int step_k;              // KM_XSTEP / KM_VSTEP: index of this step within the call
  const int *lane_order;   // lane of each CTA (or cluster) of a launch over every lane; null: in order
};

#ifdef __CUDACC__
// charge of bead b (index into the bead tables) under label lab:
// coef_charge(icharge, grep) of the reference
__device__ __forceinline__ double bead_charge(const KArgs &a, int lab, int b) {
  return (a.b_qkind && a.b_qkind[b]) ? -a.lab_zp[lab] : a.b_charge[b];
}

// neighbor_list_ele.F90:167-174: Mg-P pairs take the PMF table (DT19)
__device__ __forceinline__ bool mg_p_pair(int ti, int tj) {
  return (ti == 2 && tj == 5) || (ti == 5 && tj == 2);
}

// force_ele_DH.F90:90-94: 0-based table bin of a Mg-P distance.  Below the
// first point the reference stops; here the pair takes bin 0 and low is set.
__device__ __forceinline__ int pmf_bin(const KArgs &a, double d, bool &low) {
  if (!(d >= a.pmf_rmin)) { low = true; return 0; }
  const int ib = (int)floor((d - a.pmf_rmin) * a.pmf_rbininv);
  return min(ib, a.pmf_nbin - 1);
}
#endif

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of the 4x32 S-box with the published
// multipliers and Weyl key increments.
// Replica-exchange state kept on the device (simu_replica_exchange.F90,
// var_replica.F90), so that an exchange needs no host round trip.
struct RexState {
  double beta_global;          // beta_hbond15: the last replica's label (simu_set_dtrna.F90:58, simu_para2)
  unsigned long long counter;  // counter of the exchange's counter-based uniforms
  int idx_pair;                // odd/even pair alternation (var_replica.F90:134,165-183)
  int nacc;                    // swaps accepted by the last exchange
};

// exchange_pair_tb of one temperature dimension (var_replica.F90:165-183):
// the partner of label l (1-based) among n under the odd/even alternation
// idx_pair, 0 = no partner
__host__ __device__ inline int rex_pair(int l, int n, int idx_pair) {
  if (idx_pair == 1) return (l % 2 == 1) ? ((l + 1 <= n) ? l + 1 : 0) : l - 1;
  if (l == 1) return 0;
  return (l % 2 == 0) ? ((l + 1 <= n) ? l + 1 : 0) : l - 1;
}

struct U4 { uint32_t x, y, z, w; };

__host__ __device__ inline void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

__host__ __device__ inline U4 philox4x32(U4 ctr, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, ctr.x, hi0, lo0);
    mulhilo32(M1, ctr.z, hi1, lo1);
    U4 o;
    o.x = hi1 ^ ctr.y ^ k0;
    o.y = lo1;
    o.z = hi0 ^ ctr.w ^ k1;
    o.w = lo0;
    ctr = o;
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}

// uniform in (0, 1]: (u + 1) * 2^-32
__host__ __device__ inline double u01_open0(uint32_t u) { return ((double)u + 1.0) * 2.3283064365386963e-10; }
__host__ __device__ inline float u01f_open0(uint32_t u) { return ((float)(u >> 8) + 1.0f) * 5.9604645e-08f; }

} // namespace tis
